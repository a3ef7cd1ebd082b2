// FP64 grouped segmented-K GEMM on the FP64 tensor cores (DMMA).
//
// One launch executes every task of one stage of the block-sparse matvec
// (the reference runs them as one serial BLAS call each, src/qtensor.cpp:986-994).
// Work unit = one 64x64 tile of one output block over a range of its k-tiles:
// the CTA walks the output block's segments and their K extents, sums
// everything in registers and writes the tile once.  Units are assigned to CTAs
// on the host and laid out so that CTA c takes entries c, c+grid, ...: whole
// tiles longest first onto the least-loaded CTA, or, where that leaves the
// longest CTA a tenth or more above an even split (a stage of few, long tiles),
// the k-tiles of all tiles cut into equal per-CTA shares (stream-K).  A tile
// cut at a share boundary is computed in parts; each part stores its partial
// sum to a workspace slot, and the part that finishes last -- an atomic ticket
// after a fence, no waiting -- adds the slots in slot order and writes the
// tile, so the result does not depend on timing.
//
// Operands are staged by a 3-deep ring of cp.async copies (16-byte when a
// segment's rows are 16-byte aligned, 8-byte otherwise) and consumed by
// mma.sync m16n8k16 (FP64): Blackwell has no FP64 kind of tcgen05.mma, so
// DMMA is the FP64 tensor path.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <vector>

#include <string>

#include "../../include/dmrgx.h"
#include "grouped.h"
#include "kernels.h"

namespace dmrgx {

void set_error(const std::string& msg);

namespace {

constexpr int BM = 64, BN = 64, BK = 16, LDS = BK + 4;  // +4 doubles: conflict-free fragments
constexpr int STAGES = 3, THREADS = 128;
constexpr int kSmemBytes = STAGES * (BM + BN) * LDS * (int)sizeof(double);  // 61,440
constexpr int kSlotDoubles = BM * BN;
// cost model of the unit assignment, in k-tiles: fixed cost of a unit (prologue,
// epilogue) and extra cost of a K-split part (partial store, ticket, reduction share)
constexpr double kUnitOverhead = 6.0, kPartOverhead = 4.0;

__device__ __forceinline__ void cp16(double* sdst, const double* gsrc, int bytes) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gsrc), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp8(double* sdst, const double* gsrc, int bytes) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(gsrc), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// D = A (16x16, row) . B (16x8, col) + D; fragments as the PTX ISA lays out
// mma.m16n8k16 for .f64: a[v0 + 2 v1] = A(g + 8 v0, t + 4 v1), b[v] = B(t + 4 v, g),
// d[c] = D(g + 8 (c >> 1), 2 t + (c & 1)), g = lane / 4, t = lane % 4.
__device__ __forceinline__ void dmma16816(double (&d)[4], const double (&a)[8],
                                          const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
        "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

template <bool CPLX>
__global__ void __launch_bounds__(THREADS, 3)
grouped_gemm_nt_f64(const double* __restrict__ A, const double* __restrict__ B,
                    double* __restrict__ C, const DUnit* __restrict__ units, int nunits,
                    const DOut* __restrict__ outs, const DSeg* __restrict__ segs,
                    double* __restrict__ ws, int* __restrict__ tickets) {
  extern __shared__ __align__(16) double smem[];
  double (*sA)[BM][LDS] = reinterpret_cast<double (*)[BM][LDS]>(smem);
  double (*sB)[BN][LDS] = reinterpret_cast<double (*)[BN][LDS]>(smem + STAGES * BM * LDS);
  __shared__ int s_last;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, t = lane & 3;

  for (int ui = blockIdx.x; ui < nunits; ui += gridDim.x) {
    const DUnit u = units[ui];
    if (u.out < 0) continue;  // padding entry of the CTA assignment
    const DOut o = outs[u.out];
    const int m0 = u.tm * BM, n0 = u.tn * BN;

    // first segment and K offset of the unit's k-tile range
    int s = o.seg_begin, k0 = 0, total = 0;
    {
      const int send = o.seg_begin + o.seg_count;
      int skip = u.kt0;
      bool found = false;
      for (int x = o.seg_begin; x < send; x++) {
        const int nk = (segs[x].k + BK - 1) / BK;
        total += nk;
        if (!found && skip < nk) {
          s = x;
          k0 = skip * BK;
          found = true;
        } else if (!found) {
          skip -= nk;
        }
      }
    }
    const int n_it = max(0, min(u.kt1, total) - u.kt0);

    double acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[i][j][c] = 0.0;

    __syncthreads();  // the previous unit's last reads of the ring are done
    if (n_it > 0) {
      DSeg sg = segs[s];
      // copies of the next k-tile into ring buffer `buf`; advances (s, k0)
      auto issue = [&](int buf) {
        // 16-byte copies when every row of the segment starts on a 16-byte boundary
        const bool a16 = (((reinterpret_cast<uintptr_t>(A) >> 3) + sg.a_off) & 1) == 0 &&
                         (sg.k & 1) == 0;
        const bool b16 = (((reinterpret_cast<uintptr_t>(B) >> 3) + sg.b_off) & 1) == 0 &&
                         (sg.k & 1) == 0;
        if (a16) {
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int c = tid + THREADS * i, r = c >> 3, kk = k0 + 2 * (c & 7), row = m0 + r;
            const bool ok = row < o.m && kk < sg.k;
            cp16(&sA[buf][r][2 * (c & 7)], ok ? A + sg.a_off + (int64_t)row * sg.k + kk : A,
                 ok ? 16 : 0);
          }
        } else {
#pragma unroll
          for (int i = 0; i < 8; i++) {
            const int e = tid + THREADS * i, r = e >> 4, kk = k0 + (e & 15), row = m0 + r;
            const bool ok = row < o.m && kk < sg.k;
            cp8(&sA[buf][r][e & 15], ok ? A + sg.a_off + (int64_t)row * sg.k + kk : A,
                ok ? 8 : 0);
          }
        }
        // B rows: real, or for complex the raw rows n0/2 .. n0/2 + 31 (expanded on read)
        constexpr int BR = CPLX ? BN / 2 : BN;
        const int r0 = CPLX ? (n0 >> 1) : n0, rlim = CPLX ? (o.n >> 1) : o.n;
        if (b16) {
#pragma unroll
          for (int i = 0; i < BR * 8 / THREADS; i++) {
            const int c = tid + THREADS * i, r = c >> 3, kk = k0 + 2 * (c & 7), row = r0 + r;
            const bool ok = row < rlim && kk < sg.k;
            cp16(&sB[buf][r][2 * (c & 7)], ok ? B + sg.b_off + (int64_t)row * sg.k + kk : B,
                 ok ? 16 : 0);
          }
        } else {
#pragma unroll
          for (int i = 0; i < BR * 16 / THREADS; i++) {
            const int e = tid + THREADS * i, r = e >> 4, kk = k0 + (e & 15), row = r0 + r;
            const bool ok = row < rlim && kk < sg.k;
            cp8(&sB[buf][r][e & 15], ok ? B + sg.b_off + (int64_t)row * sg.k + kk : B,
                ok ? 8 : 0);
          }
        }
        k0 += BK;
        if (k0 >= sg.k) {
          k0 = 0;
          // next segment with a K extent (an empty one has no k-tiles in the count)
          while (++s < o.seg_begin + o.seg_count && segs[s].k <= 0) {
          }
          if (s < o.seg_begin + o.seg_count) sg = segs[s];
        }
      };

#pragma unroll
      for (int p = 0; p < STAGES - 1; p++) {
        if (p < n_it) issue(p);
        cp_commit();
      }
      for (int it = 0; it < n_it; it++) {
        cp_wait<STAGES - 2>();
        __syncthreads();  // k-tile `it` visible to all; buffer (it - 1) % STAGES free
        if (it + STAGES - 1 < n_it) issue((it + STAGES - 1) % STAGES);
        cp_commit();
        const int buf = it % STAGES;
        double a[2][8];
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
          for (int v = 0; v < 8; v++)
            a[i][v] = sA[buf][wm + 16 * i + g + 8 * (v & 1)][t + 4 * (v >> 1)];
#pragma unroll
        for (int j = 0; j < 4; j++) {
          double b[4];
          const int r = wn + 8 * j + g;
#pragma unroll
          for (int v = 0; v < 4; v++) {
            const int kk = t + 4 * v;
            if (CPLX) {
              // expanded row r of B: [Br, -Bi] (r even) or [Bi, Br] (r odd) of raw row r / 2
              const int p = r & 1;
              const double x = sB[buf][r >> 1][kk ^ p];
              b[v] = (p == 0 && (kk & 1)) ? -x : x;
            } else {
              b[v] = sB[buf][r][kk];
            }
          }
#pragma unroll
          for (int i = 0; i < 2; i++) dmma16816(acc[i][j], a[i], b);
        }
      }
      cp_wait<0>();
    }

    if (u.nparts > 1) {
      // partial sum to this part's slot; the last part adds the slots in order
      double* w = ws + (int64_t)u.slot * kSlotDoubles;
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
          for (int c = 0; c < 4; c++) w[((i * 4 + j) * 4 + c) * THREADS + tid] = acc[i][j][c];
      __threadfence();
      __syncthreads();
      const int slot0 = u.slot - u.part;
      if (tid == 0) {
        const int prev = atomicAdd(&tickets[slot0], 1);
        s_last = prev == u.nparts - 1;
        if (s_last) tickets[slot0] = 0;  // every part has counted: ready for the next launch
      }
      __syncthreads();
      if (!s_last) continue;
      __threadfence();
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
          for (int c = 0; c < 4; c++) {
            const int q = ((i * 4 + j) * 4 + c) * THREADS + tid;
            double x = 0.0;
            for (int p = 0; p < u.nparts; p++) x += __ldcg(ws + (int64_t)(slot0 + p) * kSlotDoubles + q);
            acc[i][j][c] = x;
          }
    }

    double* pc = C + o.c_off;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int row = m0 + wm + 16 * i + g + 8 * h;
        if (row >= o.m) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int col = n0 + wn + 8 * j + 2 * t;
          if (col < o.n) pc[(int64_t)row * o.n + col] = acc[i][j][2 * h];
          if (col + 1 < o.n) pc[(int64_t)row * o.n + col + 1] = acc[i][j][2 * h + 1];
        }
      }
  }
}

}  // namespace

int f64_tile_m() { return BM; }
int f64_tile_n() { return BN; }
int f64_tile_k() { return BK; }

int f64_split_mode() {
  static const int v = [] {
    const char* e = std::getenv("DMRGX_F64_SPLIT");
    if (!e || !*e) return 1;
    const int x = std::atoi(e);
    return x < 0 ? 0 : (x > 2 ? 2 : x);
  }();
  return v;
}

namespace {

struct Tile { int out, tm, tn, kt; };

// whole tiles, longest first onto the least-loaded CTA; per-CTA lists and the
// largest CTA load (k-tiles + fixed unit cost)
double assign_whole(const std::vector<Tile>& tiles, int grid, std::vector<std::vector<DUnit>>& per) {
  per.assign(grid, {});
  auto unit = [](const Tile& x) {
    DUnit u;
    u.out = x.out;
    u.tm = (int16_t)x.tm;
    u.tn = (int16_t)x.tn;
    u.kt0 = 0;
    u.kt1 = x.kt;
    return u;
  };
  bool equal = true;
  for (const Tile& x : tiles) equal = equal && x.kt == tiles[0].kt;
  if (equal) {  // all tiles alike: longest first is round robin
    for (size_t i = 0; i < tiles.size(); i++) per[i % grid].push_back(unit(tiles[i]));
    const size_t most = (tiles.size() + grid - 1) / grid;
    return most * (tiles[0].kt + kUnitOverhead);
  }
  std::vector<int> order(tiles.size());
  for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return tiles[a].kt > tiles[b].kt; });
  std::vector<std::pair<double, int>> heap;  // (load, cta), min-heap
  for (int c = 0; c < grid; c++) heap.push_back({0.0, c});
  auto cmp = [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
    return a.first != b.first ? a.first > b.first : a.second > b.second;
  };
  std::make_heap(heap.begin(), heap.end(), cmp);
  double worst = 0;
  for (int i : order) {
    const Tile& x = tiles[i];
    std::pop_heap(heap.begin(), heap.end(), cmp);
    auto& top = heap.back();
    per[top.second].push_back(unit(x));
    top.first += x.kt + kUnitOverhead;
    worst = std::max(worst, top.first);
    std::push_heap(heap.begin(), heap.end(), cmp);
  }
  return worst;
}

// stream-K style: the tiles' k-tiles in one sequence, cut into `grid` equal
// shares; a tile that crosses a share boundary becomes parts (K-split).  Pieces
// shorter than kMinPiece stay with their neighbour.  Returns the largest CTA load.
double assign_shares(const std::vector<Tile>& tiles, int grid, std::vector<std::vector<DUnit>>& per,
                     int64_t& nslots) {
  constexpr int kMinPiece = 4;
  int64_t total = 0;
  for (const Tile& x : tiles) total += x.kt;
  const int64_t q = std::max<int64_t>(kMinPiece, (total + grid - 1) / grid);
  per.assign(grid, {});
  std::vector<double> load(grid, 0.0);
  int c = 0;
  int64_t room = q;
  nslots = 0;
  for (const Tile& x : tiles) {
    std::vector<std::pair<int, int>> pieces;  // (cta, kt1) in K order
    int k = 0;
    while (k < x.kt) {
      if (room < kMinPiece && c + 1 < grid) {  // too little left in this share
        c++;
        room = q;
      }
      int take = (int)std::min<int64_t>(x.kt - k, room);
      if (c + 1 >= grid) take = x.kt - k;      // the last share takes the rest
      if (x.kt - k - take < kMinPiece) take = x.kt - k;
      pieces.push_back({c, k + take});
      k += take;
      room -= take;
      if (room <= 0 && c + 1 < grid) {
        c++;
        room = q;
      }
    }
    if (pieces.empty()) pieces.push_back({c, 0});  // no k-tiles: the tile is written as zeros
    const int parts = (int)pieces.size();
    int k0 = 0;
    for (int p = 0; p < parts; p++) {
      DUnit u;
      u.out = x.out;
      u.tm = (int16_t)x.tm;
      u.tn = (int16_t)x.tn;
      u.kt0 = k0;
      u.kt1 = pieces[p].second;
      u.slot = parts > 1 ? (int32_t)(nslots + p) : -1;
      u.part = (int16_t)p;
      u.nparts = (int16_t)parts;
      per[pieces[p].first].push_back(u);
      load[pieces[p].first] += (u.kt1 - u.kt0) + kUnitOverhead + (parts > 1 ? kPartOverhead : 0);
      k0 = pieces[p].second;
    }
    if (parts > 1) nslots += parts;
  }
  return *std::max_element(load.begin(), load.end());
}

}  // namespace

int64_t make_f64_units(const std::vector<DOut>& outs, const std::vector<DSeg>& segs, int grid,
                       int mode, std::vector<DUnit>& units) {
  units.clear();
  std::vector<int> kts(outs.size());
  size_t ntiles = 0;
  for (size_t o = 0; o < outs.size(); o++) {
    int64_t kt = 0;
    for (int s = 0; s < outs[o].seg_count; s++) kt += (segs[outs[o].seg_begin + s].k + BK - 1) / BK;
    kts[o] = (int)std::min<int64_t>(kt, INT_MAX / 2);
    ntiles += (size_t)((outs[o].m + BM - 1) / BM) * ((outs[o].n + BN - 1) / BN);
  }
  if (ntiles == 0) return 0;
  if (mode < 0) {  // tile order as listed, one unit per tile: O(tiles) host work
    units.resize(ntiles);
    size_t i = 0;
    for (size_t o = 0; o < outs.size(); o++) {
      const int tm = (outs[o].m + BM - 1) / BM, tn = (outs[o].n + BN - 1) / BN;
      for (int a = 0; a < tm; a++)
        for (int b = 0; b < tn; b++) {
          DUnit& u = units[i++];
          u.out = (int32_t)o;
          u.tm = (int16_t)a;
          u.tn = (int16_t)b;
          u.kt1 = kts[o];
        }
    }
    return 0;
  }
  std::vector<Tile> tiles;
  tiles.reserve(ntiles);
  for (size_t o = 0; o < outs.size(); o++) {
    const int tm = (outs[o].m + BM - 1) / BM, tn = (outs[o].n + BN - 1) / BN;
    for (int a = 0; a < tm; a++)
      for (int b = 0; b < tn; b++) tiles.push_back({(int)o, a, b, kts[o]});
  }
  grid = std::max(1, grid);
  std::vector<std::vector<DUnit>> per;
  int64_t nslots = 0;
  const double whole = assign_whole(tiles, grid, per);
  if (mode > 0 && tiles.size() > 0) {
    // K-split only where it shortens the longest CTA by a tenth or more
    std::vector<std::vector<DUnit>> per2;
    int64_t ns2 = 0;
    const double shares = assign_shares(tiles, grid, per2, ns2);
    if (mode == 2 || shares < 0.9 * whole) {
      per.swap(per2);
      nslots = ns2;
    }
  }
  size_t len = 0;
  for (auto& v : per) len = std::max(len, v.size());
  if (len <= 1) {  // one unit per CTA at most: no padding entries
    for (auto& v : per)
      for (auto& u : v) units.push_back(u);
    return nslots;
  }
  // CTA c's j-th unit at entry c + j * grid (the kernel's grid-stride walk)
  DUnit pad;
  pad.out = -1;
  units.assign(len * (size_t)grid, pad);
  for (int c = 0; c < grid; c++)
    for (size_t j = 0; j < per[c].size(); j++) units[j * grid + c] = per[c][j];
  return nslots;
}

cudaError_t prepare_f64_gemm() {
  // opt the kernels in to their shared memory, once per device
  static std::atomic<unsigned long long> ready{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(ready.load() & bit)) {
    e = cudaFuncSetAttribute(grouped_gemm_nt_f64<false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(grouped_gemm_nt_f64<true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    if (e != cudaSuccess) return e;
    ready.fetch_or(bit);
  }
  return cudaSuccess;
}

cudaError_t launch_grouped_f64(const double* A, const double* B, double* C, const DUnit* units,
                               int nunits, const DOut* outs, const DSeg* segs, bool cplx,
                               int grid, cudaStream_t st, double* ws, int* tickets) {
  if (nunits <= 0) return cudaSuccess;
  cudaError_t e = prepare_f64_gemm();
  if (e != cudaSuccess) return e;
  if (grid > nunits) grid = nunits;
  if (cplx)
    grouped_gemm_nt_f64<true><<<grid, THREADS, kSmemBytes, st>>>(A, B, C, units, nunits, outs,
                                                                 segs, ws, tickets);
  else
    grouped_gemm_nt_f64<false><<<grid, THREADS, kSmemBytes, st>>>(A, B, C, units, nunits, outs,
                                                                  segs, ws, tickets);
  return cudaGetLastError();
}

}  // namespace dmrgx

extern "C" int dmrgx_f64_units(int n_outs, const int* out_desc, const int* seg_k, int grid,
                               int mode, int* units, int64_t cap, int64_t* n_units,
                               int64_t* n_slots) {
  using namespace dmrgx;
  if (n_outs < 0 || (n_outs > 0 && (!out_desc || !seg_k)) || grid < 1 || !n_units || !n_slots ||
      cap < 0 || (cap > 0 && !units) || mode < -1 || mode > 2) {
    set_error("f64_units: bad argument");
    return DMRGX_E_ARG;
  }
  std::vector<DOut> outs(n_outs);
  std::vector<DSeg> segs;
  for (int i = 0; i < n_outs; i++) {
    const int m = out_desc[3 * i], n = out_desc[3 * i + 1], ns = out_desc[3 * i + 2];
    if (m < 0 || n < 0 || ns < 0 || (m + f64_tile_m() - 1) / f64_tile_m() > 32767 ||
        (n + f64_tile_n() - 1) / f64_tile_n() > 32767) {
      set_error("f64_units: bad output block extent");
      return DMRGX_E_ARG;
    }
    DOut& o = outs[i];
    o.c_off = 0;
    o.m = m;
    o.n = n;
    o.seg_begin = (int32_t)segs.size();
    o.seg_count = ns;
    for (int q = 0; q < ns; q++) {
      DSeg g;
      g.a_off = g.b_off = 0;
      g.k = seg_k[o.seg_begin + q];
      g.pad_ = 0;
      if (g.k < 0) {
        set_error("f64_units: negative K extent");
        return DMRGX_E_ARG;
      }
      segs.push_back(g);
    }
  }
  std::vector<DUnit> u;
  *n_slots = make_f64_units(outs, segs, grid, mode, u);
  *n_units = (int64_t)u.size();
  for (int64_t j = 0; j < std::min<int64_t>(cap, (int64_t)u.size()); j++) {
    const DUnit& x = u[j];
    const int v[8] = {x.out, x.tm, x.tn, x.kt0, x.kt1, x.slot, x.part, x.nparts};
    for (int q = 0; q < 8; q++) units[8 * j + q] = v[q];
  }
  return DMRGX_OK;
}
