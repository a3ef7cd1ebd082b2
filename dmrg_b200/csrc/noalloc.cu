// dmrgx_av_noalloc: the H_eff matvec without any device allocation.
//
// Who this is for: callers that cannot call cudaMalloc/cudaFree while they
// apply H_eff.  Typical cases are an eigensolver loop embedded in a host
// framework whose own allocator owns (has reserved) the device memory, so a
// raw cudaMalloc would fail or fragment it, and latency-sensitive loops that
// cannot afford the device-wide synchronisation cudaMalloc/cudaFree may
// perform.  They hold the environments, the input and the output in memory they
// already own and pass device pointers; this entry point brings the rest.
//
// How: the matvec needs one intermediate (the stage-1 result, "store") and the
// task descriptors of both stages on the device.  Both live in one file-scope
// static __device__ array, g_noalloc_scratch, reserved when the library is
// loaded on a device and held by every GPU that loads the library until the
// process exits:
//   - store: at most kStoreDoubles doubles (32 MiB);
//   - descriptors: kDescBytes bytes (4 MiB).
// Larger problems are rejected with DMRGX_E_ARG.  Host-side task lists are
// built in fixed static buffers (kMaxRows rows per stage, kMaxBlocks blocks per
// environment), so the call allocates nothing on the host either.
//
// The array is shared by every call in the process and keeps what the last call
// left in it: each call overwrites the descriptors it uses and clears the parts
// of the store no task writes.  Calls whose GPU work overlaps (different
// streams, or different host threads) race on the array; serialise them (one
// stream, or one call at a time).
//
// The array's device address is looked up with cudaGetSymbolAddress once per
// device, by the first call made while that device is current.  Every call
// uploads its task descriptors from static host buffers that the next call
// overwrites, so no call may be made while `stream` is being captured into a
// CUDA graph: such a call returns DMRGX_E_STATE.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/dmrgx.h"
#include "ctx.h"
#include "grouped.h"

namespace dmrgx {
namespace {

constexpr int64_t kStoreDoubles = int64_t(1) << 22;          // 32 MiB of doubles
constexpr int64_t kDescBytes = int64_t(4) << 20;             // 4 MiB of descriptors
constexpr int64_t kScratchBytes = kStoreDoubles * 8 + kDescBytes;
constexpr int kMaxRows = 16384;
constexpr int kMaxBlocks = 65536;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int BM = 64, BN = 64, BK = 16, LDS = BK + 4;
constexpr int THREADS = 128;

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Same tile algorithm as the context path's grouped GEMM, with the task sign
// (the reference's alpha, src/qtensor.cpp:1084) applied to A on load, because
// the caller's environment arrays are read-only here.  DSeg::pad_ holds alpha.
template <bool CPLX>
__global__ void __launch_bounds__(THREADS, 3)
noalloc_grouped_gemm(const double* __restrict__ A, const double* __restrict__ B,
                     double* __restrict__ C, const DTile* __restrict__ tiles, int ntiles,
                     const DOut* __restrict__ outs, const DSeg* __restrict__ segs) {
  __shared__ __align__(16) double sA[2][BM][LDS];
  __shared__ __align__(16) double sB[2][BN][LDS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  const int ldr = tid >> 1, ldk = (tid & 1) * 8;

  for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
    const DTile tl = tiles[ti];
    const DOut o = outs[tl.out];
    const int m0 = tl.tm * BM, n0 = tl.tn * BN;
    int total = 0;
    for (int s = 0; s < o.seg_count; s++) total += (segs[o.seg_begin + s].k + BK - 1) / BK;
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
    if (total > 0) {
      int s = o.seg_begin, k0 = 0;
      DSeg sg = segs[s];
      double ra[8], rb[8];
      auto load = [&](const DSeg& d, int kb) {
        const int row = m0 + ldr;
        const double sgn = (double)d.pad_;
        const double* pa = A + d.a_off + (int64_t)row * d.k;
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int kk = kb + ldk + i;
          ra[i] = (row < o.m && kk < d.k) ? sgn * __ldg(pa + kk) : 0.0;
        }
        const int rr = n0 + ldr;
        if (CPLX) {
          const int p = rr & 1;
          const double* pb = B + d.b_off + (int64_t)(rr >> 1) * d.k;
#pragma unroll
          for (int i = 0; i < 8; i++) {
            const int kk = kb + ldk + i;
            double v = (rr < o.n && kk < d.k) ? __ldg(pb + (kk ^ p)) : 0.0;
            rb[i] = (p == 0 && (kk & 1)) ? -v : v;
          }
        } else {
          const double* pb = B + d.b_off + (int64_t)rr * d.k;
#pragma unroll
          for (int i = 0; i < 8; i++) {
            const int kk = kb + ldk + i;
            rb[i] = (rr < o.n && kk < d.k) ? __ldg(pb + kk) : 0.0;
          }
        }
      };
      auto stash = [&](int buf) {
        double2* da = reinterpret_cast<double2*>(&sA[buf][ldr][ldk]);
        double2* db = reinterpret_cast<double2*>(&sB[buf][ldr][ldk]);
#pragma unroll
        for (int i = 0; i < 4; i++) {
          da[i] = make_double2(ra[2 * i], ra[2 * i + 1]);
          db[i] = make_double2(rb[2 * i], rb[2 * i + 1]);
        }
      };
      load(sg, 0);
      stash(0);
      __syncthreads();
      int buf = 0;
      for (int it = 0; it < total; it++) {
        const bool more = it + 1 < total;
        if (more) {
          k0 += BK;
          if (k0 >= sg.k) {
            s++;
            k0 = 0;
            sg = segs[s];
          }
          load(sg, k0);
        }
#pragma unroll
        for (int kq = 0; kq < BK / 4; kq++) {
          double a[4], b[4];
#pragma unroll
          for (int i = 0; i < 4; i++) a[i] = sA[buf][wm + i * 8 + g][kq * 4 + t];
#pragma unroll
          for (int j = 0; j < 4; j++) b[j] = sB[buf][wn + j * 8 + g][kq * 4 + t];
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
        if (more) stash(buf ^ 1);
        __syncthreads();
        buf ^= 1;
      }
    }
    double* pc = C + o.c_off;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int row = m0 + wm + i * 8 + g;
      if (row >= o.m) continue;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int col = n0 + wn + j * 8 + 2 * t;
        if (col < o.n) pc[(int64_t)row * o.n + col] = acc[i][j][0];
        if (col + 1 < o.n) pc[(int64_t)row * o.n + col + 1] = acc[i][j][1];
      }
    }
  }
}

// ---- host side: fixed buffers, no heap ----
struct HostStage {
  DTile tiles[kMaxRows * 4];
  DOut outs[kMaxRows];
  DSeg segs[kMaxRows];
  int ntiles, nouts, nsegs;
  bool full_cover;
};

std::mutex g_mu;
void* g_dev_scratch[kMaxDevices];  // device address of g_noalloc_scratch per device
int64_t g_off[kMaxBlocks + 1];
int g_order[kMaxRows];
int64_t g_tile_cost[kMaxRows * 4];
int g_tile_idx[kMaxRows * 4];
HostStage g_st[2];

// Group the task rows by output block, one DOut per block, segments in row order.
std::string plan_stage(const int* map, int nrows, const int64_t* sizes, int nblk, int f,
                       int64_t in_len, int64_t out_len, HostStage& st) {
  if (nrows > kMaxRows) return "too many task rows (limit 16384 per stage)";
  if (nblk > kMaxBlocks) return "too many environment blocks (limit 65536)";
  g_off[0] = 0;
  for (int b = 0; b < nblk; b++) {
    if (sizes[b] < 0) return "negative block size";
    g_off[b + 1] = g_off[b] + sizes[b];
  }
  for (int i = 0; i < nrows; i++) g_order[i] = i;
  std::sort(g_order, g_order + nrows, [map](int x, int y) {
    const int ox = map[7 * x + 2], oy = map[7 * y + 2];
    return ox != oy ? ox < oy : x < y;
  });
  st.nouts = st.nsegs = st.ntiles = 0;
  int64_t covered = 0;
  int64_t prev_off = -1;
  for (int q = 0; q < nrows; q++) {
    const int* r = map + 7 * g_order[q];
    const int blk = r[0], rows = r[3], cols = r[4], alpha = r[6];
    const int64_t in_beg = r[1], out_beg = r[2];
    if (blk < 0 || blk >= nblk) return "task row: block index out of range";
    if (cols <= 0 || rows < 0) return "task row: bad rows/cols";
    const int64_t S = sizes[blk], K = cols, N = rows;
    if (S % K) return "task row: block size is not a multiple of cols";
    const int64_t M = S / K;
    if (in_beg < 0 || in_beg + N * K > in_len) return "task row: input range out of bounds";
    if (out_beg < 0 || out_beg + M * N > out_len) return "task row: output range out of bounds";
    // descriptor fields are 32-bit: the caller's vector length is not capped
    // by the scratch size, so a single block's extents are checked here
    if (M * f > INT32_MAX || N * f > INT32_MAX || K * f > INT32_MAX)
      return "task row: block extent too large";
    if (M == 0 || N == 0) continue;
    if (out_beg != prev_off) {
      DOut& o = st.outs[st.nouts++];
      o.c_off = out_beg * f;
      o.m = (int32_t)M;
      o.n = (int32_t)(N * f);
      o.seg_begin = st.nsegs;
      o.seg_count = 0;
      covered += M * N;
      prev_off = out_beg;
    } else if (st.outs[st.nouts - 1].m != M || st.outs[st.nouts - 1].n != N * f) {
      return "task rows writing one output block disagree on its shape";
    }
    DSeg& sg = st.segs[st.nsegs++];
    sg.a_off = g_off[blk] * f;
    sg.b_off = in_beg * f;
    sg.k = (int32_t)(K * f);
    sg.pad_ = alpha >= 0 ? 1 : -1;
    st.outs[st.nouts - 1].seg_count++;
  }
  st.full_cover = covered == out_len;
  for (int o = 0; o < st.nouts; o++) {
    int64_t kt = 0;
    for (int s = 0; s < st.outs[o].seg_count; s++)
      kt += (st.segs[st.outs[o].seg_begin + s].k + BK - 1) / BK;
    const int tm = (st.outs[o].m + BM - 1) / BM, tn = (st.outs[o].n + BN - 1) / BN;
    if (tm > 32767 || tn > 32767) return "output block too large for the tile grid";
    for (int a = 0; a < tm; a++)
      for (int b = 0; b < tn; b++) {
        if (st.ntiles >= kMaxRows * 4) return "too many output tiles (limit 65536 per stage)";
        g_tile_cost[st.ntiles] = kt;
        DTile& t = st.tiles[st.ntiles++];
        t.out = o;
        t.tm = (int16_t)a;
        t.tn = (int16_t)b;
      }
  }
  // heaviest tiles first (ties by position), sorted through an index array
  for (int i = 0; i < st.ntiles; i++) g_tile_idx[i] = i;
  std::sort(g_tile_idx, g_tile_idx + st.ntiles, [](int x, int y) {
    return g_tile_cost[x] != g_tile_cost[y] ? g_tile_cost[x] > g_tile_cost[y] : x < y;
  });
  static DTile tmp[kMaxRows * 4];
  for (int i = 0; i < st.ntiles; i++) tmp[i] = st.tiles[g_tile_idx[i]];
  std::memcpy(st.tiles, tmp, sizeof(DTile) * st.ntiles);
  return "";
}

}  // namespace
}  // namespace dmrgx

using namespace dmrgx;

extern "C" int dmrgx_av_noalloc(int dtype, int64_t n, int64_t d_store, const int* rmap,
                                int n_rmap, const void* renv, const int64_t* renv_sizes,
                                int n_renv_blocks, const int* lmap, int n_lmap, const void* lenv,
                                const int64_t* lenv_sizes, int n_lenv_blocks, const void* in,
                                void* out, void* stream) {
  if (dtype != DMRGX_F64 && dtype != DMRGX_C128) {
    set_error("av_noalloc: dtype must be DMRGX_F64 or DMRGX_C128");
    return DMRGX_E_ARG;
  }
  if (!renv || !lenv || !in || !out || !renv_sizes || !lenv_sizes || (n_rmap && !rmap) ||
      (n_lmap && !lmap) || n < 0 || d_store < 0 || n_rmap < 0 || n_lmap < 0) {
    set_error("av_noalloc: null or negative argument");
    return DMRGX_E_ARG;
  }
  const int f = dtype == DMRGX_C128 ? 2 : 1;
  if (d_store * f > kStoreDoubles) {
    set_error("av_noalloc: intermediate of " + std::to_string(d_store * f * 8) +
              " bytes exceeds the fixed 32 MiB scratch; use dmrgx_av with a context");
    return DMRGX_E_ARG;
  }
  {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t ce = cudaStreamIsCapturing((cudaStream_t)stream, &cs);
    if (ce != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
      set_error("av_noalloc: not callable while the stream is being captured (descriptors "
                "are uploaded from host buffers that the next call reuses)");
      return ce != cudaSuccess ? DMRGX_E_CUDA : DMRGX_E_STATE;
    }
  }
  std::lock_guard<std::mutex> lock(g_mu);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_error(std::string("av_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    return DMRGX_E_CUDA;
  }
  if (!g_dev_scratch[dev]) {  // once per device, with that device current
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error(std::string("av_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return DMRGX_E_CUDA;
    }
    g_dev_scratch[dev] = p;
  }
  std::string msg = plan_stage(rmap, n_rmap, renv_sizes, n_renv_blocks, f, n, d_store, g_st[0]);
  if (msg.empty())
    msg = plan_stage(lmap, n_lmap, lenv_sizes, n_lenv_blocks, f, d_store, n, g_st[1]);
  if (!msg.empty()) {
    set_error("av_noalloc: " + msg);
    return DMRGX_E_ARG;
  }
  // descriptor region layout: [tiles1|outs1|segs1|tiles2|outs2|segs2], 256-byte aligned parts
  auto up = [](int64_t x) { return (x + 255) / 256 * 256; };
  int64_t part[6] = {up(sizeof(DTile) * g_st[0].ntiles), up(sizeof(DOut) * g_st[0].nouts),
                     up(sizeof(DSeg) * g_st[0].nsegs),   up(sizeof(DTile) * g_st[1].ntiles),
                     up(sizeof(DOut) * g_st[1].nouts),   up(sizeof(DSeg) * g_st[1].nsegs)};
  int64_t total = 0;
  for (int i = 0; i < 6; i++) total += part[i];
  if (total > kDescBytes) {
    set_error("av_noalloc: task descriptors exceed the fixed 4 MiB area");
    return DMRGX_E_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  double* store = (double*)g_dev_scratch[dev];
  unsigned char* desc = (unsigned char*)g_dev_scratch[dev] + kStoreDoubles * 8;
  unsigned char* dp[6];
  int64_t o = 0;
  for (int i = 0; i < 6; i++) {
    dp[i] = desc + o;
    o += part[i];
  }
  const void* hp[6] = {g_st[0].tiles, g_st[0].outs, g_st[0].segs,
                       g_st[1].tiles, g_st[1].outs, g_st[1].segs};
  const int64_t hb[6] = {(int64_t)sizeof(DTile) * g_st[0].ntiles, (int64_t)sizeof(DOut) * g_st[0].nouts,
                         (int64_t)sizeof(DSeg) * g_st[0].nsegs,   (int64_t)sizeof(DTile) * g_st[1].ntiles,
                         (int64_t)sizeof(DOut) * g_st[1].nouts,   (int64_t)sizeof(DSeg) * g_st[1].nsegs};
  for (int i = 0; i < 6; i++) {
    if (!hb[i]) continue;
    // pageable source: the call returns once the bytes are staged, so the
    // static host buffers may be reused by the next call
    e = cudaMemcpyAsync(dp[i], hp[i], hb[i], cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
      set_error(std::string("av_noalloc: descriptor upload: ") + cudaGetErrorString(e));
      return DMRGX_E_CUDA;
    }
  }
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int grid = nsm * 3;
  const bool cplx = f == 2;
  // stage 1 into the static store (cleared first where no task writes)
  if (!g_st[0].full_cover) {
    e = cudaMemsetAsync(store, 0, sizeof(double) * d_store * f, st);
    if (e != cudaSuccess) {
      set_error(std::string("av_noalloc: ") + cudaGetErrorString(e));
      return DMRGX_E_CUDA;
    }
  }
  if (g_st[0].ntiles) {
    const int g1 = std::min(grid, g_st[0].ntiles);
    if (cplx)
      noalloc_grouped_gemm<true><<<g1, THREADS, 0, st>>>(
          (const double*)renv, (const double*)in, store, (const DTile*)dp[0], g_st[0].ntiles,
          (const DOut*)dp[1], (const DSeg*)dp[2]);
    else
      noalloc_grouped_gemm<false><<<g1, THREADS, 0, st>>>(
          (const double*)renv, (const double*)in, store, (const DTile*)dp[0], g_st[0].ntiles,
          (const DOut*)dp[1], (const DSeg*)dp[2]);
  }
  if (!g_st[1].full_cover) {
    e = cudaMemsetAsync(out, 0, sizeof(double) * n * f, st);
    if (e != cudaSuccess) {
      set_error(std::string("av_noalloc: ") + cudaGetErrorString(e));
      return DMRGX_E_CUDA;
    }
  }
  if (g_st[1].ntiles) {
    const int g2 = std::min(grid, g_st[1].ntiles);
    if (cplx)
      noalloc_grouped_gemm<true><<<g2, THREADS, 0, st>>>(
          (const double*)lenv, store, (double*)out, (const DTile*)dp[3], g_st[1].ntiles,
          (const DOut*)dp[4], (const DSeg*)dp[5]);
    else
      noalloc_grouped_gemm<false><<<g2, THREADS, 0, st>>>(
          (const double*)lenv, store, (double*)out, (const DTile*)dp[3], g_st[1].ntiles,
          (const DOut*)dp[4], (const DSeg*)dp[5]);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("av_noalloc: launch: ") + cudaGetErrorString(e));
    return DMRGX_E_CUDA;
  }
  return 0;
}
