// FP64 grouped segmented-K GEMM on the FP64 tensor cores (DMMA, mma.sync m8n8k4).
//
// One launch executes every task of one stage of the block-sparse matvec
// (the reference runs them as one serial BLAS call each, src/qtensor.cpp:986-994).
// Work unit = one 64x64 tile of one output block; the CTA walks the output
// block's segments and their K extents, sums everything in registers and
// writes the tile once.  Tiles are listed by decreasing work; CTAs stride
// through the list (persistent grid).
//
// Blackwell has no FP64 kind of tcgen05.mma; DMMA is the FP64 tensor path.
#include <cuda_runtime.h>

#include "grouped.h"
#include "kernels.h"

namespace dmrgx {

namespace {

constexpr int BM = 64, BN = 64, BK = 16, LDS = BK + 4;  // +4 doubles: conflict-free fragments
constexpr int THREADS = 128;

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

template <bool CPLX>
__global__ void __launch_bounds__(THREADS, 3)
grouped_gemm_nt_f64(const double* __restrict__ A, const double* __restrict__ B,
                    double* __restrict__ C, const DTile* __restrict__ tiles, int ntiles,
                    const DOut* __restrict__ outs, const DSeg* __restrict__ segs) {
  __shared__ __align__(16) double sA[2][BM][LDS];
  __shared__ __align__(16) double sB[2][BN][LDS];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  const int ldr = tid >> 1, ldk = (tid & 1) * 8;  // loader: row, first k of 8

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
        const double* pa = A + d.a_off + (int64_t)row * d.k;
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int kk = kb + ldk + i;
          ra[i] = (row < o.m && kk < d.k) ? __ldg(pa + kk) : 0.0;
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

}  // namespace

int f64_tile_m() { return BM; }
int f64_tile_n() { return BN; }
int f64_tile_k() { return BK; }

cudaError_t launch_grouped_f64(const double* A, const double* B, double* C, const DTile* tiles,
                               int ntiles, const DOut* outs, const DSeg* segs, bool cplx,
                               int grid, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  if (grid > ntiles) grid = ntiles;
  if (cplx)
    grouped_gemm_nt_f64<true><<<grid, THREADS, 0, st>>>(A, B, C, tiles, ntiles, outs, segs);
  else
    grouped_gemm_nt_f64<false><<<grid, THREADS, 0, st>>>(A, B, C, tiles, ntiles, outs, segs);
  return cudaGetLastError();
}

}  // namespace dmrgx
