// Device Lanczos eigensolver behind dmrgx_eigsolve: the replacement of the
// reference's ARPACK wrapper znaupd(n, nev, Evals, Evecs, pass_val)
// (src/dsaupd.cpp:65-155 real, src/znaupd.cpp:78-197 complex): the nev lowest
// eigenvalues of H_eff (ascending) and the eigenvector of the lowest.
//
// Method: thick-restart Lanczos (Wu & Simon 2000).  The Krylov basis, all inner
// products, norms and the reorthogonalisation are FP64 on the GPU:
//   w = H v_j;  c = V^H w; w -= V c; c' = V^H w; w -= V c' (classical Gram-Schmidt
//   with one re-pass, DGKS);  alpha_j = Re(c_j + c'_j);  beta_j = |w|;
//   v_{j+1} = w / beta_j.
// A whole cycle of steps stays on the device (coefficients, alpha, beta and the
// projected matrix T live in device memory); the host reads T once per cycle,
// diagonalises it (cyclic Jacobi, FP64), and either stops or keeps the k lowest
// Ritz vectors (V <- V Y_k) plus the residual direction and goes on.
// Converged when |beta_m y_i[m]| <= tol |theta_i| for the nev lowest Ritz pairs
// (ARPACK's criterion).
//
// With a split-precision matvec the cycles run on the perturbed operator; the
// defect-correction restart then evaluates the Ritz vector with the FP64
// matvec: theta = <v, H64 v>, r = H64 v - theta v.  If |r| > tol |theta| the
// basis restarts as [v, r/|r|] with T = [[theta, |r|], [|r|, .]] (a one-vector
// thick restart whose coupling is exact) and the split-precision cycles go on.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../../include/dmrgx.h"
#include "ctx.h"
#include "devmem.h"
#include "kernels.h"

namespace dmrgx {

int run_matvec_any(dmrgx_ctx* c, const double* in, double* out, bool fp64);

namespace {

constexpr int RB = 256;        // threads per block of the vector kernels
constexpr int MAX_NCV = 64;    // basis size limit (registers of vrotate)

// part[b][j] = sum over block b's rows of conj(V[i, j]) w[i], j < k (pairs).
// V column-major with leading dimension ld (elements).
template <bool CPLX>
__global__ void __launch_bounds__(RB) vdot_partial(const double* __restrict__ V, int64_t ld, int k,
                                                   const double* __restrict__ w, int64_t n,
                                                   double* __restrict__ part) {
  __shared__ double red[RB / 32][2];
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = blockIdx.x * per, i1 = min(n, i0 + per);
  for (int j = 0; j < k; j++) {
    double sr = 0.0, si = 0.0;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
      if (CPLX) {
        const double vr = V[2 * (j * ld + i)], vi = V[2 * (j * ld + i) + 1];
        const double wr = w[2 * i], wi = w[2 * i + 1];
        sr += vr * wr + vi * wi;
        si += vr * wi - vi * wr;
      } else {
        sr += V[j * ld + i] * w[i];
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, o);
      si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if ((threadIdx.x & 31) == 0) {
      red[threadIdx.x >> 5][0] = sr;
      red[threadIdx.x >> 5][1] = si;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double tr = 0.0, ti = 0.0;
      for (int q = 0; q < RB / 32; q++) {
        tr += red[q][0];
        ti += red[q][1];
      }
      part[2 * ((int64_t)blockIdx.x * k + j)] = tr;
      part[2 * ((int64_t)blockIdx.x * k + j) + 1] = ti;
    }
    __syncthreads();
  }
}

// coef[j] = sum_b part[b][j] (fixed order); optionally T[jt][jt] += Re coef[jt]
__global__ void vdot_final(const double* __restrict__ part, int nblk, int k,
                           double* __restrict__ coef, double* __restrict__ T, int tdim, int jt) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= k) return;
  double sr = 0.0, si = 0.0;
  for (int b = 0; b < nblk; b++) {
    sr += part[2 * ((int64_t)b * k + j)];
    si += part[2 * ((int64_t)b * k + j) + 1];
  }
  coef[2 * j] = sr;
  coef[2 * j + 1] = si;
  if (T && j == jt) T[(int64_t)jt * tdim + jt] += sr;
}


// ---------------------------------------------------------------- CGS2 step, row tiles
// One Lanczos step's reorthogonalisation in three launches of lz_tile:
//   MODE 0  c1 = V^H w                        (T[j][j] += Re c1[j])
//   MODE 1  w -= V c1, then c2 = V^H w        (T[j][j] += Re c2[j])
//   MODE 2  w -= V c2, then beta = |w|        (T[j][j+1] = T[j+1][j] = beta, inv = 1/beta)
// The rows are cut into tiles of TR rows.  A block walks the tiles blockIdx.x,
// +gridDim.x, ...; for each it stages the TR x k slice of the basis and the
// TR values of w in shared memory (coalesced column reads), so a pass reads
// the basis from memory exactly once although it uses every value twice
// (subtract, then dots).  One thread per row subtracts; then warp q sums the
// columns q, q + 8, ... over the tile into the block's running sums (one warp
// per column: no atomics).  Block sums go to part[j][block]; the last block to
// finish (atomic ticket after a fence) adds them up in block order -- a fixed
// order, so results do not depend on timing -- and resets the ticket.
constexpr int TR = 128;  // rows per tile (RB >= TR: one thread per row subtracts)

// 8-byte asynchronous copy global -> shared; zero-fills when !pred (nothing read)
__device__ __forceinline__ void cp_async8(double* sdst, const double* gsrc, bool pred) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(gsrc),
               "r"(pred ? 8 : 0)
               : "memory");
}

// 16-byte asynchronous copy global -> shared of `bytes` (0, 8 or 16) valid
// bytes, the rest zero-filled; both addresses 16-byte aligned
__device__ __forceinline__ void cp_async16(double* sdst, const double* gsrc, int bytes) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gsrc), "r"(bytes)
               : "memory");
}

// true in the block that finishes last (after all partials are visible)
__device__ __forceinline__ bool lz_last(unsigned* ticket) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  return last;
}

// last block: coef[j] = sum_b part[j][b] in block order, T[jt][jt] += Re coef[jt]
__device__ __forceinline__ void lz_final_coef(const double* part, int k, double* coef, double* T,
                                              int tdim, int jt) {
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  for (int j = wp; j < k; j += RB / 32) {
    double sr = 0.0, si = 0.0;
    for (int b = lane; b < (int)gridDim.x; b += 32) {
      sr += __ldcg(part + 2 * ((int64_t)j * gridDim.x + b));
      si += __ldcg(part + 2 * ((int64_t)j * gridDim.x + b) + 1);
    }
    for (int o = 16; o > 0; o >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, o);
      si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane == 0) {
      coef[2 * j] = sr;
      coef[2 * j + 1] = si;
      if (j == jt) T[(int64_t)jt * tdim + jt] += sr;
    }
  }
}

// dynamic shared memory of lz_tile for k basis columns (bytes): two tile
// buffers (basis slice and w), the coefficients, per-warp norm partials
constexpr int LZ_BUF = 3;  // tile buffers: copies run two tiles ahead of the work
__host__ __device__ constexpr size_t lz_tile_smem(int k, bool cplx, int tr) {
  return sizeof(double) * (LZ_BUF * ((size_t)k * tr * (cplx ? 2 : 1) + tr * (cplx ? 2 : 1)) +
                           2 * MAX_NCV + RB / 32);
}
// rows per tile: TR, or TR / 2 where two TR-row buffers would not fit
__host__ __device__ constexpr int lz_tile_rows(int k, bool cplx) {
  return lz_tile_smem(k, cplx, TR) <= (200u << 10) ? TR : TR / 2;
}

constexpr int LZ_COLS = (MAX_NCV + RB / 32 - 1) / (RB / 32);  // columns per warp, at most

template <bool CPLX, int MODE, int TRT>
__global__ void __launch_bounds__(RB) lz_tile(const double* __restrict__ V, int64_t ld, int k,
                                              const double* __restrict__ cin,
                                              double* __restrict__ w, int64_t n,
                                              double* __restrict__ part, unsigned* ticket,
                                              double* __restrict__ cout, double* __restrict__ T,
                                              int tdim, int jt, double* __restrict__ inv,
                                              int vec, int rev) {
  constexpr int F = CPLX ? 2 : 1;
  constexpr int tr = TRT;
  constexpr int EPC = tr * F;          // doubles of one column in a tile
  constexpr int CPC = EPC / 2;         // 16-byte chunks of one column
  extern __shared__ double smem[];
  const size_t tsz = (size_t)k * tr * F + tr * F;  // one buffer: slice then w
  double* sc = smem + LZ_BUF * tsz;                // cin (pairs)
  double* sred = sc + 2 * MAX_NCV;                 // per-warp norm partials (MODE 2)
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  if (MODE != 0)
    for (int t = tid; t < 2 * k; t += RB) sc[t] = cin[t];
  // warp wp owns columns wp, wp + 8, ...: per-lane running sums over all tiles,
  // reduced across the warp once at the end
  double accr[LZ_COLS], acci[LZ_COLS];
#pragma unroll
  for (int q = 0; q < LZ_COLS; q++) accr[q] = acci[q] = 0.0;
  double nrm = 0.0;  // MODE 2: this thread's sum of |w|^2
  const int64_t ntiles = (n + tr - 1) / tr;
  // queue the copies of one tile into buffer b (one commit group per thread)
  auto stage = [&](int64_t tile, int b) {
    double* sV = smem + b * tsz;
    double* sw = sV + (size_t)k * tr * F;
    const int64_t i0 = tile * tr;
    const int len = (int)(n - i0 < tr ? n - i0 : tr) * F;
    if (vec) {
      // columns start 16-byte aligned (ld * F even): 16-byte chunks, thread
      // tid copies chunk tid % CPC of columns tid / CPC, + RB / CPC, ...
      const int c = tid % CPC, e = 2 * c;
      const int bytes = e + 2 <= len ? 16 : (e < len ? 8 : 0);
      const double* src = V + i0 * F + e;
      for (int j = tid / CPC; j < k; j += RB / CPC)
        cp_async16(sV + j * EPC + e, bytes ? src + (int64_t)j * ld * F : V, bytes);
    } else {
      const int e = tid % EPC;
      const double* src = V + i0 * F + e;
      for (int j = tid / EPC; j < k; j += RB / EPC)
        cp_async8(sV + j * EPC + e, e < len ? src + (int64_t)j * ld * F : V, e < len);
    }
    if (tid < CPC) {
      const int e = 2 * tid;
      const int bytes = e + 2 <= len ? 16 : (e < len ? 8 : 0);
      cp_async16(sw + e, bytes ? w + i0 * F + e : w, bytes);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  // rev: the tiles are walked from the end, so that a pass starts on the rows the
  // previous pass (the other direction) read last and L2 still holds
  auto at = [&](int64_t q) { return rev ? ntiles - 1 - q : q; };
  // tile i of this block sits in buffer i % LZ_BUF; the copies of tiles i + 1
  // and i + 2 are in flight while tile i is worked on (one commit group per
  // tile, empty past the end, so wait_group LZ_BUF - 1 always means "tile i")
  int b = 0;
#pragma unroll
  for (int u = 0; u < LZ_BUF - 1; u++) {
    const int64_t q0 = blockIdx.x + (int64_t)u * gridDim.x;
    if (q0 < ntiles) stage(at(q0), u);
    else asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  for (int64_t q = blockIdx.x; q < ntiles; q += gridDim.x) {
    const int64_t tile = at(q);
    const int64_t ahead = q + (int64_t)(LZ_BUF - 1) * gridDim.x;
    const int ba = (b + LZ_BUF - 1) % LZ_BUF;  // the buffer of tile i - 1: free
    if (ahead < ntiles) stage(at(ahead), ba);
    else asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group %0;\n" ::"n"(LZ_BUF - 1) : "memory");
    __syncthreads();  // this tile's copies (all threads') have landed; sc is set
    double* sV = smem + b * tsz;
    double* sw = sV + (size_t)k * tr * F;
    const int64_t i0 = tile * tr;
    const int len = (int)(n - i0 < tr ? n - i0 : tr) * F;  // doubles of the tile per column
    if (MODE != 0 && tid < tr) {
      const int r = tid;
      if (CPLX) {
        double ar = 0.0, ai = 0.0;
        for (int j = 0; j < k; j++) {
          const double2 v = *reinterpret_cast<const double2*>(sV + (size_t)j * tr * 2 + 2 * r);
          ar += v.x * sc[2 * j] - v.y * sc[2 * j + 1];
          ai += v.x * sc[2 * j + 1] + v.y * sc[2 * j];
        }
        const double xr = sw[2 * r] - ar, xi = sw[2 * r + 1] - ai;
        sw[2 * r] = xr;
        sw[2 * r + 1] = xi;
        if (2 * r < len) {
          w[(i0 + r) * 2] = xr;
          w[(i0 + r) * 2 + 1] = xi;
          if (MODE == 2) nrm += xr * xr + xi * xi;
        }
      } else {
        double a = 0.0;
        for (int j = 0; j < k; j++) a += sV[(size_t)j * tr + r] * sc[2 * j];
        const double x = sw[r] - a;
        sw[r] = x;
        if (r < len) {
          w[i0 + r] = x;
          if (MODE == 2) nrm += x * x;
        }
      }
    }
    if (MODE != 2) {
      __syncthreads();  // the subtracted w of the tile is in shared memory
#pragma unroll
      for (int q = 0; q < LZ_COLS; q++) {
        const int j = wp + q * (RB / 32);
        if (j >= k) break;
        for (int r = lane; r < tr; r += 32) {
          if (CPLX) {
            const double2 v = *reinterpret_cast<const double2*>(sV + (size_t)j * tr * 2 + 2 * r);
            const double xr = sw[2 * r], xi = sw[2 * r + 1];
            accr[q] += v.x * xr + v.y * xi;
            acci[q] += v.x * xi - v.y * xr;
          } else {
            accr[q] += sV[(size_t)j * tr + r] * sw[r];
          }
        }
      }
    }
    __syncthreads();  // the buffer is free for the copies LZ_BUF - 1 tiles ahead
    b = (b + 1) % LZ_BUF;
  }
  if constexpr (MODE == 2) {
    for (int o = 16; o > 0; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
    if (lane == 0) sred[wp] = nrm;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int q = 0; q < RB / 32; q++) t += sred[q];
      part[2 * blockIdx.x] = t;
    }
    if (!lz_last(ticket)) return;
    if (tid < 32) {
      double sq = 0.0;
      for (int bb = tid; bb < (int)gridDim.x; bb += 32) sq += __ldcg(part + 2 * bb);
      for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
      if (tid == 0) {
        const double beta = sqrt(fmax(sq, 0.0));
        T[(int64_t)jt * tdim + jt + 1] = beta;
        T[(int64_t)(jt + 1) * tdim + jt] = beta;
        inv[0] = beta > 1e-300 ? 1.0 / beta : 0.0;
        *ticket = 0u;
      }
    }
  } else {
#pragma unroll
    for (int q = 0; q < LZ_COLS; q++) {
      const int j = wp + q * (RB / 32);
      if (j >= k) break;
      double sr = accr[q], si = acci[q];
      for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
      }
      if (lane == 0) {
        part[2 * ((int64_t)j * gridDim.x + blockIdx.x)] = sr;
        part[2 * ((int64_t)j * gridDim.x + blockIdx.x) + 1] = si;
      }
    }
    if (!lz_last(ticket)) return;
    lz_final_coef(part, k, cout, T, tdim, jt);
    if (tid == 0) *ticket = 0u;
  }
}

// y = s * x with s = *sp (device scalar) or the host scalar sh when sp is null
__global__ void vscale(const double* __restrict__ x, const double* __restrict__ sp, double sh,
                       double* __restrict__ y, int64_t len) {
  const double s = sp ? *sp : sh;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = s * x[i];
}

// y = x - theta * v
__global__ void vresid(const double* __restrict__ x, const double* __restrict__ v, double theta,
                       double* __restrict__ y, int64_t len) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = x[i] - theta * v[i];
}

// Vout[:, q] = sum_j V[:, j] Y[j, q], q < k (Y real, column-major m x k): the
// thick restart's rotation.  Row tiles of RB rows x m columns are staged in
// shared memory by cp.async (16-byte copies when the columns are 16-byte
// aligned), then each thread forms its row's k outputs from shared memory and
// writes them (coalesced across the block).
template <bool CPLX, int TRR>
__global__ void __launch_bounds__(RB) vrotate(const double* __restrict__ V, int64_t ld, int m,
                                              const double* __restrict__ Y, int k,
                                              double* __restrict__ Vout, int64_t n, int vec) {
  constexpr int F = CPLX ? 2 : 1;
  constexpr int EPC = TRR * F;  // doubles of one column in a tile (TRR <= RB rows)
  extern __shared__ double rsm[];
  double* sY = rsm;                            // m * k
  double* sV = rsm + ((m * k + 1) & ~1);       // column j at sV[j * EPC], 16-byte aligned
  for (int t = threadIdx.x; t < m * k; t += RB) sY[t] = Y[t];
  const int64_t ntiles = (n + TRR - 1) / TRR;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t i0 = tile * TRR;
    const int len = (int)(n - i0 < TRR ? n - i0 : TRR) * F;
    __syncthreads();  // the previous tile is consumed (and sY is set)
    if (vec) {
      constexpr int CPC = EPC / 2;
      const int c = threadIdx.x % CPC, e = 2 * c;
      const int bytes = e + 2 <= len ? 16 : (e < len ? 8 : 0);
      for (int j = threadIdx.x / CPC; j < m; j += RB / CPC)
        cp_async16(sV + j * EPC + e, bytes ? V + (int64_t)j * ld * F + i0 * F + e : V, bytes);
    } else {
      const int e = threadIdx.x % EPC;
      for (int j = threadIdx.x / EPC; j < m; j += RB / EPC)
        cp_async8(sV + j * EPC + e, e < len ? V + (int64_t)j * ld * F + i0 * F + e : V, e < len);
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    const int r = threadIdx.x;
    if (r >= TRR || r * F >= len) continue;
    for (int q = 0; q < k; q++) {
      double ar = 0.0, ai = 0.0;
      for (int j = 0; j < m; j++) {
        const double y = sY[q * m + j];
        ar += sV[j * EPC + r * F] * y;
        if (CPLX) ai += sV[j * EPC + r * F + 1] * y;
      }
      Vout[(int64_t)q * ld * F + (i0 + r) * F] = ar;
      if (CPLX) Vout[(int64_t)q * ld * F + (i0 + r) * F + 1] = ai;
    }
  }
}

// dynamic shared memory of vrotate (bytes) with tiles of `rows` rows
size_t vrotate_smem(int m, int k, bool cplx, int rows) {
  return sizeof(double) * (((size_t)m * k + 1) / 2 * 2 + (size_t)m * rows * (cplx ? 2 : 1));
}
// tile rows of vrotate: RB, or RB / 2 for a wide complex basis (shared memory)
int vrotate_rows(int m, bool cplx) {
  return vrotate_smem(m, MAX_NCV, cplx, RB) <= (200u << 10) ? RB : RB / 2;
}

// Cyclic Jacobi eigen-decomposition of a small real symmetric matrix (FP64).
// A (m x m, row-major) is destroyed; w ascending; Z[j*m+q] = component j of
// eigenvector q.
void jacobi_eig(std::vector<double> A, int m, std::vector<double>& w, std::vector<double>& Z) {
  std::vector<double> V((size_t)m * m, 0.0);
  for (int i = 0; i < m; i++) V[(size_t)i * m + i] = 1.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < m; i++)
      for (int j = 0; j < m; j++) {
        const double a = A[(size_t)i * m + j];
        tot += a * a;
        if (i != j) off += a * a;
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < m - 1; p++)
      for (int q = p + 1; q < m; q++) {
        const double apq = A[(size_t)p * m + q];
        if (apq == 0.0) continue;
        const double app = A[(size_t)p * m + p], aqq = A[(size_t)q * m + q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t =
            (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int r = 0; r < m; r++) {
          const double arp = A[(size_t)r * m + p], arq = A[(size_t)r * m + q];
          A[(size_t)r * m + p] = c * arp - s * arq;
          A[(size_t)r * m + q] = s * arp + c * arq;
        }
        for (int r = 0; r < m; r++) {
          const double apr = A[(size_t)p * m + r], aqr = A[(size_t)q * m + r];
          A[(size_t)p * m + r] = c * apr - s * aqr;
          A[(size_t)q * m + r] = s * apr + c * aqr;
        }
        for (int r = 0; r < m; r++) {
          const double vrp = V[(size_t)r * m + p], vrq = V[(size_t)r * m + q];
          V[(size_t)r * m + p] = c * vrp - s * vrq;
          V[(size_t)r * m + q] = s * vrp + c * vrq;
        }
      }
  }
  std::vector<int> idx(m);
  for (int i = 0; i < m; i++) idx[i] = i;
  std::sort(idx.begin(), idx.end(),
            [&](int a, int b) { return A[(size_t)a * m + a] < A[(size_t)b * m + b]; });
  w.resize(m);
  Z.assign((size_t)m * m, 0.0);
  for (int q = 0; q < m; q++) {
    w[q] = A[(size_t)idx[q] * m + idx[q]];
    for (int j = 0; j < m; j++) Z[(size_t)j * m + q] = V[(size_t)j * m + idx[q]];
  }
}

// Symmetric eigen-decomposition of a small real matrix (FP64) in O(m^3) with a
// small constant: Householder reduction to tridiagonal form, then implicit
// symmetric QR steps with Wilkinson shifts (Golub & Van Loan, Matrix
// Computations, sections 8.3.1 and 8.3.2), rotations accumulated into the
// eigenvectors.  Same outputs as jacobi_eig: w ascending, Z[j*m+q] = component
// j of eigenvector q.  Returns false if an eigenvalue did not converge in
// 30 m steps (the caller then uses jacobi_eig).
bool tridiag_qr_eig(std::vector<double> A, int m, std::vector<double>& w, std::vector<double>& Z) {
  std::vector<double> Q((size_t)m * m, 0.0);  // Q[i*m+j]: row i, column j
  for (int i = 0; i < m; i++) Q[(size_t)i * m + i] = 1.0;
  std::vector<double> v(m), pv(m);
  // ---- A = Q T Q^T: for column k, a reflector H = I - 2 v v^T (v unit, zero
  // in rows <= k) maps A[k+1:, k] onto a multiple of e_{k+1}
  for (int k = 0; k + 2 < m; k++) {
    double nx = 0.0;
    for (int i = k + 1; i < m; i++) nx += A[(size_t)i * m + k] * A[(size_t)i * m + k];
    nx = std::sqrt(nx);
    if (nx == 0.0) continue;
    const double x0 = A[(size_t)(k + 1) * m + k];
    const double alpha = x0 >= 0 ? -nx : nx;
    for (int i = 0; i < m; i++) v[i] = 0.0;
    v[k + 1] = x0 - alpha;
    for (int i = k + 2; i < m; i++) v[i] = A[(size_t)i * m + k];
    double nv = 0.0;
    for (int i = k + 1; i < m; i++) nv += v[i] * v[i];
    nv = std::sqrt(nv);
    if (nv == 0.0) continue;
    for (int i = k + 1; i < m; i++) v[i] /= nv;
    // trailing block: A22 <- H A22 H = A22 - 2 v q^T - 2 q v^T, q = p - (v^T p) v, p = A22 v
    double vp = 0.0;
    for (int i = k + 1; i < m; i++) {
      double t = 0.0;
      for (int j = k + 1; j < m; j++) t += A[(size_t)i * m + j] * v[j];
      pv[i] = t;
      vp += v[i] * t;
    }
    for (int i = k + 1; i < m; i++) pv[i] -= vp * v[i];
    for (int i = k + 1; i < m; i++)
      for (int j = k + 1; j < m; j++)
        A[(size_t)i * m + j] -= 2.0 * (v[i] * pv[j] + pv[i] * v[j]);
    A[(size_t)(k + 1) * m + k] = A[(size_t)k * m + k + 1] = alpha;
    for (int i = k + 2; i < m; i++) A[(size_t)i * m + k] = A[(size_t)k * m + i] = 0.0;
    // Q <- Q H
    for (int i = 0; i < m; i++) {
      double t = 0.0;
      for (int j = k + 1; j < m; j++) t += Q[(size_t)i * m + j] * v[j];
      for (int j = k + 1; j < m; j++) Q[(size_t)i * m + j] -= 2.0 * t * v[j];
    }
  }
  std::vector<double> a(m), b(std::max(m - 1, 1), 0.0);
  for (int i = 0; i < m; i++) a[i] = A[(size_t)i * m + i];
  for (int i = 0; i + 1 < m; i++) b[i] = A[(size_t)(i + 1) * m + i];
  // ---- implicit symmetric QR on (a, b): chase the bulge of a Wilkinson-shifted
  // rotation down the unreduced block [l, h]; deflate negligible b from the bottom
  const double eps = std::numeric_limits<double>::epsilon();
  int h = m - 1, steps = 0;
  while (h > 0) {
    if (std::fabs(b[h - 1]) <= eps * (std::fabs(a[h - 1]) + std::fabs(a[h]))) {
      b[h - 1] = 0.0;
      h--;
      continue;
    }
    if (++steps > 30 * m) return false;
    int l = h - 1;
    while (l > 0 && std::fabs(b[l - 1]) > eps * (std::fabs(a[l - 1]) + std::fabs(a[l]))) l--;
    const double d = 0.5 * (a[h - 1] - a[h]);
    const double r0 = std::hypot(d, b[h - 1]);
    const double mu = a[h] - b[h - 1] * b[h - 1] / (d + (d >= 0 ? r0 : -r0));
    double x = a[l] - mu, z = b[l];
    for (int k = l; k < h; k++) {
      // rotation of rows / columns k, k+1 taking (x, z) to (r, 0)
      const double r = std::hypot(x, z);
      const double c = r > 0 ? x / r : 1.0, s = r > 0 ? z / r : 0.0;
      if (k > l) b[k - 1] = r;
      const double ak = a[k], ak1 = a[k + 1], bk = b[k];
      a[k] = c * c * ak + 2.0 * c * s * bk + s * s * ak1;
      a[k + 1] = s * s * ak - 2.0 * c * s * bk + c * c * ak1;
      b[k] = c * s * (ak1 - ak) + (c * c - s * s) * bk;
      if (k + 1 < h) {  // the rotation carries b[k+1] into the bulge at (k+2, k)
        z = s * b[k + 1];
        b[k + 1] *= c;
        x = b[k];
      }
      for (int i = 0; i < m; i++) {
        const double qk = Q[(size_t)i * m + k], qk1 = Q[(size_t)i * m + k + 1];
        Q[(size_t)i * m + k] = c * qk + s * qk1;
        Q[(size_t)i * m + k + 1] = -s * qk + c * qk1;
      }
    }
  }
  std::vector<int> idx(m);
  for (int i = 0; i < m; i++) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int x1, int x2) { return a[x1] < a[x2]; });
  w.resize(m);
  Z.assign((size_t)m * m, 0.0);
  for (int q = 0; q < m; q++) {
    w[q] = a[idx[q]];
    for (int j = 0; j < m; j++) Z[(size_t)j * m + q] = Q[(size_t)j * m + idx[q]];
  }
  return true;
}

struct DevMem {
  std::vector<void*> ptrs;
  cudaStream_t s = nullptr;
  ~DevMem() {
    for (void* p : ptrs) dfree(p, s);
  }
  template <class T>
  cudaError_t alloc(T*& p, size_t count) {
    T* q = nullptr;
    cudaError_t e = dalloc(&q, count, s);
    if (e == cudaSuccess) ptrs.push_back(q);
    p = q;
    return e;
  }
};

#define EIG_TRY(expr)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      set_error(std::string("eigsolve: ") + #expr + ": " + cudaGetErrorString(e_));      \
      return DMRGX_E_CUDA;                                                               \
    }                                                                                    \
  } while (0)

struct Lanczos {
  dmrgx_ctx* c;
  bool cplx;
  int64_t n, len;  // elements, doubles per vector
  int m;           // ncv
  int tdim;        // m + 1
  int grid, nblk;
  cudaStream_t s;
  DevMem mem;
  double *V, *V2, *w, *part, *part2, *coef, *coef2, *T, *inv, *Y;
  unsigned* ticket;
  int nblk2;       // blocks of the fused step kernels
  int64_t matvecs = 0, matvecs64 = 0;
  bool force64 = false;  // this solve runs its Krylov steps on the FP64 matvec

  double* col(double* M, int j) { return M + (int64_t)j * len; }

  int init() {
    mem.s = s;
    EIG_TRY(mem.alloc(V, (size_t)len * (m + 1)));
    EIG_TRY(mem.alloc(V2, (size_t)len * (m + 1)));
    EIG_TRY(mem.alloc(w, (size_t)len));
    EIG_TRY(mem.alloc(part, (size_t)2 * nblk * (m + 1)));
    EIG_TRY(mem.alloc(coef, (size_t)2 * (m + 1)));
    EIG_TRY(mem.alloc(coef2, (size_t)2 * (m + 1)));
    EIG_TRY(mem.alloc(ticket, 1));
    EIG_TRY(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s));
    EIG_TRY(mem.alloc(part2, (size_t)2 * nblk2 * (m + 1)));
    EIG_TRY(mem.alloc(T, (size_t)tdim * tdim));
    EIG_TRY(mem.alloc(inv, 2));
    EIG_TRY(mem.alloc(Y, (size_t)MAX_NCV * MAX_NCV));
    for (int k = 1; k <= m; k++) tile_blocks(k);  // before any stream capture
    return 0;
  }
  // resident blocks per SM of the row-tile kernels at basis size k (occupancy
  // calculator, registers and shared memory), cached: the persistent grid is
  // that many per SM, so no block waits for a second wave
  int occ[MAX_NCV + 2] = {0};
  int tile_blocks(int k) {
    if (!occ[k]) {
      int b = 1;
      const size_t sm = lz_tile_smem(k, cplx, lz_tile_rows(k, cplx));
      cudaError_t e =
          !cplx ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, lz_tile<false, 1, TR>, RB, sm)
          : lz_tile_rows(k, cplx) == TR
              ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, lz_tile<true, 1, TR>, RB, sm)
              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, lz_tile<true, 1, TR / 2>, RB, sm);
      occ[k] = (e == cudaSuccess && b > 0) ? std::min(b, 8) : 1;
    }
    return occ[k];
  }
  int matvec(const double* in, double* out, bool fp64) {
    matvecs++;
    if (fp64) matvecs64++;
    return run_matvec_any(c, in, out, fp64);
  }
  // coef = V[:, 0..k)^H x on the device; T[jt][jt] += Re coef[jt] when jt >= 0
  void dots(const double* Vb, int k, const double* x, int jt) {
    if (cplx)
      vdot_partial<true><<<nblk, RB, 0, s>>>(Vb, n, k, x, n, part);
    else
      vdot_partial<false><<<nblk, RB, 0, s>>>(Vb, n, k, x, n, part);
    vdot_final<<<(k + 63) / 64, 64, 0, s>>>(part, nblk, k, coef, jt >= 0 ? T : nullptr, tdim, jt);
  }

  void rotate(const double* Vin, int mm, int k, double* Vout) {
    const int rows = vrotate_rows(mm, cplx);
    const size_t sm = vrotate_smem(mm, k, cplx, rows);
    const int per_sm = (int)std::max<size_t>(1, std::min<size_t>(8, (200u << 10) / sm));
    const int64_t ntiles = (n + rows - 1) / rows;
    const int g = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)c->num_sms * per_sm));
    const int vec = (n * (cplx ? 2 : 1)) % 2 == 0;
    if (cplx && rows == RB)
      vrotate<true, RB><<<g, RB, sm, s>>>(Vin, n, mm, Y, k, Vout, n, vec);
    else if (cplx)
      vrotate<true, RB / 2><<<g, RB, sm, s>>>(Vin, n, mm, Y, k, Vout, n, vec);
    else
      vrotate<false, RB><<<g, RB, sm, s>>>(Vin, n, mm, Y, k, Vout, n, vec);
  }
  // host value of <x, x>
  int norm2(const double* x, double& out) {
    dots(x, 1, x, -1);
    double h[2];
    EIG_TRY(cudaMemcpyAsync(h, coef, sizeof(h), cudaMemcpyDeviceToHost, s));
    EIG_TRY(cudaStreamSynchronize(s));
    out = h[0];
    return 0;
  }
  // one Lanczos step j on the device: v_{j+1}, T[j][j], T[j][j+1]
  // (classical Gram-Schmidt against the whole basis, twice)
  int step(int j) {
    if (matvec(col(V, j), w, force64)) return DMRGX_E_CUDA;
    return ortho(j);
  }
  // the rest of step j once w = H v_j: CGS2 against v_0..v_j, T entries, v_{j+1}
  int ortho(int j) {
    const int k = j + 1;
    const int tr = lz_tile_rows(k, cplx);
    const size_t sm = lz_tile_smem(k, cplx, tr);
    const int64_t ntiles = (n + tr - 1) / tr;
    const int g = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)c->num_sms * tile_blocks(k)));
    const int vec = (n * (cplx ? 2 : 1)) % 2 == 0;  // columns 16-byte aligned
    if (cplx) {
      if (tr == TR) {
        lz_tile<true, 0, TR><<<g, RB, sm, s>>>(V, n, k, nullptr, w, n, part2, ticket, coef, T, tdim, j, inv, vec, (3 * j + 0) & 1);
        lz_tile<true, 1, TR><<<g, RB, sm, s>>>(V, n, k, coef, w, n, part2, ticket, coef2, T, tdim, j, inv, vec, (3 * j + 1) & 1);
        lz_tile<true, 2, TR><<<g, RB, sm, s>>>(V, n, k, coef2, w, n, part2, ticket, nullptr, T, tdim, j, inv, vec, (3 * j + 2) & 1);
      } else {
        lz_tile<true, 0, TR / 2><<<g, RB, sm, s>>>(V, n, k, nullptr, w, n, part2, ticket, coef, T, tdim, j, inv, vec, (3 * j + 0) & 1);
        lz_tile<true, 1, TR / 2><<<g, RB, sm, s>>>(V, n, k, coef, w, n, part2, ticket, coef2, T, tdim, j, inv, vec, (3 * j + 1) & 1);
        lz_tile<true, 2, TR / 2><<<g, RB, sm, s>>>(V, n, k, coef2, w, n, part2, ticket, nullptr, T, tdim, j, inv, vec, (3 * j + 2) & 1);
      }
    } else {
      lz_tile<false, 0, TR><<<g, RB, sm, s>>>(V, n, k, nullptr, w, n, part2, ticket, coef, T, tdim, j, inv, vec, (3 * j + 0) & 1);
      lz_tile<false, 1, TR><<<g, RB, sm, s>>>(V, n, k, coef, w, n, part2, ticket, coef2, T, tdim, j, inv, vec, (3 * j + 1) & 1);
      lz_tile<false, 2, TR><<<g, RB, sm, s>>>(V, n, k, coef2, w, n, part2, ticket, nullptr, T, tdim, j, inv, vec, (3 * j + 2) & 1);
    }
    vscale<<<grid, RB, 0, s>>>(w, inv, 0.0, col(V, j + 1), len);
    EIG_TRY(cudaGetLastError());
    return 0;
  }
};

// One FP64 matvec of several contexts in two launches (config 5's chains in one
// batched launch per stage): the members' stage-1 descriptors, then their
// stage-2 descriptors, merged into one grouped launch each, every offset rebased
// from the member's own buffers to one common base address.  A member reads its
// input from its din buffer and writes its output to its dout buffer; run()
// copies the Krylov vectors in and out around the launches.
struct GroupMatvec {
  cudaStream_t s = nullptr;
  std::vector<dmrgx_ctx*> cs;
  double* base = nullptr;
  DOut* d_outs[2] = {nullptr, nullptr};
  DSeg* d_segs[2] = {nullptr, nullptr};
  DUnit* d_units[2] = {nullptr, nullptr};
  double* d_ws[2] = {nullptr, nullptr};
  int* d_tickets[2] = {nullptr, nullptr};
  int nunits[2] = {0, 0};
  int grid = 0;
  bool cplx = false;
  ~GroupMatvec() { release(); }
  void release() {
    for (int q = 0; q < 2; q++) {
      dfree(d_outs[q], s);
      dfree(d_segs[q], s);
      dfree(d_units[q], s);
      dfree(d_ws[q], s);
      dfree(d_tickets[q], s);
      d_outs[q] = nullptr;
      d_segs[q] = nullptr;
      d_units[q] = nullptr;
      d_ws[q] = nullptr;
      d_tickets[q] = nullptr;
      nunits[q] = 0;
    }
  }
  int build(const std::vector<dmrgx_ctx*>& members, int grid_ctas) {
    release();
    cs = members;
    grid = grid_ctas;
    if (cs.empty()) return 0;
    cplx = cs[0]->dtype == DMRGX_C128;
    uintptr_t lo = UINTPTR_MAX;
    for (dmrgx_ctx* c : cs)
      for (void* p : {c->renv.p, c->lenv.p, c->store.p, c->din.p, c->dout.p})
        if (p) lo = std::min<uintptr_t>(lo, reinterpret_cast<uintptr_t>(p));
    base = reinterpret_cast<double*>(lo);
    auto off = [lo](const void* p) {
      return (int64_t)((reinterpret_cast<uintptr_t>(p) - lo) / sizeof(double));
    };
    for (int q = 0; q < 2; q++) {
      std::vector<DOut> outs;
      std::vector<DSeg> segs;
      for (dmrgx_ctx* c : cs) {
        const Stage& st = q == 0 ? c->st1 : c->st2;
        const int64_t a = off(q == 0 ? c->renv.p : c->lenv.p);
        const int64_t b = off(q == 0 ? c->din.p : c->store.p);
        const int64_t cc = off(q == 0 ? c->store.p : c->dout.p);
        const int s0 = (int)segs.size();
        for (DOut o : st.outs) {
          o.c_off += cc;
          o.seg_begin += s0;
          outs.push_back(o);
        }
        for (DSeg g : st.segs) {
          g.a_off += a;
          g.b_off += b;
          segs.push_back(g);
        }
      }
      // one assignment over every member's tiles, K-split like a single context's stage
      std::vector<DUnit> units;
      const int64_t nslots = make_f64_units(outs, segs, grid, f64_split_mode(), units);
      nunits[q] = (int)units.size();
      EIG_TRY(dalloc(&d_outs[q], std::max<size_t>(1, outs.size()), s));
      EIG_TRY(dalloc(&d_segs[q], std::max<size_t>(1, segs.size()), s));
      EIG_TRY(dalloc(&d_units[q], std::max<size_t>(1, units.size()), s));
      if (nslots > 0) {
        EIG_TRY(dalloc(&d_ws[q], (size_t)nslots * f64_tile_m() * f64_tile_n(), s));
        EIG_TRY(dalloc(&d_tickets[q], (size_t)nslots, s));
        EIG_TRY(cudaMemsetAsync(d_tickets[q], 0, sizeof(int) * nslots, s));
      }
      if (!outs.empty())
        EIG_TRY(cudaMemcpyAsync(d_outs[q], outs.data(), sizeof(DOut) * outs.size(),
                                cudaMemcpyHostToDevice, s));
      if (!segs.empty())
        EIG_TRY(cudaMemcpyAsync(d_segs[q], segs.data(), sizeof(DSeg) * segs.size(),
                                cudaMemcpyHostToDevice, s));
      if (!units.empty())
        EIG_TRY(cudaMemcpyAsync(d_units[q], units.data(), sizeof(DUnit) * units.size(),
                                cudaMemcpyHostToDevice, s));
    }
    EIG_TRY(cudaStreamSynchronize(s));  // the host vectors go away
    return 0;
  }
  // out_b = H_b in_b for every member b (device vectors of n_b elements)
  int run(const std::vector<const double*>& in, const std::vector<double*>& out) {
    for (size_t b = 0; b < cs.size(); b++) {
      dmrgx_ctx* c = cs[b];
      const size_t bytes = sizeof(double) * (size_t)c->n * c->f();
      EIG_TRY(cudaMemcpyAsync(c->din.p, in[b], bytes, cudaMemcpyDeviceToDevice, s));
      if (!c->st1.full_cover)
        EIG_TRY(cudaMemsetAsync(c->store.p, 0, sizeof(double) * c->d_store * c->f(), s));
      if (!c->st2.full_cover) EIG_TRY(cudaMemsetAsync(c->dout.p, 0, bytes, s));
    }
    EIG_TRY(launch_grouped_f64(base, base, base, d_units[0], nunits[0], d_outs[0], d_segs[0],
                               cplx, grid, s, d_ws[0], d_tickets[0]));
    EIG_TRY(launch_grouped_f64(base, base, base, d_units[1], nunits[1], d_outs[1], d_segs[1],
                               cplx, grid, s, d_ws[1], d_tickets[1]));
    for (size_t b = 0; b < cs.size(); b++)
      EIG_TRY(cudaMemcpyAsync(out[b], cs[b]->dout.p, sizeof(double) * (size_t)cs[b]->n * cs[b]->f(),
                              cudaMemcpyDeviceToDevice, s));
    return 0;
  }
};

// the default start vector: a fixed xorshift pattern in [-0.5, 0.5)
int eigsolve_start_pattern(Lanczos& L) {
  std::vector<double> hv(L.len);
  uint64_t x = 0x9E3779B97F4A7C15ull;
  for (int64_t i = 0; i < L.len; i++) {
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    hv[i] = (double)(x >> 11) * (1.0 / 9007199254740992.0) - 0.5;
  }
  EIG_TRY(cudaMemcpyAsync(L.V, hv.data(), sizeof(double) * L.len, cudaMemcpyHostToDevice, L.s));
  EIG_TRY(cudaStreamSynchronize(L.s));  // hv is a host temporary
  return 0;
}

// opt the row-tile kernels in to the shared memory of the largest basis
// (MAX_NCV columns, complex), once per process
bool lz_tile_attrs(const char*& why) {
  static int done = 0;  // 1 ok, -1 failed
  static const char* msg = "";
  if (!done) {
    int big = 0, bigr = 0;  // the largest over every basis size
    for (int k = 1; k <= MAX_NCV; k++) {
      big = std::max(big, (int)lz_tile_smem(k, true, lz_tile_rows(k, true)));
      bigr = std::max(bigr, (int)lz_tile_smem(k, false, lz_tile_rows(k, false)));
    }
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* fn, int bytes) {
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    };
    set((const void*)lz_tile<true, 0, TR>, big);
    set((const void*)lz_tile<true, 1, TR>, big);
    set((const void*)lz_tile<true, 2, TR>, big);
    set((const void*)lz_tile<true, 0, TR / 2>, big);
    set((const void*)lz_tile<true, 1, TR / 2>, big);
    set((const void*)lz_tile<true, 2, TR / 2>, big);
    set((const void*)lz_tile<false, 0, TR>, bigr);
    set((const void*)lz_tile<false, 1, TR>, bigr);
    set((const void*)lz_tile<false, 2, TR>, bigr);
    set((const void*)vrotate<true, RB>, 200 << 10);
    set((const void*)vrotate<true, RB / 2>, 200 << 10);
    set((const void*)vrotate<false, RB>, 200 << 10);
    done = e == cudaSuccess ? 1 : -1;
    if (e != cudaSuccess) msg = cudaGetErrorString(e);
  }
  why = msg;
  return done == 1;
}

// v0 / evec: host arrays, or device arrays on the context's device when dev_vecs
int eigsolve_impl(dmrgx_ctx* c, int nev, int ncv, double tol, int maxiter, const void* v0,
                  double* evals, void* evec, int64_t* info, bool dev_vecs) {
  const int64_t n = c->n;
  const bool cplx = c->dtype == DMRGX_C128;
  const int nev_out = nev;
  if (ncv <= 0) ncv = cplx ? 6 * nev : 4 * nev;  // the reference's ARPACK basis sizes
  ncv = std::min(ncv, MAX_NCV);
  if (ncv >= n) {
    // the basis spans the whole space: Lanczos ends on an exact invariant subspace
    ncv = (int)n;
    nev = (int)std::min<int64_t>(nev, n);
  } else if (nev >= ncv) {
    nev = std::max(1, ncv - 1);
  }
  if (tol <= 0) tol = 1e-10;
  if (maxiter <= 0) maxiter = (int)std::min<int64_t>(3 * n, 1000000);
  bool split = c->prec != DMRGX_PREC_FP64;

  const char* err_attr = "";
  Lanczos L;
  L.c = c;
  L.cplx = cplx;
  L.n = n;
  L.len = n * (cplx ? 2 : 1);
  L.m = ncv;
  L.tdim = ncv + 1;
  L.s = c->stream;
  L.grid = (int)std::max<int64_t>(1, std::min<int64_t>(c->num_sms * 8, (n + RB - 1) / RB));
  L.nblk = (int)std::max<int64_t>(1, std::min<int64_t>(c->num_sms * 4, (n + RB - 1) / RB));
  L.nblk2 = c->num_sms * 8;  // largest grid of the row-tile kernels (partials per column)
  if (!lz_tile_attrs(err_attr)) {
    set_error(std::string("eigsolve: ") + err_attr);
    return DMRGX_E_CUDA;
  }
  // before the cycles are captured: the matvec's FP64 kernel sets its attribute once
  EIG_TRY(prepare_f64_gemm());
  int rc = L.init();
  if (rc) return rc;
  const int m = L.m, td = L.tdim;

  // start vector: the caller's guess, else a fixed deterministic pattern
  if (v0 && dev_vecs) {
    EIG_TRY(cudaMemcpyAsync(L.V, v0, sizeof(double) * L.len, cudaMemcpyDeviceToDevice, L.s));
  } else if (v0) {
    EIG_TRY(cudaMemcpyAsync(L.V, v0, sizeof(double) * L.len, cudaMemcpyHostToDevice, L.s));
    EIG_TRY(cudaStreamSynchronize(L.s));  // the caller's array may go away after the call
  } else if ((rc = eigsolve_start_pattern(L))) {
    return rc;
  }
  {
    double nn;
    if ((rc = L.norm2(L.V, nn))) return rc;
    if (!(nn > 0) && dev_vecs && v0) {
      // a device guess with no weight in this layout: the default pattern instead
      if ((rc = eigsolve_start_pattern(L))) return rc;
      if ((rc = L.norm2(L.V, nn))) return rc;
    }
    if (!(nn > 0)) {
      set_error("eigsolve: zero start vector");
      return DMRGX_E_ARG;
    }
    vscale<<<L.grid, RB, 0, L.s>>>(L.V, nullptr, 1.0 / std::sqrt(nn), L.V, L.len);
  }
  // Split precision from a caller's start vector: when its FP64 residual is
  // already below kSplitGain, the split Krylov steps (floor ~1e-6) would gain
  // little before the FP64 defect corrections take over, and every Krylov step
  // costs its orthogonalisation besides the matvec: run this solve in FP64.
  if (split && v0) {
    constexpr double kSplitGain = 1e-3;
    if (L.matvec(L.V, L.w, true)) return DMRGX_E_CUDA;
    L.dots(L.V, 1, L.w, -1);
    double hth[2];
    EIG_TRY(cudaMemcpyAsync(hth, L.coef, sizeof(hth), cudaMemcpyDeviceToHost, L.s));
    EIG_TRY(cudaStreamSynchronize(L.s));
    vresid<<<L.grid, RB, 0, L.s>>>(L.w, L.V, hth[0], L.w, L.len);
    double rr;
    if ((rc = L.norm2(L.w, rr))) return rc;
    if (std::sqrt(std::max(rr, 0.0)) <= kSplitGain * std::fabs(hth[0])) {
      split = false;
      L.force64 = true;
    }
  }

  std::vector<double> Th((size_t)td * td, 0.0);
  EIG_TRY(cudaMemsetAsync(L.T, 0, sizeof(double) * td * td, L.s));
  std::vector<double> th, Z, ritz;
  int kkeep = 0, cycles = 0, corrections = 0, nconv = 0;
  double resid = 0.0;
  bool have_vec = false;  // lowest Ritz vector sits in V2[:, 0]
  // Split precision: the Krylov operator carries the split rounding (relative
  // ~1e-6..1e-5), so the first solve stops at that floor for all nev values and
  // each defect-correction cycle then converges the lowest pair only, to a
  // fraction of the current FP64 residual.  FP64: the reference's criterion.
  const double split_floor = 1e-6;
  double tol_cur = split ? std::max(tol, split_floor) : tol;
  int nev_cur = nev;

  // One Lanczos cycle (steps kkeep..m-1: matvec, two classical Gram-Schmidt
  // passes, normalisation) is captured once per (first step, basis buffer) into a
  // CUDA graph and replayed; the per-block schedule and profiling run eagerly.
  struct CycleGraph {
    int first;
    const double* V;
    cudaGraphExec_t exec;
  };
  // The instantiated graphs stay in the context (c->cycle_graphs) for the next
  // solves, keyed by (first step, basis buffer slot, basis size): a new capture
  // with the same topology -- the usual case from one site step to the next --
  // updates the old executable in place (cudaGraphExecUpdate) instead of
  // instantiating a new one.
  std::vector<CycleGraph> graphs;
  const double* v_first = L.V;  // the basis buffer V starts in (restarts swap V and V2)
  const bool use_graph = !c->per_block && !c->prof && !getenv("DMRGX_NO_GRAPH");
  auto run_cycle = [&](int first) -> int {
    if (use_graph) {
      for (auto& g : graphs)
        if (g.first == first && g.V == L.V) {
          L.matvecs += m - first;
          EIG_TRY(cudaGraphLaunch(g.exec, L.s));
          return 0;
        }
      cudaGraph_t gr = nullptr;
      if (cudaStreamBeginCapture(L.s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        int r = 0;
        for (int j = first; j < m && !r; j++) r = L.step(j);
        const cudaError_t e = cudaStreamEndCapture(L.s, &gr);
        cudaGraphExec_t ex = nullptr;
        if (!r && e == cudaSuccess && gr) {
          const int64_t key = ((int64_t)first << 20) | ((int64_t)(L.V == v_first ? 0 : 1) << 16) |
                              (int64_t)m;
          auto it = c->cycle_graphs.find(key);
          if (it != c->cycle_graphs.end()) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(it->second, gr, &info) == cudaSuccess) {
              ex = it->second;
            } else {
              cudaGetLastError();
              cudaGraphExecDestroy(it->second);
              c->cycle_graphs.erase(it);
            }
          }
          if (!ex && cudaGraphInstantiate(&ex, gr, 0) == cudaSuccess) c->cycle_graphs[key] = ex;
          else if (!ex) ex = nullptr;
        }
        if (ex) {
          cudaGraphDestroy(gr);
          graphs.push_back({first, L.V, ex});
          EIG_TRY(cudaGraphLaunch(ex, L.s));
          return 0;
        }
        if (gr) cudaGraphDestroy(gr);
        L.matvecs -= m - first;  // counted while capturing; run them eagerly below
        cudaGetLastError();
      }
    }
    for (int j = first; j < m; j++) {
      const int r = L.step(j);
      if (r) return r;
    }
    return 0;
  };

  for (;;) {
    int mm = m;  // basis size reached this cycle
    if ((rc = run_cycle(kkeep))) return rc;
    EIG_TRY(cudaMemcpyAsync(Th.data(), L.T, sizeof(double) * td * td, cudaMemcpyDeviceToHost, L.s));
    int werr = 0;
    if (split && c->err.p)
      EIG_TRY(cudaMemcpyAsync(&werr, c->err.p, sizeof(int), cudaMemcpyDeviceToHost, L.s));
    EIG_TRY(cudaStreamSynchronize(L.s));
    if (werr) {
      cudaMemsetAsync(c->err.p, 0, sizeof(int), L.s);
      set_error("eigsolve: a bounded device wait timed out in the split-precision matvec");
      return DMRGX_E_TIMEOUT;
    }
    cycles++;
    // invariant subspace: a vanishing beta ends the basis early
    for (int j = kkeep; j < m; j++) {
      const double a = std::fabs(Th[(size_t)j * td + j]);
      if (Th[(size_t)j * td + j + 1] <= 1e-14 * std::max(1.0, a)) {
        mm = j + 1;
        break;
      }
    }
    std::vector<double> A((size_t)mm * mm);
    for (int a = 0; a < mm; a++)
      for (int b = 0; b < mm; b++) A[(size_t)a * mm + b] = Th[(size_t)a * td + b];
    if (!tridiag_qr_eig(A, mm, th, Z)) jacobi_eig(A, mm, th, Z);
    const double beta_m = mm < m ? 0.0 : Th[(size_t)(m - 1) * td + m];
    const int kev = std::min(nev_cur, mm);
    nconv = 0;
    for (int q = 0; q < kev; q++) {
      const double r = std::fabs(beta_m * Z[(size_t)(mm - 1) * mm + q]);
      if (r <= tol_cur * std::max(std::fabs(th[q]), 1e-30)) nconv++;
      else break;
    }
    const bool stop = nconv >= kev || cycles >= maxiter || mm < m;
    if (stop) {
      if (corrections == 0) ritz.assign(th.begin(), th.begin() + kev);
      else ritz[0] = th[0];
      std::vector<double> Yh(mm);
      for (int a = 0; a < mm; a++) Yh[a] = Z[(size_t)a * mm + 0];
      EIG_TRY(cudaMemcpyAsync(L.Y, Yh.data(), sizeof(double) * mm, cudaMemcpyHostToDevice, L.s));
      L.rotate(L.V, mm, 1, L.V2);
      have_vec = true;
      resid = std::fabs(beta_m * Z[(size_t)(mm - 1) * mm + 0]);
      if (!split || cycles >= maxiter) break;
      // ---- defect correction: Ritz vector through the FP64 matvec
      double* v = L.V2;
      if (L.matvec(v, L.w, true)) return DMRGX_E_CUDA;
      L.dots(v, 1, L.w, -1);
      double hth[2];
      EIG_TRY(cudaMemcpyAsync(hth, L.coef, sizeof(hth), cudaMemcpyDeviceToHost, L.s));
      EIG_TRY(cudaStreamSynchronize(L.s));
      double vv;
      if ((rc = L.norm2(v, vv))) return rc;
      const double theta = hth[0] / vv;
      vresid<<<L.grid, RB, 0, L.s>>>(L.w, v, theta, L.w, L.len);
      double rr;
      if ((rc = L.norm2(L.w, rr))) return rc;
      const double rnorm = std::sqrt(std::max(rr, 0.0) / vv);
      ritz[0] = theta;
      resid = rnorm;
      if (rnorm <= tol * std::max(std::fabs(theta), 1e-30) || corrections >= 20) break;
      corrections++;
      nev_cur = 1;
      tol_cur = std::max(tol, 0.02 * rnorm / std::max(std::fabs(theta), 1e-30));
      // restart basis [v, r/|r|] with the exact coupling
      vscale<<<L.grid, RB, 0, L.s>>>(v, nullptr, 1.0 / std::sqrt(vv), L.V, L.len);
      vscale<<<L.grid, RB, 0, L.s>>>(L.w, nullptr, 1.0 / (rnorm * std::sqrt(vv)), L.col(L.V, 1),
                                     L.len);
      std::fill(Th.begin(), Th.end(), 0.0);
      Th[0] = theta;
      Th[1] = Th[(size_t)td] = rnorm;
      EIG_TRY(cudaMemcpyAsync(L.T, Th.data(), sizeof(double) * td * td, cudaMemcpyHostToDevice, L.s));
      kkeep = 1;
      have_vec = false;
      continue;
    }
    // ---- thick restart: k lowest Ritz vectors, then the residual direction
    const int k = std::min(m - 2, std::max(nev + 1, nev + (m - nev) / 2));
    std::vector<double> Yh((size_t)m * k);
    for (int q = 0; q < k; q++)
      for (int a = 0; a < m; a++) Yh[(size_t)q * m + a] = Z[(size_t)a * m + q];
    EIG_TRY(cudaMemcpyAsync(L.Y, Yh.data(), sizeof(double) * Yh.size(), cudaMemcpyHostToDevice, L.s));
    L.rotate(L.V, m, k, L.V2);
    EIG_TRY(cudaMemcpyAsync(L.col(L.V2, k), L.col(L.V, m), sizeof(double) * L.len,
                            cudaMemcpyDeviceToDevice, L.s));
    std::swap(L.V, L.V2);
    std::fill(Th.begin(), Th.end(), 0.0);
    for (int q = 0; q < k; q++) {
      Th[(size_t)q * td + q] = th[q];
      const double cpl = beta_m * Z[(size_t)(m - 1) * m + q];
      Th[(size_t)q * td + k] = cpl;
      Th[(size_t)k * td + q] = cpl;
    }
    EIG_TRY(cudaMemcpyAsync(L.T, Th.data(), sizeof(double) * td * td, cudaMemcpyHostToDevice, L.s));
    kkeep = k;
  }
  if (!have_vec) {
    set_error("eigsolve: internal error (no Ritz vector)");
    return DMRGX_E_STATE;
  }
  for (int q = 0; q < nev_out; q++) evals[q] = q < (int)ritz.size() ? ritz[q] : 0.0;
  double nn;
  if ((rc = L.norm2(L.V2, nn))) return rc;
  vscale<<<L.grid, RB, 0, L.s>>>(L.V2, nullptr, 1.0 / std::sqrt(std::max(nn, 1e-300)), L.V2, L.len);
  EIG_TRY(cudaMemcpyAsync(evec, L.V2, sizeof(double) * L.len,
                          dev_vecs ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, L.s));
  EIG_TRY(cudaStreamSynchronize(L.s));
  if (info) {
    info[0] = L.matvecs;
    info[1] = L.matvecs64;
    info[2] = cycles;
    info[3] = corrections;
    info[4] = nconv;
    std::memcpy(&info[5], &resid, sizeof(double));
  }
  if (nconv < 1 && cycles >= maxiter) {
    set_error("eigsolve: maximum number of restarts reached");
    return DMRGX_E_NOCONV;
  }
  return 0;
}

}  // namespace

// One member's solve in a lock-step group (device start / result vectors).
struct GroupArgs {
  dmrgx_ctx* c;
  int nev, ncv;
  double tol;
  const double* v0;  // device start vector or null
  double* evals;     // host, nev values
  double* evec;      // device, n elements
  int64_t* info;     // host, 6 slots, or null
  int rc;
};

// Thick-restart Lanczos (the FP64 form of eigsolve_impl) for several contexts
// at once, in lock step: every round applies H to one Krylov vector of each
// member with a single merged launch per stage (GroupMatvec), then each member
// reorthogonalises; after a cycle the host handles each member's projected
// matrix as eigsolve_impl does.  A member that has converged leaves the
// launches.  All work runs on stream s.
int eigsolve_group(std::vector<GroupArgs>& args, cudaStream_t s, int64_t* stats) {
  const char* err_attr = "";
  if (!lz_tile_attrs(err_attr)) {
    set_error(std::string("eigsolve: ") + err_attr);
    return DMRGX_E_CUDA;
  }
  struct M {
    GroupArgs* a;
    Lanczos L;
    int m = 0, td = 0, nev = 0, maxiter = 0, kkeep = 0, cycles = 0, nconv = 0;
    double tol = 1e-10, resid = 0.0;
    std::vector<double> Th, th, Z, ritz;
    bool done = false, have_vec = false;
  };
  std::vector<M> ms(args.size());
  for (size_t b = 0; b < args.size(); b++) {
    M& x = ms[b];
    GroupArgs& a = args[b];
    dmrgx_ctx* c = a.c;
    x.a = &a;
    const int64_t n = c->n;
    const bool cplx = c->dtype == DMRGX_C128;
    int nev = a.nev, ncv = a.ncv;
    if (ncv <= 0) ncv = cplx ? 6 * nev : 4 * nev;
    ncv = std::min(ncv, MAX_NCV);
    if (ncv >= n) {
      ncv = (int)n;
      nev = (int)std::min<int64_t>(nev, n);
    } else if (nev >= ncv) {
      nev = std::max(1, ncv - 1);
    }
    x.nev = nev;
    x.tol = a.tol > 0 ? a.tol : 1e-10;
    x.maxiter = (int)std::min<int64_t>(3 * n, 1000000);
    Lanczos& L = x.L;
    L.c = c;
    L.cplx = cplx;
    L.n = n;
    L.len = n * (cplx ? 2 : 1);
    L.m = ncv;
    L.tdim = ncv + 1;
    L.s = s;
    L.grid = (int)std::max<int64_t>(1, std::min<int64_t>(c->num_sms * 8, (n + RB - 1) / RB));
    L.nblk = (int)std::max<int64_t>(1, std::min<int64_t>(c->num_sms * 4, (n + RB - 1) / RB));
    L.nblk2 = c->num_sms * 8;
    int rc = L.init();
    if (rc) return rc;
    x.m = L.m;
    x.td = L.tdim;
    if (a.v0) EIG_TRY(cudaMemcpyAsync(L.V, a.v0, sizeof(double) * L.len, cudaMemcpyDeviceToDevice, s));
    else if ((rc = eigsolve_start_pattern(L))) return rc;
    double nn;
    if ((rc = L.norm2(L.V, nn))) return rc;
    if (!(nn > 0) && a.v0) {
      if ((rc = eigsolve_start_pattern(L))) return rc;
      if ((rc = L.norm2(L.V, nn))) return rc;
    }
    if (!(nn > 0)) {
      set_error("eigsolve: zero start vector");
      return DMRGX_E_ARG;
    }
    vscale<<<L.grid, RB, 0, s>>>(L.V, nullptr, 1.0 / std::sqrt(nn), L.V, L.len);
    x.Th.assign((size_t)x.td * x.td, 0.0);
    EIG_TRY(cudaMemsetAsync(L.T, 0, sizeof(double) * x.td * x.td, s));
  }
  GroupMatvec gm;
  gm.s = s;
  const int grid = args.empty() ? 1 : args[0].c->num_sms * 3;
  for (;;) {
    std::vector<int> act;
    for (size_t b = 0; b < ms.size(); b++)
      if (!ms[b].done) act.push_back((int)b);
    if (act.empty()) break;
    // one cycle: rounds t = 0, 1, ...; member b takes its step kkeep_b + t
    int rounds = 0;
    for (int b : act) rounds = std::max(rounds, ms[b].m - ms[b].kkeep);
    for (int t = 0; t < rounds; t++) {
      std::vector<dmrgx_ctx*> part;
      std::vector<const double*> in;
      std::vector<double*> out;
      std::vector<int> who;
      for (int b : act)
        if (ms[b].kkeep + t < ms[b].m) {
          part.push_back(ms[b].L.c);
          in.push_back(ms[b].L.col(ms[b].L.V, ms[b].kkeep + t));
          out.push_back(ms[b].L.w);
          who.push_back(b);
        }
      if (part != gm.cs) {
        const int rc = gm.build(part, grid);
        if (rc) return rc;
      }
      int rc = gm.run(in, out);
      if (rc) return rc;
      if (stats) {
        stats[0] += 1;                     // Krylov rounds
        stats[1] += 2;                     // grouped launches (one per stage)
        stats[2] += (int64_t)part.size();  // member matvecs served
      }
      for (int b : who) {
        ms[b].L.matvecs++;
        if ((rc = ms[b].L.ortho(ms[b].kkeep + t))) return rc;
      }
    }
    for (int b : act)
      EIG_TRY(cudaMemcpyAsync(ms[b].Th.data(), ms[b].L.T, sizeof(double) * ms[b].td * ms[b].td,
                              cudaMemcpyDeviceToHost, s));
    EIG_TRY(cudaStreamSynchronize(s));
    for (int b : act) {
      M& x = ms[b];
      Lanczos& L = x.L;
      const int m = x.m, td = x.td;
      std::vector<double>& Th = x.Th;
      int mm = m;
      x.cycles++;
      for (int j = x.kkeep; j < m; j++) {
        const double av = std::fabs(Th[(size_t)j * td + j]);
        if (Th[(size_t)j * td + j + 1] <= 1e-14 * std::max(1.0, av)) {
          mm = j + 1;
          break;
        }
      }
      std::vector<double> A((size_t)mm * mm);
      for (int r = 0; r < mm; r++)
        for (int q = 0; q < mm; q++) A[(size_t)r * mm + q] = Th[(size_t)r * td + q];
      if (!tridiag_qr_eig(A, mm, x.th, x.Z)) jacobi_eig(A, mm, x.th, x.Z);
      const std::vector<double>& th = x.th;
      const std::vector<double>& Z = x.Z;
      const double beta_m = mm < m ? 0.0 : Th[(size_t)(m - 1) * td + m];
      const int kev = std::min(x.nev, mm);
      x.nconv = 0;
      for (int q = 0; q < kev; q++) {
        const double r = std::fabs(beta_m * Z[(size_t)(mm - 1) * mm + q]);
        if (r <= x.tol * std::max(std::fabs(th[q]), 1e-30)) x.nconv++;
        else break;
      }
      if (x.nconv >= kev || x.cycles >= x.maxiter || mm < m) {
        x.ritz.assign(th.begin(), th.begin() + kev);
        std::vector<double> Yh(mm);
        for (int q = 0; q < mm; q++) Yh[q] = Z[(size_t)q * mm + 0];
        EIG_TRY(cudaMemcpyAsync(L.Y, Yh.data(), sizeof(double) * mm, cudaMemcpyHostToDevice, s));
        EIG_TRY(cudaStreamSynchronize(s));  // Yh is a host temporary
        L.rotate(L.V, mm, 1, L.V2);
        x.have_vec = true;
        x.resid = std::fabs(beta_m * Z[(size_t)(mm - 1) * mm + 0]);
        x.done = true;
        continue;
      }
      // thick restart: the k lowest Ritz vectors, then the residual direction
      const int k = std::min(m - 2, std::max(x.nev + 1, x.nev + (m - x.nev) / 2));
      std::vector<double> Yh((size_t)m * k);
      for (int q = 0; q < k; q++)
        for (int r = 0; r < m; r++) Yh[(size_t)q * m + r] = Z[(size_t)r * m + q];
      EIG_TRY(cudaMemcpyAsync(L.Y, Yh.data(), sizeof(double) * Yh.size(), cudaMemcpyHostToDevice, s));
      L.rotate(L.V, m, k, L.V2);
      EIG_TRY(cudaMemcpyAsync(L.col(L.V2, k), L.col(L.V, m), sizeof(double) * L.len,
                              cudaMemcpyDeviceToDevice, s));
      std::swap(L.V, L.V2);
      std::fill(Th.begin(), Th.end(), 0.0);
      for (int q = 0; q < k; q++) {
        Th[(size_t)q * td + q] = th[q];
        const double cpl = beta_m * Z[(size_t)(m - 1) * m + q];
        Th[(size_t)q * td + k] = cpl;
        Th[(size_t)k * td + q] = cpl;
      }
      EIG_TRY(cudaMemcpyAsync(L.T, Th.data(), sizeof(double) * td * td, cudaMemcpyHostToDevice, s));
      EIG_TRY(cudaStreamSynchronize(s));  // Yh and Th are host arrays reused below
      x.kkeep = k;
    }
  }
  for (M& x : ms) {
    Lanczos& L = x.L;
    GroupArgs& a = *x.a;
    for (int q = 0; q < a.nev; q++) a.evals[q] = q < (int)x.ritz.size() ? x.ritz[q] : 0.0;
    double nn;
    int rc = L.norm2(L.V2, nn);
    if (rc) return rc;
    vscale<<<L.grid, RB, 0, s>>>(L.V2, nullptr, 1.0 / std::sqrt(std::max(nn, 1e-300)), L.V2, L.len);
    EIG_TRY(cudaMemcpyAsync(a.evec, L.V2, sizeof(double) * L.len, cudaMemcpyDeviceToDevice, s));
    if (a.info) {
      a.info[0] = L.matvecs;
      a.info[1] = L.matvecs;
      a.info[2] = x.cycles;
      a.info[3] = 0;
      a.info[4] = x.nconv;
      std::memcpy(&a.info[5], &x.resid, sizeof(double));
    }
    a.rc = (x.nconv < 1 && x.cycles >= x.maxiter) ? DMRGX_E_NOCONV : 0;
  }
  EIG_TRY(cudaStreamSynchronize(s));
  return 0;
}

}  // namespace dmrgx

// A set of contexts whose site-step solves meet and run as one lock-step solve
// (dmrgx_set_group).  The members arrive from their own host threads; the last
// to arrive runs eigsolve_group for all of them on its stream while the others
// wait; a member that waits longer than kWaitSeconds gives up with
// DMRGX_E_TIMEOUT (a chain that failed before arriving).
struct dmrgx_group {
  int size = 0;
  std::mutex mu;
  std::condition_variable cv;
  std::vector<dmrgx::GroupArgs> pending, results;
  int64_t generation = 0;
  int64_t stats[3] = {0, 0, 0};  // Krylov rounds, grouped launches, member matvecs
  int last_rc = 0;
  std::string last_err;
};

namespace dmrgx {

constexpr int kWaitSeconds = 300;

int group_solve(dmrgx_ctx* c, int nev, int ncv, double tol, const double* v0, double* evals,
                double* evec, int64_t* info) {
  dmrgx_group* g = c->group;
  // this member's device data (plan, start vector, result buffer) is complete
  // before another stream touches it
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    set_error(std::string("eigsolve: ") + cudaGetErrorString(e));
    return DMRGX_E_CUDA;
  }
  std::unique_lock<std::mutex> lk(g->mu);
  const int64_t gen = g->generation;
  const size_t me = g->pending.size();
  g->pending.push_back(GroupArgs{c, nev, ncv, tol, v0, evals, evec, info, 0});
  if ((int)g->pending.size() == g->size) {
    std::vector<GroupArgs> work;
    work.swap(g->pending);
    lk.unlock();
    if (cudaSetDevice(c->device) != cudaSuccess) return DMRGX_E_CUDA;
    const int rc = eigsolve_group(work, c->stream, g->stats);
    const std::string msg = rc ? std::string(dmrgx_last_error()) : std::string();
    lk.lock();
    g->results = work;
    g->last_rc = rc;
    g->last_err = msg;
    g->generation++;
    g->cv.notify_all();
    if (rc) return rc;
    return work[me].rc;
  }
  if (!g->cv.wait_for(lk, std::chrono::seconds(kWaitSeconds),
                      [&] { return g->generation != gen; })) {
    set_error("eigsolve: the solve group did not assemble (a member failed or never arrived)");
    return DMRGX_E_TIMEOUT;
  }
  if (g->last_rc) {
    set_error(g->last_err);
    return g->last_rc;
  }
  if (g->results[me].rc) set_error("eigsolve: maximum number of restarts reached");
  return g->results[me].rc;
}

// the eigensolver with device start and result vectors (the site steps)
int eigsolve_device(dmrgx_ctx* c, int nev, int ncv, double tol, int maxiter, const double* v0,
                    double* evals, double* evec, int64_t* info) {
  if (!c->has_plan || nev < 1 || c->n < 1) {
    set_error("eigsolve: no plan, or nev < 1, or empty psi");
    return DMRGX_E_STATE;
  }
  return eigsolve_impl(c, nev, ncv, tol, maxiter, v0, evals, evec, info, true);
}
}  // namespace dmrgx

extern "C" int dmrgx_eigsolve(dmrgx_ctx* c, int nev, int ncv, double tol, int maxiter,
                              const void* v0, double* evals, void* evec, int64_t* info) {
  if (!c || !evals || !evec) {
    dmrgx::set_error("eigsolve: null argument");
    return DMRGX_E_ARG;
  }
  if (!c->has_plan) {
    dmrgx::set_error("eigsolve: no plan");
    return DMRGX_E_STATE;
  }
  if (nev < 1 || c->n < 1) {
    dmrgx::set_error("eigsolve: need nev >= 1 and a non-empty psi");
    return DMRGX_E_ARG;
  }
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) {
    dmrgx::set_error(std::string("eigsolve: ") + cudaGetErrorString(e));
    return DMRGX_E_CUDA;
  }
  return dmrgx::eigsolve_impl(c, nev, ncv, tol, maxiter, v0, evals, evec, info, false);
}

extern "C" int dmrgx_group_create(dmrgx_group** g, int members) {
  if (!g || members < 1) {
    dmrgx::set_error("group_create: need an output pointer and members >= 1");
    return DMRGX_E_ARG;
  }
  *g = new dmrgx_group();
  (*g)->size = members;
  return 0;
}

extern "C" void dmrgx_group_destroy(dmrgx_group* g) { delete g; }

extern "C" int dmrgx_group_stats(dmrgx_group* g, int64_t* out) {
  if (!g || !out) {
    dmrgx::set_error("group_stats: null argument");
    return DMRGX_E_ARG;
  }
  std::lock_guard<std::mutex> lk(g->mu);
  for (int q = 0; q < 3; q++) out[q] = g->stats[q];
  return 0;
}

extern "C" int dmrgx_set_group(dmrgx_ctx* c, dmrgx_group* g) {
  if (!c) {
    dmrgx::set_error("set_group: null context");
    return DMRGX_E_ARG;
  }
  c->group = g;
  return 0;
}
