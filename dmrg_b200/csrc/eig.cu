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
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dmrgx.h"
#include "ctx.h"
#include "devmem.h"

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


// ---------------------------------------------------------------- fused CGS2 step
// One Lanczos step's reorthogonalisation in three launches instead of ten:
//   lz_dots      c1 = V^H w                       (T[j][j] += Re c1[j])
//   lz_sub_dots  w -= V c1, then c2 = V^H w       (T[j][j] += Re c2[j])
//   lz_sub_norm  w -= V c2, then beta = |w|       (T[j][j+1] = T[j+1][j] = beta)
// Every block reduces its rows for CH columns at a time in registers (one block
// reduction per chunk, not per column) and writes partials part[j][block]; the
// last block to finish (atomic ticket after a fence) sums the partials of every
// column in block order -- a fixed order, so results do not depend on timing --
// and resets the ticket.
constexpr int CH = 8;  // columns per register chunk

// rows of block b: [b*per, min(n, (b+1)*per))
__device__ __forceinline__ void lz_rows(int64_t n, int64_t& i0, int64_t& i1) {
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  i0 = (int64_t)blockIdx.x * per;
  i1 = min(n, i0 + per);
}

// block-wide sums of v[0..2*CH) (pairs); thread 0 gets the results in v
__device__ __forceinline__ void block_sum(double* v, double (*red)[2 * CH]) {
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 2 * CH; q++)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < 2 * CH; q++) red[wp][q] = v[q];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < 2 * CH; q++) {
      double t = 0.0;
      for (int u = 0; u < RB / 32; u++) t += red[u][q];
      v[q] = t;
    }
  __syncthreads();
}

// partials of V[:, 0..k)^H w over this block's rows -> part[j][block]
template <bool CPLX>
__device__ __forceinline__ void lz_partial_dots(const double* __restrict__ V, int64_t ld, int k,
                                                const double* w, int64_t i0, int64_t i1,
                                                double* __restrict__ part,
                                                double (*red)[2 * CH]) {
  for (int j0 = 0; j0 < k; j0 += CH) {
    double acc[2 * CH];
#pragma unroll
    for (int q = 0; q < 2 * CH; q++) acc[q] = 0.0;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += RB) {
      if (CPLX) {
        const double wr = w[2 * i], wi = w[2 * i + 1];
#pragma unroll
        for (int jj = 0; jj < CH; jj++)
          if (j0 + jj < k) {
            const double vr = V[2 * ((j0 + jj) * ld + i)], vi = V[2 * ((j0 + jj) * ld + i) + 1];
            acc[2 * jj] += vr * wr + vi * wi;
            acc[2 * jj + 1] += vr * wi - vi * wr;
          }
      } else {
        const double wv = w[i];
#pragma unroll
        for (int jj = 0; jj < CH; jj++)
          if (j0 + jj < k) acc[2 * jj] += V[(j0 + jj) * ld + i] * wv;
      }
    }
    block_sum(acc, red);
    if (threadIdx.x == 0)
      for (int jj = 0; jj < CH && j0 + jj < k; jj++) {
        part[2 * ((int64_t)(j0 + jj) * gridDim.x + blockIdx.x)] = acc[2 * jj];
        part[2 * ((int64_t)(j0 + jj) * gridDim.x + blockIdx.x) + 1] = acc[2 * jj + 1];
      }
  }
}

// w[i] -= sum_j V[i, j] c[j] over this block's rows
template <bool CPLX>
__device__ __forceinline__ void lz_subtract(const double* __restrict__ V, int64_t ld, int k,
                                            const double* __restrict__ c, double* w, int64_t i0,
                                            int64_t i1) {
  for (int64_t i = i0 + threadIdx.x; i < i1; i += RB) {
    if (CPLX) {
      double ar = 0.0, ai = 0.0;
      for (int j = 0; j < k; j++) {
        const double vr = V[2 * (j * ld + i)], vi = V[2 * (j * ld + i) + 1];
        ar += vr * c[2 * j] - vi * c[2 * j + 1];
        ai += vr * c[2 * j + 1] + vi * c[2 * j];
      }
      w[2 * i] -= ar;
      w[2 * i + 1] -= ai;
    } else {
      double a = 0.0;
      for (int j = 0; j < k; j++) a += V[j * ld + i] * c[2 * j];
      w[i] -= a;
    }
  }
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

template <bool CPLX>
__global__ void __launch_bounds__(RB) lz_dots(const double* __restrict__ V, int64_t ld, int k,
                                              const double* __restrict__ w, int64_t n,
                                              double* __restrict__ part, unsigned* ticket,
                                              double* __restrict__ coef, double* __restrict__ T,
                                              int tdim, int jt) {
  __shared__ double red[RB / 32][2 * CH];
  int64_t i0, i1;
  lz_rows(n, i0, i1);
  lz_partial_dots<CPLX>(V, ld, k, w, i0, i1, part, red);
  if (!lz_last(ticket)) return;
  lz_final_coef(part, k, coef, T, tdim, jt);
  if (threadIdx.x == 0) *ticket = 0u;
}

template <bool CPLX>
__global__ void __launch_bounds__(RB) lz_sub_dots(const double* __restrict__ V, int64_t ld, int k,
                                                  const double* __restrict__ cin,
                                                  double* __restrict__ w, int64_t n,
                                                  double* __restrict__ part, unsigned* ticket,
                                                  double* __restrict__ cout,
                                                  double* __restrict__ T, int tdim, int jt) {
  __shared__ double red[RB / 32][2 * CH];
  int64_t i0, i1;
  lz_rows(n, i0, i1);
  lz_subtract<CPLX>(V, ld, k, cin, w, i0, i1);
  lz_partial_dots<CPLX>(V, ld, k, w, i0, i1, part, red);  // own rows: no cross-thread hazard
  if (!lz_last(ticket)) return;
  lz_final_coef(part, k, cout, T, tdim, jt);
  if (threadIdx.x == 0) *ticket = 0u;
}

template <bool CPLX>
__global__ void __launch_bounds__(RB) lz_sub_norm(const double* __restrict__ V, int64_t ld, int k,
                                                  const double* __restrict__ cin,
                                                  double* __restrict__ w, int64_t n,
                                                  double* __restrict__ part, unsigned* ticket,
                                                  double* __restrict__ T, int tdim, int j,
                                                  double* __restrict__ inv) {
  __shared__ double red[RB / 32][2 * CH];
  int64_t i0, i1;
  lz_rows(n, i0, i1);
  lz_subtract<CPLX>(V, ld, k, cin, w, i0, i1);
  double acc[2 * CH];
#pragma unroll
  for (int q = 0; q < 2 * CH; q++) acc[q] = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += RB) {
    if (CPLX) acc[0] += w[2 * i] * w[2 * i] + w[2 * i + 1] * w[2 * i + 1];
    else acc[0] += w[i] * w[i];
  }
  block_sum(acc, red);
  if (threadIdx.x == 0) part[2 * blockIdx.x] = acc[0];
  if (!lz_last(ticket)) return;
  if (threadIdx.x < 32) {
    double sq = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += 32) sq += __ldcg(part + 2 * b);
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    if (threadIdx.x == 0) {
      const double beta = sqrt(fmax(sq, 0.0));
      T[(int64_t)j * tdim + j + 1] = beta;
      T[(int64_t)(j + 1) * tdim + j] = beta;
      inv[0] = beta > 1e-300 ? 1.0 / beta : 0.0;
      *ticket = 0u;
    }
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

// Vout[:, q] = sum_j V[:, j] Y[j, q], q < k (Y real, column-major m x k)
template <bool CPLX>
__global__ void __launch_bounds__(RB) vrotate(const double* __restrict__ V, int64_t ld, int m,
                                              const double* __restrict__ Y, int k,
                                              double* __restrict__ Vout, int64_t n) {
  extern __shared__ double sY[];
  for (int t = threadIdx.x; t < m * k; t += blockDim.x) sY[t] = Y[t];
  __syncthreads();
  constexpr int F = CPLX ? 2 : 1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double x[F * MAX_NCV];
    for (int j = 0; j < m; j++) {
      x[F * j] = V[F * (j * ld + i)];
      if (CPLX) x[F * j + 1] = V[F * (j * ld + i) + 1];
    }
    for (int q = 0; q < k; q++) {
      double ar = 0.0, ai = 0.0;
      for (int j = 0; j < m; j++) {
        const double y = sY[q * m + j];
        ar += x[F * j] * y;
        if (CPLX) ai += x[F * j + 1] * y;
      }
      Vout[F * (q * ld + i)] = ar;
      if (CPLX) Vout[F * (q * ld + i) + 1] = ai;
    }
  }
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
    return 0;
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
    if (cplx)
      vrotate<true><<<grid, RB, sizeof(double) * mm * k, s>>>(Vin, n, mm, Y, k, Vout, n);
    else
      vrotate<false><<<grid, RB, sizeof(double) * mm * k, s>>>(Vin, n, mm, Y, k, Vout, n);
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
    const int k = j + 1;
    if (cplx) {
      lz_dots<true><<<nblk2, RB, 0, s>>>(V, n, k, w, n, part2, ticket, coef, T, tdim, j);
      lz_sub_dots<true><<<nblk2, RB, 0, s>>>(V, n, k, coef, w, n, part2, ticket, coef2, T, tdim, j);
      lz_sub_norm<true><<<nblk2, RB, 0, s>>>(V, n, k, coef2, w, n, part2, ticket, T, tdim, j, inv);
    } else {
      lz_dots<false><<<nblk2, RB, 0, s>>>(V, n, k, w, n, part2, ticket, coef, T, tdim, j);
      lz_sub_dots<false><<<nblk2, RB, 0, s>>>(V, n, k, coef, w, n, part2, ticket, coef2, T, tdim, j);
      lz_sub_norm<false><<<nblk2, RB, 0, s>>>(V, n, k, coef2, w, n, part2, ticket, T, tdim, j, inv);
    }
    vscale<<<grid, RB, 0, s>>>(w, inv, 0.0, col(V, j + 1), len);
    EIG_TRY(cudaGetLastError());
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
  L.nblk2 = (int)std::max<int64_t>(1, std::min<int64_t>(c->num_sms * 2, (n + 2 * RB - 1) / (2 * RB)));
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
  std::vector<CycleGraph> graphs;
  struct GraphFree {
    std::vector<CycleGraph>& g;
    ~GraphFree() {
      for (auto& x : g) cudaGraphExecDestroy(x.exec);
    }
  } graph_free{graphs};
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
        if (!r && e == cudaSuccess && gr && cudaGraphInstantiate(&ex, gr, 0) == cudaSuccess) {
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
    jacobi_eig(A, mm, th, Z);
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
