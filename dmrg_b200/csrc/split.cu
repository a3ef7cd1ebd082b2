// FP64 -> (hi, lo) operand conversion for the split-precision matvec.
//
// Each FP64 value x becomes a pair of low-precision numbers hi = rn(x),
// lo = rn(x - hi) (BF16, or TF32 held in 32-bit containers), written in the pair
// layout of split.h; padding is left untouched (it is zeroed once when the
// buffers are made).  Used once per plan for the environments and once per
// matvec for psi.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "split.h"

namespace dmrgx {

namespace {

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}

// FP64 rows -> (hi, lo) pairs in pair layout.  Each group of 64 threads converts
// one listed row (RPB rows per block); each thread keeps up to 4 loads in flight
// (the rows are short and the kernel is latency-bound otherwise).
template <int EB>
__device__ __forceinline__ void put_pair(uint8_t* row, int64_t k, double x) {
  constexpr int CH = 64 / EB;
  const int64_t h = pair_off(k, CH);
  if (EB == 2) {
    // hi from the FP32 rounding of x (any nearby BF16 value will do: lo takes
    // the exact FP64 remainder)
    __nv_bfloat16 hv = __float2bfloat16_rn((float)x);
    __nv_bfloat16 lv = __float2bfloat16_rn((float)(x - (double)__bfloat162float(hv)));
    reinterpret_cast<__nv_bfloat16*>(row)[h] = hv;
    reinterpret_cast<__nv_bfloat16*>(row)[h + CH] = lv;
  } else {
    const uint32_t hv = tf32_rna((float)x);
    const uint32_t lv = tf32_rna((float)(x - (double)__uint_as_float(hv)));
    reinterpret_cast<uint32_t*>(row)[h] = hv;
    reinterpret_cast<uint32_t*>(row)[h + CH] = lv;
  }
}

constexpr int RPB = 4;  // rows per block

template <int EB>
__global__ void __launch_bounds__(64 * RPB) pad_split_kernel(const double* __restrict__ src,
                                                             uint8_t* __restrict__ dst,
                                                             const PadJob* __restrict__ jobs,
                                                             const PadRow* __restrict__ rows,
                                                             int nrows) {
  pdl_wait();
  pdl_launch_dependents();
  const int r = blockIdx.x * RPB + (int)(threadIdx.x >> 6);
  if (r >= nrows) return;
  const PadRow pr = rows[r];
  const int tx = (int)(threadIdx.x & 63);
  const PadJob jb = jobs[pr.job];
  const int gc = jb.groups * jb.cols;
  const double* s = src + jb.src + (int64_t)pr.row * gc;
  if (jb.expand) {
    // complex row -> (re, -im, ...) and (im, re, ...)
    uint8_t* r0 = dst + (jb.dst + (int64_t)(2 * pr.row) * 2 * jb.kq) * EB;
    uint8_t* r1 = r0 + (int64_t)2 * jb.kq * EB;
    for (int e = tx; e < gc / 2; e += 64) {
      const double re = __ldg(s + 2 * e), im = __ldg(s + 2 * e + 1);
      put_pair<EB>(r0, 2 * e, re);
      put_pair<EB>(r0, 2 * e + 1, -im);
      put_pair<EB>(r1, 2 * e, im);
      put_pair<EB>(r1, 2 * e + 1, re);
    }
    return;
  }
  uint8_t* row = dst + (jb.dst + (int64_t)pr.row * 2 * jb.kq) * EB;
  // VE consecutive padded positions per thread: one 16-byte store of their hi
  // parts and one of their lo parts (positions past a group's columns are
  // padding and get zeros)
  constexpr int VE = 16 / EB;
  constexpr int CH = 64 / EB;
  const int span = jb.groups * jb.colsp;
  for (int k0 = tx * VE; k0 < span; k0 += 64 * VE) {
    double x[VE];
#pragma unroll
    for (int u = 0; u < VE; u++) {
      const int k = k0 + u, grp = k / jb.colsp, j = k - grp * jb.colsp;
      x[u] = (k < span && j < jb.cols) ? __ldg(s + (int64_t)grp * jb.cols + j) : 0.0;
    }
    uint32_t hw[4], lw[4];
    if (EB == 2) {
#pragma unroll
      for (int p = 0; p < 4; p++) {
        const __nv_bfloat16 h0 = __float2bfloat16_rn((float)x[2 * p]);
        const __nv_bfloat16 h1 = __float2bfloat16_rn((float)x[2 * p + 1]);
        const __nv_bfloat16 l0 =
            __float2bfloat16_rn((float)(x[2 * p] - (double)__bfloat162float(h0)));
        const __nv_bfloat16 l1 =
            __float2bfloat16_rn((float)(x[2 * p + 1] - (double)__bfloat162float(h1)));
        hw[p] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
        lw[p] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
      }
    } else {
#pragma unroll
      for (int p = 0; p < 4; p++) {
        hw[p] = tf32_rna((float)x[p]);
        lw[p] = tf32_rna((float)(x[p] - (double)__uint_as_float(hw[p])));
      }
    }
    const int64_t h = pair_off(k0, CH) * EB;  // bytes; 16-aligned (k0 % VE == 0)
    *reinterpret_cast<uint4*>(row + h) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    *reinterpret_cast<uint4*>(row + h + 64) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
  }
}

}  // namespace

cudaError_t launch_pad_split(int eb, const double* src, void* dst, const PadJob* jobs,
                             const PadRow* rows, int nrows, cudaStream_t st) {
  for (int r0 = 0; r0 < nrows; r0 += 1 << 28) {
    const int n = std::min(nrows - r0, 1 << 28);
    const int blocks = (n + RPB - 1) / RPB;
    const cudaError_t e =
        eb == 2 ? launch_pdl(pad_split_kernel<2>, blocks, 64 * RPB, 0, st, src, (uint8_t*)dst,
                             jobs, rows + r0, n)
                : launch_pdl(pad_split_kernel<4>, blocks, 64 * RPB, 0, st, src, (uint8_t*)dst,
                             jobs, rows + r0, n);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace dmrgx
