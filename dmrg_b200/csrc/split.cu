// FP64 -> (hi, lo) operand conversion for the split-precision matvec.
//
// Each FP64 value x becomes a pair of low-precision numbers hi = rn(x),
// lo = rn(x - hi) (BF16, or TF32 held in 32-bit containers), written into row
// layouts whose row stride is padded to 16 bytes; the padding is left untouched
// (it is zeroed once when the buffers are made).  Used once per plan for the
// environments and once per matvec for psi.
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

// FP64 rows -> (hi, lo) pairs with padded rows.  Block b converts row
// rows[b].row of job rows[b].job: element (grp, j) of the source row goes to
// dst + row*groups*colsp + grp*colsp + j.  Each thread keeps up to 4 loads in
// flight (the kernel is latency-bound on short rows otherwise).
template <int EB>
__device__ __forceinline__ void put_pair(uint8_t* hi, uint8_t* lo, int64_t d, double x) {
  if (EB == 2) {
    // hi from the FP32 rounding of x (any nearby BF16 value will do: lo takes
    // the exact FP64 remainder)
    __nv_bfloat16 h = __float2bfloat16_rn((float)x);
    __nv_bfloat16 l = __float2bfloat16_rn((float)(x - (double)__bfloat162float(h)));
    reinterpret_cast<__nv_bfloat16*>(hi)[d] = h;
    reinterpret_cast<__nv_bfloat16*>(lo)[d] = l;
  } else {
    const uint32_t h = tf32_rna((float)x);
    const uint32_t l = tf32_rna((float)(x - (double)__uint_as_float(h)));
    reinterpret_cast<uint32_t*>(hi)[d] = h;
    reinterpret_cast<uint32_t*>(lo)[d] = l;
  }
}

template <int EB>
__global__ void __launch_bounds__(64) pad_split_kernel(const double* __restrict__ src,
                                                       uint8_t* __restrict__ hi,
                                                       uint8_t* __restrict__ lo,
                                                       const PadJob* __restrict__ jobs,
                                                       const PadRow* __restrict__ rows) {
  const PadRow pr = rows[blockIdx.x];
  const PadJob jb = jobs[pr.job];
  const int gc = jb.groups * jb.cols;
  const double* s = src + jb.src + (int64_t)pr.row * gc;
  const int64_t d0 = jb.dst + (int64_t)pr.row * jb.groups * jb.colsp;
  for (int e0 = 0; e0 < gc; e0 += 4 * 64) {
    double x[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int e = e0 + u * 64 + threadIdx.x;
      x[u] = e < gc ? __ldg(s + e) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int e = e0 + u * 64 + threadIdx.x;
      if (e >= gc) break;
      const int grp = e / jb.cols, j = e - grp * jb.cols;
      put_pair<EB>(hi, lo, d0 + (int64_t)grp * jb.colsp + j, x[u]);
    }
  }
}

}  // namespace

cudaError_t launch_pad_split(int eb, const double* src, void* hi, void* lo, const PadJob* jobs,
                             const PadRow* rows, int nrows, cudaStream_t st) {
  for (int r0 = 0; r0 < nrows; r0 += 1 << 30) {
    const int n = std::min(nrows - r0, 1 << 30);
    if (eb == 2)
      pad_split_kernel<2><<<n, 64, 0, st>>>(src, (uint8_t*)hi, (uint8_t*)lo, jobs, rows + r0);
    else
      pad_split_kernel<4><<<n, 64, 0, st>>>(src, (uint8_t*)hi, (uint8_t*)lo, jobs, rows + r0);
  }
  return cudaGetLastError();
}

}  // namespace dmrgx
