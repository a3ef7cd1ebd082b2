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

// FP64 blocks -> (hi, lo) pairs with padded rows.  Element (r, grp, j) of a job
// goes to dst + r*groups*colsp + grp*colsp + j; padding is left untouched (zero).
template <int EB>
__global__ void pad_split_kernel(const double* __restrict__ src, uint8_t* __restrict__ hi,
                                 uint8_t* __restrict__ lo, const PadJob* __restrict__ jobs) {
  const PadJob jb = jobs[blockIdx.y];
  const int64_t total = (int64_t)jb.rows * jb.groups * jb.cols;
  const int gc = jb.groups * jb.cols;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / gc;
    const int rem = (int)(e - r * gc);
    const int grp = rem / jb.cols, j = rem - grp * jb.cols;
    const double x = src[jb.src + e];
    const int64_t d = jb.dst + r * (int64_t)jb.groups * jb.colsp + (int64_t)grp * jb.colsp + j;
    if (EB == 2) {
      __nv_bfloat16 h = __double2bfloat16(x);
      __nv_bfloat16 l = __double2bfloat16(x - (double)__bfloat162float(h));
      reinterpret_cast<__nv_bfloat16*>(hi)[d] = h;
      reinterpret_cast<__nv_bfloat16*>(lo)[d] = l;
    } else {
      const uint32_t h = tf32_rna((float)x);
      const uint32_t l = tf32_rna((float)(x - (double)__uint_as_float(h)));
      reinterpret_cast<uint32_t*>(hi)[d] = h;
      reinterpret_cast<uint32_t*>(lo)[d] = l;
    }
  }
}

}  // namespace

cudaError_t launch_pad_split(int eb, const double* src, void* hi, void* lo, const PadJob* jobs,
                             int njobs, int64_t max_elems, cudaStream_t st) {
  if (njobs <= 0) return cudaSuccess;
  int bx = (int)std::min<int64_t>(64, (max_elems + 255) / 256);
  if (bx < 1) bx = 1;
  for (int j0 = 0; j0 < njobs; j0 += 65535) {
    dim3 grid(bx, std::min(65535, njobs - j0));
    if (eb == 2)
      pad_split_kernel<2><<<grid, 256, 0, st>>>(src, (uint8_t*)hi, (uint8_t*)lo, jobs + j0);
    else
      pad_split_kernel<4><<<grid, 256, 0, st>>>(src, (uint8_t*)hi, (uint8_t*)lo, jobs + j0);
  }
  return cudaGetLastError();
}

}  // namespace dmrgx
