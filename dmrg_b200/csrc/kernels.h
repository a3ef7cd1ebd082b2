// Launch wrappers of the CUDA kernels (host-callable).
#pragma once
#include <cuda_runtime.h>

#include "grouped.h"

namespace dmrgx {

int f64_tile_m();
int f64_tile_n();
int f64_tile_k();

// FP64 grouped segmented GEMM (gemm_f64.cu).  cplx: interleaved complex operands.
cudaError_t launch_grouped_f64(const double* A, const double* B, double* C, const DTile* tiles,
                               int ntiles, const DOut* outs, const DSeg* segs, bool cplx,
                               int grid, cudaStream_t st);

}  // namespace dmrgx
