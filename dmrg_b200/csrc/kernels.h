// Launch wrappers of the CUDA kernels (host-callable).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "grouped.h"

namespace dmrgx {

int f64_tile_m();
int f64_tile_n();
int f64_tile_k();

// K-split mode of the matvec stages: DMRGX_F64_SPLIT, read once: 0 whole tiles
// only, 1 (default) equal shares when they shorten the longest CTA, 2 always
int f64_split_mode();

// Work units of one FP64 grouped launch over `grid` CTAs (gemm_f64.cu): every
// 64 x 64 tile of every output block, assigned longest first to the least-loaded
// CTA (mode 0); or (mode 1 when that shortens the longest CTA by a tenth, mode 2
// always) the k-tiles of all tiles cut into equal per-CTA shares, a tile that
// crosses a share boundary split along K into parts.  The units are laid out for
// the kernel's grid-stride walk.  A negative mode lists the whole tiles in order
// with no assignment (host work linear in the tiles, for one-off contractions of
// many short tiles).  Returns the number of workspace slots (and tickets) they use.
int64_t make_f64_units(const std::vector<DOut>& outs, const std::vector<DSeg>& segs, int grid,
                       int mode, std::vector<DUnit>& units);

// Opt the FP64 grouped kernel in to its shared memory on the current device (once;
// call outside any stream capture, launch_grouped_f64 also calls it).
cudaError_t prepare_f64_gemm();

// FP64 grouped segmented GEMM (gemm_f64.cu).  cplx: interleaved complex operands.
// ws / tickets: workspace of 4096 doubles and one zero-initialised int per slot
// (null when the units use none); the kernel leaves the tickets at zero.
cudaError_t launch_grouped_f64(const double* A, const double* B, double* C, const DUnit* units,
                               int nunits, const DOut* outs, const DSeg* segs, bool cplx,
                               int grid, cudaStream_t st, double* ws, int* tickets);

}  // namespace dmrgx
