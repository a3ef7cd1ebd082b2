// Split-precision (hi/lo BF16 or TF32 pairs) grouped GEMM on tcgen05: descriptors
// and launchers (split.cu: operand conversion, tc_gemm.cu: the GEMM).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "grouped.h"

namespace dmrgx {

// Pair layout of the split operands.  A row of logical length kq (a multiple of
// CH = 64 / element-bytes) is kq / CH chunks of 128 bytes, chunk c holding the hi
// parts of elements [c*CH, (c+1)*CH) followed by their lo parts; the row stride
// is 2*kq elements.  One TMA box of one 128-byte row per k-tile brings both halves.
__host__ __device__ inline int64_t pair_off(int64_t k, int ch) {
  return (k / ch) * 2 * ch + (k % ch);
}

// Output block of the split path.  Offsets/extents in elements of the arrays
// the kernel writes: the pair-layout intermediate for stage 1, the packed FP64
// psi for stage 2.
struct SOut {
  int64_t c_off;
  int32_t m, n;      // rows, columns
  int32_t ldc;       // stage 2: row stride of C.  stage 1: padded columns per row
                     // (n1p); row r, column j lands at logical k = (r % grp) * n1p + j
                     // of pair-layout row r / grp
  int32_t seg_begin, seg_count;
  int32_t tnw;       // tile width (columns per tile, <= 256, a multiple of 16)
  int32_t grp;       // stage 1: output rows per pair-layout row (MPO channels)
  int32_t rstride;   // stage 1: elements per pair-layout row (2 * kq)
  int32_t cplx;      // stage 1, complex data: write the B-expanded form (see below)
};

// Complex data.  A complex product C = A B^T is one real product of
//   A as real rows (re, im, re, im, ...) and
//   B "expanded": complex row j becomes real rows 2j = (re, -im, ...) and
//   2j+1 = (im, re, ...),
// giving real C rows (Re, Im, Re, Im, ...) -- the interleaved complex result.
// Stage 1 writes the intermediate directly in the expanded form stage 2 reads.

// One segment of an output block: tensor-map indices of its A block (m x kp) and
// B block (n x kp), its k-tile count, and the row count of the B map's box.
struct SSeg2 {
  int32_t amap, bmap;
  int32_t nkt;
  int32_t brows;
};

// Work unit: k-tiles [kt0, kt1) (over the output block's segments, in order) of
// the output tile (tm, tn).  slot >= 0: write the FP32 partial to that
// workspace slot (the tile is split along K); slot < 0: write the result.
struct SUnit {
  int32_t out;
  int16_t tm, tn;
  int32_t kt0, kt1;
  int32_t slot, pad_;
};

// A K-split output tile: its partials are workspace slots [slot0, slot0+nslots).
struct SRed {
  int32_t out;
  int16_t tm, tn;
  int32_t slot0, nslots;
};

// One block of the reduction launch: rows [r0, r0+rows) of K-split tile `red`.
struct SRedBlk {
  int32_t red, r0;
};

// One block of the conversion launch: row `row` of conversion job `job`.
struct PadRow {
  int32_t job, row;
};

// FP64 -> (hi, lo) conversion job: rows x (groups x cols) source elements;
// source element (g, j) of a row goes to logical k = g * colsp + j of a
// pair-layout destination row of kq elements (colsp >= cols, kq >= groups * colsp;
// the gaps stay zero).
struct PadJob {
  int64_t src, dst;
  int32_t rows, groups, cols, colsp;
  int32_t kq;
  int32_t expand;  // complex B operand: each source row (cols doubles = cols/2 complex)
                   // becomes the two expanded destination rows 2*row, 2*row + 1
};

// Kernel configurations: cfg 0 tiles up to 256 columns with a 4-deep ring, cfg 1
// up to 128 columns with a 7-deep ring (one CTA per SM); cfg 2 up to 128 / 3-deep
// and cfg 3 up to 64 / 4-deep (two CTAs per SM).
int tc_configs();
int tc_cfg_tn(int cfg);
int tc_cfg_stages(int cfg);
int tc_cfg_ctas_per_sm(int cfg);
int tc_smem_bytes(int cfg);
int tc_tile_m();
int tc_tile_n();        // workspace row stride (floats): the widest tile of any cfg
int tc_ktile_bytes();

// Convert the rows listed in `rows` (64 threads each) into pair layout.
cudaError_t launch_pad_split(int eb, const double* src, void* dst, const PadJob* jobs,
                             const PadRow* rows, int nrows, cudaStream_t st);

// Shared-memory opt-in of the GEMM kernels on the current device; call before
// launch_tc_gemm (not during a stream capture).
cudaError_t prepare_tc_gemm();

// One stage: the warp-specialized TMA/tcgen05 kernel of configuration cfg, CTA c
// running units [cta_begin[c], cta_begin[c+1]) in order, then the reduction of
// K-split tiles.
// Programmatic dependent launch (sm_90+): a kernel launched with launch_pdl may
// start while the previous kernel on the stream drains; pdl_wait() blocks until
// that kernel has completed and its writes are visible (a no-op for a plain
// launch), pdl_launch_dependents() lets the next such kernel start.
__device__ __forceinline__ void pdl_wait() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
}
__device__ __forceinline__ void pdl_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), int grid, int block, size_t smem,
                       cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

cudaError_t launch_tc_gemm(int eb, bool out_split, int cfg, const CUtensorMap* maps,
                           const SUnit* units, const int* cta_begin, int nctas, const SOut* outs,
                           const SSeg2* segs, void* c_pair, double* c64, float* ws,
                           const SRed* reds, const SRedBlk* redblk, int nredblk, int* err,
                           cudaStream_t st);

}  // namespace dmrgx
