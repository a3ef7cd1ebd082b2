// Device descriptors of one stage of the block-sparse matvec, executed as a
// grouped, segmented-K GEMM:  for every output block o
//     C_o[M x N] = sum_{s in segs(o)} A_s[M x K_s] . B_s[N x K_s]^T
// with A_s, B_s, C_o dense row-major and K contiguous in both operands (the
// reference's 'N','T' contraction, src/tensor.cpp:698-718).  All the
// reference's task rows that write one output block become that block's segments,
// summed in one pass, so there is no accumulation across launches and no atomics.
//
// Complex (interleaved re,im) blocks run as real GEMMs: A is read as M x 2K real,
// B is expanded on load to 2N x 2K real rows [Br,-Bi] / [Bi,Br], and C comes out
// as M x 2N real = M x N complex interleaved.  All offsets/extents below are in
// real (double) units.
#pragma once
#include <cstdint>

namespace dmrgx {

struct DOut {
  int64_t c_off;     // offset of C_o in the output buffer
  int32_t m, n;      // rows, real columns (2N for complex)
  int32_t seg_begin, seg_count;
};

struct DSeg {
  int64_t a_off;     // offset of A_s in the operand-A buffer (row stride = k)
  int64_t b_off;     // offset of B_s in the operand-B buffer (row stride = k)
  int32_t k;         // real K (2K for complex)
  int32_t pad_;
};

struct DTile {
  int32_t out;       // index into DOut
  int16_t tm, tn;    // tile coordinates inside the output block
};

// One work unit of the FP64 grouped kernel: tile (tm, tn) of output block `out`
// over the k-tiles [kt0, kt1) of the block's segments taken in order.  A tile cut
// along K into `nparts` parts stores part `part`'s partial sum to workspace slot
// `slot` (64 x 64 doubles); its parts own slots slot - part ... slot - part +
// nparts - 1, and the ticket at index slot - part counts them.  out < 0 marks a
// padding entry of the CTA assignment.
struct DUnit {
  int32_t out = -1;
  int16_t tm = 0, tn = 0;
  int32_t kt0 = 0, kt1 = 0;
  int32_t slot = -1;           // -1: the whole K range, written directly
  int16_t part = 0, nparts = 1;
};

}  // namespace dmrgx
