// The dmrgx context: device copies of the environments, the two-stage matvec
// plan and its scratch, one CUDA stream.  Internal header.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "grouped.h"
#include "qmeta.h"

namespace dmrgx {

void set_error(const std::string& msg);

// one stage of the matvec on the device
struct Stage {
  std::vector<DOut> outs;
  std::vector<DSeg> segs;
  std::vector<DTile> tiles;
  DOut* d_outs = nullptr;
  DSeg* d_segs = nullptr;
  DTile* d_tiles = nullptr;
  bool full_cover = true;   // every element of the output is written by some tile
  int64_t a_len = 0;        // real length of operand-A image
  void free_device();
};

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t b);
  void release();
};

}  // namespace dmrgx

struct dmrgx_ctx {
  int dtype = 0;       // DMRGX_F64 / DMRGX_C128
  int device = 0;
  int prec = 0;        // DMRGX_PREC_*
  int num_sms = 148;
  cudaStream_t stream = nullptr;

  bool has_plan = false;
  int64_t n = 0, d_store = 0, flops = 0;
  std::vector<dmrgx::MapRow> rmap, lmap;
  std::vector<std::vector<int>> psi_dim, psi_sym;
  int n_store_blocks = 0;
  dmrgx::Stage st1, st2;

  dmrgx::DevBuf renv, lenv, store, din, dout;  // device
  double* h_in = nullptr;                       // pinned staging
  double* h_out = nullptr;
  size_t h_cap = 0;

  int f() const { return dtype == 1 ? 2 : 1; }  // doubles per element
};
