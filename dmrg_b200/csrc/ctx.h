// The dmrgx context: device copies of the environments, the two-stage matvec
// plan and its scratch, one CUDA stream.  Internal header.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <map>
#include <vector>

#include "grouped.h"
#include "qmeta.h"
#include "split.h"

namespace dmrgx {

void set_error(const std::string& msg);

// one task row as a plain GEMM: C[M x N] += sign A[M x K] B[N x K]^T, offsets in
// doubles (A in the environment image, which already carries the row's sign)
struct PlainRow {
  int64_t a_off, b_off, c_off;
  int32_t M, N, K, sign;
};

// one stage of the matvec on the device
struct Stage {
  std::vector<PlainRow> rows;  // the same work as one GEMM per task row
  std::vector<DOut> outs;
  std::vector<DSeg> segs;
  std::vector<DUnit> units;   // CTA assignment of the FP64 grouped kernel
  int64_t nslots = 0;          // K-split workspace slots the units use
  DOut* d_outs = nullptr;
  DSeg* d_segs = nullptr;
  DUnit* d_units = nullptr;
  double* d_ws = nullptr;      // nslots x 4096 doubles
  int* d_tickets = nullptr;    // nslots, zero between launches
  bool full_cover = true;   // every element of the output is written by some tile
  int64_t a_len = 0;        // real length of operand-A image
  cudaStream_t st = nullptr; // stream of the device arrays
  void free_device();
};

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t b);
  void release();
};

// The split-precision form of a plan: descriptors of one stage.
struct SplitStage {
  std::vector<SOut> outs;
  std::vector<SSeg2> segs;
  std::vector<SUnit> units;      // grouped by CTA
  std::vector<int> cta_begin;    // CTA c runs units [cta_begin[c], cta_begin[c+1])
  std::vector<SRed> reds;
  std::vector<SRedBlk> redblk;
  std::vector<CUtensorMap> maps;
  SOut* d_outs = nullptr;
  SSeg2* d_segs = nullptr;
  SUnit* d_units = nullptr;
  int* d_cta_begin = nullptr;
  SRed* d_reds = nullptr;
  SRedBlk* d_redblk = nullptr;
  CUtensorMap* d_maps = nullptr;
  int nslots = 0;
  bool full_cover = true;
  // operand blocks of the stage's tensor maps: device address, logical padded
  // K, rows, and whether it is a B operand (box rows = the tile width)
  struct MapReq {
    uint8_t* base;
    int64_t kq, rows;
    bool b_side;
  };
  std::vector<MapReq> req;
  // tiling in use (chosen by the autotuner): kernel configuration, halving of
  // blocks that fit one tile, scale of the K-split threshold
  int cfg = 0;
  bool halve = false;
  double cap_scale = 1.0;
  bool tuned = false;            // true: measured for this plan; false: from the cache / default
  cudaStream_t st = nullptr;     // stream of the device arrays
  void free_device();
};

// Split-precision plan: (hi, lo) operand images in the pair layout of split.h
// (one buffer each) and the two stages.
struct SplitPlan {
  int eb = 0;                      // element bytes of the pairs: 2 BF16, 4 TF32 (0 = none)
  SplitStage s1, s2;
  int64_t a1_len = 0, a2_len = 0, psi_len = 0, store_len = 0;   // elements (hi and lo)
  std::vector<PadJob> psi_jobs;    // per-matvec FP64 psi -> (hi, lo)
  std::vector<PadRow> psi_rows;
  PadJob* d_psi_jobs = nullptr;
  PadRow* d_psi_rows = nullptr;
  void free_device();
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
  // task lists the stages run: the main pair's rows (the reference's rmap / lmap)
  // followed, on a periodic chain, by the edge pair's remap / lemap rows with
  // block indices shifted past the main environments' blocks and store offsets
  // past the main store (src/core.cpp:27-30, :241-247)
  std::vector<dmrgx::MapRow> rmap, lmap;
  int64_t n_rmap_main = 0, n_lmap_main = 0, d_store_main = 0;
  int r_blocks_main = 0, l_blocks_main = 0;
  int boundary = 0;    // DMRGX_BOUNDARY_* of dmrgx_dmrg
  int eig_nev = 6, eig_ncv = 0;  // site-step eigensolver of dmrgx_dmrg (dmrgx_set_solver)
  bool predict = false;
  std::vector<std::vector<int>> psi_dim, psi_sym;
  int n_store_blocks = 0;
  dmrgx::Stage st1, st2;

  dmrgx::DevBuf renv, lenv, store, din, dout;  // device
  dmrgx::SplitPlan sp;                            // split-precision form (built on demand)
  dmrgx::DevBuf sa1, sa2, spsi, sstore, sws, err;  // split-precision buffers
  bool prof = false;                            // per-launch event timing
  std::vector<cudaEvent_t> prof_ev;             // 4 per timed matvec
  void prof_mark();                             // record one event if profiling

  bool per_block = false;                       // DMRGX_SCHED_PER_BLOCK: one GEMM per task row
  void* blas = nullptr;                         // cuBLAS handle of the per-block schedule
  // wall seconds of the plan-building parts, summed since the last dmrgx_dmrg
  // began: [0] sector bookkeeping and task lists, [1] FP64 images and
  // descriptors (uploads included), [2] split-precision images and
  // descriptors, [3] autotuning
  double t_plan_part[4] = {0, 0, 0, 0};
  // solve group of this context's site steps (dmrgx_set_group), or null
  struct dmrgx_group* group = nullptr;
  // instantiated Lanczos cycle graphs kept between solves (eig.cu)
  std::map<int64_t, cudaGraphExec_t> cycle_graphs;
  // results of the last dmrgx_svd: U and V (metadata, values) and the spectrum
  std::vector<int> svd_um, svd_vm;
  std::vector<double> svd_uv, svd_vv, svd_s;
  void* run = nullptr;                          // state of the last dmrgx_dmrg (MPS, centre)
  void (*run_free)(void*) = nullptr;

  int f() const { return dtype == 1 ? 2 : 1; }  // doubles per element
};
