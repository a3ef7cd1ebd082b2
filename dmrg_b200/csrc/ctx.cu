// C ABI of libdmrgx: contexts, plans, the H_eff matvec.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <string>

#include "../../include/dmrgx.h"
#include "ctx.h"
#include "devmem.h"
#include "kernels.h"
#include "qtensor.h"
#include "split.h"

using namespace dmrgx;

namespace dmrgx {

double wall_now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int build_split_plan(dmrgx_ctx* c, int eb);
int run_matvec_split(dmrgx_ctx* c, const double* in, double* out);
int run_matvec_plain(dmrgx_ctx* c, const double* in, double* out);
void plain_release(dmrgx_ctx* c);

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }

void Stage::free_device() {
  dfree(d_outs, st);
  dfree(d_segs, st);
  dfree(d_units, st);
  dfree(d_ws, st);
  dfree(d_tickets, st);
  d_outs = nullptr;
  d_segs = nullptr;
  d_units = nullptr;
  d_ws = nullptr;
  d_tickets = nullptr;
}

cudaError_t DevBuf::ensure(size_t b) {
  if (b <= bytes && p) return cudaSuccess;
  release();
  cudaError_t e = cudaMalloc(&p, b ? b : 16);
  if (e == cudaSuccess) bytes = b;
  return e;
}

}  // namespace dmrgx

void dmrgx_ctx::prof_mark() {
  if (!prof) return;
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, stream);
  prof_ev.push_back(e);
}

namespace dmrgx {

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

}  // namespace dmrgx

#define CUDA_TRY(expr)                                                              \
  do {                                                                              \
    cudaError_t e_ = (expr);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      set_error(std::string(#expr) + ": " + cudaGetErrorString(e_));                \
      return DMRGX_E_CUDA;                                                          \
    }                                                                               \
  } while (0)

#define ARG_CHECK(cond, msg)  \
  do {                        \
    if (!(cond)) {            \
      set_error(msg);         \
      return DMRGX_E_ARG;     \
    }                         \
  } while (0)

namespace {
using dmrgx::wall_now;

// Environment image on the host with the task signs folded into the blocks:
// a block used only with alpha=-1 is stored negated, a block used with both
// signs gets a negated copy appended.  plus/minus: real offsets per block.
struct EnvImage {
  std::vector<double> vals;        // host values (empty when built on the device)
  std::vector<int64_t> plus, minus;
  int64_t len = 0;                 // doubles
};

EnvImage make_image(const double* src, const std::vector<int64_t>& off,
                    const std::vector<int64_t>& size, const std::vector<MapRow>& rows, int f) {
  const size_t nb = size.size();
  std::vector<int> use(nb, 0);
  for (auto& r : rows) use[r.blk] |= (r.alpha >= 0 ? 1 : 2);
  EnvImage im;
  int64_t total = off.empty() ? 0 : off.back();
  int64_t extra = 0;
  for (size_t b = 0; b < nb; b++)
    if (use[b] == 3) extra += size[b];
  im.len = (total + extra) * f;
  if (src) {
    im.vals.resize((size_t)im.len);
    std::memcpy(im.vals.data(), src, sizeof(double) * (size_t)total * f);
  }
  im.plus.assign(nb, -1);
  im.minus.assign(nb, -1);
  int64_t tail = total * f;
  for (size_t b = 0; b < nb; b++) {
    const int64_t o = off[b] * f, s = size[b] * f;
    if (use[b] == 2) {
      if (src)
        for (int64_t i = 0; i < s; i++) im.vals[o + i] = -im.vals[o + i];
      im.minus[b] = o;
    } else if (use[b] == 3) {
      im.plus[b] = o;
      if (src)
        for (int64_t i = 0; i < s; i++) im.vals[tail + i] = -im.vals[o + i];
      im.minus[b] = tail;
      tail += s;
    } else {
      im.plus[b] = o;
    }
  }
  return im;
}

std::string build_stage(const std::vector<MapRow>& rows, const std::vector<int64_t>& blk_size,
                        const EnvImage& im, int f, int64_t in_len, int64_t out_len, Stage& st,
                        int64_t& flops, int grid) {
  st.outs.clear();
  st.segs.clear();
  st.units.clear();
  st.rows.clear();
  std::map<int64_t, int> by_off;  // output offset -> out index
  std::vector<std::vector<DSeg>> per_out;
  for (auto& r : rows) {
    if (r.blk < 0 || r.blk >= (int)blk_size.size()) return "task row: block index out of range";
    if (r.cols <= 0 || r.rows < 0) return "task row: bad rows/cols";
    const int64_t S = blk_size[r.blk];
    const int64_t K = r.cols, N = r.rows;
    if (S % K) return "task row: block size is not a multiple of cols";
    const int64_t M = S / K;
    if (r.in_beg < 0 || r.in_beg + N * K > in_len) return "task row: input range out of bounds";
    if (r.out_beg < 0 || r.out_beg + M * N > out_len) return "task row: output range out of bounds";
    if (M * f > INT32_MAX || N * f > INT32_MAX || K * f > INT32_MAX)
      return "task row: block extent too large";
    // an empty output block writes nothing (and shares its offset with the next block)
    if (M == 0 || N == 0) continue;
    auto it = by_off.find(r.out_beg);
    int oi;
    if (it == by_off.end()) {
      oi = (int)st.outs.size();
      by_off[r.out_beg] = oi;
      DOut o;
      o.c_off = r.out_beg * f;
      o.m = (int32_t)M;
      o.n = (int32_t)(N * f);
      o.seg_begin = 0;
      o.seg_count = 0;
      st.outs.push_back(o);
      per_out.emplace_back();
    } else {
      oi = it->second;
      if (st.outs[oi].m != M || st.outs[oi].n != N * f)
        return "task rows writing one output block disagree on its shape";
    }
    DSeg sg;
    sg.a_off = r.alpha >= 0 ? im.plus[r.blk] : im.minus[r.blk];
    // the image holds the block with the row's sign applied, so alpha is +1
    st.rows.push_back({sg.a_off, r.in_beg * f, r.out_beg * f, (int32_t)M, (int32_t)N,
                       (int32_t)K, 1});
    sg.b_off = r.in_beg * f;
    sg.k = (int32_t)(K * f);
    sg.pad_ = 0;
    per_out[oi].push_back(sg);
    flops += 2 * M * N * K * (f == 2 ? 4 : 1);
  }
  int64_t covered = 0;
  for (size_t o = 0; o < st.outs.size(); o++) {
    st.outs[o].seg_begin = (int32_t)st.segs.size();
    st.outs[o].seg_count = (int32_t)per_out[o].size();
    st.segs.insert(st.segs.end(), per_out[o].begin(), per_out[o].end());
    covered += (int64_t)st.outs[o].m * st.outs[o].n / f;
  }
  st.full_cover = covered == out_len;
  const int BM = f64_tile_m(), BN = f64_tile_n();
  for (const DOut& o : st.outs)
    if ((o.m + BM - 1) / BM > 32767 || (o.n + BN - 1) / BN > 32767)
      return "output block too large for the tile grid";
  st.nslots = make_f64_units(st.outs, st.segs, grid, f64_split_mode(), st.units);
  return "";
}

int upload_stage(Stage& st, cudaStream_t s) {
  st.free_device();
  st.st = s;
  CUDA_TRY(dalloc(&st.d_outs, st.outs.size(), s));
  CUDA_TRY(dalloc(&st.d_segs, st.segs.size(), s));
  CUDA_TRY(dalloc(&st.d_units, st.units.size(), s));
  if (st.nslots > 0) {
    CUDA_TRY(dalloc(&st.d_ws, (size_t)st.nslots * f64_tile_m() * f64_tile_n(), s));
    CUDA_TRY(dalloc(&st.d_tickets, (size_t)st.nslots, s));
    CUDA_TRY(cudaMemsetAsync(st.d_tickets, 0, sizeof(int) * st.nslots, s));
  }
  if (!st.outs.empty())
    CUDA_TRY(cudaMemcpyAsync(st.d_outs, st.outs.data(), sizeof(DOut) * st.outs.size(),
                             cudaMemcpyHostToDevice, s));
  if (!st.segs.empty())
    CUDA_TRY(cudaMemcpyAsync(st.d_segs, st.segs.data(), sizeof(DSeg) * st.segs.size(),
                             cudaMemcpyHostToDevice, s));
  if (!st.units.empty())
    CUDA_TRY(cudaMemcpyAsync(st.d_units, st.units.data(), sizeof(DUnit) * st.units.size(),
                             cudaMemcpyHostToDevice, s));
  return 0;
}

// Device image of an environment with the signs folded in, gathered from a
// device tensor (the site-step path: environments never leave the GPU).
int device_image(dmrgx_ctx* c, const QTensor& T, const EnvImage& im, double* dst) {
  const int f = c->f();
  std::vector<GOut> go;
  std::vector<GSrc> gs;
  for (size_t b = 0; b < im.plus.size(); b++) {
    const int64_t sz = T.bsize((int)b);
    if (sz == 0) continue;
    for (int sgn = 0; sgn < 2; sgn++) {
      const int64_t at = sgn ? im.minus[b] : im.plus[b];
      if (at < 0) continue;
      GSrc g;
      std::memset(&g, 0, sizeof(g));
      g.src_off = T.off[b];
      g.strides[0] = 1;
      g.sign = sgn ? -1.0 : 1.0;
      gs.push_back(g);
      GOut o;
      std::memset(&o, 0, sizeof(o));
      o.dst_off = at / f;
      o.size = sz;
      o.rank = 1;
      o.dims[0] = (int32_t)sz;
      o.dst_strides[0] = 1;
      o.src_begin = (int32_t)gs.size() - 1;
      o.src_count = 1;
      go.push_back(o);
    }
  }
  CUDA_TRY(launch_gather(T.d, dst, go, gs, f == 2, c->stream));
  return 0;
}

// One (R~, L~) pair of the matvec with its own task lists, environment blocks
// and intermediate: the main pair, and on a periodic chain the edge pair
// (src/core.cpp:27-30).  Values come from the host (rvals/lvals, blocks packed
// at roff/loff) or from device tensors (rdev/ldev).
struct PairSrc {
  std::vector<MapRow> rmap, lmap;
  const double* rvals = nullptr;
  const double* lvals = nullptr;
  std::vector<int64_t> roff, rsize, loff, lsize;
  const QTensor* rdev = nullptr;
  const QTensor* ldev = nullptr;
  int64_t store = 0;
};

// Common tail of the plan entry points: sign-folded env images, stage
// descriptors, device uploads, scratch.  The pairs are merged into one task
// list per stage: each pair's stage-1 rows write their own part of the
// intermediate, and its stage-2 rows are further K-segments of the psi blocks,
// which is the reference's accumulation of the edge pair into out (lemap built
// with beta = 1, src/core.cpp:247).
int finalize_plan(dmrgx_ctx* c, const std::vector<PairSrc>& pairs) {
  const double t0 = wall_now();
  const int f = c->f();
  c->has_plan = false;
  c->flops = 0;
  std::vector<MapRow> R, Lr;
  std::vector<int64_t> rsz, lsz;
  EnvImage RI, LI;
  std::vector<EnvImage> ris, lis;
  std::vector<int64_t> rimg, limg;  // image offset (doubles) of every pair
  int64_t soff = 0;
  int rb = 0, lb = 0;
  for (const PairSrc& p : pairs) {
    ris.push_back(make_image(p.rvals, p.roff, p.rsize, p.rmap, f));
    lis.push_back(make_image(p.lvals, p.loff, p.lsize, p.lmap, f));
    const EnvImage& ri = ris.back();
    const EnvImage& li = lis.back();
    for (MapRow r : p.rmap) {
      r.blk += rb;
      r.out_beg += soff;
      R.push_back(r);
    }
    for (MapRow r : p.lmap) {
      r.blk += lb;
      r.in_beg += soff;
      Lr.push_back(r);
    }
    rsz.insert(rsz.end(), p.rsize.begin(), p.rsize.end());
    lsz.insert(lsz.end(), p.lsize.begin(), p.lsize.end());
    auto merge = [](EnvImage& all, const EnvImage& one, std::vector<int64_t>& at) {
      at.push_back(all.len);
      all.vals.insert(all.vals.end(), one.vals.begin(), one.vals.end());
      for (int64_t x : one.plus) all.plus.push_back(x < 0 ? -1 : x + all.len);
      for (int64_t x : one.minus) all.minus.push_back(x < 0 ? -1 : x + all.len);
      all.len += one.len;
    };
    merge(RI, ri, rimg);
    merge(LI, li, limg);
    soff += p.store;
    rb += (int)p.rsize.size();
    lb += (int)p.lsize.size();
  }
  c->rmap = R;
  c->lmap = Lr;
  c->n_rmap_main = pairs.empty() ? 0 : (int64_t)pairs[0].rmap.size();
  c->n_lmap_main = pairs.empty() ? 0 : (int64_t)pairs[0].lmap.size();
  c->d_store_main = pairs.empty() ? 0 : pairs[0].store;
  c->r_blocks_main = pairs.empty() ? 0 : (int)pairs[0].rsize.size();
  c->l_blocks_main = pairs.empty() ? 0 : (int)pairs[0].lsize.size();
  c->d_store = soff;
  const int grid = c->num_sms * 3;
  std::string e = build_stage(c->rmap, rsz, RI, f, c->n, c->d_store, c->st1, c->flops, grid);
  if (e.empty()) e = build_stage(c->lmap, lsz, LI, f, c->d_store, c->n, c->st2, c->flops, grid);
  if (!e.empty()) {
    set_error(e);
    return DMRGX_E_ARG;
  }
  std::map<int64_t, int> so;
  for (auto& r : c->rmap) so[r.out_beg] = 1;
  c->n_store_blocks = (int)so.size();
  c->st1.a_len = RI.len;
  c->st2.a_len = LI.len;
  CUDA_TRY(cudaSetDevice(c->device));
  CUDA_TRY(c->renv.ensure(sizeof(double) * (size_t)std::max<int64_t>(1, RI.len)));
  CUDA_TRY(c->lenv.ensure(sizeof(double) * (size_t)std::max<int64_t>(1, LI.len)));
  for (size_t i = 0; i < pairs.size(); i++) {
    if (pairs[i].rdev) {
      int rc0 = device_image(c, *pairs[i].rdev, ris[i], (double*)c->renv.p + rimg[i]);
      if (rc0) return rc0;
    }
    if (pairs[i].ldev) {
      int rc0 = device_image(c, *pairs[i].ldev, lis[i], (double*)c->lenv.p + limg[i]);
      if (rc0) return rc0;
    }
  }
  CUDA_TRY(c->store.ensure(sizeof(double) * (size_t)std::max<int64_t>(1, c->d_store * f)));
  CUDA_TRY(c->din.ensure(sizeof(double) * (size_t)std::max<int64_t>(1, c->n * f)));
  CUDA_TRY(c->dout.ensure(sizeof(double) * (size_t)std::max<int64_t>(1, c->n * f)));
  if (!RI.vals.empty())
    CUDA_TRY(cudaMemcpyAsync(c->renv.p, RI.vals.data(), sizeof(double) * RI.vals.size(),
                             cudaMemcpyHostToDevice, c->stream));
  if (!LI.vals.empty())
    CUDA_TRY(cudaMemcpyAsync(c->lenv.p, LI.vals.data(), sizeof(double) * LI.vals.size(),
                             cudaMemcpyHostToDevice, c->stream));
  int rc = upload_stage(c->st1, c->stream);
  if (rc) return rc;
  rc = upload_stage(c->st2, c->stream);
  if (rc) return rc;
  // RI/LI are host temporaries: wait for the uploads before they go away
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  const double t1 = wall_now();
  c->t_plan_part[1] += t1 - t0;
  c->sp.free_device();
  c->sp = SplitPlan();
  if (c->prec != DMRGX_PREC_FP64) {
    rc = build_split_plan(c, c->prec == DMRGX_PREC_BF16X3 ? 2 : 4);
    if (rc) return rc;
  }
  c->has_plan = true;
  return 0;
}

int run_matvec_fp64(dmrgx_ctx* c, const double* in, double* out);

int run_matvec(dmrgx_ctx* c, const double* in, double* out) {
  if (c->prec != DMRGX_PREC_FP64) return run_matvec_split(c, in, out);
  if (c->per_block) return run_matvec_plain(c, in, out);
  return run_matvec_fp64(c, in, out);
}

// error word of the bounded device waits (split path); 0 = fine
int check_device_error(dmrgx_ctx* c) {
  if (!c->err.p) return 0;
  int h = 0;
  CUDA_TRY(cudaMemcpyAsync(&h, c->err.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (h) {
    set_error("a bounded device wait timed out in the split-precision matvec");
    CUDA_TRY(cudaMemsetAsync(c->err.p, 0, sizeof(int), c->stream));
    return DMRGX_E_TIMEOUT;
  }
  return 0;
}

int run_matvec_fp64(dmrgx_ctx* c, const double* in, double* out) {
  const bool cplx = c->dtype == DMRGX_C128;
  c->prof_mark();
  c->prof_mark();
  const int grid = c->num_sms * 3;
  double* store = (double*)c->store.p;
  if (!c->st1.full_cover)
    CUDA_TRY(cudaMemsetAsync(store, 0, sizeof(double) * c->d_store * c->f(), c->stream));
  CUDA_TRY(launch_grouped_f64((const double*)c->renv.p, in, store, c->st1.d_units,
                              (int)c->st1.units.size(), c->st1.d_outs, c->st1.d_segs, cplx, grid,
                              c->stream, c->st1.d_ws, c->st1.d_tickets));
  c->prof_mark();
  if (!c->st2.full_cover)
    CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double) * c->n * c->f(), c->stream));
  CUDA_TRY(launch_grouped_f64((const double*)c->lenv.p, store, out, c->st2.d_units,
                              (int)c->st2.units.size(), c->st2.d_outs, c->st2.d_segs, cplx, grid,
                              c->stream, c->st2.d_ws, c->st2.d_tickets));
  c->prof_mark();
  return 0;
}

}  // namespace

namespace dmrgx {
int matvec_fp64(dmrgx_ctx* c, const double* in, double* out) {
  if (!c->has_plan) {
    set_error("matvec: no plan");
    return DMRGX_E_STATE;
  }
  return run_matvec_fp64(c, in, out);
}

// The step functions' bookkeeping (src/core.cpp:236-247): psi layout from
// generate_dim_sym, rmap / lmap of the main pair and, on a periodic chain,
// remap / lemap of the edge pair against the same psi layout (its own
// intermediate; lemap with beta = 1, so the edge pair accumulates into out).
std::string step_maps(const Group& G, const QMeta& L, const QMeta& R, const QMeta* Le,
                      const QMeta* Re, int l_num, int r_num, int sector,
                      std::vector<std::vector<int>>& dim, std::vector<std::vector<int>>& sym,
                      std::vector<MapRow>& rm, std::vector<MapRow>& lm, int64_t& d_store,
                      std::vector<MapRow>& erm, std::vector<MapRow>& elm, int64_t& e_store) {
  std::vector<std::vector<int>> dim_ret, sym_ret;
  generate_dim_sym(G, L, l_num - 1, R, r_num, sector, dim, sym);
  std::string e = get_map(G, R, dim, sym, r_num, 0, false, dim_ret, sym_ret, rm);
  if (!e.empty()) return "rmap: " + e;
  d_store = get_dimension(dim_ret, sym_ret);
  e = get_map(G, L, dim_ret, sym_ret, l_num, 0, true, dim, sym, lm);
  if (!e.empty()) return "lmap: " + e;
  erm.clear();
  elm.clear();
  e_store = 0;
  if (Le && Re) {
    e = get_map(G, *Re, dim, sym, r_num, 0, false, dim_ret, sym_ret, erm);
    if (!e.empty()) return "remap: " + e;
    e_store = get_dimension(dim_ret, sym_ret);
    e = get_map(G, *Le, dim_ret, sym_ret, l_num, 1, true, dim, sym, elm);
    if (!e.empty()) return "lemap: " + e;
  }
  return "";
}

// Plan from device tensors (the site step): same bookkeeping as
// dmrgx_plan_build, environment images gathered on the device.  Le / Re: the
// edge pair of a periodic chain, or null.
int plan_build_device(dmrgx_ctx* c, const QTensor& L, const QTensor& R, int l_num, int r_num,
                      int sector, const Group& G, const QTensor* Le, const QTensor* Re) {
  if (L.f != c->f() || R.f != c->f() || (Le && Le->f != c->f()) || (Re && Re->f != c->f())) {
    set_error("plan: tensor element type differs from the context's");
    return DMRGX_E_ARG;
  }
  const double t0 = wall_now();
  const bool pbc = Le && Re;
  std::vector<PairSrc> pairs(pbc ? 2 : 1);
  std::vector<std::vector<int>> dim, sym;
  std::vector<MapRow> erm, elm;
  int64_t es = 0;
  std::string e = step_maps(G, L.m, R.m, pbc ? &Le->m : nullptr, pbc ? &Re->m : nullptr, l_num,
                            r_num, sector, dim, sym, pairs[0].rmap, pairs[0].lmap,
                            pairs[0].store, erm, elm, es);
  if (!e.empty()) {
    set_error("plan: " + e);
    return DMRGX_E_ARG;
  }
  if (pbc) {
    pairs[1].rmap = erm;
    pairs[1].lmap = elm;
    pairs[1].store = es;
  }
  c->n = get_dimension(dim, sym);
  c->psi_dim = dim;
  c->psi_sym = sym;
  auto dev = [](PairSrc& p, const QTensor& Ro, const QTensor& Lo) {
    p.rdev = &Ro;
    p.ldev = &Lo;
    p.roff = Ro.off;
    p.loff = Lo.off;
    p.rsize.resize(Ro.m.syms.size());
    p.lsize.resize(Lo.m.syms.size());
    for (size_t b = 0; b < p.rsize.size(); b++) p.rsize[b] = Ro.bsize((int)b);
    for (size_t b = 0; b < p.lsize.size(); b++) p.lsize[b] = Lo.bsize((int)b);
  };
  dev(pairs[0], R, L);
  if (pbc) dev(pairs[1], *Re, *Le);
  c->t_plan_part[0] += wall_now() - t0;
  return finalize_plan(c, pairs);
}

int run_matvec_any(dmrgx_ctx* c, const double* in, double* out, bool fp64) {
  if (fp64 && c->per_block) return run_matvec_plain(c, in, out);
  return fp64 ? run_matvec_fp64(c, in, out) : run_matvec(c, in, out);
}
}  // namespace dmrgx

extern "C" {

const char* dmrgx_last_error(void) { return g_err.c_str(); }
const char* dmrgx_version(void) { return "dmrgx 0.1 (sm_100a)"; }

int dmrgx_ctx_create(dmrgx_ctx** out, int dtype, int device) {
  ARG_CHECK(out != nullptr, "ctx_create: null output pointer");
  ARG_CHECK(dtype == DMRGX_F64 || dtype == DMRGX_C128, "ctx_create: dtype must be F64 or C128");
  int ndev = 0;
  CUDA_TRY(cudaGetDeviceCount(&ndev));
  ARG_CHECK(device >= 0 && device < ndev, "ctx_create: no such CUDA device");
  CUDA_TRY(cudaSetDevice(device));
  dmrgx_ctx* c = new dmrgx_ctx();
  c->dtype = dtype;
  c->device = device;
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e == cudaSuccess) c->num_sms = prop.multiProcessorCount;
  if (e == cudaSuccess && prop.major < 10) {
    delete c;
    set_error("ctx_create: this library is built for sm_100a (Blackwell B200)");
    return DMRGX_E_CUDA;
  }
  if (e == cudaSuccess && !library_pool(device)) {
    delete c;
    set_error("ctx_create: cannot create the library's device memory pool");
    return DMRGX_E_CUDA;
  }
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    set_error(std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    return DMRGX_E_CUDA;
  }
  *out = c;
  return 0;
}

void dmrgx_ctx_destroy(dmrgx_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  if (c->run_free) c->run_free(c->run);
  c->run = nullptr;
  plain_release(c);
  c->st1.free_device();
  c->st2.free_device();
  for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
  for (auto& g : c->cycle_graphs) cudaGraphExecDestroy(g.second);
  c->sp.free_device();
  for (DevBuf* b : {&c->sa1, &c->sa2, &c->spsi, &c->sstore, &c->sws, &c->err})
    b->release();
  c->renv.release();
  c->lenv.release();
  c->store.release();
  c->din.release();
  c->dout.release();
  cudaStreamDestroy(c->stream);
  delete c;
}

int dmrgx_set_precision(dmrgx_ctx* c, int prec) {
  ARG_CHECK(c, "null context");
  ARG_CHECK(prec == DMRGX_PREC_FP64 || prec == DMRGX_PREC_BF16X3 || prec == DMRGX_PREC_TF32X3,
            "set_precision: unknown precision");
  if (prec == c->prec) return 0;
  ARG_CHECK(prec == DMRGX_PREC_FP64 || !c->per_block,
            "set_precision: the per-block schedule is FP64 only");
  c->prec = prec;
  c->sp.free_device();
  c->sp = SplitPlan();
  if (c->has_plan && prec != DMRGX_PREC_FP64) {
    CUDA_TRY(cudaSetDevice(c->device));
    int rc = build_split_plan(c, prec == DMRGX_PREC_BF16X3 ? 2 : 4);
    if (rc) {
      c->has_plan = false;
      return rc;
    }
  }
  return 0;
}

int dmrgx_matvec_launches(dmrgx_ctx* c, int* out) {
  ARG_CHECK(c && out, "matvec_launches: null argument");
  ARG_CHECK(c->has_plan, "matvec_launches: no plan");
  if (c->prec != DMRGX_PREC_FP64)
    *out = 3 + (c->sp.s1.redblk.empty() ? 0 : 1) + (c->sp.s2.redblk.empty() ? 0 : 1);
  else if (c->per_block)
    *out = (int)(c->st1.rows.size() + c->st2.rows.size());
  else
    *out = (c->st1.units.empty() ? 0 : 1) + (c->st2.units.empty() ? 0 : 1);
  return 0;
}

int dmrgx_split_tuning(dmrgx_ctx* c, int* out, int cap) {
  ARG_CHECK(c && out && cap >= 8, "split_tuning: need a context and 8 slots");
  ARG_CHECK(c->has_plan && c->sp.eb != 0, "split_tuning: no split-precision plan");
  const SplitStage* st[2] = {&c->sp.s1, &c->sp.s2};
  for (int i = 0; i < 2; i++) {
    out[4 * i] = st[i]->cfg;
    out[4 * i + 1] = st[i]->halve ? 1 : 0;
    out[4 * i + 2] = st[i]->cap_scale >= 1e6 ? -100 : (int)(st[i]->cap_scale * 100 + 0.5);
    out[4 * i + 3] = st[i]->tuned ? 1 : 0;
  }
  return 0;
}

int dmrgx_set_schedule(dmrgx_ctx* c, int schedule) {
  ARG_CHECK(c, "null context");
  ARG_CHECK(schedule == DMRGX_SCHED_GROUPED || schedule == DMRGX_SCHED_PER_BLOCK,
            "set_schedule: unknown schedule");
  ARG_CHECK(schedule == DMRGX_SCHED_GROUPED || c->prec == DMRGX_PREC_FP64,
            "set_schedule: the per-block schedule is FP64 only");
  c->per_block = schedule == DMRGX_SCHED_PER_BLOCK;
  return 0;
}

namespace {
void put_rows(const MapRow* rows, int64_t n, int* o) {
  for (int64_t i = 0; i < n; i++) {
    const MapRow& r = rows[i];
    int* p = o + 7 * i;
    p[0] = r.blk;
    p[1] = (int)r.in_beg;
    p[2] = (int)r.out_beg;
    p[3] = r.rows;
    p[4] = r.cols;
    p[5] = r.beta;
    p[6] = r.alpha;
  }
}

void rows_of(const int* m, int nr, std::vector<MapRow>& out) {
  out.resize(nr);
  for (int i = 0; i < nr; i++) {
    const int* r = m + 7 * i;
    out[i] = MapRow{r[0], r[1], r[2], r[3], r[4], r[5], r[6]};
  }
}

// host environment values + metadata -> one pair's block table
void host_pair(PairSrc& p, const QMeta& Ro, const void* rv, const QMeta& Lo, const void* lv) {
  p.rvals = (const double*)rv;
  p.lvals = (const double*)lv;
  p.roff = Ro.block_offsets();
  p.loff = Lo.block_offsets();
  p.rsize.resize(Ro.syms.size());
  p.lsize.resize(Lo.syms.size());
  for (size_t b = 0; b < p.rsize.size(); b++) p.rsize[b] = Ro.block_size((int)b);
  for (size_t b = 0; b < p.lsize.size(); b++) p.lsize[b] = Lo.block_size((int)b);
}

// block sizes as the caller gives them -> packed offsets; false on a negative size
bool sized_pair(const int64_t* sz, int nb, std::vector<int64_t>& size, std::vector<int64_t>& off) {
  size.assign(sz, sz + nb);
  off.assign(nb + 1, 0);
  for (int b = 0; b < nb; b++) {
    if (size[b] < 0) return false;
    off[b + 1] = off[b] + size[b];
  }
  return true;
}

int plan_build_common(dmrgx_ctx* c, const int* lenv_meta, const void* lenv_vals,
                      const int* renv_meta, const void* renv_vals, const int* ledge_meta,
                      const void* ledge_vals, const int* redge_meta, const void* redge_vals,
                      int l_num, int r_num, int sector, int group_n, int fermion,
                      const char* who) {
  const std::string w = who;
  ARG_CHECK(c, "null context");
  ARG_CHECK(lenv_vals && renv_vals, w + ": null environment values");
  const bool pbc = ledge_meta || redge_meta;
  ARG_CHECK(!pbc || (ledge_meta && redge_meta && ledge_vals && redge_vals),
            w + ": null edge metadata or values");
  Group G;
  ARG_CHECK(make_group(group_n, fermion, G), w + ": group_n out of range");
  QMeta L, R, Le, Re;
  std::string e = L.parse(lenv_meta);
  ARG_CHECK(e.empty(), w + ": lenv metadata: " + e);
  e = R.parse(renv_meta);
  ARG_CHECK(e.empty(), w + ": renv metadata: " + e);
  if (pbc) {
    e = Le.parse(ledge_meta);
    ARG_CHECK(e.empty(), w + ": ledge metadata: " + e);
    e = Re.parse(redge_meta);
    ARG_CHECK(e.empty(), w + ": redge metadata: " + e);
    ARG_CHECK(Le.nleg() >= l_num && Re.nleg() >= r_num, w + ": edge legs out of range");
  }
  ARG_CHECK(l_num >= 2 && l_num <= L.nleg() && r_num >= 1 && r_num <= R.nleg(),
            w + ": l_num/r_num out of range");
  std::vector<PairSrc> pairs(pbc ? 2 : 1);
  std::vector<std::vector<int>> dim, sym;
  std::vector<MapRow> erm, elm;
  int64_t es = 0;
  e = step_maps(G, L, R, pbc ? &Le : nullptr, pbc ? &Re : nullptr, l_num, r_num, sector, dim,
                sym, pairs[0].rmap, pairs[0].lmap, pairs[0].store, erm, elm, es);
  ARG_CHECK(e.empty(), w + ": " + e);
  c->n = get_dimension(dim, sym);
  c->psi_dim = dim;
  c->psi_sym = sym;
  host_pair(pairs[0], R, renv_vals, L, lenv_vals);
  if (pbc) {
    pairs[1].rmap = erm;
    pairs[1].lmap = elm;
    pairs[1].store = es;
    host_pair(pairs[1], Re, redge_vals, Le, ledge_vals);
  }
  return finalize_plan(c, pairs);
}

int build_maps_common(const int* lenv_meta, const int* renv_meta, const int* ledge_meta,
                      const int* redge_meta, int l_num, int r_num, int sector, int group_n,
                      int fermion, int64_t* info, int* rmap, int64_t rmap_cap, int* lmap,
                      int64_t lmap_cap, int* remap, int64_t remap_cap, int* lemap,
                      int64_t lemap_cap, const char* who) {
  const std::string w = who;
  ARG_CHECK(info, w + ": null info");
  const bool pbc = ledge_meta || redge_meta;
  ARG_CHECK(!pbc || (ledge_meta && redge_meta), w + ": null edge metadata");
  Group G;
  ARG_CHECK(make_group(group_n, fermion, G), w + ": group_n out of range");
  QMeta L, R, Le, Re;
  std::string e = L.parse(lenv_meta);
  ARG_CHECK(e.empty(), w + ": lenv metadata: " + e);
  e = R.parse(renv_meta);
  ARG_CHECK(e.empty(), w + ": renv metadata: " + e);
  if (pbc) {
    e = Le.parse(ledge_meta);
    ARG_CHECK(e.empty(), w + ": ledge metadata: " + e);
    e = Re.parse(redge_meta);
    ARG_CHECK(e.empty(), w + ": redge metadata: " + e);
    ARG_CHECK(Le.nleg() >= l_num && Re.nleg() >= r_num, w + ": edge legs out of range");
  }
  ARG_CHECK(l_num >= 2 && l_num <= L.nleg() && r_num >= 1 && r_num <= R.nleg(),
            w + ": l_num/r_num out of range");
  std::vector<std::vector<int>> dim, sym;
  std::vector<MapRow> rr, lr, er, el;
  int64_t ds = 0, es = 0;
  e = step_maps(G, L, R, pbc ? &Le : nullptr, pbc ? &Re : nullptr, l_num, r_num, sector, dim,
                sym, rr, lr, ds, er, el, es);
  ARG_CHECK(e.empty(), w + ": " + e);
  info[0] = get_dimension(dim, sym);
  info[1] = ds;
  info[2] = (int64_t)rr.size();
  info[3] = (int64_t)lr.size();
  if (pbc) {
    info[4] = es;
    info[5] = (int64_t)er.size();
    info[6] = (int64_t)el.size();
  }
  if (!rmap || !lmap) return 0;
  ARG_CHECK(rmap_cap >= (int64_t)rr.size() && lmap_cap >= (int64_t)lr.size(),
            w + ": map buffer too small");
  put_rows(rr.data(), (int64_t)rr.size(), rmap);
  put_rows(lr.data(), (int64_t)lr.size(), lmap);
  if (pbc && remap && lemap) {
    ARG_CHECK(remap_cap >= (int64_t)er.size() && lemap_cap >= (int64_t)el.size(),
              w + ": map buffer too small");
    put_rows(er.data(), (int64_t)er.size(), remap);
    put_rows(el.data(), (int64_t)el.size(), lemap);
  }
  return 0;
}

int from_maps_common(dmrgx_ctx* c, int64_t n, int64_t d_store, const int* rmap, int n_rmap,
                     const void* renv_vals, const int64_t* renv_sizes, int n_renv_blocks,
                     const int* lmap, int n_lmap, const void* lenv_vals,
                     const int64_t* lenv_sizes, int n_lenv_blocks, bool pbc, int64_t e_store,
                     const int* remap, int n_remap, const void* redge_vals,
                     const int64_t* redge_sizes, int n_redge_blocks, const int* lemap,
                     int n_lemap, const void* ledge_vals, const int64_t* ledge_sizes,
                     int n_ledge_blocks, const char* who) {
  const std::string w = who;
  ARG_CHECK(c, "null context");
  ARG_CHECK(n >= 0 && d_store >= 0 && e_store >= 0, w + ": negative length");
  ARG_CHECK((n_rmap == 0 || rmap) && (n_lmap == 0 || lmap), w + ": null map");
  ARG_CHECK(n_rmap >= 0 && n_lmap >= 0 && n_renv_blocks >= 0 && n_lenv_blocks >= 0,
            w + ": negative count");
  ARG_CHECK(renv_vals && lenv_vals && renv_sizes && lenv_sizes,
            w + ": null environment arrays");
  std::vector<PairSrc> pairs(pbc ? 2 : 1);
  rows_of(rmap, n_rmap, pairs[0].rmap);
  rows_of(lmap, n_lmap, pairs[0].lmap);
  pairs[0].store = d_store;
  pairs[0].rvals = (const double*)renv_vals;
  pairs[0].lvals = (const double*)lenv_vals;
  ARG_CHECK(sized_pair(renv_sizes, n_renv_blocks, pairs[0].rsize, pairs[0].roff) &&
                sized_pair(lenv_sizes, n_lenv_blocks, pairs[0].lsize, pairs[0].loff),
            w + ": negative block size");
  if (pbc) {
    ARG_CHECK((n_remap == 0 || remap) && (n_lemap == 0 || lemap), w + ": null edge map");
    ARG_CHECK(n_remap >= 0 && n_lemap >= 0 && n_redge_blocks >= 0 && n_ledge_blocks >= 0,
              w + ": negative count");
    ARG_CHECK(redge_vals && ledge_vals && redge_sizes && ledge_sizes,
              w + ": null edge arrays");
    rows_of(remap, n_remap, pairs[1].rmap);
    rows_of(lemap, n_lemap, pairs[1].lmap);
    pairs[1].store = e_store;
    pairs[1].rvals = (const double*)redge_vals;
    pairs[1].lvals = (const double*)ledge_vals;
    ARG_CHECK(sized_pair(redge_sizes, n_redge_blocks, pairs[1].rsize, pairs[1].roff) &&
                  sized_pair(ledge_sizes, n_ledge_blocks, pairs[1].lsize, pairs[1].loff),
              w + ": negative block size");
  }
  c->n = n;
  c->psi_dim.clear();
  c->psi_sym.clear();
  return finalize_plan(c, pairs);
}
}  // namespace

int dmrgx_set_solver(dmrgx_ctx* c, int nev, int ncv, int predict) {
  ARG_CHECK(c, "null context");
  ARG_CHECK(nev >= 1 && nev <= 6, "set_solver: nev must be 1..6");
  ARG_CHECK(ncv == 0 || (ncv > nev && ncv <= 64), "set_solver: ncv must be 0 or nev < ncv <= 64");
  // a start vector close to the lowest eigenvector spans the other eigenvectors
  // only weakly: excited values can come out missing or wrong
  ARG_CHECK(!predict || nev == 1, "set_solver: prediction needs nev = 1");
  c->eig_nev = nev;
  c->eig_ncv = ncv;
  c->predict = predict != 0;
  return 0;
}

int dmrgx_set_boundary(dmrgx_ctx* c, int boundary) {
  ARG_CHECK(c, "null context");
  ARG_CHECK(boundary == DMRGX_BOUNDARY_OPEN || boundary == DMRGX_BOUNDARY_PERIODIC,
            "set_boundary: unknown boundary");
  c->boundary = boundary;
  return 0;
}

int dmrgx_plan_build(dmrgx_ctx* c, const int* lenv_meta, const void* lenv_vals,
                     const int* renv_meta, const void* renv_vals, int l_num, int r_num,
                     int sector, int group_n, int fermion) {
  return plan_build_common(c, lenv_meta, lenv_vals, renv_meta, renv_vals, nullptr, nullptr,
                           nullptr, nullptr, l_num, r_num, sector, group_n, fermion,
                           "plan_build");
}

int dmrgx_plan_build_pbc(dmrgx_ctx* c, const int* lenv_meta, const void* lenv_vals,
                         const int* renv_meta, const void* renv_vals, const int* ledge_meta,
                         const void* ledge_vals, const int* redge_meta, const void* redge_vals,
                         int l_num, int r_num, int sector, int group_n, int fermion) {
  ARG_CHECK(ledge_meta && redge_meta, "plan_build_pbc: null edge metadata");
  return plan_build_common(c, lenv_meta, lenv_vals, renv_meta, renv_vals, ledge_meta,
                           ledge_vals, redge_meta, redge_vals, l_num, r_num, sector, group_n,
                           fermion, "plan_build_pbc");
}

int dmrgx_build_maps(const int* lenv_meta, const int* renv_meta, int l_num, int r_num,
                     int sector, int group_n, int fermion, int64_t* info, int* rmap,
                     int64_t rmap_cap, int* lmap, int64_t lmap_cap) {
  return build_maps_common(lenv_meta, renv_meta, nullptr, nullptr, l_num, r_num, sector,
                           group_n, fermion, info, rmap, rmap_cap, lmap, lmap_cap, nullptr, 0,
                           nullptr, 0, "build_maps");
}

int dmrgx_build_maps_pbc(const int* lenv_meta, const int* renv_meta, const int* ledge_meta,
                         const int* redge_meta, int l_num, int r_num, int sector, int group_n,
                         int fermion, int64_t* info, int* rmap, int64_t rmap_cap, int* lmap,
                         int64_t lmap_cap, int* remap, int64_t remap_cap, int* lemap,
                         int64_t lemap_cap) {
  ARG_CHECK(ledge_meta && redge_meta, "build_maps_pbc: null edge metadata");
  return build_maps_common(lenv_meta, renv_meta, ledge_meta, redge_meta, l_num, r_num, sector,
                           group_n, fermion, info, rmap, rmap_cap, lmap, lmap_cap, remap,
                           remap_cap, lemap, lemap_cap, "build_maps_pbc");
}

int dmrgx_plan_from_maps(dmrgx_ctx* c, int64_t n, int64_t d_store, const int* rmap, int n_rmap,
                         const void* renv_vals, const int64_t* renv_sizes, int n_renv_blocks,
                         const int* lmap, int n_lmap, const void* lenv_vals,
                         const int64_t* lenv_sizes, int n_lenv_blocks) {
  return from_maps_common(c, n, d_store, rmap, n_rmap, renv_vals, renv_sizes, n_renv_blocks,
                          lmap, n_lmap, lenv_vals, lenv_sizes, n_lenv_blocks, false, 0, nullptr,
                          0, nullptr, nullptr, 0, nullptr, 0, nullptr, nullptr, 0,
                          "plan_from_maps");
}

int dmrgx_plan_from_maps_pbc(dmrgx_ctx* c, int64_t n, int64_t d_store, const int* rmap,
                             int n_rmap, const void* renv_vals, const int64_t* renv_sizes,
                             int n_renv_blocks, const int* lmap, int n_lmap,
                             const void* lenv_vals, const int64_t* lenv_sizes, int n_lenv_blocks,
                             int64_t e_store, const int* remap, int n_remap,
                             const void* redge_vals, const int64_t* redge_sizes,
                             int n_redge_blocks, const int* lemap, int n_lemap,
                             const void* ledge_vals, const int64_t* ledge_sizes,
                             int n_ledge_blocks) {
  return from_maps_common(c, n, d_store, rmap, n_rmap, renv_vals, renv_sizes, n_renv_blocks,
                          lmap, n_lmap, lenv_vals, lenv_sizes, n_lenv_blocks, true, e_store,
                          remap, n_remap, redge_vals, redge_sizes, n_redge_blocks, lemap,
                          n_lemap, ledge_vals, ledge_sizes, n_ledge_blocks,
                          "plan_from_maps_pbc");
}

int dmrgx_plan_info(dmrgx_ctx* c, int64_t* out) {
  ARG_CHECK(c && out, "null argument");
  if (!c->has_plan) {
    set_error("plan_info: no plan");
    return DMRGX_E_STATE;
  }
  out[0] = c->n;
  out[1] = c->d_store_main;
  out[2] = c->n_rmap_main;
  out[3] = c->n_lmap_main;
  out[4] = c->flops;
  out[5] = (int64_t)c->psi_sym.size();
  out[6] = c->n_store_blocks;
  return 0;
}

int dmrgx_plan_edge_info(dmrgx_ctx* c, int64_t* out) {
  ARG_CHECK(c && out, "null argument");
  if (!c->has_plan) {
    set_error("plan_edge_info: no plan");
    return DMRGX_E_STATE;
  }
  out[0] = c->d_store - c->d_store_main;
  out[1] = (int64_t)c->rmap.size() - c->n_rmap_main;
  out[2] = (int64_t)c->lmap.size() - c->n_lmap_main;
  return 0;
}

int dmrgx_plan_maps(dmrgx_ctx* c, int* rmap, int* lmap) {
  ARG_CHECK(c && rmap && lmap, "null argument");
  if (!c->has_plan) {
    set_error("plan_maps: no plan");
    return DMRGX_E_STATE;
  }
  put_rows(c->rmap.data(), c->n_rmap_main, rmap);
  put_rows(c->lmap.data(), c->n_lmap_main, lmap);
  return 0;
}

int dmrgx_plan_edge_maps(dmrgx_ctx* c, int* remap, int* lemap) {
  ARG_CHECK(c && remap && lemap, "null argument");
  if (!c->has_plan) {
    set_error("plan_edge_maps: no plan");
    return DMRGX_E_STATE;
  }
  // undo the merge shifts: edge rows against the edge pair's own blocks and store
  std::vector<MapRow> er(c->rmap.begin() + c->n_rmap_main, c->rmap.end());
  std::vector<MapRow> el(c->lmap.begin() + c->n_lmap_main, c->lmap.end());
  for (auto& r : er) {
    r.blk -= c->r_blocks_main;
    r.out_beg -= c->d_store_main;
  }
  for (auto& r : el) {
    r.blk -= c->l_blocks_main;
    r.in_beg -= c->d_store_main;
  }
  put_rows(er.data(), (int64_t)er.size(), remap);
  put_rows(el.data(), (int64_t)el.size(), lemap);
  return 0;
}

int dmrgx_plan_psi_layout(dmrgx_ctx* c, int* out, int64_t cap) {
  ARG_CHECK(c && out, "null argument");
  const auto& d = c->psi_dim;
  const auto& s = c->psi_sym;
  int64_t need = 2 + (int64_t)d.size() + (int64_t)s.size() * (int64_t)d.size();
  for (auto& x : d) need += (int64_t)x.size();
  ARG_CHECK(cap >= need, "plan_psi_layout: buffer too small");
  int64_t k = 0;
  out[k++] = (int)d.size();
  out[k++] = (int)s.size();
  for (auto& x : d) out[k++] = (int)x.size();
  for (auto& x : d)
    for (int v : x) out[k++] = v;
  for (auto& b : s)
    for (int v : b) out[k++] = v;
  return 0;
}

int dmrgx_av(dmrgx_ctx* c, const void* in, void* out, int mem) {
  ARG_CHECK(c, "null context");
  ARG_CHECK(in && out, "av: null vector");
  if (!c->has_plan) {
    set_error("av: no plan");
    return DMRGX_E_STATE;
  }
  CUDA_TRY(cudaSetDevice(c->device));
  const size_t bytes = sizeof(double) * (size_t)c->n * c->f();
  if (mem == DMRGX_MEM_DEVICE) return run_matvec(c, (const double*)in, (double*)out);
  ARG_CHECK(mem == DMRGX_MEM_HOST, "av: mem must be DMRGX_MEM_HOST or DMRGX_MEM_DEVICE");
  // host arrays: the driver stages pageable copies itself (pipelined), which
  // beats a serial memcpy through our own pinned buffers
  CUDA_TRY(cudaMemcpyAsync(c->din.p, in, bytes, cudaMemcpyHostToDevice, c->stream));
  int rc = run_matvec(c, (const double*)c->din.p, (double*)c->dout.p);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(out, c->dout.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return check_device_error(c);
}

int dmrgx_profile(dmrgx_ctx* c, int enable) {
  ARG_CHECK(c, "null context");
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
  c->prof_ev.clear();
  c->prof = enable != 0;
  return 0;
}

int dmrgx_profile_read(dmrgx_ctx* c, double* out, int cap) {
  ARG_CHECK(c && out && cap >= 4, "profile_read: need a context and 4 output slots");
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < cap; i++) out[i] = 0.0;
  const size_t n = c->prof_ev.size() / 4;
  for (size_t m = 0; m < n; m++) {
    for (int k = 0; k < 3; k++) {
      float ms = 0.f;
      CUDA_TRY(cudaEventElapsedTime(&ms, c->prof_ev[4 * m + k], c->prof_ev[4 * m + k + 1]));
      out[1 + k] += ms;
    }
  }
  out[0] = (double)n;
  return 0;
}

void* dmrgx_stream(dmrgx_ctx* c) { return c ? (void*)c->stream : nullptr; }

int dmrgx_sync(dmrgx_ctx* c) {
  ARG_CHECK(c, "null context");
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return check_device_error(c);
}

}  // extern "C"
