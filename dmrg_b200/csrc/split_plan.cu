// Split-precision form of a matvec plan, derived from the FP64 plan of the same
// context: (hi, lo) operand images in the pair layout of split.h, one TMA tensor
// map per operand block, and K-split work units for the warp-specialized tcgen05
// kernel (tc_gemm.cu).
//
// Stage 1 (store = renv (x) psi):
//   A1 = renv blocks, M1 x K1 -> pair rows of kq = K1 rounded up to a k-tile
//   B1 = psi blocks as stage 1 views them, N1 x K1 -> pair rows, split every matvec
//   C1 = the intermediate, M1 x N1, written by the epilogue as (hi, lo) pairs
// Stage 2 (out = lenv (x) store):
//   the intermediate block (M1 x N1) is read as N2 x (D x N1p) with D = M1 / N2
//   (its rows are the stage-2 rows times the MPO channel, src/core.cpp:188-192);
//   N1p = N1 rounded up to 16 bytes, each stage-2 row one pair row of
//   kq2 = D x N1p rounded up to a k-tile
//   A2 = lenv blocks M2 x (D x N1) -> pair rows of kq2, zeros in each slice's padding
//   C2 = packed FP64 psi.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <functional>
#include <map>
#include <mutex>
#include <string>

#include "../../include/dmrgx.h"
#include "ctx.h"
#include "devmem.h"
#include "split.h"

namespace dmrgx {

double wall_now();  // steady-clock seconds (ctx.cu)

void SplitStage::free_device() {
  for (void* p : {(void*)d_outs, (void*)d_segs, (void*)d_units, (void*)d_cta_begin, (void*)d_reds,
                  (void*)d_redblk, (void*)d_maps})
    dfree(p, st);
  d_outs = nullptr;
  d_segs = nullptr;
  d_units = nullptr;
  d_cta_begin = nullptr;
  d_reds = nullptr;
  d_redblk = nullptr;
  d_maps = nullptr;
}

void SplitPlan::free_device() {
  s1.free_device();
  s2.free_device();
  dfree(d_psi_jobs, s1.st);
  dfree(d_psi_rows, s1.st);
  d_psi_jobs = nullptr;
  d_psi_rows = nullptr;
}

namespace {

#define SP_TRY(expr)                                                                   \
  do {                                                                                 \
    cudaError_t e_ = (expr);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      set_error(std::string("split plan: ") + #expr + ": " + cudaGetErrorString(e_));  \
      return DMRGX_E_CUDA;                                                             \
    }                                                                                  \
  } while (0)

int64_t rup(int64_t x, int64_t p) { return (x + p - 1) / p * p; }

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  // resolved once, thread-safe (function-local static)
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return (PFN_cuTensorMapEncodeTiled_v12000)p;
    return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
  }();
  return fn;
}

// Tensor map of one pair-layout block: dims (2 kq elements, rows), box (one
// 128-byte chunk per row, box_rows), 128-byte swizzle.
bool make_map(CUtensorMap* m, int eb, void* base, int64_t kq, int64_t rows, int box_rows,
              std::string& why) {
  auto fn = encode_fn();
  if (!fn) {
    why = "cuTensorMapEncodeTiled is not available from the driver";
    return false;
  }
  const cuuint64_t dims[2] = {(cuuint64_t)(2 * kq), (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)(2 * kq * eb)};
  const cuuint32_t box[2] = {(cuuint32_t)(tc_ktile_bytes() / eb), (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1, 1};
  CUresult r = fn(m, eb == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                  2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    why = "cuTensorMapEncodeTiled failed (code " + std::to_string((int)r) + ")";
    return false;
  }
  return true;
}

// Tile width (columns of one work unit) of an output block with n columns for a
// kernel whose widest tile is tn: the fewest tiles that cover n, of equal width
// rounded up to 16; `halve` cuts a block that fits one tile into two when it is
// wider than 64 (more, smaller units).
int tile_width(int n, int tn, bool halve) {
  int k = (int)((n + tn - 1) / tn);
  if (halve && k == 1 && n > 64) k = 2;
  k = std::max(k, 1);
  return (int)std::min<int64_t>(tn, rup((n + k - 1) / k, 16));
}

// Work units of one stage and their assignment to CTAs.
// Cost of a unit (SM clock cycles, rough): the larger of its MMA issue time
// (6 MMAs of N/2 cycles per k-tile) and its operand bytes at ~48 B/cycle, plus a
// fixed 800.  Tiles costlier than cap_scale x half the mean CTA load are cut
// along K (partials + fixed-order reduction).  Units go to CTAs longest-first
// onto the least-loaded CTA.
void make_units(SplitStage& st, int num_sms, double cap_scale) {
  const int TM = tc_tile_m();
  const int A_B = TM * tc_ktile_bytes();
  struct T { int out, tm, tn, kt; double per_kt; };
  std::vector<T> tiles;
  double total = 0;
  for (size_t o = 0; o < st.outs.size(); o++) {
    const SOut& so = st.outs[o];
    int kt = 0;
    for (int q = 0; q < so.seg_count; q++) kt += st.segs[so.seg_begin + q].nkt;
    const int brows = so.seg_count ? st.segs[so.seg_begin].brows : so.tnw;
    const int tm = (so.m + TM - 1) / TM, tn = (so.n + so.tnw - 1) / so.tnw;
    for (int a = 0; a < tm; a++)
      for (int b = 0; b < tn; b++) {
        const int ncols = std::min(so.tnw, so.n - b * so.tnw);
        const int nmma = (int)rup(ncols, 16);
        const double per = std::max(3.0 * nmma, (A_B + 1.0 * brows * tc_ktile_bytes()) / 48.0);
        tiles.push_back({(int)o, a, b, kt, per});
        total += kt * per + 800;
      }
  }
  const double cap = cap_scale * std::max(4000.0, 0.5 * total / std::max(1, num_sms));
  struct U { double cost; SUnit u; };
  std::vector<U> us;
  st.reds.clear();
  st.redblk.clear();
  int slot = 0;
  for (auto& t : tiles) {
    const double c = t.kt * t.per_kt;
    int parts = 1;
    if (c > cap && t.kt > 1) parts = (int)std::min<double>(t.kt, std::ceil(c / cap));
    if (parts > 1) {
      SRed r;
      r.out = t.out;
      r.tm = (int16_t)t.tm;
      r.tn = (int16_t)t.tn;
      r.slot0 = slot;
      r.nslots = parts;
      const int rows = std::min(TM, st.outs[t.out].m - t.tm * TM);
      for (int r0 = 0; r0 < rows; r0 += 4) st.redblk.push_back(SRedBlk{(int)st.reds.size(), r0});
      st.reds.push_back(r);
    }
    for (int p = 0; p < parts; p++) {
      SUnit u;
      u.out = t.out;
      u.tm = (int16_t)t.tm;
      u.tn = (int16_t)t.tn;
      u.kt0 = (int)((int64_t)t.kt * p / parts);
      u.kt1 = (int)((int64_t)t.kt * (p + 1) / parts);
      u.slot = parts > 1 ? slot++ : -1;
      u.pad_ = 0;
      us.push_back({(u.kt1 - u.kt0) * t.per_kt + 800, u});
    }
  }
  std::stable_sort(us.begin(), us.end(), [](const U& x, const U& y) { return x.cost > y.cost; });
  const int nctas = (int)std::min<size_t>(num_sms, us.size());
  std::vector<std::vector<SUnit>> per(nctas);
  std::vector<double> load(nctas, 0.0);
  for (auto& x : us) {
    int best = 0;
    for (int c = 1; c < nctas; c++)
      if (load[c] < load[best]) best = c;
    load[best] += x.cost;
    per[best].push_back(x.u);
  }
  st.units.clear();
  st.cta_begin.assign(1, 0);
  for (int c = 0; c < nctas; c++) {
    st.units.insert(st.units.end(), per[c].begin(), per[c].end());
    st.cta_begin.push_back((int)st.units.size());
  }
  st.nslots = slot;
}

template <class V, class P>
int upload_vec(const std::vector<V>& v, P*& d, cudaStream_t s) {
  dfree(d, s);
  d = nullptr;
  SP_TRY(dalloc(&d, v.size(), s));
  if (!v.empty()) SP_TRY(cudaMemcpyAsync(d, v.data(), sizeof(V) * v.size(), cudaMemcpyHostToDevice, s));
  return 0;
}

int upload(SplitStage& st, cudaStream_t s) {
  st.st = s;
  int rc = upload_vec(st.outs, st.d_outs, s);
  if (!rc) rc = upload_vec(st.segs, st.d_segs, s);
  if (!rc) rc = upload_vec(st.units, st.d_units, s);
  if (!rc) rc = upload_vec(st.cta_begin, st.d_cta_begin, s);
  if (!rc) rc = upload_vec(st.reds, st.d_reds, s);
  if (!rc) rc = upload_vec(st.redblk, st.d_redblk, s);
  if (!rc) rc = upload_vec(st.maps, st.d_maps, s);
  return rc;
}

std::vector<PadRow> rows_of(const std::vector<PadJob>& jobs) {
  std::vector<PadRow> r;
  for (size_t j = 0; j < jobs.size(); j++)
    for (int i = 0; i < jobs[j].rows; i++) r.push_back(PadRow{(int)j, i});
  return r;
}

int run_jobs(int eb, const double* src, void* dst, const std::vector<PadJob>& jobs,
             cudaStream_t s) {
  if (jobs.empty()) return 0;
  PadJob* d = nullptr;
  PadRow* dr = nullptr;
  const std::vector<PadRow> rows = rows_of(jobs);
  SP_TRY(dalloc(&d, jobs.size(), s));
  SP_TRY(dalloc(&dr, rows.size(), s));
  SP_TRY(cudaMemcpyAsync(d, jobs.data(), sizeof(PadJob) * jobs.size(), cudaMemcpyHostToDevice, s));
  if (!rows.empty())
    SP_TRY(cudaMemcpyAsync(dr, rows.data(), sizeof(PadRow) * rows.size(), cudaMemcpyHostToDevice, s));
  SP_TRY(launch_pad_split(eb, src, dst, d, dr, (int)rows.size(), s));
  dfree(d, s);
  dfree(dr, s);
  return 0;
}

}  // namespace

// Apply one tiling to a stage: tile widths, B-box rows, tensor maps, work units,
// workspace; uploads the descriptors.
int configure_stage(dmrgx_ctx* c, SplitStage& st, int cfg, bool halve, double cap_scale) {
  const int tn = tc_cfg_tn(cfg);
  st.cfg = cfg;
  st.halve = halve;
  st.cap_scale = cap_scale;
  for (auto& o : st.outs) o.tnw = tile_width(o.n, tn, halve);
  st.maps.resize(st.req.size());
  std::string why;
  for (size_t i = 0; i < st.req.size(); i++) {
    const auto& r = st.req[i];
    const int box = r.b_side ? tile_width((int)r.rows, tn, halve) : tc_tile_m();
    if (!make_map(&st.maps[i], c->sp.eb, r.base, r.kq, r.rows, box, why)) {
      set_error("split plan: " + why);
      return DMRGX_E_CUDA;
    }
  }
  for (auto& g : st.segs) {
    const auto& r = st.req[g.bmap];
    g.brows = tile_width((int)r.rows, tn, halve);
  }
  make_units(st, c->num_sms * tc_cfg_ctas_per_sm(cfg), cap_scale);
  const int slots = std::max(1, st.nslots);
  SP_TRY(c->sws.ensure((size_t)slots * tc_tile_m() * tc_tile_n() * sizeof(float)));
  return upload(st, c->stream);
}

namespace {

// Autotuner of the split stages.  Key: the stage's block-shape histogram (the
// multiset of output blocks' rows, columns and K-tile counts, rounded) and the
// element type.  On a miss every candidate tiling -- kernel configuration
// (tc_cfg_*: four tile-width / ring-depth / CTAs-per-SM choices), halving of
// one-tile blocks, K-split threshold x {1, 2, 4, none} -- is timed with CUDA events on the
// context's stream (best of three launches after one warm-up, on the plan's own
// buffers) and the fastest is kept for every later plan with the same histogram,
// and for plans of the same coarse class (stage_class).
struct TuneVal {
  int cfg;
  bool halve;
  double cap_scale;
};
std::map<uint64_t, TuneVal> g_tune;
std::mutex g_tune_mu;

uint64_t stage_key(const SplitStage& st, int eb, int which) {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&h](uint64_t v) { h ^= v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2); };
  mix((uint64_t)eb);
  mix((uint64_t)which);
  // shapes rounded (rows and columns to 64, K-tiles to 4) and sorted, so plans whose
  // sector sizes differ a little share one entry
  std::vector<uint64_t> shp;
  for (const auto& o : st.outs) {
    int kt = 0;
    for (int q = 0; q < o.seg_count; q++) kt += st.segs[o.seg_begin + q].nkt;
    shp.push_back(((uint64_t)rup(o.m, 64) << 40) | ((uint64_t)rup(o.n, 64) << 20) |
                  (uint64_t)rup(kt, 4));
  }
  std::sort(shp.begin(), shp.end());
  for (uint64_t v : shp) mix(v);
  return h;
}

// Coarse class of a stage, for plans whose histograms differ but whose shape is
// alike (the same chain position a sweep later, a neighbouring site): the
// half-octave buckets of the number of 128-row output tiles, the total and the
// longest output's K-tile counts, and the widest output's column count rounded
// to 64.  A tuning measured for one plan of a class is reused for the others
// without timing them: along a sweep the exact histograms rarely repeat, and
// timing every candidate on every new one cost more than it saved.
uint64_t stage_class(const SplitStage& st, int eb, int which) {
  int64_t tiles = 0, totkt = 0, maxkt = 0, maxn = 0;
  for (const auto& o : st.outs) {
    int64_t kt = 0;
    for (int q = 0; q < o.seg_count; q++) kt += st.segs[o.seg_begin + q].nkt;
    tiles += (o.m + 127) / 128;
    totkt += kt;
    maxkt = std::max(maxkt, kt);
    maxn = std::max<int64_t>(maxn, o.n);
  }
  auto hb = [](int64_t x) {
    return (uint64_t)std::lround(2.0 * std::log2((double)std::max<int64_t>(x, 1)));
  };
  return (uint64_t)eb | ((uint64_t)which << 4) | (hb(tiles) << 8) | (hb(totkt) << 16) |
         (hb(maxkt) << 24) | ((uint64_t)rup((int)maxn, 64) << 32);
}
std::map<uint64_t, TuneVal> g_tune_class;

int launch_stage(dmrgx_ctx* c, int which) {
  SplitPlan& sp = c->sp;
  SplitStage& st = which == 1 ? sp.s1 : sp.s2;
  uint8_t* stb = (uint8_t*)c->sstore.p;
  SP_TRY(launch_tc_gemm(sp.eb, which == 1, st.cfg, st.d_maps, st.d_units, st.d_cta_begin,
                        (int)st.cta_begin.size() - 1, st.d_outs, st.d_segs,
                        which == 1 ? stb : nullptr, which == 1 ? nullptr : (double*)c->dout.p,
                        (float*)c->sws.p, st.d_reds, st.d_redblk, (int)st.redblk.size(),
                        (int*)c->err.p, c->stream));
  return 0;
}

}  // namespace

constexpr double kTuneMinFlops = 2e8;  // useful flops of a stage worth tuning

int tune_stage(dmrgx_ctx* c, int which) {
  SplitPlan& sp = c->sp;
  SplitStage& st = which == 1 ? sp.s1 : sp.s2;
  const bool def_halve = which == 1;
  const char* env = getenv("DMRGX_TUNE");
  if (env && env[0] == '0') {
    st.tuned = false;
    return configure_stage(c, st, 0, def_halve, 1.0);
  }
  const uint64_t key = stage_key(st, sp.eb, which);
  const uint64_t cls = stage_class(st, sp.eb, which);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it == g_tune.end()) {
      auto ic = g_tune_class.find(cls);
      if (ic != g_tune_class.end()) it = g_tune.emplace(key, ic->second).first;
    }
    if (it != g_tune.end()) {
      st.tuned = false;
      return configure_stage(c, st, it->second.cfg, it->second.halve, it->second.cap_scale);
    }
  }
  // a stage this small runs in a few microseconds whatever the tiling: measuring
  // 18 tilings would cost more than it could save (the small-bond steps near
  // the chain ends), so it keeps the default
  {
    const Stage& fs = which == 1 ? c->st1 : c->st2;
    double fl = 0;
    for (const PlainRow& r : fs.rows) fl += 2.0 * r.M * r.N * r.K;
    if (fl < kTuneMinFlops) {
      st.tuned = false;
      return configure_stage(c, st, 0, def_halve, 1.0);
    }
  }
  cudaEvent_t e0, e1;
  SP_TRY(cudaEventCreate(&e0));
  SP_TRY(cudaEventCreate(&e1));
  TuneVal best{0, def_halve, 1.0};
  float best_ms = 1e30f;
  int rc = 0;
  auto trial = [&](int cfg, bool hv, double cs) {
    rc = configure_stage(c, st, cfg, hv, cs);
    if (rc) return;
    rc = launch_stage(c, which);  // warm-up
    float ms = 1e30f;
    for (int r = 0; r < 2 && !rc; r++) {
      cudaEventRecord(e0, c->stream);
      rc = launch_stage(c, which);
      cudaEventRecord(e1, c->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) rc = DMRGX_E_CUDA;
      float t = 0;
      cudaEventElapsedTime(&t, e0, e1);
      ms = std::min(ms, t);
    }
    if (!rc && ms < best_ms) {
      best_ms = ms;
      best = TuneVal{cfg, hv, cs};
    }
  };
  // every configuration and halving with the K-split threshold at its default
  // and off (1e9), then the other thresholds for the best of those
  for (int cfg = 0; cfg < tc_configs() && !rc; cfg++)
    for (int hv = 0; hv < 2 && !rc; hv++)
      for (double cs : {1.0, 1e9})
        if (!rc) trial(cfg, hv != 0, cs);
  const TuneVal b1 = best;
  for (double cs : {2.0, 4.0})
    if (!rc) trial(b1.cfg, b1.halve, cs);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  int h = 0;
  SP_TRY(cudaMemcpyAsync(&h, c->err.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  SP_TRY(cudaStreamSynchronize(c->stream));
  if (h) {
    set_error("split plan: a bounded device wait timed out while tuning");
    return DMRGX_E_TIMEOUT;
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = best;
    g_tune_class[cls] = best;
  }
  rc = configure_stage(c, st, best.cfg, best.halve, best.cap_scale);
  st.tuned = true;
  return rc;
}

int build_split_plan(dmrgx_ctx* c, int eb) {
  const double t0 = wall_now();
  SplitPlan& sp = c->sp;
  sp.free_device();
  sp = SplitPlan();
  const int f = c->f();  // complex data: real view of A, expanded B (split.h)
  const int64_t P = 16 / eb;   // padding of stage-1 output rows (16 bytes)
  const int64_t CH = 64 / eb;  // elements per half-chunk of the pair layout = per k-tile
  const Stage& f1 = c->st1;
  const Stage& f2 = c->st2;
  struct MapReq { int which; int64_t off, kq, rows; int box_rows; };  // which: 0 a1,1 psi,2 a2,3 store
  std::vector<MapReq> req1, req2;

  // MPO channels per stage-1 output block: stage 2 reads a store block
  // [D*N2 x N1] as [N2 x D*N1]
  std::map<int64_t, std::pair<int, int>> st_shape;  // FP64 store offset -> (M1, N1)
  for (size_t o = 0; o < f1.outs.size(); o++) st_shape[f1.outs[o].c_off] = {f1.outs[o].m, f1.outs[o].n};
  std::map<int64_t, int> st_grp;
  for (size_t o = 0; o < f2.outs.size(); o++) {
    const DOut& d = f2.outs[o];
    for (int q = 0; q < d.seg_count; q++) {
      const DSeg& g = f2.segs[d.seg_begin + q];
      auto is = st_shape.find(g.b_off);
      if (is == st_shape.end()) {
        set_error("split plan: a stage-2 task reads no stage-1 output block");
        return DMRGX_E_ARG;
      }
      const int M1 = is->second.first, N1 = is->second.second;
      if (N1 <= 0 || g.k % N1 != 0 || (int64_t)(g.k / N1) * (d.n / f) != M1) {
        set_error("split plan: stage-2 K does not factor as channels x stage-1 columns");
        return DMRGX_E_ARG;
      }
      auto ig = st_grp.find(g.b_off);
      if (ig != st_grp.end() && ig->second != g.k / N1) {
        set_error("split plan: a store block is read with two channel counts");
        return DMRGX_E_ARG;
      }
      st_grp[g.b_off] = g.k / N1;
    }
  }

  // ---- stage 1 layout
  std::map<int64_t, int> a1_map, psi_map;
  std::map<int64_t, int64_t> st_off, st_kq;
  std::vector<PadJob> a1_jobs;
  int64_t a1_len = 0, psi_len = 0, st_len = 0;
  for (size_t o = 0; o < f1.outs.size(); o++) {
    const DOut& d = f1.outs[o];
    SOut so;
    auto ig = st_grp.find(d.c_off);
    const int D = ig == st_grp.end() ? 1 : ig->second;
    if (d.m % D) {
      set_error("split plan: stage-1 rows are not a multiple of the channel count");
      return DMRGX_E_ARG;
    }
    const int64_t n1p = rup(d.n, P), kq2 = rup(D * n1p, CH);
    if (st_off.find(d.c_off) == st_off.end()) {
      st_off[d.c_off] = st_len;
      st_kq[d.c_off] = kq2;
      st_len += (int64_t)f * (d.m / D) * 2 * kq2;  // complex: two expanded rows each
    }
    so.c_off = st_off[d.c_off];
    so.m = d.m;
    so.n = d.n;
    so.ldc = (int32_t)n1p;
    so.grp = D;
    so.cplx = f == 2 ? 1 : 0;
    so.rstride = (int32_t)(2 * kq2);
    so.seg_begin = (int32_t)sp.s1.segs.size();
    so.seg_count = d.seg_count;
    so.tnw = 0;  // set by configure_stage
    for (int q = 0; q < d.seg_count; q++) {
      const DSeg& g = f1.segs[d.seg_begin + q];
      const int64_t kq = rup(g.k, CH);
      SSeg2 ss;
      auto ia = a1_map.find(g.a_off);
      if (ia == a1_map.end()) {
        a1_jobs.push_back(PadJob{g.a_off, a1_len, d.m, 1, g.k, g.k, (int32_t)kq, 0});
        a1_map[g.a_off] = (int)req1.size();
        req1.push_back({0, a1_len, kq, d.m, 128});
        a1_len += (int64_t)d.m * 2 * kq;
      }
      ss.amap = a1_map[g.a_off];
      auto ib = psi_map.find(g.b_off);
      if (ib == psi_map.end()) {
        sp.psi_jobs.push_back(
            PadJob{g.b_off, psi_len, d.n / f, 1, g.k, g.k, (int32_t)kq, f == 2 ? 1 : 0});
        psi_map[g.b_off] = (int)req1.size();
        req1.push_back({1, psi_len, kq, d.n, 0});
        psi_len += (int64_t)d.n * 2 * kq;
      }
      ss.bmap = psi_map[g.b_off];
      ss.nkt = (int32_t)(kq / CH);
      ss.brows = 0;  // set by configure_stage
      sp.s1.segs.push_back(ss);
    }
    sp.s1.outs.push_back(so);
  }
  sp.s1.full_cover = f1.full_cover;

  // ---- stage 2 layout
  std::map<int64_t, int> a2_map, stb_map;
  std::vector<PadJob> a2_jobs;
  int64_t a2_len = 0;
  for (size_t o = 0; o < f2.outs.size(); o++) {
    const DOut& d = f2.outs[o];
    SOut so;
    so.c_off = d.c_off;
    so.m = d.m;
    so.n = d.n;
    so.ldc = d.n;
    so.grp = 1;
    so.rstride = 0;
    so.cplx = 0;
    so.seg_begin = (int32_t)sp.s2.segs.size();
    so.seg_count = d.seg_count;
    so.tnw = 0;
    for (int q = 0; q < d.seg_count; q++) {
      const DSeg& g = f2.segs[d.seg_begin + q];
      const int N1 = st_shape[g.b_off].second;
      const int D = g.k / N1;
      const int64_t n1p = rup(N1, P), kq2 = st_kq[g.b_off];
      SSeg2 ss;
      auto ia = a2_map.find(g.a_off);
      if (ia == a2_map.end()) {
        a2_jobs.push_back(PadJob{g.a_off, a2_len, d.m, D, N1, (int32_t)n1p, (int32_t)kq2, 0});
        a2_map[g.a_off] = (int)req2.size();
        req2.push_back({2, a2_len, kq2, d.m, 128});
        a2_len += (int64_t)d.m * 2 * kq2;
      }
      ss.amap = a2_map[g.a_off];
      auto ib = stb_map.find(g.b_off);
      if (ib == stb_map.end()) {
        stb_map[g.b_off] = (int)req2.size();
        req2.push_back({3, st_off[g.b_off], kq2, d.n, 0});
      }
      ss.bmap = stb_map[g.b_off];
      ss.nkt = (int32_t)(kq2 / CH);
      ss.brows = 0;
      sp.s2.segs.push_back(ss);
    }
    sp.s2.outs.push_back(so);
  }
  sp.s2.full_cover = f2.full_cover;
  auto len = [eb](int64_t n) { return rup(std::max<int64_t>(n, 1), 256 / eb); };
  sp.a1_len = len(a1_len);
  sp.a2_len = len(a2_len);
  sp.psi_len = len(psi_len);
  sp.store_len = len(st_len);
  sp.psi_rows = rows_of(sp.psi_jobs);

  // ---- device buffers and images
  cudaStream_t s = c->stream;
  SP_TRY(c->sa1.ensure(sp.a1_len * eb));
  SP_TRY(c->sa2.ensure(sp.a2_len * eb));
  SP_TRY(c->spsi.ensure(sp.psi_len * eb));
  SP_TRY(c->sstore.ensure(sp.store_len * eb));
  SP_TRY(prepare_tc_gemm());
  SP_TRY(c->err.ensure(16));
  SP_TRY(cudaMemsetAsync(c->sa1.p, 0, sp.a1_len * eb, s));
  SP_TRY(cudaMemsetAsync(c->sa2.p, 0, sp.a2_len * eb, s));
  SP_TRY(cudaMemsetAsync(c->spsi.p, 0, sp.psi_len * eb, s));
  SP_TRY(cudaMemsetAsync(c->sstore.p, 0, sp.store_len * eb, s));
  SP_TRY(cudaMemsetAsync(c->err.p, 0, 16, s));
  uint8_t* a1 = (uint8_t*)c->sa1.p;
  uint8_t* a2 = (uint8_t*)c->sa2.p;
  uint8_t* psi = (uint8_t*)c->spsi.p;
  uint8_t* stb = (uint8_t*)c->sstore.p;
  int rc = run_jobs(eb, (const double*)c->renv.p, a1, a1_jobs, s);
  if (rc) return rc;
  rc = run_jobs(eb, (const double*)c->lenv.p, a2, a2_jobs, s);
  if (rc) return rc;
  // images complete before the tuner's timed launches
  SP_TRY(cudaStreamSynchronize(s));
  // ---- operand blocks of the tensor maps
  auto to_req = [&](const std::vector<MapReq>& req, SplitStage& st) {
    st.req.clear();
    for (const MapReq& r : req) {
      uint8_t* base = r.which == 0 ? a1 : r.which == 1 ? psi : r.which == 2 ? a2 : stb;
      st.req.push_back({base + r.off * eb, r.kq, r.rows, r.which == 1 || r.which == 3});
    }
  };
  to_req(req1, sp.s1);
  to_req(req2, sp.s2);
  sp.eb = eb;
  rc = upload_vec(sp.psi_jobs, sp.d_psi_jobs, s);
  if (!rc) rc = upload_vec(sp.psi_rows, sp.d_psi_rows, s);
  SP_TRY(cudaStreamSynchronize(s));
  const double t1 = wall_now();
  if (!rc) rc = tune_stage(c, 1);
  if (!rc) rc = tune_stage(c, 2);
  if (rc) return rc;
  SP_TRY(cudaStreamSynchronize(s));
  c->t_plan_part[2] += t1 - t0;
  c->t_plan_part[3] += wall_now() - t1;
  return 0;
}

int run_matvec_split(dmrgx_ctx* c, const double* in, double* out) {
  SplitPlan& sp = c->sp;
  cudaStream_t s = c->stream;
  const int eb = sp.eb;
  uint8_t* psi = (uint8_t*)c->spsi.p;
  uint8_t* stb = (uint8_t*)c->sstore.p;
  c->prof_mark();
  SP_TRY(launch_pad_split(eb, in, psi, sp.d_psi_jobs, sp.d_psi_rows, (int)sp.psi_rows.size(),
                          s));
  c->prof_mark();
  SP_TRY(launch_tc_gemm(eb, true, sp.s1.cfg, sp.s1.d_maps, sp.s1.d_units, sp.s1.d_cta_begin,
                        (int)sp.s1.cta_begin.size() - 1, sp.s1.d_outs, sp.s1.d_segs, stb, nullptr,
                        (float*)c->sws.p, sp.s1.d_reds, sp.s1.d_redblk,
                        (int)sp.s1.redblk.size(), (int*)c->err.p, s));
  c->prof_mark();
  if (!sp.s2.full_cover) SP_TRY(cudaMemsetAsync(out, 0, sizeof(double) * c->n, s));
  SP_TRY(launch_tc_gemm(eb, false, sp.s2.cfg, sp.s2.d_maps, sp.s2.d_units, sp.s2.d_cta_begin,
                        (int)sp.s2.cta_begin.size() - 1, sp.s2.d_outs, sp.s2.d_segs, nullptr,
                        out, (float*)c->sws.p, sp.s2.d_reds, sp.s2.d_redblk,
                        (int)sp.s2.redblk.size(), (int*)c->err.p, s));
  c->prof_mark();
  return 0;
}

}  // namespace dmrgx
