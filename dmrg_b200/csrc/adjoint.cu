// Adjoint of the two-site effective-Hamiltonian contraction.
//
// The matvec of the site step (src/core.cpp:22-31) runs two batches of block
// GEMMs from the task lists of qtensor::get_map (src/qtensor.cpp:997-1119):
//   stage 1  store[out] += alpha Rop_blk[M1 x K1] psi[in: N1 x K1]^T
//   stage 2  out[out]   += alpha Lop_blk[M2 x K2] store[in: N2 x K2]^T
// and E = <psi, out> is linear in each operator, so
//   dE/dLop_blk = sum_rows alpha conj(psi_out)[M2 x N2] store[N2 x K2]
//   dE/dstore   = sum_rows alpha conj(psi_out)^T[N2 x M2] Lop_blk[M2 x K2]
//   dE/dRop_blk = sum_rows alpha dstore_out[M1 x N1] psi[N1 x K1].
// Each is one grouped NT GEMM on the FP64 DMMA kernel (gemm_f64.cu) over
// operand copies that a gather kernel transposes, conjugates and signs.
//
// The fused operators are linear in the MPO tensor W with the reference's
// fermion sign per block pair (src/qtensor.cpp:930-968):
//   L~[x,s,b,y,s'] = sum_a sign env[x,a,y] W[a,s,b,s']          (src/core.cpp:188-189)
//   R~[s,x,a,s',y] = sum_b sign env[x,b,y] W[a,s,b,s']          (src/core.cpp:190-192)
// so dE/dW = sum_pairs sign sum_{x,y} env[x,.,y] dE/dfused[.,x,.,y,.], a
// reduction over the environment's bond indices run as the same grouped GEMM
// (one output per pair and slab of x, summed on the host in a fixed order).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>

#include "../../include/dmrgx.h"
#include "adjoint.h"
#include "devmem.h"
#include "kernels.h"

namespace dmrgx {
namespace {

GOut gout(int64_t dst_off, const std::vector<int64_t>& dims, const std::vector<int64_t>& dstr,
          int src_begin, int src_count) {
  GOut o;
  std::memset(&o, 0, sizeof(o));
  o.dst_off = dst_off;
  o.rank = (int)dims.size();
  o.size = 1;
  for (int k = 0; k < o.rank; k++) {
    o.dims[k] = (int32_t)dims[k];
    o.dst_strides[k] = dstr[k];
    o.size *= dims[k];
  }
  o.src_begin = src_begin;
  o.src_count = src_count;
  return o;
}

GSrc gsrc(int64_t off, const std::vector<int64_t>& strides, double sign, bool conj) {
  GSrc g;
  std::memset(&g, 0, sizeof(g));
  g.src_off = off;
  for (size_t k = 0; k < strides.size(); k++) g.strides[k] = strides[k];
  g.sign = sign;
  g.conj = conj ? 1 : 0;
  return g;
}

// scoped device array of doubles (stream-ordered)
struct DevArr {
  double* p = nullptr;
  cudaStream_t s = nullptr;
  explicit DevArr(cudaStream_t st) : s(st) {}
  cudaError_t alloc(int64_t n) { return dalloc(&p, (size_t)std::max<int64_t>(1, n), s); }
  ~DevArr() { dfree(p, s); }
};

int64_t label_key(const std::vector<int>& st, const std::vector<std::vector<int>>& dim) {
  int64_t loc = 0;
  for (size_t q = 0; q < dim.size(); q++) loc = loc * (int64_t)dim[q].size() + st[q];
  return loc;
}

// outputs in first-use order with their segment lists -> grouped descriptors
struct Grouper {
  std::vector<DOut> outs;
  std::vector<std::vector<DSeg>> per;
  std::map<int64_t, int> at;
  int out(int64_t key, int64_t c_off, int64_t m, int64_t n) {
    auto it = at.find(key);
    if (it != at.end()) return it->second;
    DOut o;
    o.c_off = c_off;
    o.m = (int32_t)m;
    o.n = (int32_t)n;
    o.seg_begin = 0;
    o.seg_count = 0;
    outs.push_back(o);
    per.emplace_back();
    at[key] = (int)outs.size() - 1;
    return (int)outs.size() - 1;
  }
  void seg(int o, int64_t a_off, int64_t b_off, int64_t k) {
    DSeg s;
    s.a_off = a_off;
    s.b_off = b_off;
    s.k = (int32_t)k;
    s.pad_ = 0;
    per[o].push_back(s);
  }
  void flatten(std::vector<DOut>& o, std::vector<DSeg>& s) {
    o = outs;
    s.clear();
    for (size_t i = 0; i < o.size(); i++) {
      o[i].seg_begin = (int32_t)s.size();
      o[i].seg_count = (int32_t)per[i].size();
      s.insert(s.end(), per[i].begin(), per[i].end());
    }
  }
};

// Host-side range checks of every descriptor before a launch (lengths in
// elements; f doubles per element).  A bookkeeping mistake becomes an error
// return, never an out-of-range device access.
bool gemm_in_range(const std::vector<DOut>& outs, const std::vector<DSeg>& segs, int64_t alen,
                   int64_t blen, int64_t clen, int f) {
  for (auto& o : outs) {
    if (o.m < 0 || o.n < 0 || o.n % f) return false;
    if (o.c_off < 0 || o.c_off + (int64_t)o.m * o.n > clen * f) return false;
    if (o.seg_begin < 0 || o.seg_begin + o.seg_count > (int)segs.size()) return false;
    for (int q = 0; q < o.seg_count; q++) {
      const DSeg& s = segs[o.seg_begin + q];
      if (s.k < 0 || s.k % f || s.a_off < 0 || s.b_off < 0) return false;
      if (s.a_off + (int64_t)o.m * s.k > alen * f) return false;
      if (s.b_off + (int64_t)(o.n / f) * s.k > blen * f) return false;
    }
  }
  return true;
}

bool gather_in_range(const std::vector<GOut>& go, const std::vector<GSrc>& gs, int64_t srclen,
                     int64_t dstlen) {
  for (auto& o : go) {
    if (o.rank < 1 || o.rank > 8 || o.src_begin < 0 || o.src_begin + o.src_count > (int)gs.size())
      return false;
    int64_t dmax = o.dst_off, cnt = 1;
    bool empty = false;
    for (int k = 0; k < o.rank; k++) {
      if (o.dims[k] <= 0) empty = true;
      dmax += (int64_t)(o.dims[k] - 1) * o.dst_strides[k];
      cnt *= o.dims[k];
    }
    if (empty) {
      if (o.size != 0) return false;
      continue;
    }
    if (cnt != o.size || o.dst_off < 0 || dmax >= dstlen) return false;
    for (int q = 0; q < o.src_count; q++) {
      const GSrc& g = gs[o.src_begin + q];
      int64_t smax = g.src_off;
      for (int k = 0; k < o.rank; k++) smax += (int64_t)(o.dims[k] - 1) * g.strides[k];
      if (g.src_off < 0 || smax >= srclen) return false;
    }
  }
  return true;
}

}  // namespace

int heff_adjoint(dmrgx_ctx* c, const Engine& E, const QTensor& Lop, const QTensor& Rop,
                 const double* psi, bool want_l, bool want_r, QTPtr& gl, QTPtr& gr,
                 double& energy, double& norm2, std::string& err) {
  const int f = c->f();
  const bool cplx = f == 2;
  const int64_t n = c->n;
  const cudaStream_t st = E.stream;
  DevArr out(st);
  if (out.alloc(n * f) != cudaSuccess) {
    err = "adjoint: allocation failed";
    return DMRGX_E_CUDA;
  }
  int rc = matvec_fp64(c, psi, out.p);  // leaves store = Rop (x) psi in c->store
  if (rc) {
    err = "adjoint: matvec failed";
    return rc;
  }
  {
    std::vector<double> hp((size_t)(n * f)), ho((size_t)(n * f));
    cudaMemcpyAsync(hp.data(), psi, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(ho.data(), out.p, sizeof(double) * ho.size(), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
      err = "adjoint: copy failed";
      return DMRGX_E_CUDA;
    }
    double er = 0, nn = 0;
    for (int64_t i = 0; i < n; i++) {
      if (cplx) {
        const double pr = hp[2 * i], pi = hp[2 * i + 1], orr = ho[2 * i], oi = ho[2 * i + 1];
        er += pr * orr + pi * oi;
        nn += pr * pr + pi * pi;
      } else {
        er += hp[i] * ho[i];
        nn += hp[i] * hp[i];
      }
    }
    norm2 = nn;
    energy = nn > 0 ? er / nn : 0.0;
  }
  const double* store = (const double*)c->store.p;
  cudaError_t e = cudaSuccess;

  // conj(psi) and -conj(psi): the A operand of dE/dLop carries alpha by choice of image
  DevArr cpsi(st);
  if (want_l) {
    if (cpsi.alloc(2 * n * f) != cudaSuccess) {
      err = "adjoint: allocation failed";
      return DMRGX_E_CUDA;
    }
    std::vector<GOut> go = {gout(0, {n}, {1}, 0, 1), gout(n, {n}, {1}, 1, 1)};
    std::vector<GSrc> gs = {gsrc(0, {1}, 1.0, true), gsrc(0, {1}, -1.0, true)};
    if (!gather_in_range(go, gs, n, 2 * n)) {
      err = "adjoint: conj(psi) descriptors out of range";
      return DMRGX_E_STATE;
    }
    e = launch_gather(psi, cpsi.p, go, gs, cplx, st);
  }

  if (want_l && e == cudaSuccess) {
    // transposed store blocks [K x N], one per distinct input block of stage 2
    std::map<int64_t, int64_t> st_at;
    std::vector<GOut> go;
    std::vector<GSrc> gs;
    int64_t stl = 0;
    for (auto& r : c->lmap) {
      const int64_t K = r.cols, N = r.rows, M = Lop.bsize(r.blk) / std::max(1, r.cols);
      if (M == 0 || N == 0 || K == 0 || st_at.count(r.in_beg)) continue;
      st_at[r.in_beg] = stl;
      gs.push_back(gsrc(r.in_beg, {1, K}, 1.0, false));
      go.push_back(gout(stl, {K, N}, {N, 1}, (int)gs.size() - 1, 1));
      stl += K * N;
    }
    if (!gather_in_range(go, gs, c->d_store, stl)) {
      err = "adjoint: store transpose descriptors out of range";
      return DMRGX_E_STATE;
    }
    DevArr stT(st);
    e = stT.alloc(stl * f);
    if (e == cudaSuccess && !go.empty()) e = launch_gather(store, stT.p, go, gs, cplx, st);
    gl = std::make_shared<QTensor>();
    gl->m = Lop.m;
    gl->f = f;
    if (e == cudaSuccess) e = gl->alloc(st);
    Grouper g;
    for (auto& r : c->lmap) {
      const int64_t K = r.cols, N = r.rows, M = Lop.bsize(r.blk) / std::max(1, r.cols);
      if (M == 0 || N == 0 || K == 0) continue;
      const int o = g.out(r.blk, Lop.off[r.blk] * f, M, K * f);
      g.seg(o, ((r.alpha >= 0 ? 0 : n) + r.out_beg) * f, st_at[r.in_beg] * f, N * f);
    }
    std::vector<DOut> outs;
    std::vector<DSeg> segs;
    g.flatten(outs, segs);
    if (!gemm_in_range(outs, segs, 2 * n, stl, Lop.total(), f)) {
      err = "adjoint: dE/dLop descriptors out of range";
      return DMRGX_E_STATE;
    }
    if (e == cudaSuccess) e = qt_grouped_gemm(E, cpsi.p, stT.p, gl->d, outs, segs);
  }

  if (want_r && e == cudaSuccess) {
    // dE/dstore[N x K] per stage-2 input block = sum alpha conj(psi_out)^T Lop_blk
    std::map<std::pair<int64_t, int>, int64_t> pt_at;  // (psi out block, sign) -> offset
    std::map<int, int64_t> lt_at;                      // Lop block -> offset
    std::vector<GOut> go, go2;
    std::vector<GSrc> gs, gs2;
    int64_t ptl = 0, ltl = 0;
    for (auto& r : c->lmap) {
      const int64_t K = r.cols, N = r.rows, M = Lop.bsize(r.blk) / std::max(1, r.cols);
      if (M == 0 || N == 0 || K == 0) continue;
      const int sg = r.alpha >= 0 ? 1 : -1;
      if (!pt_at.count({r.out_beg, sg})) {
        pt_at[{r.out_beg, sg}] = ptl;
        gs.push_back(gsrc(r.out_beg, {1, N}, (double)sg, true));
        go.push_back(gout(ptl, {N, M}, {M, 1}, (int)gs.size() - 1, 1));
        ptl += N * M;
      }
      if (!lt_at.count(r.blk)) {
        lt_at[r.blk] = ltl;
        gs2.push_back(gsrc(Lop.off[r.blk], {1, K}, 1.0, false));
        go2.push_back(gout(ltl, {K, M}, {M, 1}, (int)gs2.size() - 1, 1));
        ltl += K * M;
      }
    }
    if (!gather_in_range(go, gs, n, ptl) || !gather_in_range(go2, gs2, Lop.total(), ltl)) {
      err = "adjoint: transpose descriptors out of range";
      return DMRGX_E_STATE;
    }
    DevArr pT(st), lT(st), dstore(st);
    e = pT.alloc(ptl * f);
    if (e == cudaSuccess) e = lT.alloc(ltl * f);
    if (e == cudaSuccess) e = dstore.alloc(c->d_store * f);
    if (e == cudaSuccess) e = cudaMemsetAsync(dstore.p, 0, sizeof(double) * std::max<int64_t>(1, c->d_store * f), st);
    if (e == cudaSuccess && !go.empty()) e = launch_gather(psi, pT.p, go, gs, cplx, st);
    if (e == cudaSuccess && !go2.empty()) e = launch_gather(Lop.d, lT.p, go2, gs2, cplx, st);
    {
      Grouper g;
      for (auto& r : c->lmap) {
        const int64_t K = r.cols, N = r.rows, M = Lop.bsize(r.blk) / std::max(1, r.cols);
        if (M == 0 || N == 0 || K == 0) continue;
        const int sg = r.alpha >= 0 ? 1 : -1;
        const int o = g.out(r.in_beg, r.in_beg * f, N, K * f);
        g.seg(o, pt_at[{r.out_beg, sg}] * f, lt_at[r.blk] * f, M * f);
      }
      std::vector<DOut> outs;
      std::vector<DSeg> segs;
      g.flatten(outs, segs);
      if (!gemm_in_range(outs, segs, ptl, ltl, c->d_store, f)) {
        err = "adjoint: dE/dstore descriptors out of range";
        return DMRGX_E_STATE;
      }
      if (e == cudaSuccess) e = qt_grouped_gemm(E, pT.p, lT.p, dstore.p, outs, segs);
    }
    // dE/dRop_blk[M1 x K1] = sum alpha dstore_out[M1 x N1] psi_in[N1 x K1]
    std::map<std::pair<int64_t, int>, int64_t> qt_at;
    go.clear();
    gs.clear();
    int64_t qtl = 0;
    for (auto& r : c->rmap) {
      const int64_t K = r.cols, N = r.rows, M = Rop.bsize(r.blk) / std::max(1, r.cols);
      if (M == 0 || N == 0 || K == 0) continue;
      const int sg = r.alpha >= 0 ? 1 : -1;
      if (qt_at.count({r.in_beg, sg})) continue;
      qt_at[{r.in_beg, sg}] = qtl;
      gs.push_back(gsrc(r.in_beg, {1, K}, (double)sg, false));
      go.push_back(gout(qtl, {K, N}, {N, 1}, (int)gs.size() - 1, 1));
      qtl += K * N;
    }
    if (!gather_in_range(go, gs, n, qtl)) {
      err = "adjoint: psi transpose descriptors out of range";
      return DMRGX_E_STATE;
    }
    DevArr qT(st);
    if (e == cudaSuccess) e = qT.alloc(qtl * f);
    if (e == cudaSuccess && !go.empty()) e = launch_gather(psi, qT.p, go, gs, cplx, st);
    gr = std::make_shared<QTensor>();
    gr->m = Rop.m;
    gr->f = f;
    if (e == cudaSuccess) e = gr->alloc(st);
    Grouper g;
    for (auto& r : c->rmap) {
      const int64_t K = r.cols, N = r.rows, M = Rop.bsize(r.blk) / std::max(1, r.cols);
      if (M == 0 || N == 0 || K == 0) continue;
      const int sg = r.alpha >= 0 ? 1 : -1;
      const int o = g.out(r.blk, Rop.off[r.blk] * f, M, K * f);
      g.seg(o, r.out_beg * f, qt_at[{r.in_beg, sg}] * f, N * f);
    }
    std::vector<DOut> outs;
    std::vector<DSeg> segs;
    g.flatten(outs, segs);
    if (!gemm_in_range(outs, segs, c->d_store, qtl, Rop.total(), f)) {
      err = "adjoint: dE/dRop descriptors out of range";
      return DMRGX_E_STATE;
    }
    if (e == cudaSuccess) e = qt_grouped_gemm(E, dstore.p, qT.p, gr->d, outs, segs);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("adjoint: ") + cudaGetErrorString(e);
    return DMRGX_E_CUDA;
  }
  return 0;
}

int fusion_adjoint(const Engine& E, const QTensor& env, const QTensor& W, const QTensor& gfused,
                   bool right, std::vector<double>& gw, std::string& err) {
  const int f = E.f;
  if (W.m.nleg() != 4 || env.m.nleg() != 3) {
    err = "fusion adjoint: expected a 3-leg environment and a 4-leg MPO tensor";
    return DMRGX_E_ARG;
  }
  for (int leg : {1, 3})
    for (int d : W.m.dims[leg])
      if (d != 1) {
        err = "fusion adjoint: MPO physical sectors must hold one state each";
        return DMRGX_E_ARG;
      }
  QMeta Wm = W.m;  // W.exchange(0, 2) keeps the block order
  if (right) {
    std::swap(Wm.dims[0], Wm.dims[2]);
    std::swap(Wm.dirs[0], Wm.dirs[2]);
    for (auto& s : Wm.syms) std::swap(s[0], s[2]);
  }
  const auto pairs = fuse_pairs(E.G, env.m, 1, Wm, 0, right);
  std::map<int64_t, int> key2blk;
  for (size_t b = 0; b < gfused.m.syms.size(); b++)
    key2blk[label_key(gfused.m.syms[b], gfused.m.dims)] = (int)b;
  struct Task {
    int wblk, I, J;
    double sign;
    int64_t part;  // offset of this pair's first slab result
    int nslab;
  };
  std::vector<Task> tasks;
  Grouper g;
  int64_t partl = 0;
  const int SLAB = 16;  // x values per grouped output
  for (auto& p : pairs) {
    std::vector<int> sym = p.sym;
    if (right) std::swap(sym[0], sym[1]);
    else std::swap(sym[3], sym[4]);
    auto it = key2blk.find(label_key(sym, gfused.m.dims));
    if (it == key2blk.end()) {
      err = "fusion adjoint: fused block missing";
      return DMRGX_E_STATE;
    }
    const int o = it->second;
    const auto& se = env.m.syms[p.l];
    const int64_t X = env.m.dims[0][se[0]], I = env.m.dims[1][se[1]], Y = env.m.dims[2][se[2]];
    const auto& sw = W.m.syms[p.r];
    const int64_t Da = W.m.dims[0][sw[0]], Db = W.m.dims[2][sw[2]];
    const int64_t J = right ? Da : Db;
    if (I != (right ? Db : Da)) {
      err = "fusion adjoint: bond dimensions disagree";
      return DMRGX_E_STATE;
    }
    if (X == 0 || Y == 0 || I == 0 || J == 0) continue;
    const int64_t gx = J * Y;  // fused block [x, J, y] (unit physical legs)
    Task t{p.r, (int)I, (int)J, p.sign, partl, (int)((X + SLAB - 1) / SLAB)};
    for (int sl = 0; sl < t.nslab; sl++) {
      const int oi = g.out((int64_t)tasks.size() * 65536 + sl, partl * f, I, J * f);
      partl += I * J;
      for (int64_t x = (int64_t)sl * SLAB; x < std::min<int64_t>(X, (int64_t)(sl + 1) * SLAB); x++)
        g.seg(oi, (env.off[p.l] + x * I * Y) * f, (gfused.off[o] + x * gx) * f, Y * f);
    }
    tasks.push_back(t);
  }
  if (tasks.empty()) return 0;
  std::vector<DOut> outs;
  std::vector<DSeg> segs;
  g.flatten(outs, segs);
  if (!gemm_in_range(outs, segs, env.total(), gfused.total(), partl, f)) {
    err = "fusion adjoint: descriptors out of range";
    return DMRGX_E_STATE;
  }
  DevArr part(E.stream);
  cudaError_t e = part.alloc(partl * f);
  if (e == cudaSuccess) e = qt_grouped_gemm(E, env.d, gfused.d, part.p, outs, segs);
  std::vector<double> hp((size_t)(partl * f));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hp.data(), part.p, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost,
                        E.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
  if (e != cudaSuccess) {
    err = std::string("fusion adjoint: ") + cudaGetErrorString(e);
    return DMRGX_E_CUDA;
  }
  for (auto& t : tasks) {
    const int64_t Db = W.m.dims[2][W.m.syms[t.wblk][2]];
    for (int sl = 0; sl < t.nslab; sl++)
      for (int i = 0; i < t.I; i++)
        for (int j = 0; j < t.J; j++) {
          const int64_t a = right ? j : i, b = right ? i : j;  // W block [a, 1, b, 1]
          const int64_t w = (W.off[t.wblk] + a * Db + b) * f;
          const int64_t src = (t.part + (int64_t)sl * t.I * t.J + (int64_t)i * t.J + j) * f;
          for (int q = 0; q < f; q++) gw[w + q] += t.sign * hp[src + q];
        }
  }
  return 0;
}

int edge_adjoint(const QTensor& gedge, const QTensor& W, bool right, std::vector<double>& gw,
                 cudaStream_t s, std::string& err) {
  const int f = gedge.f;
  if (W.m.dims[0].size() != 1 || W.m.dims[2].size() != 1 || gedge.m.nleg() != 3) {
    err = "edge adjoint: MPO bond legs must have one sector";
    return DMRGX_E_ARG;
  }
  const int64_t Db = W.m.dims[2][0], Da = W.m.dims[0][0];
  std::vector<double> hv((size_t)(gedge.total() * f));
  if (!hv.empty()) {
    cudaMemcpyAsync(hv.data(), gedge.d, sizeof(double) * hv.size(), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
      err = "edge adjoint: copy failed";
      return DMRGX_E_CUDA;
    }
  }
  for (size_t eb = 0; eb < gedge.m.syms.size(); eb++) {
    const auto& le = gedge.m.syms[eb];
    // left edge [s, b, s'] = W[D-1, s, b, s'];  right edge [s, a, s'] = W[a, s, 0, s']
    std::vector<int> wl = right ? std::vector<int>{le[1], le[0], 0, le[2]}
                                : std::vector<int>{0, le[0], le[1], le[2]};
    int wb = -1;
    for (size_t b = 0; b < W.m.syms.size(); b++)
      if (W.m.syms[b] == wl) wb = (int)b;
    if (wb < 0) {
      err = "edge adjoint: edge block without an MPO block";
      return DMRGX_E_STATE;
    }
    const int64_t cnt = gedge.bsize((int)eb);
    for (int64_t k = 0; k < cnt; k++) {
      const int64_t welem = right ? k * Db : (Da - 1) * Db + k;
      for (int q = 0; q < f; q++) gw[(W.off[wb] + welem) * f + q] += hv[(gedge.off[eb] + k) * f + q];
    }
  }
  return 0;
}

}  // namespace dmrgx
