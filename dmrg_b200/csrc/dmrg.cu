// DMRG site steps and sweep schedule on the device (the callers around the
// matvec): the reference's two_sites / update_two / move2right / move2left
// (src/core.cpp:88-474) and dmrg() (src/functions.cpp:157-227), for the shipped
// models' MPOs (src/operators.cpp).  Every step builds L~ and R~ by the env (x)
// MPO fusion, solves for the lowest state with the device Lanczos solver
// (split precision + FP64 defect correction when the context asks for it),
// truncates by the block SVD and updates the environments; all tensors stay on
// the GPU.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/dmrgx.h"
#include "adjoint.h"
#include "ctx.h"
#include "devmem.h"
#include "qtensor.h"

namespace dmrgx {

int plan_build_device(dmrgx_ctx* c, const QTensor& L, const QTensor& R, int l_num, int r_num,
                      int sector, const Group& G, const QTensor* Le = nullptr,
                      const QTensor* Re = nullptr);
int group_solve(dmrgx_ctx* c, int nev, int ncv, double tol, const double* v0, double* evals,
                double* evec, int64_t* info);
int eigsolve_device(dmrgx_ctx* c, int nev, int ncv, double tol, int maxiter, const double* v0,
                    double* evals, double* evec, int64_t* info);

namespace {

constexpr double REF_PI = 3.14159265359;  // the reference's PI (global.h:25)
using cplx = std::complex<double>;

// ---------------------------------------------------------------- model MPOs
// Host form of a small block-sparse tensor built entry by entry.
struct HostQT {
  QMeta m;
  std::vector<std::vector<cplx>> blocks;
  void add_block(const std::vector<int>& sym, const std::vector<int>& shape) {
    m.syms.push_back(sym);
    int64_t n = 1;
    for (int v : shape) n *= v;
    blocks.emplace_back((size_t)n, cplx(0, 0));
  }
  // value of the last added block at a 4-index position of shape (D,1,D,1)
  void set(int D, int i0, int i2, cplx v) { blocks.back()[(size_t)i0 * D + i2] = v; }
};

// reference qtensor::take(n, k) followed by simplify() (src/qtensor.cpp:401-447)
HostQT take(const HostQT& A, int n, int k) {
  HostQT R;
  const int nl = A.m.nleg();
  for (int l = 0; l < nl; l++)
    if (l != n) {
      R.m.dims.push_back(A.m.dims[l]);
      R.m.dirs.push_back(A.m.dirs[l]);
    }
  for (size_t b = 0; b < A.m.syms.size(); b++) {
    std::vector<int> shape(nl);
    for (int l = 0; l < nl; l++) shape[l] = A.m.dims[l][A.m.syms[b][l]];
    int64_t r = 1;
    for (int l = n + 1; l < nl; l++) r *= shape[l];
    const int64_t cnt = (int64_t)A.blocks[b].size() / shape[n];
    std::vector<cplx> v(cnt);
    bool nz = false;
    for (int64_t i = 0; i < cnt; i++) {
      v[i] = A.blocks[b][((i / r) * shape[n] + k) * r + (i % r)];
      if (std::abs(v[i]) > 1e-10) nz = true;
    }
    if (!nz) continue;
    std::vector<int> sym;
    for (int l = 0; l < nl; l++)
      if (l != n) sym.push_back(A.m.syms[b][l]);
    R.m.syms.push_back(sym);
    R.blocks.push_back(v);
  }
  return R;
}

// reference qtensor::exchange(a, b) on a host tensor
HostQT exchange(const HostQT& A, int a, int b) {
  HostQT R = A;
  std::swap(R.m.dims[a], R.m.dims[b]);
  std::swap(R.m.dirs[a], R.m.dirs[b]);
  const int nl = A.m.nleg();
  for (size_t blk = 0; blk < A.m.syms.size(); blk++) {
    std::swap(R.m.syms[blk][a], R.m.syms[blk][b]);
    std::vector<int> sh(nl), nsh;
    for (int l = 0; l < nl; l++) sh[l] = A.m.dims[l][A.m.syms[blk][l]];
    nsh = sh;
    std::swap(nsh[a], nsh[b]);
    std::vector<int64_t> st(nl, 1), nst(nl, 1);
    for (int l = nl - 2; l >= 0; l--) {
      st[l] = st[l + 1] * sh[l + 1];
      nst[l] = nst[l + 1] * nsh[l + 1];
    }
    const int64_t cnt = (int64_t)A.blocks[blk].size();
    for (int64_t e = 0; e < cnt; e++) {
      std::vector<int> idx(nl);
      int64_t r = e;
      for (int l = nl - 1; l >= 0; l--) {
        idx[l] = (int)(r % sh[l]);
        r /= sh[l];
      }
      std::swap(idx[a], idx[b]);
      int64_t ne = 0;
      for (int l = 0; l < nl; l++) ne += idx[l] * nst[l];
      R.blocks[blk][ne] = A.blocks[blk][e];
    }
  }
  return R;
}

// model: 0 Kitaev(t, p, u)  (src/operators.cpp:406-431)
//        1 XYZ(jx, jy, jz)   (src/operators.cpp:361-391)
//        2 Potts3(f, j, p, t) (src/operators.cpp:301-350)
//        3 XYZ(jx, jy, jz) with a real MPO: sigma_y (x) sigma_y = -(i sigma_y) (x)
//          (i sigma_y) and i sigma_y = [[0, 1], [-1, 0]] is real, so the reference's
//          complex XYZ MPO becomes real with the same spectrum
// XYZ (1 and 3) take an optional fourth parameter h, a field h sum_i sigma^z_i in
// the on-site slot W[D-1, s, 0, s]; the reference has no field, and at h = 0 the
// MPO is the reference's entry for entry.
bool build_mpo(int model, const double* par, HostQT& W) {
  W = HostQT();
  const cplx I(0, 1);
  if (model == 0) {
    const double t = par[0], p = par[1], u = par[2];
    W.m.dims = {{4}, {1, 1}, {4}, {1, 1}};
    W.m.dirs = {0, -1, 0, 1};
    W.add_block({0, 0, 0, 0}, {4, 1, 4, 1});
    W.set(4, 0, 0, 1); W.set(4, 3, 3, 1);
    W.add_block({0, 0, 0, 1}, {4, 1, 4, 1});
    W.set(4, 1, 0, 1); W.set(4, 3, 1, -p); W.set(4, 3, 2, -t);
    W.add_block({0, 1, 0, 0}, {4, 1, 4, 1});
    W.set(4, 2, 0, 1); W.set(4, 3, 1, t); W.set(4, 3, 2, p);
    W.add_block({0, 1, 0, 1}, {4, 1, 4, 1});
    W.set(4, 0, 0, 1); W.set(4, 3, 0, -2 * u); W.set(4, 3, 3, 1);
    return true;
  }
  if (model == 1) {
    const double jx = par[0], jy = par[1], jz = par[2], h = par[3];
    W.m.dims = {{5}, {1, 1}, {5}, {1, 1}};
    W.m.dirs = {0, 0, 0, 0};
    W.add_block({0, 0, 0, 0}, {5, 1, 5, 1});
    W.set(5, 0, 0, 1); W.set(5, 3, 0, 1); W.set(5, 4, 3, jz); W.set(5, 4, 4, 1);
    W.set(5, 4, 0, h);
    W.add_block({0, 0, 0, 1}, {5, 1, 5, 1});
    W.set(5, 1, 0, 1); W.set(5, 2, 0, -I); W.set(5, 4, 1, jx); W.set(5, 4, 2, -I * jy);
    W.add_block({0, 1, 0, 0}, {5, 1, 5, 1});
    W.set(5, 1, 0, 1); W.set(5, 2, 0, I); W.set(5, 4, 1, jx); W.set(5, 4, 2, I * jy);
    W.add_block({0, 1, 0, 1}, {5, 1, 5, 1});
    W.set(5, 0, 0, 1); W.set(5, 3, 0, -1); W.set(5, 4, 3, -jz); W.set(5, 4, 4, 1);
    W.set(5, 4, 0, -h);
    return true;
  }
  if (model == 3) {
    const double jx = par[0], jy = par[1], jz = par[2], h = par[3];
    W.m.dims = {{5}, {1, 1}, {5}, {1, 1}};
    W.m.dirs = {0, 0, 0, 0};
    W.add_block({0, 0, 0, 0}, {5, 1, 5, 1});
    W.set(5, 0, 0, 1); W.set(5, 3, 0, 1); W.set(5, 4, 3, jz); W.set(5, 4, 4, 1);
    W.set(5, 4, 0, h);
    W.add_block({0, 0, 0, 1}, {5, 1, 5, 1});
    W.set(5, 1, 0, 1); W.set(5, 2, 0, 1); W.set(5, 4, 1, jx); W.set(5, 4, 2, -jy);
    W.add_block({0, 1, 0, 0}, {5, 1, 5, 1});
    W.set(5, 1, 0, 1); W.set(5, 2, 0, -1); W.set(5, 4, 1, jx); W.set(5, 4, 2, jy);
    W.add_block({0, 1, 0, 1}, {5, 1, 5, 1});
    W.set(5, 0, 0, 1); W.set(5, 3, 0, -1); W.set(5, 4, 3, -jz); W.set(5, 4, 4, 1);
    W.set(5, 4, 0, -h);
    return true;
  }
  if (model == 2) {
    const double f = par[0], j = par[1], p = par[2], t = par[3];
    W.m.dims = {{4}, {1, 1, 1}, {4}, {1, 1, 1}};
    W.m.dirs = {0, 0, 0, 0};
    const cplx vs = -j * cplx(std::cos(t), std::sin(t));
    const cplx vd = -j * cplx(std::cos(t), -std::sin(t));
    auto diag = [&](int q) {
      W.set(4, 0, 0, 1);
      W.set(4, 3, 0, -2 * f * std::cos(p + 2 * REF_PI * q / 3));
      W.set(4, 3, 3, 1);
    };
    auto s_op = [&]() { W.set(4, 1, 0, 1); W.set(4, 3, 2, vs); };
    auto sd_op = [&]() { W.set(4, 2, 0, 1); W.set(4, 3, 1, vd); };
    W.add_block({0, 0, 0, 0}, {4, 1, 4, 1}); diag(0);
    W.add_block({0, 0, 0, 1}, {4, 1, 4, 1}); s_op();
    W.add_block({0, 0, 0, 2}, {4, 1, 4, 1}); sd_op();
    W.add_block({0, 1, 0, 0}, {4, 1, 4, 1}); sd_op();
    W.add_block({0, 1, 0, 1}, {4, 1, 4, 1}); diag(1);
    W.add_block({0, 1, 0, 2}, {4, 1, 4, 1}); s_op();
    W.add_block({0, 2, 0, 0}, {4, 1, 4, 1}); s_op();
    W.add_block({0, 2, 0, 1}, {4, 1, 4, 1}); sd_op();
    W.add_block({0, 2, 0, 2}, {4, 1, 4, 1}); diag(2);
    return true;
  }
  return false;
}

// qtensor::id(bulk_mpo) (src/qtensor.cpp:157-184): the operator that carries an
// edge environment across a bulk site on a periodic chain.  Legs and directions
// of the bulk MPO W, except legs 0 and 2, which take the edge environment's MPO
// leg (leg 1); one block (s0, s1, s0, s1) per pair of sectors with
// delta(i0, i2) delta(i1, i3).  Blocks of zero size are left out (they hold no
// values).
HostQT edge_identity(const QMeta& edge, const QMeta& W) {
  HostQT R;
  R.m.dims = W.dims;
  R.m.dirs = W.dirs;
  R.m.dims[0] = R.m.dims[2] = edge.dims[1];
  R.m.dirs[0] = R.m.dirs[2] = edge.dirs[1];
  for (int s0 = 0; s0 < (int)R.m.dims[0].size(); s0++)
    for (int s1 = 0; s1 < (int)R.m.dims[1].size(); s1++) {
      const int a = R.m.dims[0][s0], b = R.m.dims[1][s1];
      if (a == 0 || b == 0) continue;
      R.add_block({s0, s1, s0, s1}, {a, b, a, b});
      for (int i0 = 0; i0 < a; i0++)
        for (int i1 = 0; i1 < b; i1++)
          R.blocks.back()[(((size_t)i0 * b + i1) * a + i0) * b + i1] = cplx(1, 0);
    }
  return R;
}

QTPtr upload(const HostQT& H, int f, cudaStream_t s, std::string& err) {
  auto T = std::make_shared<QTensor>();
  T->m = H.m;
  T->f = f;
  if (T->alloc(s) != cudaSuccess) {
    err = "allocation failed";
    return nullptr;
  }
  std::vector<double> v((size_t)T->total() * f);
  size_t k = 0;
  for (auto& b : H.blocks)
    for (auto& x : b) {
      v[k++] = x.real();
      if (f == 2) v[k++] = x.imag();
    }
  if (!v.empty()) cudaMemcpyAsync(T->d, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice, s);
  cudaStreamSynchronize(s);
  return T;
}

// singular values per step kept for dmrgx_singular (the reference's NSI, global.h)
constexpr int kSingularRow = 20;

struct Run {
  dmrgx_ctx* c;
  Engine E;
  int L;
  QTPtr bulk, ledge, redge;  // mpo[i], mpo[0], mpo[L-1]
  std::vector<QTPtr> env;    // mps(i): block environments
  std::vector<QTPtr> site;   // mps[i]: U (left of the centre) or V (right of it)
  int sector;
  int m_cut = 0;             // bond cutoff of the sweeps
  // one-site centre of the state after the last step: psi[b_{c-1}, s_c, b_{c+1}]
  // (left legs absent at c = 0, right ones at c = L-1)
  int center = -1;
  QTPtr cpsi;
  int model = 0;
  std::vector<double> par;   // model parameters of the MPO in use
  // periodic chain (the reference's PBC build): edge environments mps.edge(i),
  // seeded at 0 and L-1 with the drivers' edge operators (src/mps.h add_edge)
  bool pbc = false;
  std::vector<QTPtr> edge;
  // eigensolver of the site steps: eigenvalues wanted (the reference's NEV = 6,
  // global.h:21), Krylov basis (0: the reference's 4 nev / 6 nev), prediction
  int eig_nev = 6, eig_ncv = 0;
  bool predict = false;
  QTPtr guess;                               // start vector of the next solve
  int last_kind = 0, last_center = -1;       // 1 move2right, 2 move2left
  QTPtr last_psi, last_U, last_V;
  std::map<std::pair<std::vector<int>, int>, QTPtr> edge_ids;  // id(W) by (dims, dir) of leg 1
  // per-step records
  std::vector<int> lr;
  std::vector<double> energies, trunc;
  std::vector<double> entropy;  // per step, print_singular's S
  std::vector<double> sv;       // per step, the first 20 singular values (0 past |s|)
  std::vector<int> nsv;         // per step, |s|
  std::vector<int64_t> matvecs;
  std::vector<double> step_s;  // wall seconds of every step
  std::vector<double> step_split;  // per step: eigensolver, SVD, env update, fusion, plan
  double t_eig = 0, t_svd = 0, t_env = 0, t_fuse = 0, t_plan = 0;
  std::string err;

  const QTensor& mpo(int i) const { return i == 0 ? *ledge : (i == L - 1 ? *redge : *bulk); }

  static double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
  }

  // plan of a step (timed); Le / Re: the edge pair of a periodic chain
  int plan(const QTensor& Lop, const QTensor& Rop, int ln, int rn, int sec, const Group& G,
           const QTensor* Le = nullptr, const QTensor* Re = nullptr) {
    const double t0 = now();
    const int rc = plan_build_device(c, Lop, Rop, ln, rn, sec, G, Le, Re);
    t_plan += now() - t0;
    return rc;
  }

  // lowest state of the current plan -> psi tensor (written by the eigensolver on
  // the device); records energies.  With a predicted centre (guess) the solve
  // starts from it, else from the solver's fixed pattern.
  int solve(int l, int r, QTPtr& psi) {
    const double t0 = now();
    std::vector<double> ev(std::max(6, eig_nev), 0.0);
    int64_t info[6];
    psi = std::make_shared<QTensor>();
    psi->m.dims = c->psi_dim;
    psi->m.syms = c->psi_sym;
    psi->m.dirs.assign(c->psi_dim.size(), 0);
    psi->f = c->f();
    if (psi->alloc(E.stream) != cudaSuccess) {
      err = "psi allocation failed";
      return DMRGX_E_CUDA;
    }
    if (psi->total() != c->n) {
      err = "psi layout mismatch";
      return DMRGX_E_STATE;
    }
    double* v0 = nullptr;
    if (guess) {
      // a guess whose blocks do not fit this plan is dropped, not an error
      if (dalloc(&v0, (size_t)std::max<int64_t>(1, c->n * c->f()), E.stream) != cudaSuccess) {
        v0 = nullptr;
      } else if (to_plan(*guess, v0)) {
        dfree(v0, E.stream);
        v0 = nullptr;
        err.clear();
      }
      guess.reset();
    }
    int rc;
    if (c->group) {
      // one lock-step solve with the group's other contexts (FP64 grouped matvec)
      if (c->prec != DMRGX_PREC_FP64 || c->per_block) {
        err = "a solve group needs FP64 contexts on the grouped schedule";
        if (v0) dfree(v0, E.stream);
        return DMRGX_E_STATE;
      }
      rc = group_solve(c, eig_nev, eig_ncv, 1e-10, v0, ev.data(), psi->d, info);
    } else {
      rc = eigsolve_device(c, eig_nev, eig_ncv, 1e-10, 0, v0, ev.data(), psi->d, info);
    }
    if (v0) dfree(v0, E.stream);
    if (rc) {
      err = std::string("eigsolve: ") + dmrgx_last_error();
      return rc;
    }
    lr.push_back(l);
    lr.push_back(r);
    const int nrec = (int)std::min<int64_t>(std::min(6, eig_nev), c->n);
    for (int q = 0; q < 6; q++) energies.push_back(q < nrec ? ev[q] : 0.0);
    matvecs.push_back(info[0]);
    t_eig += now() - t0;
    return 0;
  }

  // White's wavefunction prediction of the next step's one-site centre from the
  // last step's psi = U S V (the reference starts every solve from ARPACK's
  // random vector instead, src/dsaupd.cpp:97):
  //   right move after a right move (centre c -> c+1):  (U^+ psi) . B_{c+1}
  //   left move after a left move (centre c -> c-1):    A_{c-1} . (psi V^+)
  //   turn at a chain end (same centre site):           psi
  // B_{c+1} / A_{c-1}: the site tensors the previous sweep left there.
  void remember(int kind, const QTPtr& psi, const QTPtr& U, const QTPtr& V) {
    last_kind = kind;
    last_center = center;
    last_psi = predict ? psi : nullptr;
    last_U = predict ? U : nullptr;
    last_V = predict ? V : nullptr;
  }
  void predict_center(int kind, int next_center) {
    guess.reset();
    if (!predict || !last_psi) return;
    const double t0 = now();
    if (kind != last_kind && next_center == last_center) {
      guess = last_psi;
    } else if (kind == 1 && last_kind == 1 && next_center == last_center + 1 &&
               site[next_center]) {
      auto Uc = qt_copy(E, *last_U);
      qt_conjugate(E, *Uc);
      QTPtr sv = qt_contract_mat(E, *Uc, *last_psi, 'T', 'N', 2, err);
      if (sv) guess = qt_contract_mat(E, *sv, *site[next_center], 'N', 'N', 1, err);
    } else if (kind == 2 && last_kind == 2 && next_center == last_center - 1 &&
               site[next_center]) {
      auto Vc = qt_copy(E, *last_V);
      qt_conjugate(E, *Vc);
      QTPtr us = qt_contract_mat(E, *last_psi, *Vc, 'N', 'T', 2, err);
      if (us) guess = qt_contract_mat(E, *site[next_center], *us, 'N', 'N', 1, err);
    }
    if (!guess) err.clear();  // no prediction: the solve starts from the default
    t_eig += now() - t0;
  }

  int svd(const QTensor& psi, int num, int cutoff, QTPtr& U, QTPtr& V) {
    const double t0 = now();
    std::vector<double> s;
    if (qt_svd(E, psi, num, cutoff, U, V, s, err)) return DMRGX_E_CUDA;
    // print_singular's figures (src/useful.cpp:75-102), same expressions and
    // summation order: entropy S = -sum s^2 log(s^2 + TOL) over the whole
    // spectrum (TOL = 1e-10, global.h), the first NSI = 20 values, and the
    // truncation error 1 - sum_{i < min(cutoff, |s|)} s_i^2
    double S = 0.0;
    for (size_t i = 0; i < s.size(); i++) S += -s[i] * s[i] * std::log(s[i] * s[i] + 1e-10);
    entropy.push_back(S);
    for (int i = 0; i < kSingularRow; i++) sv.push_back(i < (int)s.size() ? s[i] : 0.0);
    nsv.push_back((int)s.size());
    double e = 1.0;
    const int64_t k = std::min<int64_t>(cutoff, (int64_t)s.size());
    for (int64_t i = 0; i < k; i++) e -= s[i] * s[i];
    trunc.push_back(e);
    t_svd += now() - t0;
    return 0;
  }

  // L_new = (lenv U)^T conj(U)...: src/core.cpp:266-268
  QTPtr left_update(const QTensor& lenv, QTensor& U, int num) {
    const double t0 = now();
    QTPtr vec = qt_contract_mat(E, lenv, U, 'N', 'N', num, err);
    if (!vec) return nullptr;
    auto Uc = qt_copy(E, U);
    qt_conjugate(E, *Uc);
    QTPtr out = qt_contract_mat(E, *Uc, *vec, 'T', 'N', num, err);
    t_env += now() - t0;
    return out;
  }
  // src/core.cpp:269-271
  QTPtr right_update(const QTensor& renv, QTensor& V, int num) {
    const double t0 = now();
    QTPtr vec = qt_contract_mat(E, renv, V, 'N', 'T', num, err);
    if (!vec) return nullptr;
    auto Vc = qt_copy(E, V);
    qt_conjugate(E, *Vc);
    QTPtr out = qt_contract_mat(E, *Vc, *vec, 'N', 'N', num, err);
    t_env += now() - t0;
    return out;
  }
  // lenv = (mps(l-1) ._1 W_l).exchange(3,4)   (src/core.cpp:188-189)
  QTPtr fuse_left(int l) {
    const double t0 = now();
    QTPtr o = qt_contract_legs(E, *env[l - 1], 1, mpo(l), 0, false, 3, 4, err);
    t_fuse += now() - t0;
    return o;
  }
  // renv = (mps(r+1) ._1 W_r.exchange(0,2), change).exchange(0,1)   (src/core.cpp:190-192)
  QTPtr fuse_right(int r) {
    const double t0 = now();
    QTPtr ope = qt_exchange(E, mpo(r), 0, 2, err);
    if (!ope) return nullptr;
    QTPtr o = qt_contract_legs(E, *env[r + 1], 1, *ope, 0, true, 0, 1, err);
    t_fuse += now() - t0;
    return o;
  }

  // periodic chain: the edge environment carried across a bulk site,
  //   ledge = (edge(l-1) ._1 ope).exchange(3,4)          (src/core.cpp:193-197)
  //   redge = (edge(r+1) ._1 ope, change).exchange(0,1)   (src/core.cpp:198-199)
  // ope = e.id(W) of the edge environment e the step names: edge(l-1) for both
  // sides in update_two and move2right, edge(r+1) in move2left (:302, :418)
  QTPtr edge_op(const QTensor& e) {
    auto key = std::make_pair(e.m.dims[1], e.m.dirs[1]);
    auto it = edge_ids.find(key);
    if (it != edge_ids.end()) return it->second;
    QTPtr o = upload(edge_identity(e.m, bulk->m), c->f(), E.stream, err);
    if (o) edge_ids[key] = o;
    return o;
  }
  QTPtr fuse_edge_left(int l, const QTPtr& ope) {
    const double t0 = now();
    QTPtr o = ope ? qt_contract_legs(E, *edge[l - 1], 1, *ope, 0, false, 3, 4, err) : nullptr;
    t_fuse += now() - t0;
    return o;
  }
  QTPtr fuse_edge_right(int r, const QTPtr& ope) {
    const double t0 = now();
    QTPtr o = ope ? qt_contract_legs(E, *edge[r + 1], 1, *ope, 0, true, 0, 1, err) : nullptr;
    t_fuse += now() - t0;
    return o;
  }

  // src/core.cpp:88-172
  int two_sites(int l, int r, int cutoff) {
    const QTensor& le = mpo(l);
    const QTensor& re = mpo(r);
    // on a periodic chain the edge pair is edge(l), edge(r) (src/core.cpp:96-99)
    QTPtr lx = pbc ? edge[l] : nullptr, rx = pbc ? edge[r] : nullptr;
    int rc = plan(le, re, 2, 1, sector, E.G, lx.get(), rx.get());
    if (rc) return fail(rc);
    QTPtr psi, U, V;
    if ((rc = solve(l, r, psi))) return rc;
    if ((rc = svd(*psi, 1, cutoff, U, V))) return rc;
    env[l] = left_update(le, *U, 1);
    env[r] = right_update(re, *V, 1);
    if (pbc) {
      edge[l] = left_update(*lx, *U, 1);   // src/core.cpp:161-170
      edge[r] = right_update(*rx, *V, 1);
      if (!edge[l] || !edge[r]) return DMRGX_E_CUDA;
    }
    site[l] = U;
    site[r] = V;
    center = -1;
    remember(0, nullptr, nullptr, nullptr);
    return env[l] && env[r] ? 0 : DMRGX_E_CUDA;
  }
  // src/core.cpp:182-283
  int update_two(int l, int r, int cutoff) {
    QTPtr le = fuse_left(l), re = fuse_right(r);
    if (!le || !re) return DMRGX_E_CUDA;
    QTPtr lx, rx;
    if (pbc) {
      QTPtr ope = edge_op(*edge[l - 1]);
      lx = fuse_edge_left(l, ope);
      rx = fuse_edge_right(r, ope);
      if (!lx || !rx) return DMRGX_E_CUDA;
    }
    int rc = plan(*le, *re, 3, 2, sector, E.G, lx.get(), rx.get());
    if (rc) return fail(rc);
    QTPtr psi, U, V;
    if ((rc = solve(l, r, psi))) return rc;
    if ((rc = svd(*psi, 2, cutoff, U, V))) return rc;
    env[l] = left_update(*le, *U, 2);
    env[r] = right_update(*re, *V, 2);
    if (pbc) {
      edge[l] = left_update(*lx, *U, 2);   // src/core.cpp:272-281
      edge[r] = right_update(*rx, *V, 2);
      if (!edge[l] || !edge[r]) return DMRGX_E_CUDA;
    }
    site[l] = U;
    site[r] = V;
    center = -1;
    remember(0, nullptr, nullptr, nullptr);
    return env[l] && env[r] ? 0 : DMRGX_E_CUDA;
  }
  // src/core.cpp:293-378
  int move2right(int l, int r, int cutoff) {
    QTPtr le = fuse_left(l);
    if (!le) return DMRGX_E_CUDA;
    QTPtr lx, rx;
    if (pbc) {  // src/core.cpp:302-307
      lx = fuse_edge_left(l, edge_op(*edge[l - 1]));
      rx = edge[r];
      if (!lx || !rx) return DMRGX_E_CUDA;
    }
    int rc = plan(*le, *env[r], 3, 1, sector, E.G, lx.get(), rx.get());
    if (rc) return fail(rc);
    predict_center(1, l);
    QTPtr psi, U, V;
    if ((rc = solve(l, r, psi))) return rc;
    if ((rc = svd(*psi, 2, cutoff, U, V))) return rc;
    env[l] = left_update(*le, *U, 2);
    if (pbc && !(edge[l] = left_update(*lx, *U, 2))) return DMRGX_E_CUDA;  // :371-376
    site[l] = U;
    center = l;  // psi[a_{l-1}, s_l, b_r]: centre at l, right block from r = l + 1
    cpsi = psi;
    remember(1, psi, U, V);
    return env[l] ? 0 : DMRGX_E_CUDA;
  }
  // src/core.cpp:388-474
  int move2left(int l, int r, int cutoff) {
    QTPtr re = fuse_right(r);
    if (!re) return DMRGX_E_CUDA;
    QTPtr lx, rx;
    if (pbc) {  // src/core.cpp:398-403
      lx = edge[l];
      rx = fuse_edge_right(r, edge_op(*edge[r + 1]));
      if (!lx || !rx) return DMRGX_E_CUDA;
    }
    int rc = plan(*env[l], *re, 2, 2, sector, E.G, lx.get(), rx.get());
    if (rc) return fail(rc);
    predict_center(2, r);
    QTPtr psi, U, V;
    if ((rc = solve(l, r, psi))) return rc;
    if ((rc = svd(*psi, 1, cutoff, U, V))) return rc;
    env[r] = right_update(*re, *V, 2);
    if (pbc && !(edge[r] = right_update(*rx, *V, 2))) return DMRGX_E_CUDA;  // :467-472
    site[r] = V;
    center = r;  // psi[b_l, s_r, a_{r+1}]: centre at r, left block through l = r - 1
    cpsi = psi;
    remember(2, psi, U, V);
    return env[r] ? 0 : DMRGX_E_CUDA;
  }
  int fail(int rc) {
    err = std::string("plan: ") + dmrgx_last_error();
    return rc;
  }

  // ------------------------------------------------------------ state after the sweeps
  QTPtr fuse_left_of(const QTensor& e, const QTensor& W) {
    return qt_contract_legs(E, e, 1, W, 0, false, 3, 4, err);
  }
  QTPtr fuse_right_of(const QTensor& e, const QTensor& W) {
    QTPtr ope = qt_exchange(E, W, 0, 2, err);
    if (!ope) return nullptr;
    return qt_contract_legs(E, e, 1, *ope, 0, true, 0, 1, err);
  }

  // Plan operands of the one-site centre c: the move2right form
  // (L~_c or the left edge, right block c+1) for c < L-1, and
  // (left block L-2, right edge) at c = L-1.
  struct Form {
    QTPtr lop, rop;
    int ln = 0, rn = 0;
  };
  int form_at(int cc, const QTPtr& W, const QTPtr& le, const QTPtr& re,
              const std::vector<QTPtr>& ev, Form& F) {
    if (cc < L - 1) {
      F.lop = cc == 0 ? le : (ev[cc - 1] ? fuse_left_of(*ev[cc - 1], *W) : nullptr);
      F.rop = ev[cc + 1];
      F.ln = cc == 0 ? 2 : 3;
      F.rn = 1;
    } else {
      F.lop = ev[L - 2];
      F.rop = re;
      F.ln = 2;
      F.rn = 1;
    }
    if (!F.lop || !F.rop) {
      if (err.empty()) err = "an environment of the centre is missing";
      return DMRGX_E_STATE;
    }
    return 0;
  }

  // centre tensor (any block order) -> the current plan's packed psi layout
  int to_plan(const QTensor& psi, double* dst) {
    const int f = c->f();
    if (psi.m.nleg() != (int)c->psi_dim.size()) {
      err = "centre tensor and plan disagree on the number of legs";
      return DMRGX_E_STATE;
    }
    std::map<std::vector<int>, int> at;
    for (size_t b = 0; b < psi.m.syms.size(); b++) at[psi.m.syms[b]] = (int)b;
    std::vector<GOut> go;
    std::vector<GSrc> gs;
    int64_t off = 0;
    for (auto& sym : c->psi_sym) {
      int64_t sz = 1;
      for (size_t l = 0; l < sym.size(); l++) sz *= c->psi_dim[l][sym[l]];
      auto it = at.find(sym);
      if (it != at.end() && sz > 0) {
        if (psi.bsize(it->second) != sz) {
          err = "centre block size differs from the plan's";
          return DMRGX_E_STATE;
        }
        GSrc g;
        std::memset(&g, 0, sizeof(g));
        g.src_off = psi.off[it->second];
        g.strides[0] = 1;
        g.sign = 1.0;
        gs.push_back(g);
        GOut o;
        std::memset(&o, 0, sizeof(o));
        o.dst_off = off;
        o.size = sz;
        o.rank = 1;
        o.dims[0] = (int32_t)sz;
        o.dst_strides[0] = 1;
        o.src_begin = (int32_t)gs.size() - 1;
        o.src_count = 1;
        go.push_back(o);
      }
      off += sz;
    }
    if (off != c->n) {
      err = "plan layout size mismatch";
      return DMRGX_E_STATE;
    }
    if (cudaMemsetAsync(dst, 0, sizeof(double) * std::max<int64_t>(1, c->n * f), E.stream) !=
            cudaSuccess ||
        launch_gather(psi.d, dst, go, gs, f == 2, E.stream) != cudaSuccess) {
      err = "centre relayout failed";
      return DMRGX_E_CUDA;
    }
    return 0;
  }

  // <psi|H|psi> / <psi|psi> at the centre with the given operators, and the
  // adjoints of the centre's Lop / Rop when asked
  int eval_center(const QTPtr& W, const QTPtr& le, const QTPtr& re, const std::vector<QTPtr>& ev,
                  bool want_l, bool want_r, Form& F, QTPtr& gl, QTPtr& gr, double& en,
                  double& nn) {
    int rc = form_at(center, W, le, re, ev, F);
    if (rc) return rc;
    rc = plan_build_device(c, *F.lop, *F.rop, F.ln, F.rn, sector, E.G);
    if (rc) return fail(rc);
    double* d = nullptr;
    if (dalloc(&d, (size_t)std::max<int64_t>(1, c->n * c->f()), E.stream) != cudaSuccess) {
      err = "centre allocation failed";
      return DMRGX_E_CUDA;
    }
    rc = to_plan(*cpsi, d);
    if (!rc) rc = heff_adjoint(c, E, *F.lop, *F.rop, d, want_l, want_r, gl, gr, en, nn, err);
    dfree(d, E.stream);
    return rc;
  }

  // SVD of the centre that drops no weight above the sweeps' cutoff
  int center_svd(int num, QTPtr& U, QTPtr& V, double& disc) {
    std::vector<double> s;
    if (qt_svd(E, *cpsi, num, m_cut, U, V, s, err)) return DMRGX_E_CUDA;
    disc = 0;
    for (size_t i = (size_t)std::min<int64_t>(m_cut, (int64_t)s.size()); i < s.size(); i++)
      disc += s[i] * s[i];
    return 0;
  }

  // move the one-site centre without changing the state: psi = U S V,
  // new site tensor, environment update, psi' = A_{c-1} (psi V^+)  or  (U^+ psi) B_{c+1}
  int move_left(double& disc) {
    const int c0 = center;
    const int nr = c0 == L - 1 ? 1 : 2;
    QTPtr U, V;
    int rc = center_svd(1, U, V, disc);
    if (rc) return rc;
    QTPtr rt = c0 == L - 1 ? redge : fuse_right_of(*env[c0 + 1], *bulk);
    if (!rt) return DMRGX_E_CUDA;
    env[c0] = right_update(*rt, *V, nr);
    site[c0] = V;
    auto Vc = qt_copy(E, *V);
    if (!Vc || qt_conjugate(E, *Vc)) return DMRGX_E_CUDA;
    QTPtr us = qt_contract_mat(E, *cpsi, *Vc, 'N', 'T', nr, err);
    if (!us || !env[c0]) return DMRGX_E_CUDA;
    QTPtr nxt = qt_contract_mat(E, *site[c0 - 1], *us, 'N', 'N', 1, err);
    if (!nxt) return DMRGX_E_CUDA;
    nxt->m.dirs.assign(nxt->m.nleg(), 0);
    cpsi = nxt;
    center = c0 - 1;
    return 0;
  }
  int move_right(double& disc, QTPtr lt) {
    const int c0 = center;
    const int nl = c0 == 0 ? 1 : 2;
    QTPtr U, V;
    int rc = center_svd(nl, U, V, disc);
    if (rc) return rc;
    if (!lt) lt = c0 == 0 ? ledge : fuse_left_of(*env[c0 - 1], *bulk);
    if (!lt) return DMRGX_E_CUDA;
    env[c0] = left_update(*lt, *U, nl);
    site[c0] = U;
    auto Uc = qt_copy(E, *U);
    if (!Uc || qt_conjugate(E, *Uc)) return DMRGX_E_CUDA;
    QTPtr sv = qt_contract_mat(E, *Uc, *cpsi, 'T', 'N', nl, err);
    if (!sv || !env[c0]) return DMRGX_E_CUDA;
    QTPtr nxt = qt_contract_mat(E, *sv, *site[c0 + 1], 'N', 'N', 1, err);
    if (!nxt) return DMRGX_E_CUDA;
    nxt->m.dirs.assign(nxt->m.nleg(), 0);
    cpsi = nxt;
    center = c0 + 1;
    return 0;
  }

  // environments of the centre rebuilt from the site tensors alone (the MPS),
  // for the MPO (W, le, re): left blocks 0..c-1, right blocks c+1..L-1
  int rebuild(const QTPtr& W, const QTPtr& le, const QTPtr& re, std::vector<QTPtr>& ev) {
    ev.assign(L, nullptr);
    const int cc = center;
    for (int k = 0; k < cc; k++) {
      if (!site[k]) {
        err = "site tensor missing";
        return DMRGX_E_STATE;
      }
      if (k == 0) {
        ev[0] = left_update(*le, *site[0], 1);
      } else {
        QTPtr lt = fuse_left_of(*ev[k - 1], *W);
        if (!lt) return DMRGX_E_CUDA;
        ev[k] = left_update(*lt, *site[k], 2);
      }
      if (!ev[k]) return DMRGX_E_CUDA;
    }
    for (int k = L - 1; k > cc; k--) {
      if (!site[k]) {
        err = "site tensor missing";
        return DMRGX_E_STATE;
      }
      if (k == L - 1) {
        ev[k] = right_update(*re, *site[k], 1);
      } else {
        QTPtr rt = fuse_right_of(*ev[k + 1], *W);
        if (!rt) return DMRGX_E_CUDA;
        ev[k] = right_update(*rt, *site[k], 2);
      }
      if (!ev[k]) return DMRGX_E_CUDA;
    }
    return 0;
  }

  // dE/dW_k for every site k by the adjoint of the centre's H_eff contraction:
  // the centre walks to the left edge, then across the chain; at each site the
  // MPO tensor sits in the centre's Lop (left edge, fused L~) or Rop (right edge).
  // gw[k]: the bulk MPO layout (edge gradients land in row D-1 / column 0).
  // checks: [0] final eigenvalue E0, [1] max |<psi|H|psi> - E0| over the centres,
  // [2] max_k |<dE/dW_k, W_k> - E0| (E is linear in each W_k), [3] max discarded weight.
  int adjoint(bool recompute, const std::vector<double>& w_host,
              std::vector<std::vector<double>>& gw, double* checks) {
    if (pbc) {
      err = "adjoint: periodic chains are not supported";
      return DMRGX_E_STATE;
    }
    if (center < 0 || !cpsi) {
      err = "adjoint: the last step left no one-site centre (the schedule must end with a move)";
      return DMRGX_E_STATE;
    }
    const int f = c->f();
    const double e0 = energies.empty() ? 0.0 : energies[energies.size() - 6];
    double edev = 0, wdev = 0, disc = 0;
    int rc;
    if (recompute) {
      std::vector<QTPtr> ev;
      for (auto& e : env) e.reset();  // drop the stored environments first
      if ((rc = rebuild(bulk, ledge, redge, ev))) return rc;
      env = ev;
    }
    gw.assign(L, std::vector<double>((size_t)(bulk->total() * f), 0.0));
    Form F;
    QTPtr gl, gr;
    double en = 0, nn = 1, d = 0;
    if ((rc = eval_center(bulk, ledge, redge, env, false, false, F, gl, gr, en, nn))) return rc;
    edev = std::fabs(en - e0);
    while (center > 0) {
      if ((rc = move_left(d))) return rc;
      disc = std::max(disc, d);
      if (center > 0) {
        if ((rc = eval_center(bulk, ledge, redge, env, false, false, F, gl, gr, en, nn))) return rc;
        edev = std::max(edev, std::fabs(en - e0));
      }
    }
    for (;;) {
      const int cc = center;
      const bool last = cc == L - 1;
      if ((rc = eval_center(bulk, ledge, redge, env, !last, last, F, gl, gr, en, nn))) return rc;
      edev = std::max(edev, std::fabs(en - e0));
      if (last) rc = edge_adjoint(*gr, *bulk, true, gw[cc], E.stream, err);
      else if (cc == 0) rc = edge_adjoint(*gl, *bulk, false, gw[cc], E.stream, err);
      else rc = fusion_adjoint(E, *env[cc - 1], *bulk, *gl, false, gw[cc], err);
      if (rc) return rc;
      for (auto& v : gw[cc]) v /= nn;
      // <dE/dW_k, W_k> = E
      double sr = 0;
      for (size_t w = 0; w < w_host.size() / f; w++)
        sr += f == 2 ? gw[cc][2 * w] * w_host[2 * w] - gw[cc][2 * w + 1] * w_host[2 * w + 1]
                     : gw[cc][w] * w_host[w];
      wdev = std::max(wdev, std::fabs(sr - e0));
      if (last) break;
      if ((rc = move_right(d, cc == 0 ? ledge : F.lop))) return rc;
      disc = std::max(disc, d);
    }
    if (checks) {
      checks[0] = e0;
      checks[1] = edev;
      checks[2] = wdev;
      checks[3] = disc;
    }
    return 0;
  }

  // <Psi|H(W)|Psi> of the current state for another MPO of the same shape
  int expect(const QTPtr& W, const QTPtr& le, const QTPtr& re, double& value) {
    if (pbc) {
      err = "expect: periodic chains are not supported";
      return DMRGX_E_STATE;
    }
    if (center < 0 || !cpsi) {
      err = "expect: no state (run dmrg first)";
      return DMRGX_E_STATE;
    }
    std::vector<QTPtr> ev;
    int rc = rebuild(W, le, re, ev);
    if (rc) return rc;
    Form F;
    QTPtr gl, gr;
    double nn = 1;
    return eval_center(W, le, re, ev, false, false, F, gl, gr, value, nn);
  }

  // the reference schedule dmrg() (src/functions.cpp:157-227)
  // one site step with its wall time recorded
  template <class F>
  int timed(F&& f) {
    const double t0 = now();
    const double before[5] = {t_eig, t_svd, t_env, t_fuse, t_plan};
    const int r = f();
    if (!r) {
      step_s.push_back(now() - t0);
      const double after[5] = {t_eig, t_svd, t_env, t_fuse, t_plan};
      for (int q = 0; q < 5; q++) step_split.push_back(after[q] - before[q]);
    }
    return r;
  }

  int dmrg(int cutoff, int sweep) {
    int pre_cutoff = 10;
    if (sweep == -1) pre_cutoff = cutoff;
    const int pre_sweep = cutoff / 100;
    int rc = timed([&] { return two_sites(0, L - 1, cutoff * 10); });
    if (rc) return rc;
    for (int i = 1; i < L / 2; i++)
      if ((rc = timed([&] { return update_two(i, L - i - 1, pre_cutoff); }))) return rc;
    if (sweep != -1)
      for (int i = L / 2; i < L - 1; i++)
        if ((rc = timed([&] { return move2right(i, i + 1, pre_cutoff); }))) return rc;
    if (sweep != -1)
      for (int s = 0; s < pre_sweep - 1; s++) {
        for (int i = L - 2; i > 0; i--)
          if ((rc = timed([&] { return move2left(i - 1, i, 100 * (s + 1)); }))) return rc;
        for (int i = 1; i < L - 1; i++)
          if ((rc = timed([&] { return move2right(i, i + 1, 100 * (s + 1)); }))) return rc;
      }
    for (int s = 0; s < sweep; s++) {
      for (int i = L - 2; i > 0; i--)
        if ((rc = timed([&] { return move2left(i - 1, i, cutoff); }))) return rc;
      for (int i = 1; i < L - 1; i++)
        if ((rc = timed([&] { return move2right(i, i + 1, cutoff); }))) return rc;
    }
    if (sweep != -1)
      for (int i = L - 2; i >= L / 2; i--)
        if ((rc = timed([&] { return move2left(i - 1, i, cutoff); }))) return rc;
    return 0;
  }
};

int model_nparams(int model) { return model == 0 ? 3 : 4; }

std::vector<double> flatten(const HostQT& W, int f) {
  std::vector<double> v;
  for (auto& b : W.blocks)
    for (auto& x : b) {
      v.push_back(x.real());
      if (f == 2) v.push_back(x.imag());
    }
  return v;
}

// the three device MPO tensors of a parameter set: bulk, left edge, right edge
// (left() = take(0, D-1), right() = take(2, 0).exchange(0, 1), src/qtensor.cpp:449-463)
bool mpo_set(int model, const double* par, int f, cudaStream_t st, QTPtr& bulk, QTPtr& le,
             QTPtr& re, HostQT* host, std::string& err) {
  HostQT W;
  if (!build_mpo(model, par, W)) {
    err = "unknown model";
    return false;
  }
  const int D = W.m.dims[0][0];
  bulk = upload(W, f, st, err);
  le = upload(take(W, 0, D - 1), f, st, err);
  re = upload(exchange(take(W, 2, 0), 0, 1), f, st, err);
  if (host) *host = W;
  return bulk && le && re;
}

void free_run(void* p) { delete static_cast<Run*>(p); }

// A run with the model's MPO on the context's device: what dmrgx_dmrg and
// dmrgx_load_state share.  nullptr (err set) on bad arguments.
Run* make_run(dmrgx_ctx* c, int model, int L, int m, int sector, const double* params,
              int nparams, std::string& err) {
  if (model < 0 || model > 3) {
    err = "unknown model";
    return nullptr;
  }
  const bool real_model = model == 0 || model == 3;
  if (real_model != (c->dtype == DMRGX_F64)) {
    err = "Kitaev and real XYZ run on F64 contexts, XYZ and Potts on C128";
    return nullptr;
  }
  Run* R = new Run;
  R->c = c;
  R->L = L;
  R->sector = sector;
  R->m_cut = m;
  R->model = model;
  R->E.stream = c->stream;
  R->E.device = c->device;
  R->E.num_sms = c->num_sms;
  R->E.f = c->f();
  R->par.assign(8, 0.0);
  for (int i = 0; i < nparams && i < 8; i++) R->par[i] = params[i];
  R->E.G.n = model == 2 ? 3 : 2;
  R->E.G.fermion = model == 0;
  cudaSetDevice(c->device);
  if (!mpo_set(model, R->par.data(), c->f(), c->stream, R->bulk, R->ledge, R->redge, nullptr,
               err)) {
    delete R;
    return nullptr;
  }
  R->env.assign(L, nullptr);
  R->site.assign(L, nullptr);
  return R;
}

// ---------------------------------------------------------------- checkpoint
// Text form of a block-sparse tensor: metadata lines (legs and blocks; sector
// sizes per leg; directions; block labels), then one line per block in the
// reference's tensor::write_file format (src/tensor.cpp:249-257: the number of
// indices, the extents, the values, 32 significant digits; complex values as
// "(re,im)", std::complex's stream form), which tensor::read_file
// (src/tensor.cpp:260-271) reads back.
bool write_qt(std::ostream& o, const QTensor& T, cudaStream_t st) {
  const QMeta& m = T.m;
  std::vector<double> v((size_t)T.total() * T.f);
  if (!v.empty() &&
      (cudaMemcpyAsync(v.data(), T.d, sizeof(double) * v.size(), cudaMemcpyDeviceToHost, st) !=
           cudaSuccess ||
       cudaStreamSynchronize(st) != cudaSuccess))
    return false;
  o << m.nleg() << " " << m.syms.size() << "\n";
  for (auto& d : m.dims) {
    o << d.size();
    for (int x : d) o << " " << x;
    o << "\n";
  }
  for (int l = 0; l < m.nleg(); l++) o << (l ? " " : "") << m.dirs[l];
  o << "\n";
  for (auto& sy : m.syms) {
    for (int l = 0; l < m.nleg(); l++) o << (l ? " " : "") << sy[l];
    o << "\n";
  }
  o.precision(32);
  for (size_t b = 0; b < m.syms.size(); b++) {
    o << m.nleg();
    for (int l = 0; l < m.nleg(); l++) o << " " << m.dims[l][m.syms[b][l]];
    for (int64_t i = T.off[b]; i < T.off[b + 1]; i++) {
      if (T.f == 2) o << " " << std::complex<double>(v[2 * i], v[2 * i + 1]);
      else o << " " << v[i];
    }
    o << "\n";
  }
  return (bool)o;
}

QTPtr read_qt(std::istream& in, int f, cudaStream_t st, std::string& err) {
  auto T = std::make_shared<QTensor>();
  QMeta& m = T->m;
  int nleg = 0;
  int64_t nblk = 0;
  if (!(in >> nleg >> nblk) || nleg < 1 || nleg > 8 || nblk < 0 || nblk > (1 << 24)) {
    err = "bad tensor header";
    return nullptr;
  }
  m.dims.resize(nleg);
  for (auto& d : m.dims) {
    int ns = 0;
    if (!(in >> ns) || ns < 0 || ns > 4096) {
      err = "bad sector count";
      return nullptr;
    }
    d.resize(ns);
    for (int& x : d)
      if (!(in >> x) || x < 0) {
        err = "bad sector size";
        return nullptr;
      }
  }
  m.dirs.resize(nleg);
  for (int& x : m.dirs)
    if (!(in >> x)) {
      err = "bad direction";
      return nullptr;
    }
  m.syms.assign((size_t)nblk, std::vector<int>(nleg));
  for (auto& sy : m.syms)
    for (int l = 0; l < nleg; l++)
      if (!(in >> sy[l]) || sy[l] < 0 || sy[l] >= (int)m.dims[l].size()) {
        err = "bad block label";
        return nullptr;
      }
  T->f = f;
  if (T->alloc(st) != cudaSuccess) {
    err = "allocation failed";
    return nullptr;
  }
  std::vector<double> v((size_t)T->total() * f);
  for (int64_t b = 0; b < nblk; b++) {
    int n = 0;
    if (!(in >> n) || n != nleg) {
      err = "block index count differs from the tensor's legs";
      return nullptr;
    }
    for (int l = 0; l < nleg; l++) {
      int e = 0;
      if (!(in >> e) || e != m.dims[l][m.syms[b][l]]) {
        err = "block extent differs from its sector size";
        return nullptr;
      }
    }
    for (int64_t i = T->off[b]; i < T->off[b + 1]; i++) {
      if (f == 2) {
        std::complex<double> z;
        if (!(in >> z)) {
          err = "bad complex value";
          return nullptr;
        }
        v[2 * i] = z.real();
        v[2 * i + 1] = z.imag();
      } else if (!(in >> v[i])) {
        err = "bad value";
        return nullptr;
      }
    }
  }
  if (!v.empty() &&
      (cudaMemcpyAsync(T->d, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice, st) !=
           cudaSuccess ||
       cudaStreamSynchronize(st) != cudaSuccess)) {
    err = "upload failed";
    return nullptr;
  }
  return T;
}

}  // namespace
}  // namespace dmrgx

using namespace dmrgx;

extern "C" int dmrgx_dmrg(dmrgx_ctx* c, int model, int L, int m, int sweeps, int sector,
                          const double* params, int nparams, double* energies, double* trunc,
                          int* steps_lr, int64_t* matvecs, int64_t cap, int64_t* nsteps,
                          double* seconds) {
  if (!c || !params || !nsteps || L < 4) {
    set_error("dmrg: bad arguments (need a context, parameters and L >= 4)");
    return DMRGX_E_ARG;
  }
  if (c->run_free) c->run_free(c->run);
  c->run = nullptr;
  c->run_free = nullptr;
  std::string err;
  Run* R = make_run(c, model, L, m, sector, params, nparams, err);
  if (!R) {
    set_error("dmrg: " + err);
    return DMRGX_E_ARG;
  }
  R->eig_nev = c->eig_nev;
  R->eig_ncv = c->eig_ncv;
  R->predict = c->predict;
  if (c->boundary == DMRGX_BOUNDARY_PERIODIC) {
    // the drivers' edge operators: kitaev.cpp:42-45 H_Kitaev(t, -p, 0),
    // xyz.cpp:39-42 H_XYZ(jx, jy, jz) (no field), potts.cpp:44-47 H_Potts3(0, j, p, t)
    std::vector<double> ep(R->par);
    if (model == 0) {
      ep[1] = -ep[1];
      ep[2] = 0.0;
    } else if (model == 2) {
      ep[0] = 0.0;
    } else {
      ep[3] = 0.0;
    }
    QTPtr eb, el, er;
    if (!mpo_set(model, ep.data(), c->f(), c->stream, eb, el, er, nullptr, err)) {
      delete R;
      set_error("dmrg: edge operators: " + err);
      return DMRGX_E_CUDA;
    }
    R->pbc = true;
    R->edge.assign(L, nullptr);
    R->edge[0] = el;
    R->edge[L - 1] = er;
  }
  for (double& x : c->t_plan_part) x = 0.0;
  const double t0 = Run::now();
  int rc = R->dmrg(m, sweeps);
  const double t1 = Run::now();
  if (rc) {
    set_error("dmrg: " + R->err);
    delete R;
    return rc;
  }
  const int64_t ns = (int64_t)R->trunc.size();
  *nsteps = ns;
  for (int64_t i = 0; i < ns && i < cap; i++) {
    if (energies)
      for (int q = 0; q < 6; q++) energies[6 * i + q] = R->energies[6 * i + q];
    if (trunc) trunc[i] = R->trunc[i];
    if (steps_lr) {
      steps_lr[2 * i] = R->lr[2 * i];
      steps_lr[2 * i + 1] = R->lr[2 * i + 1];
    }
    if (matvecs) matvecs[i] = R->matvecs[i];
  }
  if (seconds) {
    seconds[0] = t1 - t0;
    seconds[1] = R->t_eig;
    seconds[2] = R->t_svd;
    seconds[3] = R->t_env;
    seconds[4] = R->t_fuse;
  }
  c->run = R;  // the final state stays for dmrgx_adjoint / dmrgx_expect
  c->run_free = free_run;
  return 0;
}

extern "C" int dmrgx_adjoint(dmrgx_ctx* c, int recompute, double* dE_dparams, int nparams,
                             double* dE_dW, int64_t w_cap, int64_t* w_len, double* checks,
                             double* seconds) {
  if (!c || !c->run) {
    set_error("adjoint: no state (run dmrgx_dmrg on this context first)");
    return DMRGX_E_STATE;
  }
  Run* R = static_cast<Run*>(c->run);
  const int f = c->f();
  const int np = model_nparams(R->model);
  if (nparams < 0 || nparams > np) {
    set_error("adjoint: the model has fewer parameters than asked for");
    return DMRGX_E_ARG;
  }
  const int64_t wl = R->bulk->total() * f;
  if (w_len) *w_len = wl;
  if (dE_dW && w_cap < (int64_t)R->L * wl) {
    set_error("adjoint: dE_dW needs L * w_len doubles");
    return DMRGX_E_ARG;
  }
  cudaSetDevice(c->device);
  HostQT W0;
  std::string err;
  build_mpo(R->model, R->par.data(), W0);
  const std::vector<double> w0 = flatten(W0, f);
  const int prec = c->prec;
  c->prec = DMRGX_PREC_FP64;  // the adjoint runs on the FP64 plan only
  std::vector<std::vector<double>> gw;
  const double t0 = Run::now();
  R->err.clear();
  int rc = R->adjoint(recompute != 0, w0, gw, checks);
  const double t1 = Run::now();
  c->prec = prec;
  if (rc) {
    set_error("adjoint: " + R->err);
    return rc;
  }
  if (dE_dW)
    for (int k = 0; k < R->L; k++) std::copy(gw[k].begin(), gw[k].end(), dE_dW + (int64_t)k * wl);
  // dE/dp = sum_k <dE/dW_k, dW/dp>; W is affine in every parameter but the Potts
  // angles, which take a central difference of the MPO entries (step 1e-5)
  for (int p = 0; p < nparams; p++) {
    const bool affine = !(R->model == 2 && p >= 2);
    const double h = affine ? 1.0 : 1e-5;
    std::vector<double> pp = R->par, pm = R->par;
    pp[p] += h;
    if (!affine) pm[p] -= h;
    HostQT Wp, Wm;
    build_mpo(R->model, pp.data(), Wp);
    build_mpo(R->model, pm.data(), Wm);
    const std::vector<double> vp = flatten(Wp, f), vm = flatten(Wm, f);
    const double den = affine ? h : 2 * h;
    double acc = 0;
    for (int k = 0; k < R->L; k++)
      for (size_t w = 0; w < vp.size() / f; w++) {
        if (f == 2) {
          const double dr = (vp[2 * w] - vm[2 * w]) / den, di = (vp[2 * w + 1] - vm[2 * w + 1]) / den;
          acc += gw[k][2 * w] * dr - gw[k][2 * w + 1] * di;
        } else {
          acc += gw[k][w] * (vp[w] - vm[w]) / den;
        }
      }
    dE_dparams[p] = acc;
  }
  if (seconds) seconds[0] = t1 - t0;
  return 0;
}

extern "C" int dmrgx_expect(dmrgx_ctx* c, const double* params, int nparams, double* value) {
  if (!c || !c->run || !params || !value) {
    set_error("expect: bad arguments or no state (run dmrgx_dmrg first)");
    return DMRGX_E_ARG;
  }
  Run* R = static_cast<Run*>(c->run);
  std::vector<double> par(8, 0.0);
  for (int i = 0; i < nparams && i < 8; i++) par[i] = params[i];
  cudaSetDevice(c->device);
  QTPtr W, le, re;
  std::string err;
  if (!mpo_set(R->model, par.data(), c->f(), c->stream, W, le, re, nullptr, err)) {
    set_error("expect: " + err);
    return DMRGX_E_CUDA;
  }
  const int prec = c->prec;
  c->prec = DMRGX_PREC_FP64;
  R->err.clear();
  int rc = R->expect(W, le, re, *value);
  c->prec = prec;
  if (rc) {
    set_error("expect: " + R->err);
    return rc;
  }
  return 0;
}

extern "C" int dmrgx_svd(dmrgx_ctx* c, const int* meta, const void* vals, int num, int cutoff,
                         int group_n, int fermion, int64_t* sizes) {
  if (!c || !meta || !vals || !sizes) {
    set_error("svd: null argument");
    return DMRGX_E_ARG;
  }
  Engine E;
  E.stream = c->stream;
  E.device = c->device;
  E.num_sms = c->num_sms;
  E.f = c->f();
  if (!make_group(group_n, fermion, E.G)) {
    set_error("svd: group_n must be >= 1 or DMRGX_GROUP_Z2CUBED");
    return DMRGX_E_ARG;
  }
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) {
    set_error(std::string("svd: ") + cudaGetErrorString(e));
    return DMRGX_E_CUDA;
  }
  std::string err;
  QTPtr A = qt_from_host(E, meta, vals, err);
  if (!A) {
    set_error("svd: " + err);
    return DMRGX_E_ARG;
  }
  QTPtr U, V;
  std::vector<double> sv;
  if (qt_svd(E, *A, num, cutoff, U, V, sv, err)) {
    set_error("svd: " + err);
    return err.rfind("svd: the number", 0) == 0 ? DMRGX_E_ARG : DMRGX_E_CUDA;
  }
  if (qt_to_host(*U, c->svd_um, c->svd_uv, c->stream) ||
      qt_to_host(*V, c->svd_vm, c->svd_vv, c->stream)) {
    set_error("svd: copy of the results failed");
    return DMRGX_E_CUDA;
  }
  c->svd_s = sv;
  sizes[0] = (int64_t)c->svd_um.size();
  sizes[1] = (int64_t)c->svd_uv.size() / c->f();
  sizes[2] = (int64_t)c->svd_vm.size();
  sizes[3] = (int64_t)c->svd_vv.size() / c->f();
  sizes[4] = (int64_t)c->svd_s.size();
  return 0;
}

extern "C" int dmrgx_svd_result(dmrgx_ctx* c, int* u_meta, void* u_vals, int* v_meta,
                                void* v_vals, double* s) {
  if (!c) {
    set_error("svd_result: null context");
    return DMRGX_E_ARG;
  }
  if (c->svd_um.empty()) {
    set_error("svd_result: no dmrgx_svd result on this context");
    return DMRGX_E_STATE;
  }
  if (u_meta) std::memcpy(u_meta, c->svd_um.data(), sizeof(int) * c->svd_um.size());
  if (u_vals) std::memcpy(u_vals, c->svd_uv.data(), sizeof(double) * c->svd_uv.size());
  if (v_meta) std::memcpy(v_meta, c->svd_vm.data(), sizeof(int) * c->svd_vm.size());
  if (v_vals) std::memcpy(v_vals, c->svd_vv.data(), sizeof(double) * c->svd_vv.size());
  if (s) std::memcpy(s, c->svd_s.data(), sizeof(double) * c->svd_s.size());
  return 0;
}

extern "C" int dmrgx_singular(dmrgx_ctx* c, double* entropy, double* s20, int* nsv, int64_t cap,
                              int64_t* nsteps) {
  if (!c || !c->run || !nsteps) {
    set_error("singular: no finished dmrgx_dmrg run on this context");
    return DMRGX_E_STATE;
  }
  Run* R = static_cast<Run*>(c->run);
  const int64_t ns = (int64_t)R->entropy.size();
  *nsteps = ns;
  for (int64_t i = 0; i < ns && i < cap; i++) {
    if (entropy) entropy[i] = R->entropy[i];
    if (nsv) nsv[i] = R->nsv[i];
    if (s20)
      for (int q = 0; q < kSingularRow; q++) s20[kSingularRow * i + q] = R->sv[kSingularRow * i + q];
  }
  return 0;
}

extern "C" int dmrgx_step_split(dmrgx_ctx* c, double* out, int64_t cap, int64_t* nsteps) {
  if (!c || !c->run || !nsteps) {
    set_error("step_split: no finished dmrgx_dmrg run on this context");
    return DMRGX_E_STATE;
  }
  Run* R = static_cast<Run*>(c->run);
  const int64_t ns = (int64_t)R->step_s.size();
  *nsteps = ns;
  for (int64_t i = 0; i < ns && i < cap && out; i++)
    for (int q = 0; q < 5; q++) out[5 * i + q] = R->step_split[5 * i + q];
  return 0;
}

extern "C" int dmrgx_step_seconds(dmrgx_ctx* c, double* out, int64_t cap, int64_t* nsteps) {
  if (!c || !c->run || !nsteps) {
    set_error("step_seconds: no state (run dmrgx_dmrg on this context first)");
    return DMRGX_E_STATE;
  }
  const Run* R = static_cast<const Run*>(c->run);
  *nsteps = (int64_t)R->step_s.size();
  for (int64_t i = 0; out && i < *nsteps && i < cap; i++) out[i] = R->step_s[i];
  return 0;
}

extern "C" int dmrgx_run_seconds(dmrgx_ctx* c, double* out, int cap) {
  if (!c || !c->run || !out || cap < 6) {
    set_error("run_seconds: need a context with a dmrgx_dmrg state and 6 slots");
    return DMRGX_E_ARG;
  }
  const Run* R = static_cast<const Run*>(c->run);
  double tot = 0;
  for (double x : R->step_s) tot += x;
  out[0] = tot;
  out[1] = R->t_eig;
  out[2] = R->t_svd;
  out[3] = R->t_env;
  out[4] = R->t_fuse;
  out[5] = R->t_plan;
  for (int q = 0; q < 4 && 6 + q < cap; q++) out[6 + q] = c->t_plan_part[q];
  return 0;
}

extern "C" int dmrgx_save_state(dmrgx_ctx* c, const char* path) {
  if (!c || !path) {
    set_error("save_state: null argument");
    return DMRGX_E_ARG;
  }
  if (!c->run) {
    set_error("save_state: no state (run dmrgx_dmrg or dmrgx_load_state first)");
    return DMRGX_E_STATE;
  }
  Run* R = static_cast<Run*>(c->run);
  if (R->pbc) {
    set_error("save_state: periodic chains are not supported");
    return DMRGX_E_STATE;
  }
  if (R->center < 0 || !R->cpsi) {
    set_error("save_state: the last step left no one-site centre");
    return DMRGX_E_STATE;
  }
  std::ofstream o(path);
  if (!o) {
    set_error(std::string("save_state: cannot open ") + path);
    return DMRGX_E_ARG;
  }
  const double e0 = R->energies.empty() ? 0.0 : R->energies[R->energies.size() - 6];
  o.precision(17);
  o << "dmrgx-mps 1\n";
  o << "model " << R->model << " L " << R->L << " sector " << R->sector << " m " << R->m_cut
    << " center " << R->center << " f " << c->f() << " energy " << e0 << "\n";
  o << "params " << R->par.size();
  for (double p : R->par) o << " " << p;
  o << "\n";
  bool ok = true;
  for (int k = 0; k < R->L && ok; k++) {
    if (k == R->center || !R->site[k]) continue;
    o << "site " << k << "\n";
    ok = write_qt(o, *R->site[k], c->stream);
    o.precision(17);
  }
  if (ok) {
    o << "centre\n";
    ok = write_qt(o, *R->cpsi, c->stream);
  }
  o << "end\n";
  if (!ok || !o) {
    set_error(std::string("save_state: writing ") + path + " failed");
    return DMRGX_E_CUDA;
  }
  return 0;
}

extern "C" int dmrgx_load_state(dmrgx_ctx* c, const char* path) {
  if (!c || !path) {
    set_error("load_state: null argument");
    return DMRGX_E_ARG;
  }
  std::ifstream in(path);
  if (!in) {
    set_error(std::string("load_state: cannot open ") + path);
    return DMRGX_E_ARG;
  }
  std::string tag, k1, k2, k3, k4, k5, k6, k7;
  int ver = 0, model = -1, L = 0, sector = 0, m = 0, center = -1, f = 0, np = 0;
  double e0 = 0;
  if (!(in >> tag >> ver) || tag != "dmrgx-mps" || ver != 1 ||
      !(in >> k1 >> model >> k2 >> L >> k3 >> sector >> k4 >> m >> k5 >> center >> k6 >> f >>
        k7 >> e0) ||
      k1 != "model" || k2 != "L" || k3 != "sector" || k4 != "m" || k5 != "center" ||
      k6 != "f" || k7 != "energy" || !(in >> tag >> np) || tag != "params" ||
      np < 0 || np > 8 || L < 4 || center < 0 || center >= L) {
    set_error("load_state: not a dmrgx state file (bad header)");
    return DMRGX_E_ARG;
  }
  if (f != c->f()) {
    set_error("load_state: element type of the file differs from the context's");
    return DMRGX_E_ARG;
  }
  std::vector<double> par((size_t)np);
  for (double& p : par)
    if (!(in >> p)) {
      set_error("load_state: bad parameters");
      return DMRGX_E_ARG;
    }
  std::string err;
  Run* R = make_run(c, model, L, m, sector, par.data(), np, err);
  if (!R) {
    set_error("load_state: " + err);
    return DMRGX_E_ARG;
  }
  int rc = 0;
  for (;;) {
    if (!(in >> tag)) {
      err = "truncated file";
      break;
    }
    if (tag == "end") break;
    if (tag == "site") {
      int k = -1;
      if (!(in >> k) || k < 0 || k >= L) {
        err = "bad site index";
        break;
      }
      R->site[k] = read_qt(in, f, c->stream, err);
      if (!R->site[k]) break;
    } else if (tag == "centre") {
      R->cpsi = read_qt(in, f, c->stream, err);
      if (!R->cpsi) break;
    } else {
      err = "unknown record " + tag;
      break;
    }
  }
  if (tag == "end" && err.empty() && !R->cpsi) err = "no centre tensor";
  if (tag == "end" && err.empty()) {
    R->center = center;
    R->energies.assign(6, 0.0);
    R->energies[0] = e0;
    std::vector<QTPtr> ev;
    rc = R->rebuild(R->bulk, R->ledge, R->redge, ev);
    if (!rc) R->env = ev;
    else err = R->err;
  }
  if (!err.empty() || rc) {
    delete R;
    set_error("load_state: " + (err.empty() ? std::string("environment rebuild failed") : err));
    return rc ? rc : DMRGX_E_ARG;
  }
  if (c->run_free) c->run_free(c->run);
  c->run = R;
  c->run_free = free_run;
  return 0;
}
