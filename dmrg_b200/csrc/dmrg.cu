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
#include <string>
#include <vector>

#include "../../include/dmrgx.h"
#include "ctx.h"
#include "qtensor.h"

namespace dmrgx {

int plan_build_device(dmrgx_ctx* c, const QTensor& L, const QTensor& R, int l_num, int r_num,
                      int sector, const Group& G);

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
    const double jx = par[0], jy = par[1], jz = par[2];
    W.m.dims = {{5}, {1, 1}, {5}, {1, 1}};
    W.m.dirs = {0, 0, 0, 0};
    W.add_block({0, 0, 0, 0}, {5, 1, 5, 1});
    W.set(5, 0, 0, 1); W.set(5, 3, 0, 1); W.set(5, 4, 3, jz); W.set(5, 4, 4, 1);
    W.add_block({0, 0, 0, 1}, {5, 1, 5, 1});
    W.set(5, 1, 0, 1); W.set(5, 2, 0, -I); W.set(5, 4, 1, jx); W.set(5, 4, 2, -I * jy);
    W.add_block({0, 1, 0, 0}, {5, 1, 5, 1});
    W.set(5, 1, 0, 1); W.set(5, 2, 0, I); W.set(5, 4, 1, jx); W.set(5, 4, 2, I * jy);
    W.add_block({0, 1, 0, 1}, {5, 1, 5, 1});
    W.set(5, 0, 0, 1); W.set(5, 3, 0, -1); W.set(5, 4, 3, -jz); W.set(5, 4, 4, 1);
    return true;
  }
  if (model == 3) {
    const double jx = par[0], jy = par[1], jz = par[2];
    W.m.dims = {{5}, {1, 1}, {5}, {1, 1}};
    W.m.dirs = {0, 0, 0, 0};
    W.add_block({0, 0, 0, 0}, {5, 1, 5, 1});
    W.set(5, 0, 0, 1); W.set(5, 3, 0, 1); W.set(5, 4, 3, jz); W.set(5, 4, 4, 1);
    W.add_block({0, 0, 0, 1}, {5, 1, 5, 1});
    W.set(5, 1, 0, 1); W.set(5, 2, 0, 1); W.set(5, 4, 1, jx); W.set(5, 4, 2, -jy);
    W.add_block({0, 1, 0, 0}, {5, 1, 5, 1});
    W.set(5, 1, 0, 1); W.set(5, 2, 0, -1); W.set(5, 4, 1, jx); W.set(5, 4, 2, jy);
    W.add_block({0, 1, 0, 1}, {5, 1, 5, 1});
    W.set(5, 0, 0, 1); W.set(5, 3, 0, -1); W.set(5, 4, 3, -jz); W.set(5, 4, 4, 1);
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

struct Run {
  dmrgx_ctx* c;
  Engine E;
  int L;
  QTPtr bulk, ledge, redge;  // mpo[i], mpo[0], mpo[L-1]
  std::vector<QTPtr> env;    // mps(i): block environments
  int sector;
  // per-step records
  std::vector<int> lr;
  std::vector<double> energies, trunc;
  std::vector<int64_t> matvecs;
  double t_eig = 0, t_svd = 0, t_env = 0, t_fuse = 0;
  std::string err;

  const QTensor& mpo(int i) const { return i == 0 ? *ledge : (i == L - 1 ? *redge : *bulk); }

  static double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
  }

  // lowest state of the current plan -> psi tensor; records energies
  int solve(int l, int r, QTPtr& psi) {
    const double t0 = now();
    std::vector<double> ev(6);
    std::vector<double> vec((size_t)c->n * c->f());
    int64_t info[6];
    int rc = dmrgx_eigsolve(c, 6, 0, 1e-10, 0, nullptr, ev.data(), vec.data(), info);
    if (rc) {
      err = std::string("eigsolve: ") + dmrgx_last_error();
      return rc;
    }
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
    cudaMemcpyAsync(psi->d, vec.data(), sizeof(double) * vec.size(), cudaMemcpyHostToDevice,
                    E.stream);
    cudaStreamSynchronize(E.stream);
    lr.push_back(l);
    lr.push_back(r);
    for (int q = 0; q < 6; q++) energies.push_back(q < (int)std::min<int64_t>(6, c->n) ? ev[q] : 0.0);
    matvecs.push_back(info[0]);
    t_eig += now() - t0;
    return 0;
  }

  int svd(const QTensor& psi, int num, int cutoff, QTPtr& U, QTPtr& V) {
    const double t0 = now();
    std::vector<double> s;
    if (qt_svd(E, psi, num, cutoff, U, V, s, err)) return DMRGX_E_CUDA;
    // truncation error of print_singular (src/useful.cpp:97-101)
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

  // src/core.cpp:88-172
  int two_sites(int l, int r, int cutoff) {
    const QTensor& le = mpo(l);
    const QTensor& re = mpo(r);
    int rc = plan_build_device(c, le, re, 2, 1, sector, E.G);
    if (rc) return fail(rc);
    QTPtr psi, U, V;
    if ((rc = solve(l, r, psi))) return rc;
    if ((rc = svd(*psi, 1, cutoff, U, V))) return rc;
    env[l] = left_update(le, *U, 1);
    env[r] = right_update(re, *V, 1);
    return env[l] && env[r] ? 0 : DMRGX_E_CUDA;
  }
  // src/core.cpp:182-283
  int update_two(int l, int r, int cutoff) {
    QTPtr le = fuse_left(l), re = fuse_right(r);
    if (!le || !re) return DMRGX_E_CUDA;
    int rc = plan_build_device(c, *le, *re, 3, 2, sector, E.G);
    if (rc) return fail(rc);
    QTPtr psi, U, V;
    if ((rc = solve(l, r, psi))) return rc;
    if ((rc = svd(*psi, 2, cutoff, U, V))) return rc;
    env[l] = left_update(*le, *U, 2);
    env[r] = right_update(*re, *V, 2);
    return env[l] && env[r] ? 0 : DMRGX_E_CUDA;
  }
  // src/core.cpp:293-378
  int move2right(int l, int r, int cutoff) {
    QTPtr le = fuse_left(l);
    if (!le) return DMRGX_E_CUDA;
    int rc = plan_build_device(c, *le, *env[r], 3, 1, sector, E.G);
    if (rc) return fail(rc);
    QTPtr psi, U, V;
    if ((rc = solve(l, r, psi))) return rc;
    if ((rc = svd(*psi, 2, cutoff, U, V))) return rc;
    env[l] = left_update(*le, *U, 2);
    return env[l] ? 0 : DMRGX_E_CUDA;
  }
  // src/core.cpp:388-474
  int move2left(int l, int r, int cutoff) {
    QTPtr re = fuse_right(r);
    if (!re) return DMRGX_E_CUDA;
    int rc = plan_build_device(c, *env[l], *re, 2, 2, sector, E.G);
    if (rc) return fail(rc);
    QTPtr psi, U, V;
    if ((rc = solve(l, r, psi))) return rc;
    if ((rc = svd(*psi, 1, cutoff, U, V))) return rc;
    env[r] = right_update(*re, *V, 2);
    return env[r] ? 0 : DMRGX_E_CUDA;
  }
  int fail(int rc) {
    err = std::string("plan: ") + dmrgx_last_error();
    return rc;
  }

  // the reference schedule dmrg() (src/functions.cpp:157-227)
  int dmrg(int cutoff, int sweep) {
    int pre_cutoff = 10;
    if (sweep == -1) pre_cutoff = cutoff;
    const int pre_sweep = cutoff / 100;
    int rc = two_sites(0, L - 1, cutoff * 10);
    if (rc) return rc;
    for (int i = 1; i < L / 2; i++)
      if ((rc = update_two(i, L - i - 1, pre_cutoff))) return rc;
    if (sweep != -1)
      for (int i = L / 2; i < L - 1; i++)
        if ((rc = move2right(i, i + 1, pre_cutoff))) return rc;
    if (sweep != -1)
      for (int s = 0; s < pre_sweep - 1; s++) {
        for (int i = L - 2; i > 0; i--)
          if ((rc = move2left(i - 1, i, 100 * (s + 1)))) return rc;
        for (int i = 1; i < L - 1; i++)
          if ((rc = move2right(i, i + 1, 100 * (s + 1)))) return rc;
      }
    for (int s = 0; s < sweep; s++) {
      for (int i = L - 2; i > 0; i--)
        if ((rc = move2left(i - 1, i, cutoff))) return rc;
      for (int i = 1; i < L - 1; i++)
        if ((rc = move2right(i, i + 1, cutoff))) return rc;
    }
    if (sweep != -1)
      for (int i = L - 2; i >= L / 2; i--)
        if ((rc = move2left(i - 1, i, cutoff))) return rc;
    return 0;
  }
};

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
  Run R;
  R.c = c;
  R.L = L;
  R.sector = sector;
  R.E.stream = c->stream;
  R.E.device = c->device;
  R.E.num_sms = c->num_sms;
  R.E.f = c->f();
  double par[8] = {0};
  for (int i = 0; i < nparams && i < 8; i++) par[i] = params[i];
  HostQT W;
  if (!build_mpo(model, par, W)) {
    set_error("dmrg: unknown model");
    return DMRGX_E_ARG;
  }
  const bool real_model = model == 0 || model == 3;
  if (real_model != (c->dtype == DMRGX_F64)) {
    set_error("dmrg: Kitaev and real XYZ run on F64 contexts, XYZ and Potts on C128");
    return DMRGX_E_ARG;
  }
  R.E.G.n = model == 2 ? 3 : 2;
  R.E.G.fermion = model == 0;
  // edges: left() = take(0, D-1), right() = take(2, 0).exchange(0, 1) (src/qtensor.cpp:449-463)
  const int D = W.m.dims[0][0];
  HostQT le = take(W, 0, D - 1);
  HostQT re = exchange(take(W, 2, 0), 0, 1);
  std::string err;
  cudaSetDevice(c->device);
  R.bulk = upload(W, c->f(), c->stream, err);
  R.ledge = upload(le, c->f(), c->stream, err);
  R.redge = upload(re, c->f(), c->stream, err);
  if (!R.bulk || !R.ledge || !R.redge) {
    set_error("dmrg: " + err);
    return DMRGX_E_CUDA;
  }
  R.env.assign(L, nullptr);
  const double t0 = Run::now();
  int rc = R.dmrg(m, sweeps);
  const double t1 = Run::now();
  if (rc) {
    set_error("dmrg: " + R.err);
    return rc;
  }
  const int64_t ns = (int64_t)R.trunc.size();
  *nsteps = ns;
  for (int64_t i = 0; i < ns && i < cap; i++) {
    if (energies)
      for (int q = 0; q < 6; q++) energies[6 * i + q] = R.energies[6 * i + q];
    if (trunc) trunc[i] = R.trunc[i];
    if (steps_lr) {
      steps_lr[2 * i] = R.lr[2 * i];
      steps_lr[2 * i + 1] = R.lr[2 * i + 1];
    }
    if (matvecs) matvecs[i] = R.matvecs[i];
  }
  if (seconds) {
    seconds[0] = t1 - t0;
    seconds[1] = R.t_eig;
    seconds[2] = R.t_svd;
    seconds[3] = R.t_env;
    seconds[4] = R.t_fuse;
  }
  return 0;
}
