// The site-step eigensolver of the reference DMRG code (clover199/DMRG) on the
// GPU through libdmrgx: a drop-in for its two ARPACK wrappers,
//   void znaupd(int n, int nev, double* Evals, double* Evecs, lanczos<double>&)
//       (src/dsaupd.cpp:65-155, real, dsaupd 'SA')
//   void znaupd(int n, int nev, double* Evals, complex<double>* Evecs,
//               lanczos<complex<double> >&)
//       (src/znaupd.cpp:78-197, complex, znaupd 'SR')
// declared in include/basic.h:12,28-29 and called by every step function
// (src/core.cpp:139,251,353,450,591).
//
// A maintainer copies this file into the reference's src/, drops dsaupd.o and
// znaupd.o from the makefile's objects, links -ldmrgx instead of -larpack and
// adds one friend declaration to include/qtensor.h (the blocks are private):
//   template <typename T> friend struct qt_access;
//
// Each call hands the step's own task lists (pass_val.rmap / lmap, built by
// get_map, src/qtensor.cpp:997-1119) and environment blocks to
// dmrgx_plan_from_maps, then solves on the device with the reference's
// settings: nev values, basis 4 nev (real) / 6 nev (complex), tolerance 1e-10,
// the lowest eigenvector in Evecs.  Errors are reported on cerr and the run goes
// on, as the reference's wrappers do.
//
// Environment: DMRGX_PREC=bf16x3 or tf32x3 selects split-precision matvecs
// (FP64 Krylov basis and defect correction); the default is FP64.
#include <algorithm>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <vector>

#include "val_for_lanczos.h"
#include "dmrgx.h"

template <typename T>
struct qt_access {
  // blocks packed in block order (each row-major) and their element counts
  static void pack(const qtensor<T>& q, std::vector<T>& vals, std::vector<int64_t>& sizes) {
    for (size_t b = 0; b < q.val_.size(); b++) {
      sizes.push_back((int64_t)q.val_[b].val_.size());
      vals.insert(vals.end(), q.val_[b].val_.begin(), q.val_[b].val_.end());
    }
  }
};

namespace {

int dropin_precision() {
  const char* p = std::getenv("DMRGX_PREC");
  if (p && !std::strcmp(p, "bf16x3")) return DMRGX_PREC_BF16X3;
  if (p && !std::strcmp(p, "tf32x3")) return DMRGX_PREC_TF32X3;
  return DMRGX_PREC_FP64;
}

template <typename T>
void dropin_solve(int n, int nev, double* Evals, T* Evecs, lanczos<T>& pv, int dtype) {
  static dmrgx_ctx* ctx[2] = {0, 0};  // one context per element type, kept for the run
  if (!ctx[dtype]) {
    if (dmrgx_ctx_create(&ctx[dtype], dtype, 0) ||
        dmrgx_set_precision(ctx[dtype], dropin_precision())) {
      std::cerr << "dmrgx: " << dmrgx_last_error() << std::endl;
      return;
    }
  }
  std::vector<T> rv, lv;
  std::vector<int64_t> rs, ls;
  qt_access<T>::pack(pv.renv, rv, rs);
  qt_access<T>::pack(pv.lenv, lv, ls);
  std::vector<int> rmap, lmap;  // the reference's own task lists, 7 ints per row
  for (size_t i = 0; i < pv.rmap.size(); i++)
    rmap.insert(rmap.end(), pv.rmap[i].begin(), pv.rmap[i].end());
  for (size_t i = 0; i < pv.lmap.size(); i++)
    lmap.insert(lmap.end(), pv.lmap[i].begin(), pv.lmap[i].end());
  int64_t d_store = 0;  // end of the furthest intermediate block
  for (size_t i = 0; i < pv.rmap.size(); i++) {
    const std::vector<int>& r = pv.rmap[i];
    d_store = std::max<int64_t>(d_store, r[2] + (rs[r[0]] / r[4]) * (int64_t)r[3]);
  }
  if (dmrgx_plan_from_maps(ctx[dtype], n, d_store, rmap.data(), (int)pv.rmap.size(), rv.data(),
                           rs.data(), (int)rs.size(), lmap.data(), (int)pv.lmap.size(),
                           lv.data(), ls.data(), (int)ls.size()) ||
      dmrgx_eigsolve(ctx[dtype], nev, 0, 1e-10, 0, NULL, Evals, Evecs, NULL))
    std::cerr << "dmrgx: " << dmrgx_last_error() << std::endl;
}

}  // namespace

void znaupd(int n, int nev, double* Evals, double* Evecs, lanczos<double>& pass_val) {
  dropin_solve(n, nev, Evals, Evecs, pass_val, DMRGX_F64);
}

void znaupd(int n, int nev, double* Evals, std::complex<double>* Evecs,
            lanczos<std::complex<double> >& pass_val) {
  dropin_solve(n, nev, Evals, Evecs, pass_val, DMRGX_C128);
}
