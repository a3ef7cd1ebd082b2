// Adjoint of the two-site effective-Hamiltonian contraction with respect to its
// operators and, through the env (x) MPO fusion, with respect to the MPO
// tensors.  Internal header.
#pragma once
#include <string>
#include <vector>

#include "ctx.h"
#include "qtensor.h"

namespace dmrgx {

// FP64 matvec of the context's current plan (device in/out, plan layout of psi)
int matvec_fp64(dmrgx_ctx* c, const double* in, double* out);

// E = <psi, Lop (x)_{l_num} (Rop (x)_{r_num} psi)> for the plan that
// plan_build_device(c, Lop, Rop, ...) left in c; psi is a device vector in the
// plan's layout.  Returns energy = Re E / <psi, psi> and, when asked,
// gl = dE/dLop (metadata of Lop) and gr = dE/dRop (metadata of Rop), the
// holomorphic derivatives (E is linear in each operator, no conjugates).
int heff_adjoint(dmrgx_ctx* c, const Engine& E, const QTensor& Lop, const QTensor& Rop,
                 const double* psi, bool want_l, bool want_r, QTPtr& gl, QTPtr& gr,
                 double& energy, double& norm2, std::string& err);

// dE/dW of a fused operator, accumulated into gw (host, layout of W: W.total()
// elements, f doubles each):
//   right = false: fused = (env ._1 W).exchange(3,4)                (src/core.cpp:188-189)
//   right = true : fused = (env ._1 W.exchange(0,2), change).exchange(0,1)  (:190-192)
int fusion_adjoint(const Engine& E, const QTensor& env, const QTensor& W, const QTensor& gfused,
                   bool right, std::vector<double>& gw, std::string& err);

// dE/dW of an edge operator used directly as Lop / Rop:
//   right = false: edge = W.take(0, D-1)                     (src/qtensor.cpp:449-454)
//   right = true : edge = W.take(2, 0).exchange(0, 1)        (src/qtensor.cpp:457-463)
int edge_adjoint(const QTensor& gedge, const QTensor& W, bool right, std::vector<double>& gw,
                 cudaStream_t s, std::string& err);

}  // namespace dmrgx
