"""torch.autograd wrapper of the DMRG ground-state energy, for gradient checks.

forward runs the reference dmrg() schedule on the GPU (dmrgx_dmrg) and returns
the final step's lowest energy; backward returns grad_output * dE/dparams from
the adjoint effective-Hamiltonian contractions (dmrgx_adjoint).  The gradient is
computed eagerly in forward (one adjoint sweep over the final state).  This is
test plumbing around the C ABI, not a training path: there is no second
derivative and no batching over the parameter tensor."""
import numpy as np
import torch

from . import native

_REAL = ("kitaev", "xyz_real")


class GroundEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, model, L, m, sweeps, sector, recompute):
        c = native.Context(native.F64 if model in _REAL else native.C128)
        p = params.detach().cpu().numpy().astype(np.float64)
        r = c.dmrg(model, L, m, sweeps, p, sector=sector)
        g = c.adjoint(nparams=p.size, recompute=recompute)["dE_dparams"]
        ctx.save_for_backward(torch.as_tensor(g, dtype=params.dtype))
        return params.new_tensor(float(r["energies"][-1, 0]))

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g.to(grad_out.device), None, None, None, None, None, None


def ground_energy(params, model, L, m, sweeps, sector=0, recompute=False):
    """E0(params) with dE0/dparams through autograd.  model: 'kitaev' (t, p, u),
    'xyz' / 'xyz_real' (jx, jy, jz[, h]), 'potts' (f, j, p, t)."""
    return GroundEnergy.apply(params, model, L, m, sweeps, sector, recompute)
