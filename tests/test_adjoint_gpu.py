"""dE/dJ from the adjoint effective-Hamiltonian contractions (dmrgx_adjoint).

Three independent checks per model:
  * Hellmann-Feynman: <Psi|dH/dp|Psi> evaluated by dmrgx_expect with the MPO of
    the unit coupling e_p (each shipped Hamiltonian is linear in its couplings
    with no constant term) on the same state -- equal to the adjoint value up
    to rounding (1e-9 relative);
  * central finite differences of whole DMRG runs, step 1e-4, to 1e-6 relative
    (Kitaev: of the exact BdG energy instead);
  * internal: every centre the adjoint sweep visits has the same energy, and
    <dE/dW_k, W_k> = E for every site (E is linear in each MPO tensor)."""
import numpy as np
import pytest
import torch

from dmrg_b200 import native
from dmrg_b200.autograd import ground_energy
from oracle import exact

pytestmark = pytest.mark.gpu


def _run(model, par, L, m, n, sector=0):
    ctx = native.Context(native.F64 if model in ("kitaev", "xyz_real") else native.C128)
    r = ctx.dmrg(model, L, m, n, par, sector=sector)
    return ctx, float(r["energies"][-1, 0])


def _check_internal(a):
    e0, edev, wdev, disc = a["checks"]
    assert edev < 1e-10 * abs(e0), a["checks"]
    assert wdev < 1e-10 * abs(e0), a["checks"]
    assert disc < 1e-20, a["checks"]


def test_xyz_adjoint_hf_fd():
    par = [1.0, 0.8, 0.5, 0.0]
    L, m, n = 16, 32, 4
    ctx, e0 = _run("xyz_real", par, L, m, n)
    a = ctx.adjoint()
    _check_internal(a)
    g = a["dE_dparams"]
    for p in range(4):
        unit = np.zeros(4)
        unit[p] = 1.0
        hf = ctx.expect(unit)
        assert abs(hf - g[p]) <= 1e-9 * abs(g[p]) + 1e-11, (p, hf, g[p])
    # dE/dh = <sum_i sigma^z_i> = 0: the global spin flip maps the sector to itself
    assert abs(g[3]) < 1e-8
    # whole-run central differences on Jz
    h = 1e-4
    _, ep = _run("xyz_real", [1.0, 0.8, 0.5 + h, 0.0], L, m, n)
    _, em = _run("xyz_real", [1.0, 0.8, 0.5 - h, 0.0], L, m, n)
    fd = (ep - em) / (2 * h)
    print("xyz dE/dJz adjoint", g[2], "fd", fd, "checks", a["checks"], a["seconds"])
    assert abs(fd - g[2]) < 1e-6 * abs(g[2])
    # environments rebuilt from the MPS give the same gradient
    b = ctx.adjoint(recompute=True)
    _check_internal(b)
    assert np.abs(b["dE_dparams"] - g).max() < 1e-9 * np.abs(g).max()


def test_xyz_complex_adjoint_matches_real_gauge():
    """The complex reference MPO and the real re-gauged one give one gradient."""
    par = [1.0, 0.8, 0.5, 0.0]
    cr, _ = _run("xyz_real", par, 12, 24, 3)
    cc, _ = _run("xyz", par, 12, 24, 3)
    gr = cr.adjoint()["dE_dparams"]
    a = cc.adjoint()
    _check_internal(a)
    gc = a["dE_dparams"]
    assert np.abs(gr - gc).max() < 1e-8 * np.abs(gr).max(), (gr, gc)


def test_kitaev_adjoint_against_bdg():
    """Fermion signs: gradients against the exact free-fermion energy."""
    par = [1.0, 1.0, 0.25]
    L = 16
    ctx, e0 = _run("kitaev", par, L, 32, 4)
    assert abs(e0 - exact.kitaev_bdg(L, *par)) < 1e-10 * abs(e0)
    a = ctx.adjoint()
    _check_internal(a)
    g = a["dE_dparams"]
    h = 1e-5
    for p in range(3):
        pp, pm = list(par), list(par)
        pp[p] += h
        pm[p] -= h
        fd = (exact.kitaev_bdg(L, *pp) - exact.kitaev_bdg(L, *pm)) / (2 * h)
        unit = np.zeros(3)
        unit[p] = 1.0
        hf = ctx.expect(unit)
        print("kitaev p", p, "adjoint", g[p], "hf", hf, "bdg fd", fd)
        assert abs(hf - g[p]) <= 1e-9 * abs(g[p]) + 1e-11
        assert abs(fd - g[p]) < 1e-7 * abs(g[p]) + 1e-9


def test_potts_adjoint_complex():
    par = [1.0, 1.0, 0.0, 0.0]
    L, m, n = 12, 32, 3
    ctx, e0 = _run("potts", par, L, m, n)
    a = ctx.adjoint()
    _check_internal(a)
    g = a["dE_dparams"]
    for p, unit in ((0, [1.0, 0.0, 0.0, 0.0]), (1, [0.0, 1.0, 0.0, 0.0])):
        hf = ctx.expect(unit)
        assert abs(hf - g[p]) <= 1e-9 * abs(g[p]) + 1e-11, (p, hf, g[p])
    h = 1e-4
    for p in range(4):
        pp, pm = list(par), list(par)
        pp[p] += h
        pm[p] -= h
        fd = (_run("potts", pp, L, m, n)[1] - _run("potts", pm, L, m, n)[1]) / (2 * h)
        print("potts p", p, "adjoint", g[p], "fd", fd)
        assert abs(fd - g[p]) < 1e-6 * max(abs(g[p]), 1.0)


def test_autograd_function():
    J = torch.tensor([1.0, 0.8, 0.5, 0.0], dtype=torch.float64, requires_grad=True)
    E = ground_energy(J, "xyz_real", 12, 24, 3)
    (gJ,) = torch.autograd.grad(E, J)
    h = 1e-4
    for p in range(3):
        pp = J.detach().clone()
        pm = J.detach().clone()
        pp[p] += h
        pm[p] -= h
        fd = (ground_energy(pp, "xyz_real", 12, 24, 3) - ground_energy(pm, "xyz_real", 12, 24, 3)) / (2 * h)
        assert abs(float(fd) - float(gJ[p])) < 1e-6 * abs(float(gJ[p]))
