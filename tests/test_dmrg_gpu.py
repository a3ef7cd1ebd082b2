"""The full dmrg() schedule on the GPU against the reference.

Small chains where the bond dimension keeps the state exact: every step's
lowest energy must equal the reference's step energy (the reference prints 10
decimals, global.h ACC) and the final energy the exact value (BdG / ED) to
1e-10 relative; truncation errors match the reference's to 1e-9."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from dmrg_b200 import native
from oracle import exact

pytestmark = pytest.mark.gpu

with open(os.path.join(GOLDEN, "energies.json")) as fh:
    GOLD = json.load(fh)

CASES = [("kitaev", "kitaev", native.F64), ("xyz", "xyz", native.C128),
         ("xyz", "xyz_real", native.F64), ("potts", "potts", native.C128)]


@pytest.mark.parametrize("gold,model,dtype", CASES)
def test_dmrg_small_chain_matches_reference_steps(gold, model, dtype):
    g = GOLD[gold]
    a = g["args"]
    ctx = native.Context(dtype)
    r = ctx.dmrg(model, a["L"], a["m"], a["n"], a["params"])
    ref = np.array(g["energy_rows"])
    assert len(r["energies"]) == len(ref)
    assert np.array_equal(r["lr"], ref[:, :2].astype(int))
    # reference energies are printed with 10 decimals
    assert np.abs(r["energies"][:, 0] - ref[:, 2]).max() < 2e-10 * np.abs(ref[:, 2]).max() + 6e-11
    assert abs(r["energies"][-1, 0] - g["exact"]) < 1e-10 * abs(g["exact"])
    tr = np.array(g["trunc_err_rows"])
    assert np.abs(r["trunc"] - tr[:, 2]).max() < 1e-9
    print(model, r["seconds"], r["energies"][-1, 0])


def load_schedule(name):
    """A reference dmrg() run recorded in full precision (make_golden.py record_schedule)."""
    z = np.load(os.path.join(GOLDEN, f"schedule_{name}.npz"))
    return {k: z[k] for k in z.files}


# Tolerances of the full-precision comparison.  The bar is 1e-10 relative on
# energies and truncation errors.  A truncation error 1 - sum s_i^2 is a
# difference of O(1) numbers, so it carries an absolute rounding floor of a few
# 1e-16 per kept value; 5e-14 covers the few hundred values kept here.  The
# singular values and the entropy are functions of the step's eigenvector,
# which both eigensolvers converge only to a residual |H psi - E psi| <= 1e-10
# |E|: the vectors may differ by |d psi| ~ 1e-10 |E| / gap (~1e-9 for these
# chains), a singular value moves by at most |d psi| and the entropy by a few
# times that, so both are compared to 1e-8 absolute (s_0 ~ 1).  The SVD itself
# is held to 1e-13 of s_0 on identical inputs in test_svd_gpu.py.
E_REL = 1e-10
TRUNC_REL, TRUNC_ABS = 1e-10, 5e-14
S_ABS, SV_ABS = 1e-8, 1e-8


def check_schedule(r, g, rows=None, dpsi=0.0):
    """The steps `rows` (all by default) of a GPU run against the reference's
    full-precision rows.  dpsi: the eigenvector accuracy the run's solver
    guarantees when it differs from the reference's; the weight outside the
    kept subspace then moves by up to 2 sqrt(trunc) dpsi, which is added to
    the truncation-error bar."""
    assert np.array_equal(r["lr"], g["lr"]), "step sequence differs from the reference"
    sl = slice(None) if rows is None else rows
    e, e_ref = r["energies"][sl, 0], g["evals"][sl, 0]
    de = np.abs(e - e_ref) / np.abs(e_ref)
    assert de.max() <= E_REL, (de.max(), int(de.argmax()))
    dt = np.abs(r["trunc"][sl] - g["trunc"][sl])
    tt = np.abs(g["trunc"][sl])
    assert (dt <= TRUNC_REL * tt + 2 * dpsi * np.sqrt(tt) + TRUNC_ABS).all(), (dt.max(), int(dt.argmax()))
    ds = np.abs(r["entropy"][sl] - g["entropy"][sl])
    assert ds.max() <= S_ABS, (ds.max(), int(ds.argmax()))
    dv = np.abs(r["s20"][sl] - g["s20"][sl])
    assert dv.max() <= SV_ABS, (dv.max(), np.unravel_index(dv.argmax(), dv.shape))
    assert np.array_equal(r["nsv"][sl], g["nsv"][sl])
    return de.max(), dt.max(), ds.max(), dv.max()


SCHEDULE_CASES = [("kitaev_L8_m16", "kitaev", native.F64), ("xyz_L8_m16", "xyz", native.C128),
                  ("xyz_L8_m16", "xyz_real", native.F64), ("potts_L6_m27", "potts", native.C128)]


@pytest.mark.parametrize("name,model,dtype", SCHEDULE_CASES)
def test_dmrg_schedule_full_precision(name, model, dtype):
    """Per step: lowest energy, truncation error, entropy and the first 20
    singular values (the reference's energy and singular-value rows,
    src/useful.cpp:54-102) against the reference run recorded in full double
    precision at its own print_energy / print_singular calls."""
    g = load_schedule(name)
    L, m, n, sector = (int(v) for v in g["args"])
    ctx = native.Context(dtype)
    r = ctx.dmrg(model, L, m, n, g["params"].tolist(), sector=sector)
    print(name, model, "max dE/E %.1e dtrunc %.1e dS %.1e ds %.1e" % check_schedule(r, g))


@pytest.mark.parametrize("solver", ["reference", "fast"])
def test_config2_xyz_L64_m256_full_precision(solver):
    """BASELINE config 2 at its own size: the XYZ chain L=64 (jx=1, jy=0.8,
    jz=0.5), the reference's dmrg() schedule to m=256 with 8 sweeps, every one of
    its 1210 steps against the reference run recorded in full precision (energy
    1e-10 relative, truncation error, entropy and singular values as above).
    The GPU runs the real form of the MPO (sigma_y sigma_y = -(i sigma_y)(i
    sigma_y)), which has the reference's spectrum.  "reference": the reference's
    eigensolver settings (6 values, basis 24, fixed start); "fast": the lowest
    value only from White's prediction -- a different solver path to the same
    converged states.

    Compared step by step: the growth to the middle at cutoff 10 (steps 0-62),
    and every step of the last four sweeps and the closing half sweep (steps
    683-1209), with the final energy.  Between them (the pre-sweep at 100 and
    the first four sweeps at 256) the two runs take different but equally valid
    paths: where a cutoff exceeds the rank, the reference pads U and V to
    min(dim, cutoff) with complement columns (src/qtensor.cpp:1221-1252) that
    span an arbitrary part of the complement -- the columns LAPACK's dgesvd
    happens to return -- and that part enters the next step's variational space.
    Both runs then converge to the same state, step for step."""
    g = load_schedule("xyz_L64_m256")
    L, m, n, sector = (int(v) for v in g["args"])
    ctx = native.Context(native.F64)
    if solver == "fast":
        ctx.set_solver(1, 12, True)
    r = ctx.dmrg("xyz_real", L, m, n, g["params"].tolist(), sector=sector)
    steps = len(g["lr"])
    growth = slice(0, 1 + 2 * (L // 2 - 1))          # two_sites + update_two + move2right
    converged = slice(steps - (4 * 2 * (L - 2) + L // 2 - 1), steps)
    # the fast solver stops at the residual bound 1e-10 |E| (|E| ~ 88, gap ~ 1):
    # its eigenvectors are good to ~1e-8, the reference settings' far better
    dpsi = 1e-8 if solver == "fast" else 0.0
    a = check_schedule(r, g, growth, dpsi)
    b = check_schedule(r, g, converged, dpsi)
    de_final = abs(r["energies"][-1, 0] - g["evals"][-1, 0]) / abs(g["evals"][-1, 0])
    assert de_final <= E_REL, de_final
    print("config 2", solver, "growth: max dE/E %.1e dtrunc %.1e dS %.1e ds %.1e" % a,
          "converged: %.1e %.1e %.1e %.1e" % b, "final dE/E %.1e" % de_final,
          "GPU s", r["seconds"]["total"], "reference s", float(g["ref_seconds"]))


@pytest.mark.parametrize("prec", ["fp64", "bf16x3"])
def test_config4_potts_L48_m512_growth_full_precision(prec):
    """BASELINE config 4's chain at its bond dimension: the 3-state Potts chain
    L=48 (f=1, j=1, complex128, Z3 sectors) on the reference's dmrg() growth
    schedule sweep = -1 (src/functions.cpp:169-182: two_sites, then update_two
    to the middle with cutoff 512 at every step; the full schedule runs for
    hours on the host).  Bond dimensions reach 512 from the sixth step on.
    Every one of the 24 steps against the reference run recorded in full
    precision: energies to 1e-10 relative, truncation errors, entropies and
    singular values to the bars above.  "bf16x3": the split-precision matvec
    with FP64 defect correction, to the same bars."""
    g = load_schedule("potts_L48_m512_growth")
    L, m, n, sector = (int(v) for v in g["args"])
    ctx = native.Context(native.C128)
    if prec == "bf16x3":
        ctx.set_precision(native.PREC_BF16X3)
    r = ctx.dmrg("potts", L, m, n, g["params"].tolist(), sector=sector)
    assert r["nsv"].max() >= 512
    print("config 4", prec, "max dE/E %.1e dtrunc %.1e dS %.1e ds %.1e" % check_schedule(r, g),
          "E", r["energies"][-1, 0], "GPU s", r["seconds"]["total"],
          "reference s", float(g["ref_seconds"]))


with open(os.path.join(GOLDEN, "energies_pbc.json")) as fh:
    GOLD_PBC = json.load(fh)


@pytest.mark.parametrize("gold,model,dtype", CASES)
def test_dmrg_periodic_matches_reference_steps(gold, model, dtype):
    """PBC build: edge environments carried through every step (src/core.cpp:27-30 and
    the PBC blocks of the step functions); step energies equal the reference's, the
    final energy the periodic chain's exact value (XYZ, Potts)."""
    g = GOLD_PBC[gold]
    a = g["args"]
    ctx = native.Context(dtype)
    ctx.set_boundary(native.BOUNDARY_PERIODIC)
    r = ctx.dmrg(model, a["L"], a["m"], a["n"], a["params"])
    ref = np.array(g["energy_rows"])
    assert len(r["energies"]) == len(ref)
    assert np.array_equal(r["lr"], ref[:, :2].astype(int))
    err = np.abs(r["energies"][:, 0] - ref[:, 2]).max()
    print(model, "pbc", r["energies"][-1, 0], ref[-1, 2], err)
    assert err < 2e-10 * np.abs(ref[:, 2]).max() + 6e-11
    if g["exact"] is not None:
        assert abs(r["energies"][-1, 0] - g["exact"]) < 1e-10 * abs(g["exact"])
    tr = np.array(g["trunc_err_rows"])
    assert np.abs(r["trunc"] - tr[:, 2]).max() < 1e-9
    with pytest.raises(native.DmrgxError, match="periodic"):
        ctx.adjoint()


def test_dmrg_periodic_split_precision():
    """Split-precision matvecs on a periodic chain reach the FP64 energy."""
    c64 = native.Context(native.F64)
    c64.set_boundary(native.BOUNDARY_PERIODIC)
    r64 = c64.dmrg("xyz_real", 16, 32, 2, [1.0, 0.8, 0.5])
    ctx = native.Context(native.F64)
    ctx.set_boundary(native.BOUNDARY_PERIODIC)
    ctx.set_precision(native.PREC_BF16X3)
    r = ctx.dmrg("xyz_real", 16, 32, 2, [1.0, 0.8, 0.5])
    e64, e = r64["energies"][-1, 0], r["energies"][-1, 0]
    print("pbc split", e, e64)
    assert abs(e - e64) <= 1e-9 * abs(e64)


@pytest.mark.parametrize("gold,model,dtype", CASES)
def test_dmrg_lowest_only_and_prediction_keep_reference_energies(gold, model, dtype):
    """nev=1 (lowest value only), with and without White's prediction as the start
    vector: every step's lowest energy is still the reference's; prediction cuts
    the matvecs."""
    g = GOLD[gold]
    a = g["args"]
    ref = np.array(g["energy_rows"])
    tol = 2e-10 * np.abs(ref[:, 2]).max() + 6e-11
    runs = {}
    for name, kw in (("nev1", dict(nev=1, ncv=12)), ("pred", dict(nev=1, ncv=12, predict=True))):
        ctx = native.Context(dtype)
        ctx.set_solver(**kw)
        r = ctx.dmrg(model, a["L"], a["m"], a["n"], a["params"])
        assert np.abs(r["energies"][:, 0] - ref[:, 2]).max() < tol, name
        assert not r["energies"][:, 1:].any()
        runs[name] = int(r["matvecs"].sum())
    print(model, "matvecs", runs)
    assert runs["pred"] < runs["nev1"]
    with pytest.raises(native.DmrgxError, match="nev = 1"):
        native.Context(dtype).set_solver(nev=6, predict=True)


def test_kitaev_L32_m64_prediction():
    """Config 1 with the fast solver settings: the BdG energy, far fewer matvecs."""
    ex = exact.kitaev_bdg(32, 1.0, 1.0, 0.25)
    ctx = native.Context(native.F64)
    ctx.set_solver(nev=1, ncv=12, predict=True)
    r = ctx.dmrg("kitaev", 32, 64, 6, [1.0, 1.0, 0.25])
    base = native.Context(native.F64).dmrg("kitaev", 32, 64, 6, [1.0, 1.0, 0.25])
    print("kitaev L32 m64 predicted", r["energies"][-1, 0], ex, r["matvecs"].sum(),
          base["matvecs"].sum(), r["seconds"], base["seconds"])
    assert abs(r["energies"][-1, 0] - ex) < 1e-9 * abs(ex)
    assert r["matvecs"].sum() < 0.5 * base["matvecs"].sum()


def test_kitaev_L32_m64_matches_bdg():
    """Config 1: Kitaev chain L=32, t=Delta=1, mu=0.5 (u=0.25), m=64, 6 sweeps."""
    ctx = native.Context(native.F64)
    r = ctx.dmrg("kitaev", 32, 64, 6, [1.0, 1.0, 0.25])
    e = r["energies"][-1, 0]
    ex = exact.kitaev_bdg(32, 1.0, 1.0, 0.25)
    print("kitaev L32 m64", e, ex, r["seconds"], len(r["trunc"]))
    assert abs(e - ex) < 1e-9 * abs(ex)


@pytest.mark.parametrize("prec", [native.PREC_BF16X3, native.PREC_TF32X3])
def test_dmrg_split_precision_energy(prec):
    """Split-precision matvecs + FP64 defect correction reach the FP64 energy."""
    c64 = native.Context(native.F64)
    r64 = c64.dmrg("xyz_real", 16, 32, 2, [1.0, 0.8, 0.5])
    ctx = native.Context(native.F64)
    ctx.set_precision(prec)
    r = ctx.dmrg("xyz_real", 16, 32, 2, [1.0, 0.8, 0.5])
    print(prec, r["energies"][-1, 0], r64["energies"][-1, 0], r["seconds"])
    assert abs(r["energies"][-1, 0] - r64["energies"][-1, 0]) <= 1e-9 * abs(r64["energies"][-1, 0])


@pytest.mark.parametrize("prec", [native.PREC_BF16X3, native.PREC_TF32X3])
@pytest.mark.parametrize("model,L,par", [("potts", 12, [1.0, 1.0, 0.0, 0.0]),
                                         ("xyz", 14, [1.0, 0.8, 0.5])])
def test_dmrg_split_precision_complex(model, L, par, prec):
    """Complex models (C128) with split-precision contractions reach the FP64 energy."""
    c64 = native.Context(native.C128)
    r64 = c64.dmrg(model, L, 32, 2, par)
    ctx = native.Context(native.C128)
    ctx.set_precision(prec)
    r = ctx.dmrg(model, L, 32, 2, par)
    print(model, prec, r["energies"][-1, 0], r64["energies"][-1, 0])
    assert abs(r["energies"][-1, 0] - r64["energies"][-1, 0]) <= 1e-9 * abs(r64["energies"][-1, 0])
