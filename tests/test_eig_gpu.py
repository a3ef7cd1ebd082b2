"""Device eigensolver (dmrgx_eigsolve) against the reference's ARPACK results.

On every golden step the lowest Ritz value must match the reference's
(SciPy-ARPACK on the reference av, tol 1e-10) to 1e-10 relative, and the
returned vector must be an eigenvector of the FP64 operator to the stated
tolerance.  With split precision the defect-correction restart must bring the
energy to within 1e-9 relative of the FP64 solve."""
import numpy as np
import pytest

from conftest import MODELS, load_steps
from dmrg_b200 import native

pytestmark = pytest.mark.gpu


def residual(ctx64, v, e):
    hv = ctx64.av(v)
    return np.linalg.norm(hv - e * v) / abs(e)


@pytest.mark.parametrize("model", MODELS)
def test_eigsolve_fp64_matches_reference(model):
    for st in load_steps(model):
        ctx = native.Context(native.C128 if st["complex"] else native.F64)
        ctx.plan_build(st["lenv"], st["renv"], st["l_num"], st["r_num"], st["sector"],
                       st["group_n"], st["fermion"])
        ev, vec, info = ctx.eigsolve(nev=6)
        ref = st["evals"]
        k = min(len(ref), ctx.n)
        print(model, ctx.n, ev[:3], ref[:3], info)
        assert abs(ev[0] - ref[0]) <= 1e-10 * abs(ref[0])
        assert np.allclose(ev[:k], ref[:k], rtol=1e-8, atol=1e-8)
        assert abs(np.linalg.norm(vec) - 1) < 1e-12
        assert residual(ctx, vec, ev[0]) < 1e-8


@pytest.mark.parametrize("prec", [native.PREC_BF16X3, native.PREC_TF32X3])
def test_eigsolve_split_defect_correction(prec):
    st = load_steps("kitaev")[0]
    ref = native.Context(native.F64)
    ref.plan_build(st["lenv"], st["renv"], st["l_num"], st["r_num"], st["sector"],
                   st["group_n"], st["fermion"])
    e64, v64, _ = ref.eigsolve(nev=6)
    ctx = native.Context(native.F64)
    ctx.set_precision(prec)
    ctx.plan_build(st["lenv"], st["renv"], st["l_num"], st["r_num"], st["sector"],
                   st["group_n"], st["fermion"])
    ev, vec, info = ctx.eigsolve(nev=6)
    print(prec, ev[0], e64[0], info)
    assert abs(ev[0] - e64[0]) <= 1e-9 * abs(e64[0])
    assert residual(ref, vec, ev[0]) < 1e-8


def test_eigsolve_start_vector_and_small_space():
    """A start vector is honoured (one cycle when it is already the ground state)
    and a space smaller than the basis is solved exactly."""
    st = load_steps("xyz")[0]
    ctx = native.Context(native.C128)
    ctx.plan_build(st["lenv"], st["renv"], st["l_num"], st["r_num"], st["sector"],
                   st["group_n"], st["fermion"])
    ev, vec, info = ctx.eigsolve(nev=6)
    ev2, vec2, info2 = ctx.eigsolve(nev=1, v0=vec)
    assert abs(ev2[0] - ev[0]) <= 1e-10 * abs(ev[0])
    assert info2["matvecs"] <= info["matvecs"]
