"""Split-precision matvec (tcgen05, hi/lo pairs, FP32 accumulation) against FP64.

Stated error bound of one matvec, relative in the 2-norm: 5e-5 for both BF16
and TF32 pairs (3 products).  The dropped lo*lo term is ~2^-16 (BF16) / ~2^-22
(TF32) of a product and the intermediate is re-split after stage 1; measured on
B200: BF16 6e-6..1e-5, TF32 5e-7 (m<=64) .. 1.5e-5 (m=1024, long K: the FP32
accumulation of the TF32 path dominates).  The checks below use this bound."""
import numpy as np
import pytest

from conftest import load_microbench_m64, load_steps
from dmrg_b200 import native, workloads

pytestmark = pytest.mark.gpu
BOUND = {native.PREC_BF16X3: 5e-5, native.PREC_TF32X3: 5e-5}


def rel(y, ref):
    return np.linalg.norm(y - ref) / np.linalg.norm(ref)


@pytest.mark.parametrize("prec", [native.PREC_BF16X3, native.PREC_TF32X3])
def test_split_microbench_m64_against_reference(prec):
    mb = load_microbench_m64()
    ctx = native.Context(native.F64)
    ctx.set_precision(prec)
    ctx.plan_build(mb["lenv"], mb["renv"], 3, 2, mb["sector"], mb["group_n"], 0)
    e = rel(ctx.av(mb["x"]), mb["ax"])
    print("m64 rel err", prec, e)
    assert e < BOUND[prec]


@pytest.mark.parametrize("prec", [native.PREC_BF16X3, native.PREC_TF32X3])
@pytest.mark.parametrize("m", [9, 35, 256, 1024])
def test_split_against_fp64(prec, m):
    w = workloads.microbench(m, seed=m)
    ref_ctx = native.Context(native.F64)
    ref_ctx.plan_build(w["lenv"], w["renv"], 3, 2, w["sector"], 32, 0)
    ctx = native.Context(native.F64)
    ctx.set_precision(prec)
    ctx.plan_build(w["lenv"], w["renv"], 3, 2, w["sector"], 32, 0)
    for seed in (1, 2):
        x = workloads.random_psi(ctx.n, seed=seed)
        e = rel(ctx.av(x), ref_ctx.av(x))
        print("m", m, "prec", prec, "rel err", e)
        assert e < BOUND[prec]


def test_split_switch_precision_on_existing_plan():
    """set_precision after plan_build rebuilds the split form; back to FP64 is exact."""
    mb = load_microbench_m64()
    ctx = native.Context(native.F64)
    ctx.plan_build(mb["lenv"], mb["renv"], 3, 2, mb["sector"], mb["group_n"], 0)
    y64 = ctx.av(mb["x"])
    ctx.set_precision(native.PREC_TF32X3)
    assert rel(ctx.av(mb["x"]), y64) < BOUND[native.PREC_TF32X3]
    ctx.set_precision(native.PREC_FP64)
    assert np.abs(ctx.av(mb["x"]) - y64).max() == 0.0


@pytest.mark.parametrize("model", ["kitaev"])
def test_split_real_physical_steps(model):
    for st in load_steps(model):
        ctx = native.Context(native.F64)
        ctx.set_precision(native.PREC_TF32X3)
        ctx.plan_build(st["lenv"], st["renv"], st["l_num"], st["r_num"], st["sector"],
                       st["group_n"], st["fermion"])
        assert rel(ctx.av(st["x"]), st["ax"]) < BOUND[native.PREC_TF32X3]


@pytest.mark.parametrize("prec", [native.PREC_BF16X3, native.PREC_TF32X3])
@pytest.mark.parametrize("model", ["xyz", "potts"])
def test_split_complex_physical_steps(model, prec):
    """Complex contractions as one real split GEMM with the B operand expanded."""
    for st in load_steps(model):
        ctx = native.Context(native.C128)
        ctx.set_precision(prec)
        ctx.plan_build(st["lenv"], st["renv"], st["l_num"], st["r_num"], st["sector"],
                       st["group_n"], st["fermion"])
        e = rel(ctx.av(st["x"]), st["ax"])
        assert e < BOUND[prec], (model, e)


@pytest.mark.parametrize("prec", [native.PREC_BF16X3, native.PREC_TF32X3])
@pytest.mark.parametrize("m", [35, 256])
def test_split_complex_against_fp64(prec, m):
    a, b = workloads.microbench(m, seed=m), workloads.microbench(m, seed=m + 1)
    lenv = (a["lenv"][0], a["lenv"][1] + 1j * b["lenv"][1])
    renv = (a["renv"][0], a["renv"][1] - 0.5j * b["renv"][1])
    ref_ctx = native.Context(native.C128)
    ref_ctx.plan_build(lenv, renv, 3, 2, a["sector"], 32, 0)
    ctx = native.Context(native.C128)
    ctx.set_precision(prec)
    ctx.plan_build(lenv, renv, 3, 2, a["sector"], 32, 0)
    rng = np.random.default_rng(m)
    x = rng.standard_normal(ctx.n) + 1j * rng.standard_normal(ctx.n)
    e = rel(ctx.av(x), ref_ctx.av(x))
    print("complex m", m, "prec", prec, "rel err", e)
    assert e < BOUND[prec]
