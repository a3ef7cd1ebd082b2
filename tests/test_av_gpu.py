"""H_eff matvec on the GPU (FP64 path) against the reference.

Tolerance: FP64 with a different summation order than BLAS; every check is
max|y - y_ref| <= 1e-13 * max|y_ref| (1e-12 at the m=1024 size)."""
import numpy as np
import pytest

from conftest import MODELS, load_microbench_m64, load_steps, load_z2cubed
from dmrg_b200 import native, workloads
from oracle import restate

pytestmark = pytest.mark.gpu
TOL = 1e-13


def block_sizes(meta):
    q = restate.QT.from_ibuf(meta, np.zeros(10 ** 8))
    return np.array([b.size for b in q.blocks], np.int64)


def close(y, ref, tol=TOL):
    scale = max(np.abs(ref).max(), 1e-300)
    return np.abs(y - ref).max() <= tol * scale


@pytest.mark.parametrize("model", MODELS)
def test_av_plan_build_matches_reference(model):
    for st in load_steps(model):
        ctx = native.Context(native.C128 if st["complex"] else native.F64)
        ctx.plan_build(st["lenv"], st["renv"], st["l_num"], st["r_num"], st["sector"],
                       st["group_n"], st["fermion"])
        r, l = ctx.maps()
        assert np.array_equal(r, st["rmap"]) and np.array_equal(l, st["lmap"])
        assert close(ctx.av(st["x"]), st["ax"])
        ctx.close()


@pytest.mark.parametrize("model", MODELS)
def test_av_from_reference_maps(model):
    """The drop-in entry: the reference's own rmap/lmap and env blocks."""
    for st in load_steps(model):
        ctx = native.Context(native.C128 if st["complex"] else native.F64)
        n = st["x"].size
        rs, ls = block_sizes(st["renv"][0]), block_sizes(st["lenv"][0])
        # d_store = end of the furthest stage-1 output block
        d_store = 0
        for row in st["rmap"]:
            M = rs[row[0]] // row[4]
            d_store = max(d_store, row[2] + M * row[3])
        ctx.plan_from_maps(n, d_store, st["rmap"], st["renv"][1], rs, st["lmap"], st["lenv"][1], ls)
        assert close(ctx.av(st["x"]), st["ax"])
        ctx.close()


def test_av_microbench_m64():
    mb = load_microbench_m64()
    ctx = native.Context(native.F64)
    ctx.plan_build(mb["lenv"], mb["renv"], 3, 2, mb["sector"], mb["group_n"], 0)
    assert ctx.n == mb["n"]
    assert close(ctx.av(mb["x"]), mb["ax"])


@pytest.mark.parametrize("model", MODELS)
def test_av_periodic_edge_pair(model):
    """PBC: both pairs in one plan, from metadata and from the reference's own maps."""
    for st in load_steps(model, pbc=True):
        dt = native.C128 if st["complex"] else native.F64
        ctx = native.Context(dt)
        ctx.plan_build_pbc(st["lenv"], st["renv"], st["ledge"], st["redge"], st["l_num"],
                           st["r_num"], st["sector"], st["group_n"], st["fermion"])
        r, l = ctx.maps()
        es, re_, le_ = ctx.edge_maps()
        assert np.array_equal(r, st["rmap"]) and np.array_equal(l, st["lmap"])
        assert np.array_equal(re_, st["remap"]) and np.array_equal(le_, st["lemap"])
        assert close(ctx.av(st["x"]), st["ax"])
        ctx.close()
        # the drop-in: the reference's task lists and blocks of both pairs
        def d_store_of(rmap, sizes):
            d = 0
            for row in rmap:
                d = max(d, row[2] + sizes[row[0]] // row[4] * row[3])
            return d
        rs, ls = block_sizes(st["renv"][0]), block_sizes(st["lenv"][0])
        rxs, lxs = block_sizes(st["redge"][0]), block_sizes(st["ledge"][0])
        ctx = native.Context(dt)
        ctx.plan_from_maps_pbc(st["x"].size, d_store_of(st["rmap"], rs), st["rmap"],
                               st["renv"][1], rs, st["lmap"], st["lenv"][1], ls,
                               d_store_of(st["remap"], rxs), st["remap"], st["redge"][1], rxs,
                               st["lemap"], st["ledge"][1], lxs)
        assert close(ctx.av(st["x"]), st["ax"])
        for prec in (native.PREC_BF16X3, native.PREC_TF32X3):
            ctx.set_precision(prec)
            assert close(ctx.av(st["x"]), st["ax"], 5e-5)
        ctx.close()


def test_av_z2cubed():
    """Z2 x Z2 x Z2 (S4E) plans, real and complex, FP64 and split precision."""
    for z in load_z2cubed():
        dt = native.C128 if z["complex"] else native.F64
        for prec, tol in ((native.PREC_FP64, TOL), (native.PREC_BF16X3, 5e-5),
                          (native.PREC_TF32X3, 5e-5)):
            ctx = native.Context(dt)
            ctx.set_precision(prec)
            ctx.plan_build(z["lenv"], z["renv"], z["l_num"], z["r_num"], z["sector"],
                           native.GROUP_Z2CUBED, z["fermion"])
            r, l = ctx.maps()
            assert np.array_equal(r, z["rmap"]) and np.array_equal(l, z["lmap"])
            y = ctx.av(z["x"])
            assert close(y, z["ax"], tol), (z["complex"], prec,
                                             np.abs(y - z["ax"]).max() / np.abs(z["ax"]).max())
            ctx.close()


def test_av_microbench_full_size_against_restatement():
    w = workloads.microbench(1024)
    ctx = native.Context(native.F64)
    ctx.plan_build(w["lenv"], w["renv"], 3, 2, w["sector"], 32, 0)
    assert ctx.n == 599964 and ctx.flops == 3861687920
    le = restate.QT.from_ibuf(*w["lenv"])
    re_ = restate.QT.from_ibuf(*w["renv"])
    rmap, lmap = ctx.maps()
    x = workloads.random_psi(ctx.n, seed=2)
    store = np.zeros(ctx.d_store)
    restate.contract_map(re_, store, x, rmap, 2)
    ref = np.zeros(ctx.n)
    restate.contract_map(le, ref, store, lmap, 3)
    y = ctx.av(x)
    assert close(y, ref, 1e-12)
    # linearity at full size
    x2 = workloads.random_psi(ctx.n, seed=3)
    y2 = ctx.av(x2)
    y3 = ctx.av(2.0 * x - 0.5 * x2)
    assert close(y3, 2.0 * y - 0.5 * y2, 1e-12)


@pytest.mark.parametrize("cplx", [False, True])
def test_av_large_blocks_against_restatement(cplx):
    """Blocks of ~340 rows and columns (three U(1) sectors at m=1024, the shape of
    a sweep's middle steps), many tiles per block and K up to ~1000 per segment.
    Real and complex (environment values given complex phases), against the
    numpy restatement and the per-block library schedule, 1e-12 relative."""
    w = workloads.microbench(1024, qmax=1, width=1e9)
    lm, lv = w["lenv"]
    rm, rv = w["renv"]
    if cplx:
        rng = np.random.default_rng(5)
        lv = lv * np.exp(1j * rng.uniform(0, 2 * np.pi, lv.size))
        rv = rv * np.exp(1j * rng.uniform(0, 2 * np.pi, rv.size))
    ctx = native.Context(native.C128 if cplx else native.F64)
    ctx.plan_build((lm, lv), (rm, rv), 3, 2, w["sector"], 32, 0)
    le = restate.QT.from_ibuf(lm, lv)
    re_ = restate.QT.from_ibuf(rm, rv)
    rmap, lmap = ctx.maps()
    assert max(le.blocks[r[0]].size // r[4] for r in lmap) >= 256
    x = workloads.random_psi(ctx.n, seed=2, complex_=cplx)
    store = np.zeros(ctx.d_store, x.dtype)
    restate.contract_map(re_, store, x, rmap, 2)
    ref = np.zeros(ctx.n, x.dtype)
    restate.contract_map(le, ref, store, lmap, 3)
    y = ctx.av(x)
    assert close(y, ref, 1e-12)
    ctx.set_schedule(native.SCHED_PER_BLOCK)
    assert close(ctx.av(x), y, 1e-12)
    ctx.close()


@pytest.mark.parametrize("model", MODELS)
def test_av_is_hermitian_on_physical_steps(model):
    """<u|H v> = <H u|v>: the reference's check_hermitian (src/core.cpp:40-83) as a
    size-independent property (bosonic models need the sign fix)."""
    rng = np.random.default_rng(0)
    for st in load_steps(model):
        ctx = native.Context(native.C128 if st["complex"] else native.F64)
        ctx.plan_build(st["lenv"], st["renv"], st["l_num"], st["r_num"], st["sector"],
                       st["group_n"], st["fermion"])
        u = rng.standard_normal(ctx.n) + (1j * rng.standard_normal(ctx.n) if st["complex"] else 0)
        v = rng.standard_normal(ctx.n) + (1j * rng.standard_normal(ctx.n) if st["complex"] else 0)
        a = np.vdot(u, ctx.av(v))
        b = np.vdot(ctx.av(u), v)
        assert abs(a - b) <= 1e-11 * max(abs(a), 1.0)


def test_av_small_odd_and_empty_blocks():
    """Tiny, odd and zero-size sectors: m=2..7 microbench structures."""
    for m in (9, 13, 21, 35):
        w = workloads.microbench(m, seed=m)
        ctx = native.Context(native.F64)
        ctx.plan_build(w["lenv"], w["renv"], 3, 2, w["sector"], 32, 0)
        le = restate.QT.from_ibuf(*w["lenv"])
        re_ = restate.QT.from_ibuf(*w["renv"])
        rc = restate.build_context(restate.Group(32), le, re_, 3, 2, w["sector"])
        x = workloads.random_psi(rc.n, seed=m)
        assert close(ctx.av(x), restate.av(rc, x))


def test_av_device_pointers():
    import torch
    mb = load_microbench_m64()
    ctx = native.Context(native.F64)
    ctx.plan_build(mb["lenv"], mb["renv"], 3, 2, mb["sector"], mb["group_n"], 0)
    x = torch.tensor(mb["x"], device="cuda:0")
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    ctx.av_device(x.data_ptr(), y.data_ptr())
    ctx.sync()
    assert close(y.cpu().numpy(), mb["ax"])


@pytest.mark.parametrize("model", MODELS)
def test_av_per_block_schedule_matches_reference(model):
    """The plain FP64 path (one cuBLAS GEMM per task row) on the same plans."""
    for st in load_steps(model):
        ctx = native.Context(native.C128 if st["complex"] else native.F64)
        ctx.set_schedule(native.SCHED_PER_BLOCK)
        ctx.plan_build(st["lenv"], st["renv"], st["l_num"], st["r_num"], st["sector"],
                       st["group_n"], st["fermion"])
        assert close(ctx.av(st["x"]), st["ax"])
        ctx.close()


def test_av_per_block_microbench_m64():
    mb = load_microbench_m64()
    ctx = native.Context(native.F64)
    ctx.set_schedule(native.SCHED_PER_BLOCK)
    ctx.plan_build(mb["lenv"], mb["renv"], 3, 2, mb["sector"], mb["group_n"], 0)
    assert close(ctx.av(mb["x"]), mb["ax"])
    with pytest.raises(native.DmrgxError):
        ctx.set_precision(native.PREC_BF16X3)  # the per-block schedule is FP64 only
