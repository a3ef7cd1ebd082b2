"""dmrgx_av_noalloc: the matvec entry point that allocates nothing.

It exists for callers that cannot call cudaMalloc/cudaFree while applying H_eff
(an eigensolver loop inside a framework whose allocator has reserved the device
memory, or a loop that cannot take the synchronisation allocation may cause).
Its intermediate lives in a fixed static device array shared by all calls, so
the checks run it several times in a row, on different problems, against the
context entry point (dmrgx_plan_from_maps + dmrgx_av) with the same tolerance
as the other matvec tests: max|y - y_ref| <= 1e-13 max|y_ref|.

This file is collected last on purpose (name order), so a run that stops at the
first failure has already run every other test.
"""
import numpy as np
import pytest

from conftest import load_microbench_m64, load_steps
from dmrg_b200 import native
from oracle import restate

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _sizes(meta):
    q = restate.QT.from_ibuf(meta, np.zeros(10 ** 7))
    return np.array([b.size for b in q.blocks], np.int64)


def _problem(kind):
    if kind == "microbench":
        p = load_microbench_m64()
        d_store = p["d_store"]
    else:
        # "xyz": complex, every sign +1; "kitaev": real, fermionic, with rows of
        # sign -1 in rmap (the signs are applied as the operands are loaded)
        p = load_steps(kind)[2 if kind == "kitaev" else 0]
        rs = _sizes(p["renv"][0])
        d_store = max(int(r[2] + rs[r[0]] // r[4] * r[3]) for r in p["rmap"])
    p = dict(p)
    p["d_store"] = d_store
    p["rsizes"] = _sizes(p["renv"][0])
    p["lsizes"] = _sizes(p["lenv"][0])
    p["dtype"] = native.C128 if np.iscomplexobj(p["lenv"][1]) else native.F64
    return p


def _context_result(p, x):
    ctx = native.Context(p["dtype"])
    ctx.plan_from_maps(x.size, p["d_store"], p["rmap"], p["renv"][1], p["rsizes"], p["lmap"],
                       p["lenv"][1], p["lsizes"])
    y = ctx.av(x)
    ctx.close()
    return y


def _noalloc_result(p, x):
    import torch
    dev = torch.device("cuda:0")
    renv = torch.from_numpy(np.ascontiguousarray(p["renv"][1])).to(dev)
    lenv = torch.from_numpy(np.ascontiguousarray(p["lenv"][1])).to(dev)
    xin = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    out = torch.full_like(xin, float("nan"))      # stale garbage must not survive
    stream = torch.cuda.current_stream(dev).cuda_stream
    native.av_noalloc(p["dtype"], x.size, p["d_store"], p["rmap"], renv.data_ptr(),
                      p["rsizes"], p["lmap"], lenv.data_ptr(), p["lsizes"], xin.data_ptr(),
                      out.data_ptr(), stream)
    torch.cuda.synchronize(dev)
    return out.cpu().numpy()


def _close(y, ref):
    return np.abs(y - ref).max() <= TOL * max(np.abs(ref).max(), 1e-300)


def test_noalloc_matches_context_entry_on_consecutive_calls():
    mb, xyz, kit = _problem("microbench"), _problem("xyz"), _problem("kitaev")
    assert (kit["rmap"][:, 6] < 0).any()            # the sign branch is exercised
    rng = np.random.default_rng(42)
    calls = []
    # repeated, then other problems (complex; fermionic signs), then back
    for p in (mb, mb, xyz, kit, kit, mb):
        n = p["x"].size
        x = rng.standard_normal(n)
        if p["dtype"] == native.C128:
            x = x + 1j * rng.standard_normal(n)
        calls.append((p, x))
    for p, x in calls:
        ref = _context_result(p, x)
        got = _noalloc_result(p, x)
        assert _close(got, ref), np.abs(got - ref).max()


def test_noalloc_matches_reference_golden():
    for kind in ("microbench", "kitaev"):
        p = _problem(kind)
        for _ in range(2):
            assert _close(_noalloc_result(p, p["x"]), p["ax"])


def test_noalloc_rejects_oversized_intermediate():
    import torch
    p = _problem("microbench")
    buf = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    with pytest.raises(native.DmrgxError, match="exceeds the fixed 32 MiB scratch"):
        native.av_noalloc(native.F64, p["x"].size, 5 * 2 ** 20, p["rmap"], buf.data_ptr(),
                          p["rsizes"], p["lmap"], buf.data_ptr(), p["lsizes"], buf.data_ptr(),
                          buf.data_ptr(), 0)
