"""The oracle itself, pinned against the reference's golden outputs (CPU only)."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, MODELS, load_microbench_m64, load_steps, load_z2cubed
from oracle import exact, restate


def _ctx(st):
    G = restate.Group(st["group_n"], bool(st["fermion"]))
    le = restate.QT.from_ibuf(*st["lenv"])
    re_ = restate.QT.from_ibuf(*st["renv"])
    lx = restate.QT.from_ibuf(*st["ledge"]) if "ledge" in st else None
    rx = restate.QT.from_ibuf(*st["redge"]) if "redge" in st else None
    return restate.build_context(G, le, re_, st["l_num"], st["r_num"], st["sector"], lx, rx)


@pytest.mark.parametrize("model", MODELS)
def test_restatement_maps_and_av_match_reference(model):
    for st in load_steps(model):
        ctx = _ctx(st)
        assert np.array_equal(ctx.rmap, st["rmap"])
        assert np.array_equal(ctx.lmap, st["lmap"])
        y = restate.av(ctx, st["x"])
        assert np.allclose(y, st["ax"], rtol=0, atol=1e-13 * np.abs(st["ax"]).max())


@pytest.mark.parametrize("model", MODELS)
def test_reference_ritz_pair(model):
    """The captured Ritz vector is an eigenvector of the captured operator."""
    for st in load_steps(model):
        ctx = _ctx(st)
        v = st["evec"] / np.linalg.norm(st["evec"])
        hv = restate.av(ctx, v)
        e = np.vdot(v, hv).real
        assert abs(e - st["evals"][0]) < 1e-8 * max(1.0, abs(e))
        assert np.linalg.norm(hv - e * v) < 1e-6 * max(1.0, abs(e))


@pytest.mark.parametrize("model", MODELS)
def test_restatement_periodic_edge_pair(model):
    """PBC build: remap/lemap of the edge pair and av with both pairs (src/core.cpp:27-30)."""
    for st in load_steps(model, pbc=True):
        ctx = _ctx(st)
        assert np.array_equal(ctx.rmap, st["rmap"]) and np.array_equal(ctx.lmap, st["lmap"])
        assert np.array_equal(ctx.remap, st["remap"])
        assert np.array_equal(ctx.lemap, st["lemap"])
        assert len(st["remap"]) and len(st["lemap"])
        y = restate.av(ctx, st["x"])
        assert np.allclose(y, st["ax"], rtol=0, atol=1e-13 * np.abs(st["ax"]).max())
        # the captured Ritz vector is an eigenvector of the operator with both pairs
        v = st["evec"] / np.linalg.norm(st["evec"])
        hv = restate.av(ctx, v)
        e = np.vdot(v, hv).real
        assert abs(e - st["evals"][0]) < 1e-8 * max(1.0, abs(e))


def test_periodic_energies_pin_reference_runs():
    """The PBC reference runs end at the periodic chain's exact energy."""
    with open(os.path.join(GOLDEN, "energies_pbc.json")) as fh:
        en = json.load(fh)
    ex = {"xyz": exact.xyz_ed(8, 1.0, 0.8, 0.5, 0, periodic=True),
          "potts": exact.potts_ed(6, 1.0, 1.0, 0, periodic=True)}
    for m, e in ex.items():
        assert abs(en[m]["exact"] - e) < 1e-12
        assert abs(en[m]["final_energy"] - e) < 2e-10 * abs(e) + 1e-10
    assert en["kitaev"]["exact"] is None


def test_restatement_microbench_m64():
    mb = load_microbench_m64()
    ctx = _ctx(dict(mb, l_num=3, r_num=2))
    assert ctx.n == mb["n"] and ctx.d_store == mb["d_store"]
    assert np.array_equal(ctx.rmap, mb["rmap"]) and np.array_equal(ctx.lmap, mb["lmap"])
    y = restate.av(ctx, mb["x"])
    assert np.allclose(y, mb["ax"], rtol=0, atol=1e-13 * np.abs(mb["ax"]).max())


def test_restatement_z2cubed():
    """Z2 x Z2 x Z2 fusion and parity table (S4E build), real and complex."""
    for z in load_z2cubed():
        ctx = _ctx(z)
        assert ctx.n == z["n"] and ctx.d_store == z["d_store"]
        assert np.array_equal(ctx.rmap, z["rmap"]) and np.array_equal(ctx.lmap, z["lmap"])
        assert set(np.unique(z["rmap"][:, 6])) == {-1, 1}  # both parity signs occur
        y = restate.av(ctx, z["x"])
        assert np.allclose(y, z["ax"], rtol=0, atol=1e-13 * np.abs(z["ax"]).max())


def test_z2cubed_rule():
    """XOR fusion with -b standing for b; parity odd exactly for labels 2..5."""
    G = restate.Group(-8, True)
    for a in range(8):
        for b in range(8):
            assert G.ss(a, b) == a ^ b and G.ss(a, -b) == a ^ b
    assert [G.ff(a) for a in range(8)] == [0, 0, 1, 1, 1, 1, 0, 0]
    assert restate.Group(-8, False).ff(3) == 0


def test_tensor_text_format_pinned_to_reference_reader(tmp_path):
    """The restated tensor::write_file / read_file pair against the reference's own
    read_file (src/tensor.cpp:260-296), real and complex, including a zero extent."""
    from oracle import refbind
    if not refbind.available("xyz"):
        pytest.skip("oracle/_ref not built in this checkout")
    R = refbind.Ref("xyz")
    rng = np.random.default_rng(4)
    for cplx in (0, 1):
        for ext in ([3, 1, 4], [2, 5], [1, 0, 2]):
            v = rng.standard_normal(int(np.prod(ext)))
            if cplx:
                v = v + 1j * rng.standard_normal(v.size)
            v = v * 10.0 ** rng.integers(-12, 12, v.size)
            line = restate.format_tensor_text(ext, v, bool(cplx))
            path = tmp_path / f"t{cplx}_{len(ext)}.txt"
            path.write_text(line + "\n")
            idx, ref_vals = R.tensor_read(cplx, str(path))
            e2, mine, _ = restate.read_tensor_text(line.split(), 0, bool(cplx))
            assert list(idx[: len(ext)]) == ext == e2
            assert np.array_equal(ref_vals, v) and np.array_equal(mine, v)


def test_state_file_reader(tmp_path):
    """The oracle's reader of dmrgx state files on a hand-made file: header fields,
    parameters, block metadata and one block line per block (tensor::write_file)."""
    blk = restate.format_tensor_text([2, 1, 3], np.arange(6.0) - 2.5, False)
    zero = restate.format_tensor_text([1, 0, 3], np.zeros(0), False)
    text = "\n".join([
        "dmrgx-mps 1",
        "model 3 L 4 sector 0 m 8 center 1 f 1 energy -1.25",
        "params 3 1 0.8 0.5",
        "centre",
        "3 2", "2 2 1", "2 1 0", "1 3", "0 0 0",
        "0 0 0", "1 1 0",
        blk, zero,
        "end", ""])
    path = tmp_path / "s.txt"
    path.write_text(text)
    st = restate.read_state(str(path))
    assert st["header"] == dict(model=3, L=4, sector=0, m=8, center=1, f=1, energy=-1.25)
    assert st["params"] == [1.0, 0.8, 0.5]
    q = st["tensors"]["centre"]
    assert q.dims == [[2, 1], [1, 0], [3]] and q.syms == [(0, 0, 0), (1, 1, 0)]
    assert np.array_equal(q.blocks[0].ravel(), np.arange(6.0) - 2.5)
    assert q.blocks[1].size == 0


def test_exact_energies_pin_reference_runs():
    with open(os.path.join(GOLDEN, "energies.json")) as fh:
        en = json.load(fh)
    ex = {"kitaev": exact.kitaev_bdg(8, 1.0, 1.0, 0.25),
          "xyz": exact.xyz_ed(8, 1.0, 0.8, 0.5, 0),
          "potts": exact.potts_ed(6, 1.0, 1.0, 0)}
    for m in MODELS:
        assert abs(en[m]["exact"] - ex[m]) < 1e-12
        # the reference prints 10 digits after the point (global.h ACC)
        assert abs(en[m]["final_energy"] - ex[m]) < 2e-10 * abs(ex[m]) + 1e-10


def test_restatement_against_live_reference():
    """When the reference build is present, restatement == reference on fresh inputs."""
    from oracle import refbind
    if not refbind.available("u1"):
        pytest.skip("oracle/_ref not built in this checkout")
    from dmrg_b200 import workloads
    w = workloads.microbench(48, seed=5)
    R = refbind.Ref("u1")
    le, re_ = R.py_to_qt(0, *w["lenv"]), R.py_to_qt(0, *w["renv"])
    info = (refbind.C.c_int * 4)()
    box = R.lib.oref_pv_build(0, le, re_, 3, 2, w["sector"], info)
    rmap, lmap = R.pv_maps(0, box, dict(n_rmap=info[2], n_lmap=info[3]))
    x = workloads.random_psi(info[0], seed=3)
    y = np.zeros_like(x)
    R.lib.oref_av(0, box, x.ctypes.data, y.ctypes.data)
    ctx = _ctx(dict(lenv=w["lenv"], renv=w["renv"], l_num=3, r_num=2, sector=w["sector"],
                    group_n=32, fermion=0))
    assert np.array_equal(ctx.rmap, rmap) and np.array_equal(ctx.lmap, lmap)
    assert np.allclose(restate.av(ctx, x), y, rtol=0, atol=1e-13 * np.abs(y).max())
    R.lib.oref_pv_free(0, box)
