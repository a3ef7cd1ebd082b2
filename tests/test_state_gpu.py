"""State checkpoints (dmrgx_save_state / dmrgx_load_state).

A state written after a run and read into a fresh context is the same state:
<Psi|H|Psi> and the adjoint gradient on the loaded state equal those on the
original (1e-12 / 1e-10 relative), and writing it again gives the same file.
Every block line is read back by the restated tensor::read_file and, when the
oracle build is present, by the reference's own read_file (src/tensor.cpp:285-296)."""
import numpy as np
import pytest

from dmrg_b200 import native
from oracle import refbind, restate

pytestmark = pytest.mark.gpu

CASES = [("xyz_real", native.F64, [1.0, 0.8, 0.5, 0.0]),
         ("xyz", native.C128, [1.0, 0.8, 0.5, 0.0]),
         ("kitaev", native.F64, [1.0, 1.0, 0.25])]


@pytest.mark.parametrize("model,dtype,par", CASES)
def test_save_load_round_trip(model, dtype, par, tmp_path):
    ctx = native.Context(dtype)
    r = ctx.dmrg(model, 12, 16, 2, par)
    e0 = float(r["energies"][-1, 0])
    ev = ctx.expect(par)
    g = ctx.adjoint(nparams=len(par))["dE_dparams"]
    p1 = tmp_path / "state1.txt"
    ctx.save_state(str(p1))

    st = restate.read_state(str(p1))
    assert st["header"]["L"] == 12 and st["header"]["f"] == (2 if dtype == native.C128 else 1)
    assert abs(st["header"]["energy"] - e0) <= 1e-15 * abs(e0)
    assert "centre" in st["tensors"] and len(st["tensors"]) == 12

    c2 = native.Context(dtype)
    c2.load_state(str(p1))
    ev2 = c2.expect(par)
    assert abs(ev2 - ev) <= 1e-12 * abs(ev), (ev, ev2)
    assert abs(ev2 - e0) <= 1e-9 * abs(e0)
    g2 = c2.adjoint(nparams=len(par))["dE_dparams"]
    assert np.abs(g2 - g).max() <= 1e-10 * np.abs(g).max()

    # loading does not change the state: the file written again is identical
    p2 = tmp_path / "state2.txt"
    ctx3 = native.Context(dtype)
    ctx3.load_state(str(p1))
    ctx3.save_state(str(p2))
    assert p1.read_text() == p2.read_text()

    # block lines through the reference's own reader
    if refbind.available("xyz"):
        R = refbind.Ref("xyz")
        for ln in block_lines(p1.read_text())[:8]:
            one = tmp_path / "one.txt"
            one.write_text(ln + "\n")
            ext, vals = R.tensor_read(int(dtype == native.C128), str(one))
            e2, mine, _ = restate.read_tensor_text(ln.split(), 0, dtype == native.C128)
            assert list(ext[: len(e2)]) == e2 and np.array_equal(vals, mine)


def block_lines(text):
    """The one-line blocks of a state file, found by walking its record layout:
    header, parameters, then per tensor its name, "nleg nblk", nleg sector lines,
    the directions, nblk label lines and nblk block lines."""
    ls = text.splitlines()
    i, out = 3, []
    while ls[i] != "end":
        nleg, nblk = (int(t) for t in ls[i + 1].split())
        i += 2 + nleg + 1 + nblk
        out += ls[i: i + nblk]
        i += nblk
    return out


def test_load_errors(tmp_path):
    ctx = native.Context(native.F64)
    bad = tmp_path / "bad.txt"
    bad.write_text("not a state\n")
    with pytest.raises(native.DmrgxError, match="bad header"):
        ctx.load_state(str(bad))
    with pytest.raises(native.DmrgxError, match="cannot open"):
        ctx.load_state(str(tmp_path / "missing.txt"))
    with pytest.raises(native.DmrgxError, match="no state"):
        ctx.save_state(str(tmp_path / "x.txt"))
    c = native.Context(native.C128)
    c.dmrg("xyz", 8, 8, 1, [1.0, 0.8, 0.5])
    c.save_state(str(tmp_path / "c.txt"))
    with pytest.raises(native.DmrgxError, match="element type"):
        ctx.load_state(str(tmp_path / "c.txt"))
