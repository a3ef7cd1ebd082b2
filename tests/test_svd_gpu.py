"""Block SVD with truncation on the GPU (dmrgx_svd) against the reference's
qtensor::svd (src/qtensor.cpp:1122-1262) on the same inputs.

Fixtures (tests/golden/svd.npz, made by make_golden.py svd): the lowest Ritz
vectors of captured Kitaev / XYZ / Potts steps, whose spectra fall to 1e-15 and
exact zeros, and a graded-spectrum U(1) tensor with values far below 1e-8 s_0.

Bars:
  * U and V metadata (legs, sectors, blocks, directions) identical;
  * the whole spectrum to 1e-13 s_0;
  * every kept singular vector whose value is separated from its neighbours in
    its sector by at least 1e-5 s_0 to 1e-10 up to a phase, with V's row
    carrying the opposite phase (a vector's error is ~1e-16 s_0 / gap, so
    vectors of clustered values are compared through the projector on their
    cluster instead);
  * every sector block of U and V unitary to 1e-12 (the complement columns the
    reference pads with are arbitrary, but must complete the kept ones).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from dmrg_b200 import native
from oracle import restate

pytestmark = pytest.mark.gpu

Z = np.load(os.path.join(GOLDEN, "svd.npz"))
CASES = [str(c) for c in Z["cases"]]
S_TOL = 1e-13
VEC_TOL = 1e-10
GAP = 1e-5


def _qt(meta, vals):
    return restate.QT.from_ibuf(meta, vals)


def _sectors(q, k_last):
    """k label -> matrix of the sector's singular vectors (U: columns, V: rows),
    blocks stacked in block order."""
    out = {}
    for sym, b in zip(q.syms, q.blocks):
        if k_last:
            lab = sym[-1]
            mat = b.reshape(-1, b.shape[-1])
            out[lab] = mat if lab not in out else np.vstack([out[lab], mat])
        else:
            lab = sym[0]
            mat = b.reshape(b.shape[0], -1)
            out[lab] = mat if lab not in out else np.hstack([out[lab], mat])
    return out


@pytest.mark.parametrize("name", CASES)
def test_block_svd_matches_reference(name):
    p = name + "_"
    num, cutoff, gn, ferm, cplx = (int(v) for v in Z[p + "args"])
    ctx = native.Context(native.C128 if cplx else native.F64)
    (um, uv), (vm, vv), s = ctx.svd(Z[p + "meta"], Z[p + "vals"], num, cutoff, gn, ferm)
    ctx.close()
    assert np.array_equal(um, Z[p + "u_meta"]), "U metadata differs"
    assert np.array_equal(vm, Z[p + "v_meta"]), "V metadata differs"
    s_ref = Z[p + "s"]
    s0 = s_ref[0]
    assert s.shape == s_ref.shape
    ds = np.abs(s - s_ref).max() / s0
    assert ds <= S_TOL, ds
    cut = s_ref[cutoff] if 0 < cutoff < s_ref.size else 0.0  # largest discarded value
    U, Ur = _sectors(_qt(um, uv), True), _sectors(_qt(um, Z[p + "u_vals"]), True)
    V, Vr = _sectors(_qt(vm, vv), False), _sectors(_qt(vm, Z[p + "v_vals"]), False)
    sd = _qt(Z[p + "sd_meta"], Z[p + "sd_vals"])
    # S's diagonal blocks (a, b): the kept values of the sector whose k leg is
    # labelled a in U and b in V (the labels fuse to the tensor's sector)
    kept = {sym[0]: np.diag(b) for sym, b in zip(sd.syms, sd.blocks)}
    vlab = {sym[0]: sym[1] for sym in sd.syms}
    for lab, vb in V.items():
        assert np.abs(vb @ vb.conj().T - np.eye(vb.shape[0])).max() <= 1e-12, lab
    worst, compared = 0.0, 0
    for lab, a in U.items():
        uni = np.abs(a.conj().T @ a - np.eye(a.shape[1])).max()
        assert uni <= 1e-12, (lab, uni)
        if lab not in vlab or vlab[lab] not in V:
            continue
        vb, vbr = V[vlab[lab]], Vr[vlab[lab]]
        sk = kept.get(lab, np.zeros(0))
        j = 0
        while j < sk.size:
            # the cluster of values within GAP of each other, starting at j
            e = j + 1
            while e < sk.size and sk[e - 1] - sk[e] < GAP * s0:
                e += 1
            below = sk[e] if e < sk.size else cut
            if sk[e - 1] - below >= GAP * s0 and (j == 0 or sk[j - 1] - sk[j] >= GAP * s0):
                if e == j + 1:
                    ph = np.vdot(a[:, j], Ur[lab][:, j])
                    ph /= abs(ph)
                    err_u = np.abs(a[:, j] * ph - Ur[lab][:, j]).max()
                    err_v = np.abs(vb[j] * np.conj(ph) - vbr[j]).max()
                    err = max(err_u, err_v)
                else:
                    P = a[:, j:e] @ a[:, j:e].conj().T
                    Pr = Ur[lab][:, j:e] @ Ur[lab][:, j:e].conj().T
                    err = np.abs(P - Pr).max()
                worst = max(worst, err)
                compared += e - j
            j = e
    assert compared > 0
    assert worst <= VEC_TOL, worst
    print(name, "spectrum %.1e, vectors %.1e over %d kept" % (ds, worst, compared))
