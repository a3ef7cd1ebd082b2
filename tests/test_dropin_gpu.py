"""The drop-in proven through the reference's own code.

oracle/_ref/liboref_<model>_dropin.so is the reference DMRG code built from its
unmodified sources with its two ARPACK wrappers (src/dsaupd.cpp, src/znaupd.cpp)
replaced by the maintainer's file dmrg_b200/dropin/dmrgx_znaupd.cpp, linked to
libdmrgx.so (oracle/Makefile, DROPINS).  Running the reference's dmrg()
schedule (src/functions.cpp:157-227) through it, every site step's eigenproblem
is handed to the GPU by the reference's own step functions (src/core.cpp:139,
251, 353, 450) with the reference's own task lists.  Each step's energies,
truncation error, entropy and singular values must equal those of the
reference run with ARPACK, recorded in full precision (tests/golden/
schedule_*.npz), to the bars of test_dmrg_gpu.check_schedule.
"""
import os

import numpy as np
import pytest

from oracle import refbind

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [("kitaev", "kitaev_L8_m16"), ("xyz", "xyz_L8_m16"), ("potts", "potts_L6_m27")]


def _rows(res):
    """A reference run's recorded rows in the layout of a dmrgx_dmrg result."""
    en, sv = res["en"], res["sv"]
    evals = np.zeros((len(en), 6))
    for i, e in enumerate(en):
        evals[i, :len(e["evals"])] = e["evals"]
    s20 = np.zeros((len(sv), 20))
    for i, x in enumerate(sv):
        s20[i, :min(20, len(x["s"]))] = x["s"][:20]
    return dict(lr=np.array([[e["l"], e["r"]] for e in en], np.int32), energies=evals,
                trunc=np.array([x["trunc"] for x in sv]),
                entropy=np.array([x["entropy"] for x in sv]), s20=s20,
                nsv=np.array([len(x["s"]) for x in sv], np.int32))


def test_dropin_library_binds_znaupd_to_libdmrgx():
    """CPU: the drop-in build loads, and its znaupd comes from the drop-in file
    (libdmrgx.so is among its dependencies; no ARPACK hook)."""
    import subprocess
    path = os.path.join(refbind.REFDIR, "liboref_xyz_dropin.so")
    if not os.path.exists(path):
        pytest.skip("drop-in oracle variant not built")
    dyn = subprocess.run(["readelf", "-d", path], capture_output=True, text=True).stdout
    assert "libdmrgx.so" in dyn
    syms = subprocess.run(["nm", "-D", "--undefined-only", path], capture_output=True,
                          text=True).stdout
    assert "dmrgx_plan_from_maps" in syms and "dmrgx_eigsolve" in syms
    refbind.Ref("xyz_dropin")


@pytest.mark.gpu
@pytest.mark.parametrize("model,fixture", CASES)
def test_reference_dmrg_through_dropin(model, fixture):
    from test_dmrg_gpu import check_schedule, load_schedule
    g = load_schedule(fixture)
    L, m, n, sector = (int(v) for v in g["args"])
    R = refbind.Ref(model + "_dropin")
    r = _rows(R.run(model, L, m, n, sector, g["params"].tolist()))
    print(model, "drop-in: max dE/E %.1e dtrunc %.1e dS %.1e ds %.1e" % check_schedule(r, g))
