import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def load_steps(model, pbc=False):
    """Golden per-step matvec fixtures of one model (see tests/golden/make_golden.py);
    pbc: the periodic-chain fixtures, each step with its edge pair."""
    z = np.load(os.path.join(GOLDEN, f"steps_{model}{'_pbc' if pbc else ''}.npz"))
    gn, ferm, sector = (int(v) for v in z["group"])
    out = []
    for k in range(int(z["nsteps"])):
        p = f"s{k}_"
        st = dict(
            lenv=(z[p + "lenv_meta"], z[p + "lenv_vals"]),
            renv=(z[p + "renv_meta"], z[p + "renv_vals"]),
            l_num=int(z[p + "nums"][0]), r_num=int(z[p + "nums"][1]),
            rmap=z[p + "rmap"], lmap=z[p + "lmap"], x=z[p + "x"], ax=z[p + "ax"],
            evals=z[p + "evals"], evec=z[p + "evec"],
            group_n=gn, fermion=ferm, sector=sector,
            complex=np.iscomplexobj(z[p + "lenv_vals"]))
        if pbc:
            st.update(ledge=(z[p + "ledge_meta"], z[p + "ledge_vals"]),
                      redge=(z[p + "redge_meta"], z[p + "redge_vals"]),
                      remap=z[p + "remap"], lemap=z[p + "lemap"])
        out.append(st)
    return out


def load_microbench_m64():
    z = np.load(os.path.join(GOLDEN, "microbench_m64.npz"))
    n, d_store, sector, gn = (int(v) for v in z["info"])
    return dict(lenv=(z["lenv_meta"], z["lenv_vals"]), renv=(z["renv_meta"], z["renv_vals"]),
                rmap=z["rmap"], lmap=z["lmap"], x=z["x"], ax=z["ax"], n=n, d_store=d_store,
                sector=sector, group_n=gn, l_num=3, r_num=2, fermion=0, complex=False)


def load_z2cubed():
    """Golden Z2 x Z2 x Z2 (S4E) fixtures, real then complex (tests/golden/make_golden.py)."""
    z = np.load(os.path.join(GOLDEN, "z2cubed.npz"))
    out = []
    for p in ("r_", "c_"):
        n, d_store, sector, gn, ferm, l_num, r_num = (int(v) for v in z[p + "info"])
        out.append(dict(lenv=(z[p + "lenv_meta"], z[p + "lenv_vals"]),
                        renv=(z[p + "renv_meta"], z[p + "renv_vals"]),
                        rmap=z[p + "rmap"], lmap=z[p + "lmap"], x=z[p + "x"], ax=z[p + "ax"],
                        n=n, d_store=d_store, sector=sector, group_n=gn, fermion=ferm,
                        l_num=l_num, r_num=r_num, complex=p == "c_"))
    return out


MODELS = ("kitaev", "xyz", "potts")


@pytest.fixture(scope="session")
def golden_steps():
    return {m: load_steps(m) for m in MODELS}
