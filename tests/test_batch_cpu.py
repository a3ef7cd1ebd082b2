"""Config-5 chain list: 16 XYZ chains, Jz ~ U[0.2, 1.0] from the fixed seed, four
chains at each bond dimension."""
import numpy as np

from dmrg_b200 import batch


def test_config5_chain_list():
    ch = batch.config5_chains()
    assert len(ch) == 16
    assert [c["m"] for c in ch] == [64] * 4 + [128] * 4 + [256] * 4 + [512] * 4
    jz = np.array([c["params"][2] for c in ch])
    assert np.all((jz >= 0.2) & (jz <= 1.0))
    assert all(c["L"] == 64 and c["params"][0] == 1.0 and c["params"][1] == 0.8 and
               c["params"][3] == 0.0 for c in ch)
    assert np.array_equal(jz, [c["params"][2] for c in batch.config5_chains()])
