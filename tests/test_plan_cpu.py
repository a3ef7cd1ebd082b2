"""The C ABI library on the host: it loads, exports what include/dmrgx.h
declares, and its sector bookkeeping equals the reference's bit for bit."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import MODELS, ROOT, load_microbench_m64, load_steps, load_z2cubed
from dmrg_b200 import native, workloads


def header_functions():
    txt = open(os.path.join(ROOT, "include", "dmrgx.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(dmrgx_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = native.lib()
    names = header_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(native.SIGNATURES), "ctypes table out of sync with the header"


@pytest.mark.parametrize("model", MODELS)
def test_native_maps_equal_reference(model):
    for st in load_steps(model):
        n, ds, rmap, lmap = native.build_maps(st["lenv"][0], st["renv"][0], st["l_num"],
                                              st["r_num"], st["sector"], st["group_n"],
                                              st["fermion"])
        assert np.array_equal(rmap, st["rmap"])
        assert np.array_equal(lmap, st["lmap"])
        assert n == st["x"].size


def test_native_maps_microbench_m64():
    mb = load_microbench_m64()
    n, ds, rmap, lmap = native.build_maps(mb["lenv"][0], mb["renv"][0], 3, 2, mb["sector"],
                                          mb["group_n"], 0)
    assert (n, ds) == (mb["n"], mb["d_store"])
    assert np.array_equal(rmap, mb["rmap"]) and np.array_equal(lmap, mb["lmap"])


@pytest.mark.parametrize("model", MODELS)
def test_native_maps_periodic_equal_reference(model):
    """The edge pair's task lists (src/core.cpp:241-247) of the reference's PBC build."""
    for st in load_steps(model, pbc=True):
        n, ds, rmap, lmap, es, remap, lemap = native.build_maps_pbc(
            st["lenv"][0], st["renv"][0], st["ledge"][0], st["redge"][0], st["l_num"],
            st["r_num"], st["sector"], st["group_n"], st["fermion"])
        assert n == st["x"].size
        assert np.array_equal(rmap, st["rmap"]) and np.array_equal(lmap, st["lmap"])
        assert np.array_equal(remap, st["remap"]) and np.array_equal(lemap, st["lemap"])
        assert set(np.unique(lemap[:, 5])) <= {1}  # lemap accumulates (beta = 1)


def test_periodic_bookkeeping_errors():
    st = load_steps("xyz", pbc=True)[0]
    with pytest.raises(native.DmrgxError, match="out of range"):
        native.build_maps_pbc(st["lenv"][0], st["renv"][0], st["ledge"][0], st["redge"][0], 9,
                              st["r_num"], st["sector"], st["group_n"], st["fermion"])
    bad = np.array(st["ledge"][0], np.int32)
    bad[-1] = 999  # block label out of range
    with pytest.raises(native.DmrgxError, match="ledge metadata"):
        native.build_maps_pbc(st["lenv"][0], st["renv"][0], bad, st["redge"][0], st["l_num"],
                              st["r_num"], st["sector"], st["group_n"], st["fermion"])
    # with the edge pair equal to the main pair the edge task lists repeat the main ones,
    # except that lemap accumulates (beta = 1)
    n, ds, rmap, lmap, es, remap, lemap = native.build_maps_pbc(
        st["lenv"][0], st["renv"][0], st["lenv"][0], st["renv"][0], st["l_num"], st["r_num"],
        st["sector"], st["group_n"], st["fermion"])
    assert es == ds and np.array_equal(remap, rmap)
    assert np.array_equal(lemap[:, :5], lmap[:, :5]) and (lemap[:, 5] == 1).all()


def test_native_maps_z2cubed():
    """group_n = GROUP_Z2CUBED: the reference's S4E fusion rule and parity table."""
    for z in load_z2cubed():
        n, ds, rmap, lmap = native.build_maps(z["lenv"][0], z["renv"][0], z["l_num"], z["r_num"],
                                              z["sector"], native.GROUP_Z2CUBED, z["fermion"])
        assert (n, ds) == (z["n"], z["d_store"])
        assert np.array_equal(rmap, z["rmap"]) and np.array_equal(lmap, z["lmap"])
    with pytest.raises(native.DmrgxError, match="group_n out of range"):
        native.build_maps(z["lenv"][0], z["renv"][0], 3, 2, 5, -7, 1)


def test_microbench_m1024_sizes():
    """The benchmark input has the stated size: 599,964-element psi, 190+190 tasks."""
    w = workloads.microbench(1024)
    n, ds, rmap, lmap = native.build_maps(w["lenv"][0], w["renv"][0], 3, 2, w["sector"], 32, 0)
    assert (n, ds, len(rmap), len(lmap)) == (599964, 2928712, 190, 190)
    assert w["lenv"][1].size == w["renv"][1].size == 2928712


def test_bad_metadata_is_an_error_not_a_crash():
    w = workloads.microbench(32)
    bad = np.array(w["lenv"][0], np.int32)
    bad[-1] = 999  # block label out of range
    with pytest.raises(native.DmrgxError, match="label out of range"):
        native.build_maps(bad, w["renv"][0], 3, 2, 1, 32, 0)
    with pytest.raises(native.DmrgxError, match="l_num/r_num"):
        native.build_maps(w["lenv"][0], w["renv"][0], 7, 2, 1, 32, 0)
