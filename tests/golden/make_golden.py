"""Generate the golden fixtures under tests/golden/ from the reference itself.

    make -C oracle && python tests/golden/make_golden.py

Runs the reference DMRG code (built unmodified from its sources into
oracle/_ref by oracle/Makefile) and records:

  steps_<model>.npz   per-step matvec fixtures captured inside the reference's
                      eigensolver call: both environments (metadata + values),
                      the reference task lists rmap/lmap, a seeded random psi x
                      and the reference av(x) (src/core.cpp:22-31), the six
                      lowest Ritz values and the lowest Ritz vector.  One step
                      of each kind the schedule uses: update_two (l_num,r_num)
                      = (3,2), move2right (3,1), move2left (2,2).
  microbench_m64.npz  the U(1) microbench structure at m=64 (same generator as
                      the m=1024 benchmark input), with the reference maps and
                      av(x) from the Z_32-embedded reference build.
  energies.json       final energies and truncation errors of small reference
                      runs, with the exact energies (BdG / ED) beside them.
  z2cubed.npz         random environments under the Z2 x Z2 x Z2 fusion rule
                      (workloads.random_z2cubed, real and complex), with the
                      task lists and av(x) of the reference's S4E build
                      (SYMMETRY 8, FERMION, src/useful.cpp:4-27).

  steps_<model>_pbc.npz, energies_pbc.json
                      the same for periodic chains (the reference's PBC build,
                      global.h:14), each step with its edge pair: ledge/redge
                      and the task lists remap/lemap (src/core.cpp:241-247).

  schedule_<name>.npz
                      every step of a reference dmrg() run in full double
                      precision (energies, truncation error, entropy, first 20
                      singular values), recorded at the reference's own
                      print_energy / print_singular calls: the small runs of
                      RUNS (small_full), BASELINE config 2, XYZ L=64 m=256
                      n=8 (config2; about an hour on 8 host cores), and
                      BASELINE config 4's chain, Potts3 L=48 at m=512, on the
                      reference's growth schedule sweep = -1 (config4).

  svd.npz             the reference's block SVD with truncation (qtensor::svd)
                      on captured step states and a graded-spectrum tensor:
                      inputs, U, V, the kept values per sector and the spectrum.

``python tests/golden/make_golden.py z2cubed`` regenerates only the named
fixtures (steps, microbench, z2cubed, pbc); no argument regenerates all of them.

The files are small (tens of KB) and committed; the GPU box never needs the
reference tree.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import exact, refbind  # noqa: E402
from dmrg_b200 import workloads    # noqa: E402

RUNS = {
    # model: (variant, L, m, sweeps, params, group_n, fermion, exact energy fn)
    "kitaev": ("kitaev", 8, 16, 2, [1.0, 1.0, 0.25], 2, 1,
               lambda: exact.kitaev_bdg(8, 1.0, 1.0, 0.25)),
    "xyz": ("xyz", 8, 16, 2, [1.0, 0.8, 0.5], 2, 0,
            lambda: exact.xyz_ed(8, 1.0, 0.8, 0.5, 0)),
    "potts": ("potts", 6, 27, 2, [1.0, 1.0, 0.0, 0.0], 3, 0,
              lambda: exact.potts_ed(6, 1.0, 1.0, 0)),
}


# periodic chains (the reference's PBC build); Kitaev has no closed form here
RUNS_PBC = {
    "kitaev": ("kitaev_pbc", 8, 16, 2, [1.0, 1.0, 0.25], 2, 1, lambda: None),
    "xyz": ("xyz_pbc", 8, 16, 2, [1.0, 0.8, 0.5], 2, 0,
            lambda: exact.xyz_ed(8, 1.0, 0.8, 0.5, 0, periodic=True)),
    "potts": ("potts_pbc", 6, 27, 2, [1.0, 1.0, 0.0, 0.0], 3, 0,
              lambda: exact.potts_ed(6, 1.0, 1.0, 0, periodic=True)),
}


def pick_steps(steps):
    """Last captured step of each (l_num, r_num) kind (largest bond dimension)."""
    out = {}
    for st in steps:
        k = (st["info"]["l_num"], st["info"]["r_num"])
        out[k] = st
    return [out[k] for k in sorted(out)]


def make_steps(runs=RUNS, suffix=""):
    energies = {}
    for model, (variant, L, m, n, par, gn, ferm, exact_fn) in runs.items():
        R = refbind.Ref(variant)
        cap = refbind.StepCapture(want=lambda i, info: True)
        res = R.run(model, L, m, n, 0, par, capture=cap)
        chosen = pick_steps(cap.steps)
        arrs = {}
        for k, st in enumerate(chosen):
            p = f"s{k}_"
            arrs[p + "lenv_meta"], arrs[p + "lenv_vals"] = st["lenv"]
            arrs[p + "renv_meta"], arrs[p + "renv_vals"] = st["renv"]
            arrs[p + "nums"] = np.array([st["info"]["l_num"], st["info"]["r_num"]], np.int32)
            arrs[p + "rmap"] = st["rmap"]
            arrs[p + "lmap"] = st["lmap"]
            arrs[p + "x"] = st["x"]
            arrs[p + "ax"] = st["ax"]
            arrs[p + "evals"] = st["evals"]
            arrs[p + "evec"] = st["evec"]
            if "ledge" in st:
                arrs[p + "ledge_meta"], arrs[p + "ledge_vals"] = st["ledge"]
                arrs[p + "redge_meta"], arrs[p + "redge_vals"] = st["redge"]
                arrs[p + "remap"] = st["remap"]
                arrs[p + "lemap"] = st["lemap"]
        arrs["nsteps"] = np.array(len(chosen))
        arrs["group"] = np.array([gn, ferm, 0], np.int32)  # group_n, fermion, sector
        np.savez_compressed(os.path.join(HERE, f"steps_{model}{suffix}.npz"), **arrs)
        e_exact = exact_fn()
        energies[model] = dict(
            args=dict(L=L, m=m, n=n, params=par, sector=0),
            final_energy=float(res["energy"][-1, 2]),
            energy_rows=res["energy"][:, :3].tolist(),
            trunc_err_rows=res["singular"][:, [0, 1, -1]].tolist(),
            exact=e_exact)
        print(model + suffix, "steps", len(cap.steps), "E", res["energy"][-1, 2], "exact",
              e_exact)
    with open(os.path.join(HERE, f"energies{suffix}.json"), "w") as fh:
        json.dump(energies, fh, indent=1)


def make_steps_pbc():
    """Per-step fixtures of periodic chains, with the edge pair of every step."""
    make_steps(RUNS_PBC, "_pbc")


def make_microbench():
    """The U(1) microbench at m=64 through the Z_32 reference build."""
    w = workloads.microbench(64)
    R = refbind.Ref("u1")
    le = R.py_to_qt(0, *w["lenv"])
    re_ = R.py_to_qt(0, *w["renv"])
    info = (refbind.C.c_int * 4)()
    box = R.lib.oref_pv_build(0, le, re_, 3, 2, w["sector"], info)
    n = info[0]
    pv_info = dict(l_num=3, r_num=2, n_rmap=info[2], n_lmap=info[3])
    rmap, lmap = R.pv_maps(0, box, pv_info)
    x = workloads.random_psi(n, seed=11)
    ax = np.zeros(n)
    R.lib.oref_av(0, box, x.ctypes.data, ax.ctypes.data)
    np.savez_compressed(os.path.join(HERE, "microbench_m64.npz"),
                        lenv_meta=w["lenv"][0], lenv_vals=w["lenv"][1],
                        renv_meta=w["renv"][0], renv_vals=w["renv"][1],
                        rmap=rmap, lmap=lmap, x=x, ax=ax,
                        info=np.array([n, info[1], w["sector"], w["group_n"]], np.int64))
    R.lib.oref_pv_free(0, box)
    print("microbench m=64: n", n, "d_store", info[1], "tasks", info[2], info[3])


def make_z2cubed():
    """Task lists and av(x) of the reference's S4E build on random Z2^3 inputs."""
    R = refbind.Ref("s4e")
    arrs = {}
    for cplx in (0, 1):
        w = workloads.random_z2cubed(seed=3, complex_=bool(cplx), msize=3)
        le = R.py_to_qt(cplx, *w["lenv"])
        re_ = R.py_to_qt(cplx, *w["renv"])
        info = (refbind.C.c_int * 4)()
        box = R.lib.oref_pv_build(cplx, le, re_, w["l_num"], w["r_num"], w["sector"], info)
        n = info[0]
        rmap, lmap = R.pv_maps(cplx, box, dict(n_rmap=info[2], n_lmap=info[3]))
        x = workloads.random_psi(n, seed=11, complex_=bool(cplx))
        ax = np.zeros_like(x)
        R.lib.oref_av(cplx, box, x.ctypes.data, ax.ctypes.data)
        R.lib.oref_pv_free(cplx, box)
        p = "c_" if cplx else "r_"
        arrs[p + "lenv_meta"], arrs[p + "lenv_vals"] = w["lenv"]
        arrs[p + "renv_meta"], arrs[p + "renv_vals"] = w["renv"]
        arrs[p + "rmap"], arrs[p + "lmap"], arrs[p + "x"], arrs[p + "ax"] = rmap, lmap, x, ax
        arrs[p + "info"] = np.array([n, info[1], w["sector"], w["group_n"], w["fermion"],
                                     w["l_num"], w["r_num"]], np.int64)
        print("z2cubed", "complex" if cplx else "real", "n", n, "d_store", info[1],
              "tasks", info[2], info[3])
    np.savez_compressed(os.path.join(HERE, "z2cubed.npz"), **arrs)


def record_schedule(name, variant, model, L, m, n, params, sector=0):
    """Every step of one reference dmrg() run in full double precision.

    Rows in schedule order, taken at the reference's own print_energy and
    print_singular calls (the oracle link wraps both, oracle/ref_hooks.cpp):
    (l, r), the six printed eigenvalues, the truncation error and entropy the
    reference computes (src/useful.cpp:75-102) and its first 20 singular values."""
    import time
    R = refbind.Ref(variant)
    t0 = time.time()
    res = R.run(model, L, m, n, sector, params)
    secs = time.time() - t0
    en, sv = res["en"], res["sv"]
    assert len(en) == len(sv), (len(en), len(sv))
    lr = np.array([[e["l"], e["r"]] for e in en], np.int32)
    assert np.array_equal(lr, np.array([[x["l"], x["r"]] for x in sv], np.int32))
    evals = np.zeros((len(en), 6))
    for i, e in enumerate(en):
        evals[i, :len(e["evals"])] = e["evals"]
    s20 = np.zeros((len(sv), 20))
    for i, x in enumerate(sv):
        k = min(20, len(x["s"]))
        s20[i, :k] = x["s"][:k]
    np.savez_compressed(
        os.path.join(HERE, f"schedule_{name}.npz"), lr=lr, evals=evals,
        trunc=np.array([x["trunc"] for x in sv]), entropy=np.array([x["entropy"] for x in sv]),
        cutoff=np.array([x["cutoff"] for x in sv], np.int32), s20=s20,
        nsv=np.array([len(x["s"]) for x in sv], np.int32),
        args=np.array([L, m, n, sector], np.int32), params=np.array(params, np.float64),
        ref_seconds=np.array(secs))
    print(name, "rows", len(en), "E", evals[-1, 0], "seconds", round(secs, 1))


def make_config2():
    """XYZ L=64, m=256, 8 sweeps, the reference schedule (jx=1, jy=0.8, jz=0.5)."""
    record_schedule("xyz_L64_m256", "xyz", "xyz", 64, 256, 8, [1.0, 0.8, 0.5])


def make_config4():
    """Potts3 L=48 at m=512 (f=1, j=1, p=t=0): the reference's dmrg() with
    sweep = -1, its growth schedule (two_sites, then update_two to the middle
    with cutoff 512 at every step, src/functions.cpp:169-182).  Bond dimensions
    reach 512 from the sixth step on.  About half an hour on 8 host cores."""
    record_schedule("potts_L48_m512_growth", "potts", "potts", 48, 512, -1,
                    [1.0, 1.0, 0.0, 0.0])


def make_small_full():
    """Full-precision rows of the small golden runs (same arguments as RUNS)."""
    for model, (variant, L, m, n, par, gn, ferm, exact_fn) in RUNS.items():
        record_schedule(f"{model}_L{L}_m{m}", variant, model, L, m, n, par)


def psi_meta(R, cplx, lenv, lnum, renv, rnum, sector):
    """The psi layout of a step (generate_dim_sym, src/useful.cpp:151-194) as qtensor
    metadata; psi's legs carry direction 0 (the reference's qtensor(val, dim, sym)
    constructor, src/qtensor.cpp:25-48)."""
    le = R.py_to_qt(cplx, *lenv)
    re_ = R.py_to_qt(cplx, *renv)
    need = R.lib.oref_gen_dim_sym(cplx, le, lnum, re_, rnum, sector, None, 0)
    out = np.zeros(need, np.int32)
    R.lib.oref_gen_dim_sym(cplx, le, lnum, re_, rnum, sector,
                           out.ctypes.data_as(refbind.C.POINTER(refbind.C.c_int)), need)
    nleg = int(out[0])
    head = 2 + nleg + int(out[2:2 + nleg].sum())
    return np.concatenate([out[:head], np.zeros(nleg, np.int32), out[head:]])


def reference_svd(R, cplx, meta, vals, num, cutoff):
    """The reference's qtensor::svd (src/qtensor.cpp:1122-1262) on one tensor:
    U, S (diagonal blocks: the kept values per sector) and V serialised, and the
    whole spectrum it returns."""
    C = refbind.C
    a = R.py_to_qt(cplx, meta, vals)
    U, S, V = C.c_void_p(), C.c_void_p(), C.c_void_p()
    cap = int(np.asarray(vals).size) + 16
    sv = np.zeros(cap)
    ns = R.lib.oref_svd(cplx, a, num, cutoff, C.byref(U), C.byref(S), C.byref(V),
                        sv.ctypes.data_as(C.POINTER(C.c_double)), cap)
    out = dict(u=R.qt_to_py(cplx, U.value), sdiag=R.qt_to_py(0, S.value),
               v=R.qt_to_py(cplx, V.value), s=sv[:ns].copy())
    R.lib.oref_qt_free(cplx, U.value)
    R.lib.oref_qt_free(0, S.value)
    R.lib.oref_qt_free(cplx, V.value)
    return out


def make_svd():
    """Block SVD fixtures: the reference's qtensor::svd on the same inputs the
    GPU test gives dmrgx_svd.  Inputs: the lowest Ritz vector of one captured
    step of each model (their spectra fall to 1e-15 and exact zeros), and the
    m=64 U(1) microbench psi with every block scaled by 10^-(2b mod 15) (a
    graded spectrum with values far below 1e-8 s_0), each with a cutoff that
    truncates."""
    arrs = {}
    cases = []
    for model, variant, gn, ferm in (("kitaev", "kitaev", 2, 1), ("xyz", "xyz", 2, 0),
                                     ("potts", "potts", 3, 0)):
        z = np.load(os.path.join(HERE, f"steps_{model}.npz"))
        k = int(z["nsteps"]) - 1
        p = f"s{k}_"
        cplx = int(np.iscomplexobj(z[p + "lenv_vals"]))
        R = refbind.Ref(variant)
        ln, rn = (int(v) for v in z[p + "nums"])
        meta = psi_meta(R, cplx, (z[p + "lenv_meta"], z[p + "lenv_vals"]), ln - 1,
                        (z[p + "renv_meta"], z[p + "renv_vals"]), rn, 0)
        num = 2 if meta[0] == 4 else 1
        cases.append((model, R, cplx, meta, z[p + "evec"], num, 6, gn, ferm))
    w = workloads.microbench(64)
    R = refbind.Ref("u1")
    meta = psi_meta(R, 0, w["lenv"], 2, w["renv"], 2, w["sector"])
    nblk = int(meta[1])
    nleg = int(meta[0])
    nsec = meta[2:2 + nleg]
    dims = []
    o = 2 + nleg
    for l in range(nleg):
        dims.append(meta[o:o + nsec[l]])
        o += nsec[l]
    sym = meta[o + nleg:].reshape(nblk, nleg)
    rng = np.random.default_rng(5)
    parts = []
    for b in range(nblk):
        size = int(np.prod([dims[l][sym[b, l]] for l in range(nleg)]))
        parts.append(rng.standard_normal(size) * 10.0 ** (-((2 * b) % 15)))
    cases.append(("graded_u1", R, 0, meta, np.concatenate(parts), 2, 40, w["group_n"], 0))
    for name, R, cplx, meta, vals, num, cutoff, gn, ferm in cases:
        ref = reference_svd(R, cplx, meta, vals, num, cutoff)
        p = name + "_"
        arrs[p + "meta"], arrs[p + "vals"] = meta, vals
        arrs[p + "args"] = np.array([num, cutoff, gn, ferm, cplx], np.int32)
        arrs[p + "u_meta"], arrs[p + "u_vals"] = ref["u"]
        arrs[p + "v_meta"], arrs[p + "v_vals"] = ref["v"]
        arrs[p + "sd_meta"], arrs[p + "sd_vals"] = ref["sdiag"]
        arrs[p + "s"] = ref["s"]
        print("svd", name, "values", ref["s"].size, "s0", ref["s"][0], "min", ref["s"][-1])
    arrs["cases"] = np.array([c[0] for c in cases])
    np.savez_compressed(os.path.join(HERE, "svd.npz"), **arrs)


PARTS = {"steps": make_steps, "microbench": make_microbench, "z2cubed": make_z2cubed,
         "pbc": make_steps_pbc, "small_full": make_small_full, "svd": make_svd, "config2": make_config2,
         "config4": make_config4}


def main(parts):
    # config2 and config4 take up to an hour of host time each: only when named
    for name in parts or [p for p in PARTS if p not in ("config2", "config4")]:
        PARTS[name]()


if __name__ == "__main__":
    main(sys.argv[1:])
