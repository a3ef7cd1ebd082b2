"""Many independent DMRG chains on one GPU at once, with gradient checks.

Each chain gets its own context (its own CUDA stream, plan and buffers); a pool of
host threads drives them, so the chains' kernels interleave on the device.  With
grouped=True the chains of one bond dimension run in lock step: each site step's
eigensolve of all of them is one Lanczos whose matvecs are one grouped launch per
stage (native.Group).  The
library releases the GIL in every call (ctypes) and keeps no cross-context state
but the cuSOLVER function table and the split-tiling cache, both thread-safe; all
per-step device memory is stream-ordered, so one chain's frees never wait for
another chain's kernels.

Per chain (XYZ, jx, jy, jz, h):
  * the reference dmrg() schedule at bond dimension m (dmrgx_dmrg),
  * dE/dJz and dE/dh by the adjoint effective-Hamiltonian sweep (dmrgx_adjoint),
    optionally with the environments rebuilt from the MPS first,
  * Hellmann-Feynman <Psi|dH/dp|Psi> by dmrgx_expect with the unit coupling e_p,
  * central finite differences of whole runs at p +- step.
"""
import concurrent.futures as cf
import time

import numpy as np

from . import native

JX, JY = 1.0, 0.8


def config5_chains(seed=20261203, L=64, ms=(64, 128, 256, 512), per_m=4):
    """16 XYZ chains: Jz ~ U[0.2, 1.0] from `seed`, m in ms (per_m chains each), h = 0."""
    rng = np.random.default_rng(seed)
    jz = rng.uniform(0.2, 1.0, size=len(ms) * per_m)
    out = []
    for i, z in enumerate(jz):
        out.append(dict(chain=i, L=L, m=int(ms[i // per_m]), params=[JX, JY, float(z), 0.0]))
    return out


def _energy(spec, par, sweeps, prec, model, group=None):
    c = native.Context(native.F64 if model == "xyz_real" else native.C128)
    if prec:
        c.set_precision(prec)
    if group is not None:
        c.set_group(group)
    r = c.dmrg(model, spec["L"], spec["m"], sweeps, par)
    if group is not None:
        c.set_group(None)
    return c, r


def run_chain(spec, sweeps=2, prec=native.PREC_FP64, fd_step=1e-4, recompute=True,
              model="xyz_real", fd=True, group=None):
    t0 = time.time()
    par = list(spec["params"])
    c, r = _energy(spec, par, sweeps, prec, model, group)
    e0 = float(r["energies"][-1, 0])
    t_dmrg = time.time() - t0
    a = c.adjoint(nparams=4, recompute=recompute)
    g = a["dE_dparams"]
    hf = []
    for p in (2, 3):
        unit = np.zeros(4)
        unit[p] = 1.0
        hf.append(c.expect(unit))
    res = dict(chain=spec["chain"], L=spec["L"], m=spec["m"], jz=par[2], E0=e0,
               dE_dJz=float(g[2]), dE_dh=float(g[3]), hf_Jz=hf[0], hf_h=hf[1],
               checks=[float(x) for x in a["checks"]], t_dmrg=t_dmrg, t_adjoint=a["seconds"],
               matvecs=int(r["matvecs"].sum()))
    c.close()
    if fd:
        fds = []
        for p in (2, 3):
            pp, pm = list(par), list(par)
            pp[p] += fd_step
            pm[p] -= fd_step
            cp, rp = _energy(spec, pp, sweeps, prec, model)
            cp.close()
            cm, rm = _energy(spec, pm, sweeps, prec, model)
            cm.close()
            fds.append((float(rp["energies"][-1, 0]) - float(rm["energies"][-1, 0])) / (2 * fd_step))
        res["fd_Jz"], res["fd_h"] = fds
        res["rel_fd_Jz"] = abs(res["fd_Jz"] - res["dE_dJz"]) / abs(res["dE_dJz"])
        res["abs_fd_h"] = abs(res["fd_h"] - res["dE_dh"])
    res["rel_hf_Jz"] = abs(res["hf_Jz"] - res["dE_dJz"]) / abs(res["dE_dJz"])
    res["abs_hf_h"] = abs(res["hf_h"] - res["dE_dh"])
    res["wall"] = time.time() - t0
    return res


def run_batch(specs, workers=None, grouped=False, **kw):
    """Run every chain concurrently (one host thread and one context per chain,
    up to `workers` at a time).  Returns (results in chain order, wall seconds).

    grouped: the chains of one (L, m) form a solve group (native.Group): their
    DMRG runs meet at every site step, whose eigensolve is one lock-step Lanczos
    with one grouped FP64 matvec launch per stage for all of them.  Chains of
    different m follow different schedules (the pre-sweeps depend on m), so they
    form different groups.  Needs FP64; every chain gets its own thread, so
    every group can assemble.  The group counters come back in each result."""
    groups = {}
    if grouped:
        if kw.get("prec", native.PREC_FP64) != native.PREC_FP64:
            raise ValueError("solve groups run the FP64 matvec")
        sizes = {}
        for sp in specs:
            sizes[(sp["L"], sp["m"])] = sizes.get((sp["L"], sp["m"]), 0) + 1
        groups = {k: native.Group(v) for k, v in sizes.items()}
        workers = len(specs)
    workers = workers or len(specs)
    t0 = time.time()

    def one(sp):
        g = groups.get((sp["L"], sp["m"]))
        r = run_chain(sp, group=g, **kw)
        if g is not None:
            r["group_stats"] = dict(zip(("rounds", "launches", "member_matvecs"), g.stats()))
        return r

    with cf.ThreadPoolExecutor(max_workers=workers) as ex:
        res = list(ex.map(one, specs))
    wall = time.time() - t0
    for g in groups.values():
        g.close()
    return res, wall


def main():
    import argparse
    import json

    ap = argparse.ArgumentParser(description="16-chain gradient check (XYZ, L=64, m in {64..512})")
    ap.add_argument("--sweeps", type=int, default=2)
    ap.add_argument("--prec", default="bf16x3", choices=["fp64", "bf16x3", "tf32x3"])
    ap.add_argument("--workers", type=int, default=16)
    ap.add_argument("--L", type=int, default=64)
    ap.add_argument("--no-fd", action="store_true")
    ap.add_argument("--grouped", action="store_true",
                    help="chains of one bond dimension in one solve group (FP64)")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    prec = {"fp64": native.PREC_FP64, "bf16x3": native.PREC_BF16X3,
            "tf32x3": native.PREC_TF32X3}[a.prec]
    specs = config5_chains(L=a.L)
    if a.grouped:
        prec, a.prec = native.PREC_FP64, "fp64"
    res, wall = run_batch(specs, workers=a.workers, grouped=a.grouped, sweeps=a.sweeps, prec=prec,
                          fd=not a.no_fd)
    summary = {"wall_s": wall, "chains": len(res), "sweeps": a.sweeps, "prec": a.prec,
               "grouped": a.grouped,
               "max_rel_hf_Jz": max(r["rel_hf_Jz"] for r in res),
               "max_abs_hf_h": max(r["abs_hf_h"] for r in res)}
    if a.grouped:
        summary["groups"] = {str(r["m"]): r["group_stats"] for r in res}
    if not a.no_fd:
        summary["max_rel_fd_Jz"] = max(r["rel_fd_Jz"] for r in res)
        summary["max_abs_fd_h"] = max(r["abs_fd_h"] for r in res)
    out = {"summary": summary, "chains": res}
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(out, fh, indent=1)
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
