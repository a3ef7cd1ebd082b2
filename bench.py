"""H_eff matvec benchmark (the m=1024 U(1) microbench) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--prec fp64] [--impl dmrgx|reference]

One step = one application of the two-site effective Hamiltonian
H_eff psi = (L W)((W R) psi) to one wavefunction of the synthetic microbench
(m_l = m_r = 1024 in nine U(1) sectors, d = 2, MPO bond D = 5; 599,964-element
psi, 190 + 190 block GEMMs, 3.862 GFLOP).  Inputs are resident in HBM; L2 is
flushed (a 256 MiB write) between timed steps, outside the timed events.
Multi-GPU runs are independent replicas (one process per GPU, no collective on
the data path); the value is the total over ranks divided by the slowest
rank's device time.

Printed once by rank 0, one JSON line; see the keys below.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "H_eff matvec/s at m=1024 (U(1) microbench, two-site, D=5)"
UNIT = "matvec/s"


TRAFFIC_BF16X3 = 15.136512e6 + 24.813056e6  # bytes per matvec (both stage launches), ncu


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--prec", default="bf16x3", choices=["fp64", "bf16x3", "tf32x3"])
    p.add_argument("--impl", default="dmrgx", choices=["dmrgx", "reference"])
    p.add_argument("--cpu-sample-s", type=float, default=12.0)
    p.add_argument("--config1", type=int, default=1,
                   help="1: BASELINE config 1 (Kitaev L=32, m=64, 6 sweeps) on the GPU beside the "
                        "reference's own run on the host cores")
    p.add_argument("--config5", type=int, default=1,
                   help="1: BASELINE config 5 reduced (8 chains, m in {64, 128}) in solve groups")
    p.add_argument("--sweep", type=int, default=1,
                   help="also time the DMRG schedule (XYZ real chain) in three forms: plain "
                        "per-block FP64, grouped FP64, grouped headline precision")
    p.add_argument("--sweep-L", type=int, default=32)
    p.add_argument("--sweep-m", type=int, default=1024)
    p.add_argument("--sweep-n", type=int, default=1)
    p.add_argument("--probe", default="", choices=["", "eig", "mv"],
                   help="profiling workload instead of the benchmark: the state at the middle "
                        "of an XYZ chain (L=--sweep-L, m=--sweep-m, fast solver schedule), then "
                        "one eigensolve with the reference's settings (eig) or one matvec (mv) "
                        "in the headline precision, inside the NVTX range 'probe'")
    return p.parse_args()


def run_probe(args):
    """A sweep step's matvec / eigensolve at full size, for ncu captures
    (ncu --nvtx --nvtx-include "probe/" ...).  Prints one JSON line."""
    import time
    import torch
    from dmrg_b200 import native
    prec = {"fp64": native.PREC_FP64, "bf16x3": native.PREC_BF16X3,
            "tf32x3": native.PREC_TF32X3}[args.prec]
    c = native.Context(native.F64)
    c.set_solver(1, 12, True)
    c.dmrg("xyz_real", args.sweep_L, args.sweep_m, 0, [1.0, 0.8, 0.5])
    c._refresh()
    c.set_precision(prec)
    x = torch.randn(c.n, dtype=torch.float64, device="cuda:0")
    y = torch.empty_like(x)
    for _ in range(3):                       # split images, tuning, warm caches
        c.av_device(x.data_ptr(), y.data_ptr())
    if args.probe == "eig":
        c.eigsolve(nev=6)
    c.sync()
    torch.cuda.nvtx.range_push("probe")
    t0 = time.time()
    if args.probe == "eig":
        _, _, info = c.eigsolve(nev=6)
    else:
        c.av_device(x.data_ptr(), y.data_ptr())
        info = {"matvecs": 1}
    c.sync()
    dt = time.time() - t0
    torch.cuda.nvtx.range_pop()
    # per-launch device time of 20 more matvecs (outside the NVTX range)
    c.profile(True)
    for _ in range(20):
        c.av_device(x.data_ptr(), y.data_ptr())
    cnt, slots = c.profile_read()
    c.profile(False)
    info["stage_us"] = (slots / max(cnt, 1) * 1e3).round(1).tolist()
    info["tuning"] = [list(t) for t in c.split_tuning()] if prec != native.PREC_FP64 else None
    print(json.dumps({"probe": args.probe, "n": c.n, "gflop_per_matvec": c.flops / 1e9,
                      "precision": args.prec, "seconds": dt, "matvecs": info["matvecs"],
                      "us_per_step": dt / info["matvecs"] * 1e6,
                      "matvec_stage_us": info["stage_us"], "tuning": info["tuning"]}, default=float))


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def fp64_gemm_peak(torch, dev):
    """cuBLAS DGEMM 8192^3 burst on this GPU: the FP64 tensor-core ceiling,
    measured in-run (the driver's peak file carries no FP64 figure)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2 * n ** 3 / best / 1e12


def cpu_reference_rate(sample_s: float, w=None):
    """The reference's CPU av (src/core.cpp:22-31: get_map task lists executed as
    serial BLAS GEMMs, OpenBLAS on all host threads) on this workload.
    Uses the reference build (oracle/_ref) when present, else the numpy port."""
    from oracle import refbind
    from dmrg_b200 import workloads
    if w is None:
        w = workloads.microbench(1024)
    threads = os.cpu_count() or 1
    if refbind.available("u1"):
        R = refbind.Ref("u1")
        le, re_ = R.py_to_qt(0, *w["lenv"]), R.py_to_qt(0, *w["renv"])
        import ctypes as C
        info = (C.c_int * 4)()
        box = R.lib.oref_pv_build(0, le, re_, 3, 2, w["sector"], info)
        n = info[0]
        x = workloads.random_psi(n, seed=1)
        y = np.zeros(n)
        R.lib.oref_av(0, box, x.ctypes.data, y.ctypes.data)  # warm-up
        cnt, t0 = 0, time.perf_counter()
        while True:
            R.lib.oref_av(0, box, x.ctypes.data, y.ctypes.data)
            cnt += 1
            el = time.perf_counter() - t0
            if el >= sample_s or cnt >= 2000:
                break
        R.lib.oref_pv_free(0, box)
        return dict(value=cnt / el, unit=UNIT, cores=threads, kind="reference",
                    sample=f"{cnt} reference av() calls on the m=1024 microbench in {el:.1f} s "
                           f"(reference get_map+av built from its sources, OpenBLAS "
                           f"{threads} threads)")
    from oracle import restate
    from dmrg_b200 import native
    n, ds, rmap, lmap = native.build_maps(w["lenv"][0], w["renv"][0], 3, 2, w["sector"], 32, 0)
    le = restate.QT.from_ibuf(*w["lenv"])
    re_ = restate.QT.from_ibuf(*w["renv"])
    x = workloads.random_psi(n, seed=1)
    cnt, t0 = 0, time.perf_counter()
    while True:
        st = np.zeros(ds)
        restate.contract_map(re_, st, x, rmap, 2)
        y = np.zeros(n)
        restate.contract_map(le, y, st, lmap, 3)
        cnt += 1
        el = time.perf_counter() - t0
        if el >= sample_s or cnt >= 2000:
            break
    return dict(value=cnt / el, unit=UNIT, cores=threads, kind="port",
                sample=f"{cnt} numpy-port matvecs on the m=1024 microbench in {el:.1f} s")


def sweep_compare(native, args):
    """The reference dmrg() schedule on the GPU for the XYZ chain (jx=1, jy=0.8,
    jz=0.5, real MPO) in three forms: the plain FP64 path (one cuBLAS GEMM per
    task row), the grouped FP64 path, and the grouped headline precision.
    sweep_s = wall seconds of the last full sweep (2(L-2) site steps at bond
    dimension m, from the per-step times); schedule_s = the whole schedule."""
    prec = {"fp64": native.PREC_FP64, "bf16x3": native.PREC_BF16X3,
            "tf32x3": native.PREC_TF32X3}[args.prec]
    L = args.sweep_L
    out = {"workload": f"XYZ chain L={L}, m={args.sweep_m}, {args.sweep_n} sweep(s), "
                       "reference dmrg() schedule, real MPO", "runs": {}}
    # the reference's site-step eigensolver (nev=6 from a fixed start), then the
    # fast settings: lowest value only (nev=1, ncv=12) from White's prediction
    fast = {"nev": 1, "ncv": 12, "predict": True}
    arms = [("plain_fp64", native.SCHED_PER_BLOCK, native.PREC_FP64, None),
            ("fp64", native.SCHED_GROUPED, native.PREC_FP64, None)]
    if args.prec != "fp64":
        arms.append((args.prec, native.SCHED_GROUPED, prec, None))
    arms.append(("fp64_predicted", native.SCHED_GROUPED, native.PREC_FP64, fast))
    if args.prec != "fp64":
        arms.append((args.prec + "_predicted", native.SCHED_GROUPED, prec, fast))
    half = L // 2 - 1          # steps of the closing half sweep
    full = 2 * (L - 2)         # steps of one full sweep
    for name, sched, p, solver in arms:
        c = native.Context(native.F64)
        c.set_schedule(sched)
        c.set_precision(p)
        if solver:
            c.set_solver(**solver)
        import torch
        # ncu --nvtx --nvtx-include "sweep_<arm>/" selects one arm's launches
        torch.cuda.nvtx.range_push("sweep_" + name)
        r = c.dmrg("xyz_real", L, args.sweep_m, args.sweep_n, [1.0, 0.8, 0.5])
        torch.cuda.nvtx.range_pop()
        st = c.step_seconds()
        ns = len(st)
        last = st[ns - half - full: ns - half] if ns >= half + full else st
        sp = c.step_split()
        lsp = sp[ns - half - full: ns - half] if ns >= half + full else sp
        out["runs"][name] = {"schedule_s": float(r["seconds"]["total"]), "steps": ns,
                             "sweep_s": float(np.sum(last)),
                             "sweep_split_s": dict(zip(("eig", "svd", "env", "fuse", "plan"),
                                                       lsp.sum(axis=0).tolist())),
                             "energy": float(r["energies"][-1, 0]),
                             "matvecs": int(r["matvecs"].sum()),
                             "split_s": c.run_seconds()}
        c.close()
    runs = out["runs"]
    head = args.prec if args.prec != "fp64" else "fp64"
    out["speedup_vs_plain_fp64"] = runs["plain_fp64"]["sweep_s"] / runs[head]["sweep_s"]
    out["speedup_vs_grouped_fp64"] = runs["fp64"]["sweep_s"] / runs[head]["sweep_s"]
    out["dE_rel_vs_fp64"] = abs(runs[head]["energy"] - runs["fp64"]["energy"]) / abs(runs["fp64"]["energy"])
    # the fast solver settings against the reference's, same precision, whole schedule
    fh = head + "_predicted"
    out["predicted"] = {"solver": fast,
                        "schedule_speedup_vs_reference_solver":
                            runs[head]["schedule_s"] / runs[fh]["schedule_s"],
                        "sweep_speedup_vs_reference_solver":
                            runs[head]["sweep_s"] / runs[fh]["sweep_s"],
                        "dE_rel_vs_fp64": abs(runs[fh]["energy"] - runs["fp64"]["energy"])
                        / abs(runs["fp64"]["energy"])}
    return out


def config1_compare(native):
    """BASELINE config 1 end to end, GPU beside the reference on the host: the Kitaev
    chain L=32 (t=1, Delta=1, mu=0.5 -> u=0.25), the reference's dmrg() schedule to
    m=64 with 6 sweeps.  The reference run is its own code (oracle/_ref, ARPACK
    settings, OpenBLAS on all host threads), timed in this process; the GPU runs
    the same schedule in FP64 and BF16x3 with the reference's solver settings,
    and in FP64 with the fast settings.  Reports wall seconds, the final energies
    against the exact BdG value, and the largest per-step energy differences
    between the GPU FP64 runs and the reference."""
    from oracle import exact, refbind
    L, m, n, par = 32, 64, 6, [1.0, 1.0, 0.25]
    out = {"workload": "Kitaev chain L=32, t=1, Delta=1, mu=0.5, m=64, 6 sweeps, "
                       "reference dmrg() schedule, FP64 real"}
    runs = {}
    # the reference's solver settings in both precisions, then the fast settings
    # (lowest value only, 12-vector basis, White's prediction) in FP64
    for name, prec, fast in (("fp64", native.PREC_FP64, False),
                             ("bf16x3", native.PREC_BF16X3, False),
                             ("fp64_fast", native.PREC_FP64, True)):
        c = native.Context(native.F64)
        c.set_precision(prec)
        if fast:
            c.set_solver(1, 12, True)
        t0 = time.perf_counter()
        r = c.dmrg("kitaev", L, m, n, par)
        runs[name] = (time.perf_counter() - t0, r)
        runs[name][1]["split_s"] = c.run_seconds()
        c.close()
    e_bdg = exact.kitaev_bdg(L, *par)
    out["bdg_energy"] = e_bdg
    for name, (secs, r) in runs.items():
        e = float(r["energies"][-1, 0])
        out["gpu_" + name] = {"seconds": secs, "energy": e, "dE_rel_vs_bdg": abs(e - e_bdg) / abs(e_bdg),
                              "matvecs": int(r["matvecs"].sum()),
                              "split_s": {k: round(v, 4) for k, v in r["split_s"].items()}}
    if refbind.available("kitaev"):
        R = refbind.Ref("kitaev")
        t0 = time.perf_counter()
        res = R.run("kitaev", L, m, n, 0, par)
        secs = time.perf_counter() - t0
        e_ref = np.array([row["evals"][0] for row in res["en"]])
        out["reference"] = {"seconds": secs, "threads": os.cpu_count(), "energy": float(e_ref[-1]),
                            "kind": "reference (its own code built from its sources, ARPACK "
                                    "settings, OpenBLAS on all host threads)"}
        for name in ("fp64", "fp64_fast"):
            e_gpu = runs[name][1]["energies"][:, 0]
            if e_ref.shape == e_gpu.shape:
                out["max_step_dE_rel_%s_vs_reference" % name] = float(
                    np.max(np.abs(e_gpu - e_ref) / np.abs(e_ref)))
        for name in runs:
            out["speedup_" + name + "_vs_reference"] = secs / runs[name][0]
    return out


def config5_compare():
    """BASELINE config 5 in solve groups, reduced to fit the benchmark's time: the
    eight chains of bond dimensions 64 and 128 (XYZ L=64, Jz from seed 20261203),
    one sweep, two solve groups of four whose matvecs are one grouped launch per
    stage, then each chain's adjoint dE/dJz, dE/dh against Hellmann-Feynman.
    The full sixteen-chain run is `python -m dmrg_b200.batch --grouped`."""
    from dmrg_b200 import batch
    specs = batch.config5_chains(L=64, ms=(64, 128), per_m=4)
    res, wall = batch.run_batch(specs, grouped=True, sweeps=1, fd=False)
    return {"workload": "config 5 reduced: 8 XYZ chains L=64, m in {64, 128} x 4, 1 sweep, "
                        "FP64, two solve groups (one grouped matvec launch per stage)",
            "wall_s": wall,
            "max_rel_hf_dE_dJz": max(r["rel_hf_Jz"] for r in res),
            "max_abs_hf_dE_dh": max(r["abs_hf_h"] for r in res),
            "groups": {str(r["m"]): r["group_stats"] for r in res},
            "chains": [{"m": r["m"], "jz": r["jz"], "E0": r["E0"], "dE_dJz": r["dE_dJz"],
                        "hf_Jz": r["hf_Jz"]} for r in res]}


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    from dmrg_b200 import workloads
    w = workloads.microbench(1024)
    rates = []
    cb = cpu_reference_rate(min(2.0, args.cpu_sample_s), w)  # warm-up pass
    t0 = time.perf_counter()
    per = []
    for _ in range(args.steps):
        r = cpu_reference_rate(0.0, w)
        per.append(1.0 / r["value"])
    el = time.perf_counter() - t0
    value = args.steps / sum(per)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(per) / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "H_eff matvec microbench m=1024, 9 U(1) sectors, d=2, D=5",
                       "psi_elems": 599964, "tasks": [190, 190], "gflop_per_matvec": 3.862},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cb["cores"],
                             "kind": cb["kind"], "sample": f"{args.steps} single-matvec steps; "
                             + cb["sample"].split(";")[0]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "wall_s": el}
    print(json.dumps(line), flush=True)


def time_matvecs(torch, ctx, stream, xs, ys, flush, steps, warmup, profile=False):
    """Device time of `steps` matvecs (inputs resident, L2 flushed before each,
    outside the events).  Returns (seconds, per-slot profile or None).

    The flush writes a 256 MiB buffer and then reads a second, never-written
    256 MiB buffer: the write evicts the workload's lines, the read forces the
    write-back of the dirty flush lines, so none of that lands in the timed
    matvec."""
    fw, fr = flush

    def one(timed):
        with torch.cuda.stream(stream):
            fw.fill_(1.0)
            fr.sum()
            if timed:
                s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s.record(stream)
            ctx.av_device(xs.data_ptr(), ys.data_ptr())
            if timed:
                e.record(stream)
                return s, e
        return None

    for _ in range(warmup):
        one(False)
    torch.cuda.synchronize()
    if profile:
        ctx.profile(True)
    torch.cuda.nvtx.range_push("timed")  # ncu --nvtx --nvtx-include "timed/" selects these
    evs = [one(True) for _ in range(steps)]
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    prof = None
    if profile:
        prof = ctx.profile_read()
        ctx.profile(False)
    return sum(s.elapsed_time(e) for s, e in evs) / 1e3, prof


def main():
    args = parse()
    world, rank, local = dist_init(args)
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch
    from dmrg_b200 import native, workloads
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    if args.probe:
        run_probe(args)
        return
    prec = {"fp64": native.PREC_FP64, "bf16x3": native.PREC_BF16X3,
            "tf32x3": native.PREC_TF32X3}[args.prec]

    w = workloads.microbench(1024)
    ctx = native.Context(native.F64, local)
    ctx.set_precision(prec)
    ctx.plan_build(w["lenv"], w["renv"], 3, 2, w["sector"], 32, 0)
    n, flops = ctx.n, ctx.flops
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    ref = None
    if prec != native.PREC_FP64:   # the grouped FP64 GPU path on the same input, for the ratio
        ref = native.Context(native.F64, local)
        ref.plan_build(w["lenv"], w["renv"], 3, 2, w["sector"], 32, 0)
        ref_stream = torch.cuda.ExternalStream(ref.stream(), device=dev)
    # the plain FP64 GPU path: one cuBLAS GEMM per task row (the reference's av() loop)
    plain = native.Context(native.F64, local)
    plain.set_schedule(native.SCHED_PER_BLOCK)
    plain.plan_build(w["lenv"], w["renv"], 3, 2, w["sector"], 32, 0)
    plain_stream = torch.cuda.ExternalStream(plain.stream(), device=dev)

    xs = torch.tensor(workloads.random_psi(n, seed=5), device=dev)
    ys = torch.empty_like(xs)
    flush = (torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev),
             torch.ones(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev))
    torch.cuda.synchronize()

    try:
        clocks = Clocks("GPU-" + str(torch.cuda.get_device_properties(dev).uuid))
    except Exception:
        clocks = Clocks(local)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    dev_s, _ = time_matvecs(torch, ctx, stream, xs, ys, flush, args.steps, args.warmup)
    ck = clocks.stop()
    from dmrg_b200 import replicas
    dev_s = replicas.max_over_ranks(dev_s, dev)
    per = dev_s / args.steps
    value = world * args.steps / dev_s
    y_main = ys.cpu().numpy()

    # per-launch device times of the same workload (events between launches)
    _, prof = time_matvecs(torch, ctx, stream, xs, ys, flush, args.steps, 1, profile=True)
    cnt, slots = prof

    fp64 = None
    if ref is not None:
        ys64 = torch.empty_like(xs)
        f_s, _ = time_matvecs(torch, ref, ref_stream, xs, ys64, flush, args.steps, args.warmup)
        _, (fc, fslots) = time_matvecs(torch, ref, ref_stream, xs, ys64, flush, args.steps, 1,
                                       profile=True)
        y64 = ys64.cpu().numpy()
        rel_err = float(np.linalg.norm(y_main - y64) / np.linalg.norm(y64))
        fp64 = {"value": args.steps / f_s, "ms_per_step": 1e3 * f_s / args.steps,
                "stage_ms": [float(x / fc) for x in fslots[1:]],
                "tflops": flops / (float(fslots[1] + fslots[2]) / fc / 1e3) / 1e12}
        # the FP64 path's own roofline: the FP64 tensor-core (DMMA) ceiling, measured
        # in-run by a cuBLAS DGEMM burst (the peak file has no FP64 figure)
        pk64 = fp64_gemm_peak(torch, dev)
        fp64["roofline"] = {"bound": "tensor", "achieved": fp64["tflops"], "peak": pk64,
                            "unit": "TFLOP/s", "frac": fp64["tflops"] / pk64,
                            "kernel": "grouped_gemm_nt_f64 (stage 1 + stage 2 launches)",
                            "peak_source": "in-run cuBLAS DGEMM 8192^3 burst"}

    ysp = torch.empty_like(xs)
    p_s, _ = time_matvecs(torch, plain, plain_stream, xs, ysp, flush, args.steps, args.warmup)
    p_err = float(np.linalg.norm(ysp.cpu().numpy() - y_main) / np.linalg.norm(ysp.cpu().numpy()))
    plain_path = {"value": args.steps / p_s, "ms_per_step": 1e3 * p_s / args.steps,
                  "launches_per_step": plain.matvec_launches(),
                  "rel_err_vs_headline": p_err}

    # end to end through the C ABI with page-locked host buffers (the H2D copy of
    # psi, the matvec and the D2H copy of the result inside the timing)
    xh = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    xh[:] = workloads.random_psi(n, seed=6)
    yh = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    for _ in range(max(2, args.warmup)):
        ctx.av(xh, out=yh)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ctx.av(xh, out=yh)
    e2e_s = replicas.max_over_ranks(time.perf_counter() - t0, dev)

    if rank == 0:
        peaks, src = measured_peaks()
        gemm_s = float(slots[1] + slots[2]) / cnt / 1e3   # both stage launches of the kernel
        achieved = flops / gemm_s / 1e12
        if args.prec == "fp64":
            pk = fp64_gemm_peak(torch, dev)
            peak_note = "in-run cuBLAS DGEMM 8192^3 burst (FP64 tensor cores); no FP64 figure in MEASURED_PEAKS.json"
            kernel = "grouped_gemm_nt_f64 (stage 1 + stage 2 launches)"
        elif args.prec == "bf16x3":
            pk = peaks["bf16_tflops"]
            peak_note = f"bf16_tflops of MEASURED_PEAKS.json ({src}, burst)"
            kernel = "grouped_split_tc<bf16> (stage 1 + stage 2 launches)"
        else:
            pk = peaks["bf16_tflops"] / 2
            peak_note = f"half the bf16_tflops of MEASURED_PEAKS.json ({src}): TF32 runs at half the BF16 rate"
            kernel = "grouped_split_tc<tf32> (stage 1 + stage 2 launches)"
        cpu = cpu_reference_rate(args.cpu_sample_s, w)
        sweep = sweep_compare(native, args) if args.sweep else None
        cfg1 = config1_compare(native) if args.config1 else None
        cfg5 = config5_compare() if args.config5 else None
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.prec == "fp64" else args.prec, "data": "synthetic",
            "config": {"workload": "H_eff matvec microbench m=1024, 9 U(1) sectors, d=2, D=5",
                       "psi_elems": n, "tasks": [ctx.n_rmap, ctx.n_lmap],
                       "gflop_per_matvec": flops / 1e9, "precision": args.prec,
                       "parallelism": f"replicas x{world}",
                       "l2": "flushed before every timed step: 256 MiB write, then 256 MiB read of a clean buffer (write-back done outside the timing)"},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": pk, "unit": "TFLOP/s",
                         "frac": achieved / pk,
                         # dram__bytes_read.sum + dram__bytes_write.sum of the stage-1 and
                         # stage-2 launches of one steady-state BF16x3 matvec of this workload,
                         # one ncu capture (--nvtx-include "timed/", --set full)
                         "traffic": TRAFFIC_BF16X3 if args.prec == "bf16x3" else None,
                         "kernel": kernel,
                         "peak_source": peak_note,
                         "note": "achieved = algorithmic flops (2MNK per task, not counting the "
                                 "3 split products) / summed device time of the stage launches",
                         "stage_ms": [float(x / cnt) for x in slots]},
            "cpu_baseline": cpu,
            "e2e": {"value": world * args.steps / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": n * 8},
            "gpu_launches": ctx.matvec_launches() * args.steps,
            "clocks": ck,
        }
        if sweep is not None:
            line["sweep"] = sweep
        if cfg1 is not None:
            line["config1"] = cfg1
        if cfg5 is not None:
            line["config5"] = cfg5
        line["plain_fp64_path"] = plain_path
        line["vs_plain_fp64"] = value / plain_path["value"]
        if fp64 is not None:
            line["fp64_path"] = fp64
            line["split_vs_fp64"] = value / fp64["value"]
            line["split_rel_err"] = rel_err
            line["config"]["tuning"] = [dict(zip(("cfg", "halve", "ksplit_scale", "measured"), t))
                                        for t in ctx.split_tuning()]
        print(json.dumps(line), flush=True)
    ctx.close()
    plain.close()
    if ref is not None:
        ref.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
