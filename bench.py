#!/usr/bin/env python
"""FMM matvec throughput on B200: points/s of the directional Helmholtz FMM
(defmm's method) on the sphere workload: N = 2,000,000 points uniform on the
unit sphere, k = 2 pi 64 (128 wavelengths across the diameter), order 5,
leaf size 64; complex FP64 charges uniform in [-1, 1]^2 (seeded synthetic
data, no dataset).

One step = one matvec (P2M .. L2P + P2P) over that input.  Both arithmetic
paths are timed: plain FP64 (the drop-in) and mixed precision; `value` is the
mixed path's points/s when its relative L2 deviation from the FP64 result is
<= 1e-6 (otherwise the FP64 path's).  Inputs are resident in HBM for `value`
(CUDA events around K steps on the launching stream); `e2e` is the same
metric through the host-buffer C-ABI call (host->device copy of the charges
and device->host copy of the potentials inside the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (launched by torchrun) every rank runs an independent replica
(its own seeded charges): the matvec does not shard; value = all ranks'
points / max-over-ranks time.  --impl reference times the reference's own
CPU implementation (oracle/_ref/defmm_ref_fast, built unmodified) on a
bounded sample of the same workload, on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FMM matvec points/s on 1 B200 at rel L2 err <=1e-6: mixed/learned vs plain FP64"
UNIT = "points/s"
MIXED_TOL = 1e-6


def workload(name, rank=0):
    from defmm_b200 import workloads as W
    if name == "sphere2m":
        return W.sphere_surface(2_000_000, seed=0)
    if name == "sphere100k":
        return W.sphere_surface(100_000, seed=0, wavelengths=32)
    if name == "sphere200k":  # config-2 points per wavelength^2, for profiling
        return W.sphere_surface(200_000, seed=0, wavelengths=40)
    if name == "cube20k":
        return W.cube_surface(20_000, seed=0)
    raise KeyError(name)


def cpu_sample(name):
    """Bounded CPU sample of the same workload: same geometry and points per
    wavelength^2, N/64 points at 1/8 of the wavenumber."""
    from defmm_b200 import workloads as W
    if name == "sphere2m":
        return W.sphere_surface(2_000_000 // 64, seed=0, wavelengths=128 / 8), "sphere N=31,250, 16 wavelengths, order 5, leaf 64"
    if name == "sphere100k":
        return W.sphere_surface(100_000 // 16, seed=0, wavelengths=8), "sphere N=6,250, 8 wavelengths, order 5, leaf 64"
    return workload(name), "full workload"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev=0):
        self.dev = dev
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], p.get("bf16_tflops"), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, 1590.0, "fallback"


def run_reference(args, name):
    """Reference arm: the reference's own CPU matvec on the bounded sample."""
    from defmm_b200 import workloads as W
    from oracle import refrun
    w, desc = cpu_sample(name)
    q = W.charges(w.n, 1)
    if not refrun.available(fast=True):
        return {"impl": "reference", "unavailable": "reference build oracle/_ref/defmm_ref_fast is missing"}
    vals = []
    for i in range(args.warmup + args.steps):
        r = refrun.run(w.points, w.points, q, w.order, w.ncrit, w.kappa, lists=False, fast=True)
        if i >= args.warmup:
            vals.append(w.n / r.summary["gemv_s"])
    v = float(statistics.mean(vals))
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": name, "sample": desc},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "reference", "sample": desc},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_ragged(args, torch):
    """48 independent problems of uneven size (workloads.ragged_problems),
    mixed precision (FP32 charges and expansions): every operator's matvec
    once per step, run (a) as one graph launch of the whole batch
    (defmm_batch) and (b) one operator after another on the same stream
    (each a replayed graph).  points/s = total points per step / time,
    device-timed with CUDA events; inputs resident on the device."""
    from defmm_b200 import Batch, IBFMM_Mat, workloads as W
    P = W.ragged_problems(48, 0)
    t0 = time.perf_counter()
    ops = []
    for w in P:
        A = IBFMM_Mat()
        A.set_precision("mixed")
        A.addSourceParticles(w.points)
        A.addTargetParticles(w.points)
        A.prcmpt(w.order, w.ncrit, w.kappa)
        ops.append(A)
    setup_s = time.perf_counter() - t0
    ins = [torch.from_numpy(W.charges(w.n, 3 + i)).cuda() for i, w in enumerate(P)]
    outs = [torch.zeros(w.n, dtype=torch.complex128, device="cuda") for w in P]
    stream = torch.cuda.Stream()
    total = sum(w.n for w in P)
    dev_bytes = sum(A.info("device_bytes") for A in ops)
    sid = stream.cuda_stream

    def seq():
        for A, x, y in zip(ops, ins, outs):
            A.matvec_device(x.data_ptr(), y.data_ptr(), 1, sid)

    batches = {k: Batch(ops, [t.data_ptr() for t in ins], [t.data_ptr() for t in outs], k) for k in (1, 2, 4, 48)}
    runs = [("sequential", seq)] + [("lanes%d" % k, (lambda b=b: b.launch(sid))) for k, b in batches.items()]
    t = {}
    with torch.cuda.stream(stream):
        for name, fn in runs:
            for _ in range(args.warmup):
                fn()
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                fn()
            e1.record(stream)
            stream.synchronize()
            t[name] = e0.elapsed_time(e1) / args.steps
    best = min(batches, key=lambda k: t["lanes%d" % k])
    t["batch"] = t["lanes%d" % best]
    line = {"metric": "FMM matvec points/s, 48 independent problems in one graph launch", "impl": "ours",
            "value": total / (t["batch"] * 1e-3), "unit": "points/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t["batch"], "higher_is_better": True,
            "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "ragged48", "problems": len(P), "total_points": total,
                       "n_range": [min(w.n for w in P), max(w.n for w in P)], "orders": [4, 5, 6],
                       "precision": "mixed", "lanes": best},
            "lanes_ms": {k: t["lanes%d" % k] for k in batches},
            "sequential": {"ms_per_step": t["sequential"], "points_per_s": total / (t["sequential"] * 1e-3)},
            "setup_s": setup_s, "plan_bytes": dev_bytes}
    print(json.dumps(line), flush=True)
    batches.clear()


def run_spheroid(args, torch):
    """Spheroid with semi-axes (1, 0.5, 0.25), N = 4,000,000, density
    1 + 4|z|, 256 wavelengths along the long axis, order 6, leaf 96, mixed
    precision only: the FP64 path would hold M and L for 2 x 33.3M
    expansion slots of 216 entries (230 GB), beyond the 180 GB of one B200.
    Accuracy: FP64 direct sums at 2,000 seeded targets."""
    from defmm_b200 import IBFMM_Mat, workloads as W
    w = W.spheroid(4_000_000, seed=0)
    q = W.charges(w.n, 1)
    A = IBFMM_Mat()
    A.set_precision("mixed")
    A.addSourceParticles(w.points)
    A.addTargetParticles(w.points)
    t0 = time.perf_counter()
    A.prcmpt(w.order, w.ncrit, w.kappa)
    setup_s = time.perf_counter() - t0
    A.upload()
    info = A.info()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    dq = torch.from_numpy(q).to("cuda")
    dp = torch.empty(w.n, dtype=torch.complex128, device="cuda")
    for _ in range(args.warmup):
        A.matvec_device(dq.data_ptr(), dp.data_ptr(), 1, stream.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(0) as ck:
        e0.record(stream)
        for _ in range(args.steps):
            A.matvec_device(dq.data_ptr(), dp.data_ptr(), 1, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    A.matvec(q)
    chk = A.check_full(2000, seed=7)
    A.set_profiling(True)
    A.matvec_device(dq.data_ptr(), dp.data_ptr(), 1, stream.cuda_stream)
    torch.cuda.synchronize()
    phases = A.phase_times()
    A.set_profiling(False)
    line = {"metric": "FMM matvec points/s, mixed precision, spheroid", "impl": "ours",
            "value": w.n / (ms * 1e-3), "unit": "points/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "dtype": "f32+f64",
            "data": "synthetic",
            "config": {"workload": "spheroid4m", "n_points": w.n, "kappa": w.kappa, "order": w.order,
                       "leaf_size": w.ncrit, "precision": "mixed",
                       "fp64": "not run: M and L would need 230 GB"},
            "accuracy": {"direct_sum_2000_targets": chk}, "clocks": ck.summary(), "phases_ms": phases,
            "setup_s": setup_s, "device_bytes": A.info("device_bytes"),
            "plan": {k: info[k] for k in ["nlvl", "cpt", "slots_S", "slots_T", "far_hf", "near", "i_near",
                                          "tables", "permuted_spectra"]}}
    print(json.dumps(line), flush=True)


def run_rhs64(args, torch):
    """64 right-hand sides (complex charges with FP32-representable parts
    uniform in [-1, 1]) on the 2M-point sphere (k = 2 pi 64, order 5, leaf
    64), mixed precision: one defmm_gemv_device call with nrhs = 64 per step
    (each right-hand side replays the operator's captured graph)."""
    from defmm_b200 import IBFMM_Mat, workloads as W
    w = W.sphere_surface(2_000_000, seed=0)
    nrhs = 64
    Q = W.charges(w.n, 5, nrhs=nrhs).astype(np.complex64).astype(np.complex128)
    A = IBFMM_Mat()
    A.set_precision("mixed")
    A.addSourceParticles(w.points)
    A.addTargetParticles(w.points)
    A.prcmpt(w.order, w.ncrit, w.kappa)
    stream = torch.cuda.Stream()
    dq = torch.from_numpy(Q).to("cuda")
    dp = torch.empty((nrhs, w.n), dtype=torch.complex128, device="cuda")
    for _ in range(max(1, args.warmup - 2)):
        A.matvec_device(dq.data_ptr(), dp.data_ptr(), nrhs, stream.cuda_stream)
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(0) as ck:
        e0.record(stream)
        for _ in range(args.steps):
            A.matvec_device(dq.data_ptr(), dp.data_ptr(), nrhs, stream.cuda_stream)
        e1.record(stream)
        stream.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    one = A.matvec(Q[nrhs - 1])
    same = bool(np.array_equal(dp[nrhs - 1].cpu().numpy(), one))
    line = {"metric": "FMM matvec points/s over 64 right-hand sides, mixed precision", "impl": "ours",
            "value": nrhs * w.n / (ms * 1e-3), "unit": "points/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "ms_per_rhs": ms / nrhs, "higher_is_better": True,
            "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "rhs64", "n_points": w.n, "nrhs": nrhs, "kappa": w.kappa, "order": w.order,
                       "leaf_size": w.ncrit, "precision": "mixed"},
            "last_rhs_equals_single_call": same, "clocks": ck.summary()}
    print(json.dumps(line), flush=True)


def run_orders(args, torch):
    """Error against FP64 direct sums (2,000 seeded targets) and time per
    matvec for orders 4-7, FP64 and mixed, on the spheroid at the 4M
    workload's points per square wavelength: N = 500,000, 90.5 wavelengths
    along the long axis, leaf 96."""
    from defmm_b200 import IBFMM_Mat, workloads as W
    n = 500_000
    rows = []
    for L in (4, 5, 6, 7):
        w = W.spheroid(n, seed=0, order=L, wavelengths=256.0 * math.sqrt(n / 4_000_000))
        q = W.charges(w.n, 1)
        A = IBFMM_Mat()
        A.addSourceParticles(w.points)
        A.addTargetParticles(w.points)
        A.prcmpt(w.order, w.ncrit, w.kappa)
        stream = torch.cuda.Stream()
        dq = torch.from_numpy(q).to("cuda")
        dp = torch.empty(w.n, dtype=torch.complex128, device="cuda")
        row = {"order": L}
        out = {}
        for prec in ("fp64", "mixed"):
            A.set_precision(prec)
            for _ in range(args.warmup):
                A.matvec_device(dq.data_ptr(), dp.data_ptr(), 1, stream.cuda_stream)
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                A.matvec_device(dq.data_ptr(), dp.data_ptr(), 1, stream.cuda_stream)
            e1.record(stream)
            stream.synchronize()
            out[prec] = A.matvec(q)
            row[prec] = {"ms": e0.elapsed_time(e1) / args.steps, "vs_direct": A.check_full(2000, seed=7)}
        row["mixed_vs_fp64_rel_l2"] = float(np.linalg.norm(out["mixed"] - out["fp64"]) / np.linalg.norm(out["fp64"]))
        rows.append(row)
        del A
    line = {"metric": "FMM error vs FP64 direct sums and ms per matvec by order, spheroid", "impl": "ours",
            "unit": "relative error", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "data": "synthetic",
            "config": {"workload": "spheroid_orders", "n_points": n, "leaf_size": 96,
                       "wavelengths_long_axis": 256.0 * math.sqrt(n / 4_000_000)},
            "orders": rows}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sphere2m")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, args.workload)), flush=True)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist:
            dist.barrier()

    extra = {"ragged48": run_ragged, "spheroid4m": run_spheroid, "spheroid_orders": run_orders,
             "rhs64": run_rhs64}
    if args.workload in extra:
        if rank == 0:
            extra[args.workload](args, torch)
        return

    from defmm_b200 import IBFMM_Mat, replicas, workloads as W

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, dist, "cuda")

    w = workload(args.workload, rank)
    q = W.charges(w.n, replicas.replica_seed(rank))
    A = IBFMM_Mat()
    A.addSourceParticles(w.points)
    A.addTargetParticles(w.points)
    t0 = time.perf_counter()
    A.prcmpt(w.order, w.ncrit, w.kappa)
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    A.upload()
    upload_s = time.perf_counter() - t0
    info = A.info()
    # a dedicated stream: torch's default stream is the legacy NULL stream,
    # which the library's non-blocking streams would not order against
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    dq = torch.from_numpy(q).to("cuda")
    dp = torch.empty(w.n, dtype=torch.complex128, device="cuda")

    res = {}
    tune, tune_s = {}, 0.0
    for prec in ["fp64", "mixed"]:
        A.set_precision(prec)
        if not args.no_autotune:  # launch choices timed on this operator (defmm_autotune)
            t0 = time.perf_counter()
            A.autotune(reps=1)
            tune_s += time.perf_counter() - t0
        tune[prec] = {k: A.info(k) for k in ("m2l_threads", "m2l_pairing", "p2p_blocks_per_sm")}
        for _ in range(args.warmup):
            A.matvec_device(dq.data_ptr(), dp.data_ptr(), 1, stream.cuda_stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches = 0
        barrier()
        torch.cuda.synchronize()
        with Clocks(local) as ck:
            e0.record(stream)
            for _ in range(args.steps):
                A.matvec_device(dq.data_ptr(), dp.data_ptr(), 1, stream.cuda_stream)
                launches += A.info("launches")
            e1.record(stream)
            torch.cuda.synchronize()
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
        res[prec] = {"ms": ms, "p": dp.cpu().numpy(), "launches": launches, "clocks": ck.summary()}

    p64, p32 = res["fp64"]["p"], res["mixed"]["p"]
    err_mixed = float(np.linalg.norm(p32 - p64) / np.linalg.norm(p64))
    head = "mixed" if err_mixed <= MIXED_TOL else "fp64"
    A.set_precision(head)
    ms = res[head]["ms"]
    value = replicas.job_throughput(w.n, world, ms * 1e-3)

    # end to end through the host-buffer C-ABI call
    A.matvec(q)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        A.matvec(q)
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps)
    chk = A.check_full(2000, seed=7)  # FP64 direct sum at 2,000 seeded targets

    # per-phase device times (separate profiled runs, not part of `value`)
    phases = {}
    for prec in ["fp64", "mixed"]:
        A.set_precision(prec)
        A.set_profiling(True)
        A.matvec_device(dq.data_ptr(), dp.data_ptr(), 1, stream.cuda_stream)
        torch.cuda.synchronize()
        phases[prec] = A.phase_times()
        A.set_profiling(False)
    A.set_precision(head)

    # roofline of the dominant HBM-bound kernel, M2L (with the inverse DFT
    # fused), on the headline path.  Algorithmic bytes per matvec: every
    # source spectrum once (e P^3 per source slot), every permuted transfer
    # spectrum once, the local expansion of every target slot read and
    # written (2 e L^3), 8 B per list entry.
    hbm, bf16, src = measured_peaks()
    e = 16 if head == "fp64" else 8
    L = w.order
    PP = (2 * L - 1) ** 3
    n_far = info["far_hf"] + info["far_lf"]
    m2l_bytes = (e * PP * info["slots_S"] + e * PP * info["permuted_spectra"]
                 + 2 * e * L ** 3 * info["m2l_targets"] + 8 * n_far)
    m2l_ms = phases[head]["m2l"]
    achieved = m2l_bytes / (m2l_ms * 1e-3) / 1e9
    # the M2L kernel this run used (launch choice of the headline precision)
    lc = tune[head]
    kname = "%s<%s, %d, %d>" % ("k_m2l_pair" if lc["m2l_pairing"] else "k_m2l",
                                "double" if head == "fp64" else "float", L, lc["m2l_threads"])
    # DRAM traffic per far pair of the same kernel, measured by ncu on a
    # smaller sphere and scaled by the far pairs of this workload
    traffic = None
    tp = os.path.join(ROOT, "profiles", "m2l_traffic.json")
    if os.path.exists(tp):
        try:
            with open(tp) as f:
                tr = json.load(f).get(head, {})
            if tr.get("kernel") == kname and tr.get("bytes_per_pair") is not None:
                traffic = tr["bytes_per_pair"] * n_far
        except (OSError, ValueError):
            traffic = None
    roofline = {"bound": "hbm", "kernel": kname + " (M2L + inverse DFT, all cone batches)", "achieved": achieved,
                "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_source": src,
                "traffic": traffic, "algorithmic_bytes": m2l_bytes}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import refrun
            ws, desc = cpu_sample(args.workload)
            if refrun.available(fast=True):
                r = refrun.run(ws.points, ws.points, W.charges(ws.n, 1), ws.order, ws.ncrit, ws.kappa,
                               lists=False, fast=True)
                cpu = {"value": ws.n / r.summary["gemv_s"], "unit": UNIT, "cores": 1, "kind": "reference",
                       "sample": desc, "gemv_s": r.summary["gemv_s"]}
        except Exception as ex:  # the baseline must not sink the GPU result
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64" if head == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": args.workload, "n_points": w.n, "kappa": w.kappa, "order": w.order,
                       "leaf_size": w.ncrit, "precision": head, "parallelism": f"replicas{world}",
                       "l2": "working set per step >> L2 (126 MB): expansions and spectra are GBs"},
            "matvecs_per_s": world / (ms * 1e-3),
            "fp64": {"ms_per_step": res["fp64"]["ms"], "points_per_s": world * w.n / (res["fp64"]["ms"] * 1e-3)},
            "mixed": {"ms_per_step": res["mixed"]["ms"], "points_per_s": world * w.n / (res["mixed"]["ms"] * 1e-3),
                      "rel_l2_vs_fp64": err_mixed},
            "speedup_mixed_vs_fp64": res["fp64"]["ms"] / res["mixed"]["ms"],
            "accuracy": {"direct_sum_2000_targets": chk, "precision": head},
            "e2e": {"value": world * w.n / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 16 * w.n,
                    "d2h_bytes_per_step": 16 * w.n},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": res[head]["clocks"],
            "gpu_launches": res[head]["launches"],
            "phases_ms": phases,
            "setup_s": setup_s,
            "setup": {"prcmpt_s": setup_s, "level_walk_s": info["plan_walk_ms"] / 1e3,
                      "level_walk_on_gpu": bool(info["plan_walk_device"]), "upload_s": upload_s,
                      "autotune_s": tune_s},
            "launch": tune,
            "plan": {k: info[k] for k in ["nlvl", "cpt", "slots_S", "slots_T", "far_hf", "far_lf", "near",
                                          "i_near", "tables", "permuted_spectra", "device_bytes"]},
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
