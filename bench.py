#!/usr/bin/env python3
"""Throughput of the FP64 block-structured AMR two-phase LBM step on B200.

Workload: the rising bubble on a 256x512-cell base grid of 16x16 blocks with 3
refinement levels (finest-equivalent 2048x4096), R=128 at (1024,512), density
ratio 1000, viscosity ratio 100, Eo=10, Mo=1e-5, W=4, a regrid every 10 time
steps. Synthetic inputs: the analytic bubble of the reference's start-up,
evolved W warm-up steps.

One bench step = one regrid interval: 10 iterations of the Main_Loop body
(Fill_Ghost_Cells_C2, collision, Fill_Ghost_Cells_hg, streaming,
Macroscopic_Values_h/g, Fill_Ghost_Cells_C) with Refine_Derefine_Mesh after the
10th, run by the C ABI (amrlbm_step) as one CUDA graph. The L2 cache is flushed
between bench steps (outside the timed intervals).

value    = leaf-cell updates of all ranks / slowest rank's device time (MLUPS)
hbm_gbs  = value x 352 B (every population and macroscopic field read and
           written once per update)
e2e      = the same updates timed around upload of every leaf's fields from
           host memory -> amrlbm_step -> download of every leaf's fields and
           the diagnostics, all through the C ABI (wall clock)
--impl reference: the oracle (a C++/OpenMP restatement of the reference's
           Fortran, which cannot be compiled here) on all host cores.

Every leg checks that the state it ends on is physical (finite leaf values,
|Uy| far below the lattice sound speed, positive density, a rising bubble)
and stops with an error otherwise. cpu_baseline: the oracle is loaded with the
device's state at the start of the timed region, runs the same regrid
intervals on all host cores (its diagnostics must then equal the device's bit
for bit) and goes on to a bounded sample; a second leg runs at 4 threads, the
reference's OMP_NUM_THREADS (AMR_Rising_2D_OMP.f90:23).

Beside the FP64 value: mixed_precision (the same workload with FP16 / BF16
population storage, MLUPS), mixed_precision_error (the 64x128-base bubble in
FP16 and BF16 against FP64 at steps 1000 / 2500 / 5000: rise velocity,
centroid, mass), batched (the seeded batch of 256 uneven problems in one pool,
block size and CTAs per SM chosen by amrlbm.autotune, FP64 and FP16 MLUPS),
learned_regrid (the 8-bubble learned-regrid configuration: forecaster samples
seen and trained on, then the criterion every 10 steps against the learned
regrid every 32: regrids, escapes, misses, MLUPS).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "amr-lbm-openmp-2d_b200")
sys.path.insert(0, PKG)

METRIC = "MLUPS and HBM GB/s on 1 B200: mixed-prec batched vs FP64 plain at stated error"
BYTES_PER_UPDATE = 352  # 2 * (18 populations + C, P, Ux, Uy) * 8 B
# algorithmic bytes per leaf cell of the fused kernels (reads + writes, FP64)
BYTES_PER_UPDATE_MIXED = 104
KERNELS = {
    0: ("fill_c2_collide", 296),        # h,g,C in; h,g out
    1: ("fill_hg_stream_macro_h", 296), # h,g in; h,g,C out
    2: ("fill_c_macro_g_err", 104),     # g,C in; P,Ux,Uy out
    3: ("regrid", None),
}
WORKLOAD = "rising_bubble_base256x512_blocks16_L3_R128"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="own", choices=["own", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-long", action="store_true", help="skip the 5000-step run")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed-precision, error-report and batched legs")
    ap.add_argument("--profile-forecast", action="store_true",
                    help="profiling mode: the learned regrid's forecast on a reduced learned "
                         "workload (base 256x512, 4 bubbles), --steps regrid intervals of 32")
    ap.add_argument("--profile-precision", default=None, choices=["fp64", "fp16", "bf16"],
                    help="profiling mode: the workload in this precision for --warmup + "
                         "--steps intervals, nothing else")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--max-blks", type=int, default=0,
                    help="pool capacity (default: a fully refined tree); smaller pools "
                         "keep profiler captures small")
    return ap.parse_args()


def workload():
    import amrlbm
    return amrlbm.workload_large()


def config_dict(p, inner):
    return {"workload": WORKLOAD, "base_grid": "256x512", "block": f"{p.nx}x{p.ny}",
            "levels": p.max_levels, "finest_equivalent": "2048x4096", "radius": p.radius,
            "density_ratio": round(p.rho_h / p.rho_l, 6), "viscosity_ratio": p.visc_ratio,
            "eo": p.bo, "mo": 1e-5, "w": p.w, "m0": p.m0, "gy": p.gy,
            "start_pressure": "hydrostatic" if p.hydrostatic_start else "laplace",
            "regrid_every": p.regrid_every,
            "time_steps_per_bench_step": inner, "l2": "flushed between bench steps",
            "parallelism": "replicas"}


# bound on max |Uy| of a physical state of the workload: 5000 steps of it stay
# below 0.002 (tests/test_physics_long.py), the lattice sound speed is 0.577
U_BOUND = 0.05


def check_state(d, label):
    """Stops the bench unless the diagnostics (amrlbm_diag / the oracle's
    Output) describe a physical state."""
    import math
    bad = [k for k in ("mass", "rho_min", "u_max", "y_centroid", "rise_velocity")
           if not math.isfinite(d[k])]
    if d.get("status", 0) or bad:
        raise RuntimeError(f"{label}: non-finite state {bad} {d}")
    if not (d["u_max"] < U_BOUND and d["rho_min"] > 0.0 and d["rise_velocity"] > 0.0):
        raise RuntimeError(f"{label}: state not physical: u_max {d['u_max']}, rho_min "
                           f"{d['rho_min']}, rise velocity {d['rise_velocity']}")


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


PROFILE_FILES = {
    "fill_c2_collide": "k_fill_c_collide__rising_bubble_256x512_L3.md",
    "fill_hg_stream_macro_h": "k_fill_hg_stream__rising_bubble_256x512_L3.md",
}


def profile_traffic(kernel_name):
    """dram bytes per launch from the committed ncu summary of the kernel on
    this workload, if one exists."""
    path = os.path.join(ROOT, "profiles", PROFILE_FILES.get(kernel_name, kernel_name + ".md"))
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch_full_workload:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region: the
    sampler is started and its first sample awaited before the timed region,
    and one more sample is awaited after it."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def _lines(self):
        try:
            with open(self.path) as f:
                return [l for l in f.read().splitlines() if l.strip()]
        except OSError:
            return []

    def start(self):
        import tempfile
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.index)],
                stdout=fd, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        os.close(fd)
        t0 = time.time()
        while self.proc and not self._lines() and time.time() - t0 < 5.0:
            time.sleep(0.02)
        self.n0 = len(self._lines())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        t0 = time.time()
        while len(self._lines()) <= self.n0 and time.time() - t0 < 2.0:
            time.sleep(0.02)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        lines = self._lines()
        os.unlink(self.path)
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(backend):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def allreduce(vals, op, world, device=None):
    if world == 1:
        return vals
    import torch
    import torch.distributed as dist
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return t.tolist()


def oracle_from_device(gpu, p, threads):
    """An oracle holding the device pool's complete state (topology, free
    list, level range, every allocated block's fields)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import numpy as np
    from amrlbm import F_ALLOC
    from oracle_lib import Oracle
    orc = Oracle(p, threads)
    t = gpu.topology()
    c = gpu.counts()
    orc.set_topology(t, c["kk"])
    orc.set_level_range(c["level_min"], c["level_max"])
    ids = np.array([i + 1 for i in range(len(t["level"])) if t["flags"][i] & F_ALLOC],
                   dtype=np.int32)
    f = gpu.download_fields(ids)
    shp = dict(h=gpu.hshape, g=gpu.hshape, C=gpu.cshape, P=gpu.pshape, Ux=gpu.pshape,
               Uy=gpu.pshape)
    for i, bid in enumerate(ids):
        orc.upload_block(int(bid), *[f[k][i].reshape(shp[k], order="F")
                                     for k in ("h", "g", "C", "P", "Ux", "Uy")])
    return orc


def cpu_leg(orc, p, inner, seconds, min_chunks=0, check_after=None):
    """Regrid intervals of the oracle until `seconds` of CPU work (at least
    min_chunks); after chunk `check_after[0]` its diagnostics are handed to
    check_after[1]. Returns MLUPS, chunks, seconds."""
    updates, elapsed, chunks = 0, 0.0, 0
    ph0 = orc.phase_times()
    while chunks < min_chunks or elapsed < seconds:
        nleaf = orc.counts()["nleaf"]
        t = time.perf_counter()
        orc.main_loop(inner)
        elapsed += time.perf_counter() - t
        updates += nleaf * p.nx * p.ny * inner  # the regrid is after the last step
        chunks += 1
        if check_after and chunks == check_after[0]:
            check_after[1](orc.output())
    check_state(orc.output(), f"oracle after {chunks} intervals")
    ph = {k: v - ph0[k] for k, v in orc.phase_times().items()}
    tot = sum(ph.values()) or 1.0
    cpu_leg.phase_share = {k: round(v / tot, 4) for k, v in ph.items()}
    return updates / elapsed / 1e6, chunks, elapsed


def run_reference(args):
    world, rank, local = dist_setup("gloo")
    if rank != 0:
        return 0
    p = workload()
    inner = p.regrid_every
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle
    threads = os.cpu_count() or 1
    orc = Oracle(p, threads)
    orc.initialize_rising_bubble()
    for _ in range(args.warmup):
        orc.main_loop(inner)
    check_state(orc.output(), "reference arm after warm-up")
    updates, total = 0, 0.0
    for _ in range(args.steps):
        nleaf = orc.counts()["nleaf"]
        t = time.perf_counter()
        orc.main_loop(inner)
        total += time.perf_counter() - t
        updates += nleaf * p.nx * p.ny * inner
    check_state(orc.output(), "reference arm after the timed steps")
    v = updates / total / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "MLUPS",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(p, inner),
            "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": threads, "kind": "port",
                             "sample": f"{args.steps} bench steps of {inner} time steps of "
                                       f"the workload after {args.warmup} warm-up steps"},
            "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def mixed_error_report(checkpoints=(1000, 2500, 5000)):
    """The mixed-precision configuration's error report: the 64x128-base,
    density-ratio-10 bubble run in FP64, FP16 and BF16 storage; rise velocity,
    centroid and mass of each against FP64 at the checkpoints."""
    import amrlbm
    p = amrlbm.workload_small()
    runs = {}
    for prec in ("fp64", "fp16", "bf16"):
        g = amrlbm.AmrLbm(p)
        g.initialize_rising_bubble()
        g.set_precision(prec)
        done, out = 0, {}
        for c in checkpoints:
            g.main_loop(c - done)
            done = c
            out[c] = g.output()
        g.close()
        runs[prec] = out
    rep = {}
    for prec in ("fp16", "bf16"):
        rows = {}
        for c in checkpoints:
            a, r = runs[prec][c], runs["fp64"][c]
            check_state(a, f"{prec} run at step {c}")
            rows[str(c)] = {
                "rise_velocity_rel_err": abs(a["rise_velocity"] - r["rise_velocity"]) / abs(r["rise_velocity"]),
                "centroid_err_cells": abs(a["y_centroid"] - r["y_centroid"]),
                "mass_rel_err": abs(a["mass"] - r["mass"]) / r["mass"]}
        rep[prec] = rows
    rep["workload"] = "rising_bubble_base64x128_blocks16_L2_R32 (density ratio 10)"
    rep["bounds"] = {"rise_velocity_rel_err": 0.01, "mass_rel_err": 1e-6}
    return rep


def learned_leg(samples_target=1_000_000, eval_steps=960):
    """Learned regrid on its configuration (512x1024 base, 3 levels, 8
    bubbles R in [32, 128], density ratio 1000, Eo 20, Ar 40; interval 32,
    horizon 16): forecaster samples from a seeded run until samples_target
    leaves have been seen, training, then the same start (another seed) run
    eval_steps steps with the criterion every 10 steps, the criterion every
    32 and the learned regrid every 32; regrids, escapes (leaves the
    criterion flags at a regrid), misses and MLUPS of each."""
    import numpy as np
    import amrlbm
    p, bubbles = amrlbm.learned_workload(regrid_every=32)
    g = amrlbm.AmrLbm(p)
    g.set_bubbles(bubbles)
    g.initialize_rising_bubble()
    xs, ys, seen, pos, regrids = [], [], 0, 0, 0
    while seen < samples_target and regrids < 400:
        x, y, c = amrlbm.collect_samples(g, regrids=10, horizon=16, keep_far=0.02, seed=regrids)
        xs.append(x)
        ys.append(y)
        seen, pos, regrids = seen + c["samples"], pos + c["positives"], regrids + 10
    check_state(g.output(), "learned-regrid sample run")
    leaves0 = g.counts()["nleaf"]
    g.close()
    x, y = np.concatenate(xs), np.concatenate(ys)
    net = amrlbm.Net(seed=7, max_batch=512)
    losses = amrlbm.train_net(net, x, y, epochs=3, batch=256)
    out = {"workload": "learned_regrid_base512x1024_blocks16_L3_8bubbles_ratio1000",
           "samples_seen": int(seen), "positives": int(pos), "samples_trained": int(len(y)),
           "sample_regrids": regrids, "leaves": int(leaves0), "losses": losses}
    p2, b2 = amrlbm.learned_workload(regrid_every=32, seed=20261206)
    for name, every, use in (("criterion_every_10", 10, False), ("criterion_every_32", 32, False),
                             ("learned_every_32", 32, True)):
        p2.regrid_every = every
        s = amrlbm.AmrLbm(p2)
        s.set_bubbles(b2)
        s.initialize_rising_bubble()
        if use:  # the forecast runs inside the step's graph before each regrid
            s.set_regrid_net(net, horizon=16.0, threshold=0.5)
        c0 = s.profile_read(0)[2]
        s.sync()
        s.timer_start()
        s.main_loop(eval_steps)
        ms = s.timer_stop()
        st = s.regrid_stats()
        st["mlups"] = (s.profile_read(0)[2] - c0) / (ms / 1e3) / 1e6
        st["leaves"] = s.counts()["nleaf"]
        check_state(s.output(), name)
        out[name] = st
        s.close()
    return out, net


def long_run_leg(steps=5000):
    """The headline workload's full 5000 steps from the start-up, device-timed
    with every regrid and mesh change inside: MLUPS over the whole run, the
    leaf count along it and the final diagnostics."""
    import amrlbm
    p = workload()
    g = amrlbm.AmrLbm(p)
    g.initialize_rising_bubble()
    out = {"steps": steps, "leaves_start": g.counts()["nleaf"]}
    c0 = g.profile_read(0)[2]
    ms, done, leaves = 0.0, 0, []
    while done < steps:
        k = min(500, steps - done)
        g.sync()
        g.timer_start()
        g.main_loop(k)
        ms += g.timer_stop()
        done += k
        leaves.append(g.counts()["nleaf"])
    d = g.output()
    check_state(d, "5000-step run")
    out.update({"mlups": (g.profile_read(0)[2] - c0) / (ms / 1e3) / 1e6, "ms": ms,
                "leaves_every_500_steps": leaves,
                "diagnostics": {k: d[k] for k in ("mass", "u_max", "y_centroid", "rise_velocity")}})
    g.close()
    return out


def batch_forecaster(count=32, regrids=40, seed=20261207):
    """A forecaster for the batch's physics: samples from another seeded batch
    of `count` problems (regrids every 32 steps, labels 16 steps ahead),
    trained as in the learned-regrid leg."""
    import numpy as np
    import amrlbm
    insts = amrlbm.batch_instances(count, seed=seed)
    g = amrlbm.AmrLbm(amrlbm.batch_params(n=16, max_blks=80000, regrid_every=32), instances=insts)
    g.initialize_rising_bubble()
    x, y, c = amrlbm.collect_samples(g, regrids=regrids, horizon=16, keep_far=0.05, seed=3)
    g.close()
    net = amrlbm.Net(seed=7, max_batch=512)
    losses = amrlbm.train_net(net, x, y, epochs=4, batch=256)
    z = net.forward(x.astype(np.float32))
    recall = float(((z > 0) & (y > 0)).sum() / max(y.sum(), 1))
    return net, {"problems": count, "seed": seed, "samples_seen": c["samples"],
                 "positives": c["positives"], "samples_trained": int(len(y)),
                 "losses": losses, "train_recall": recall}


def batched_leg(count=256, steps=2000, tune_count=32):
    """Batched uneven instances, and the three layers together: the seeded
    256-problem batch (block size and CTAs per SM picked by amrlbm.autotune
    on its first tune_count problems), each run `steps` steps from the
    start-up, device-timed: the plain FP64 path with the criterion every 10
    steps; FP16 storage with the criterion every 10 and every 32 steps; FP16
    storage with the learned regrid every 32 steps (a forecaster trained on
    another seeded batch, batch_forecaster). Per instance at the end, the
    relative mass and rise-velocity differences of each FP16 run against the
    FP64 one."""
    import numpy as np
    import amrlbm
    insts = amrlbm.batch_instances(count)
    best, table = amrlbm.autotune(insts[:tune_count], "fp16", intervals=1, warmup=1)
    ctas = (best or {}).get("ctas_per_sm", 0)
    net, training = batch_forecaster()
    res = {"instances": count, "steps": steps, "block": "16x16",
           "autotune": {"best": best, "table": table}, "forecaster": training}
    ends = {}
    arms = (("fp64_criterion_every_10", "fp64", 10, False),
            ("fp16_criterion_every_10", "fp16", 10, False),
            ("fp16_criterion_every_32", "fp16", 32, False),
            ("fp16_learned_every_32", "fp16", 32, True))
    for name, prec, every, use in arms:
        g = amrlbm.AmrLbm(amrlbm.batch_params(n=16, max_blks=400000, regrid_every=every),
                          instances=insts)
        g.initialize_rising_bubble()
        c = g.counts()
        res.setdefault("leaves_start", c["nleaf"])
        res.setdefault("leaf_cells_start", c["nleaf"] * 256)
        if prec != "fp64":
            g.set_precision(prec)
            g.set_launch(ctas)
        if use:
            g.set_regrid_net(net, horizon=16.0, threshold=0.5)
        c0 = g.profile_read(0)[2]
        g.sync()
        g.timer_start()
        g.main_loop(steps)
        ms = g.timer_stop()
        st = g.regrid_stats()
        st["mlups"] = (g.profile_read(0)[2] - c0) / (ms / 1e3) / 1e6
        st["ms"] = ms
        st["leaves"] = g.counts()["nleaf"]
        d = g.output_instances()
        bad = [i for i, x in enumerate(d) if not (x["u_max"] < U_BOUND and x["rho_min"] > 0)]
        if bad:
            raise RuntimeError(f"batched {name}: instances {bad[:8]} not physical")
        ends[name] = d
        res[name] = st
        g.close()
    net.close()
    ref = ends["fp64_criterion_every_10"]
    for name in ("fp16_criterion_every_10", "fp16_criterion_every_32", "fp16_learned_every_32"):
        dm = np.array([abs(y["mass"] - x["mass"]) / abs(x["mass"]) for x, y in zip(ref, ends[name])])
        dv = np.array([abs(y["rise_velocity"] - x["rise_velocity"]) /
                       max(abs(x["rise_velocity"]), 1e-300) for x, y in zip(ref, ends[name])])
        res[name]["vs_fp64"] = {
            "mass_rel_diff": {"max": float(dm.max()), "median": float(np.median(dm)),
                              "instances_within_1e-6": int((dm <= 1e-6).sum())},
            "rise_velocity_rel_diff": {"max": float(dv.max()), "median": float(np.median(dv)),
                                       "instances_within_1pct": int((dv <= 0.01).sum())}}
        res[name]["speedup_vs_fp64"] = res[name]["mlups"] / res["fp64_criterion_every_10"]["mlups"]
    return res


def run_own(args):
    world, rank, local = dist_setup("nccl")
    import amrlbm
    import numpy as np
    dev = None
    if world > 1:
        import torch
        torch.cuda.set_device(local)
        dev = torch.device("cuda", local)
    p = workload()
    p.device = local
    if args.max_blks:
        p.max_blks = args.max_blks
    inner = p.regrid_every
    gpu = amrlbm.AmrLbm(p)
    gpu.initialize_rising_bubble()
    for _ in range(args.warmup):
        gpu.main_loop(inner)
    gpu.sync()
    check_state(gpu.output(), "after warm-up")
    # the oracle takes the state the timed region starts from (rank 0, N=1)
    orc = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        orc = oracle_from_device(gpu, p, os.cpu_count() or 1)

    def barrier():
        gpu.sync()
        if world > 1:
            import torch
            import torch.distributed as dist
            torch.cuda.synchronize()
            dist.barrier()

    # ---- device-timed region (no per-kernel events inside it)
    cells0 = gpu.profile_read(0)[2]  # leaf-cell updates so far (device counter)
    launches0 = gpu.launch_count()
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    total_ms = 0.0
    for _ in range(args.steps):
        gpu.flush_l2()
        gpu.sync()
        gpu.timer_start()
        gpu.main_loop(inner)
        total_ms += gpu.timer_stop()
    clk = clocks.stop()
    barrier()
    launches = gpu.launch_count() - launches0
    updates = gpu.profile_read(0)[2] - cells0
    diag_timed = gpu.output()
    check_state(diag_timed, "after the timed region")

    # ---- the same steps once more with CUDA events around each kernel group,
    # for the per-kernel split and the roofline of the dominant kernel
    gpu.profile(True)
    for _ in range(args.steps):
        gpu.flush_l2()
        gpu.sync()
        gpu.main_loop(inner)
    gpu.sync()
    kern = {}
    for k, (name, bpc) in KERNELS.items():
        ms, n, _ = gpu.profile_read(k)
        kern[k] = (name, bpc, ms, n)
    gpu.profile(False)
    check_state(gpu.output(), "after the per-kernel pass")
    max_ms = allreduce([total_ms], _op("max"), world, dev)[0]
    all_updates = allreduce([float(updates)], _op("sum"), world, dev)[0]
    value = all_updates / (max_ms / 1e3) / 1e6

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        # every leaf's fields in page-locked host memory (the caller's buffers)
        sizes = dict(h=int(np.prod(gpu.hshape)), g=int(np.prod(gpu.hshape)),
                     C=int(np.prod(gpu.cshape)), P=int(np.prod(gpu.pshape)),
                     Ux=int(np.prod(gpu.pshape)), Uy=int(np.prod(gpu.pshape)))
        cap = 2 * len(gpu.leaves()) + 64

        def pinned(rows, cols):
            try:
                import torch
                return torch.empty((rows, cols), dtype=torch.float64, pin_memory=True).numpy()
            except Exception:
                return np.empty((rows, cols))
        host = {k: pinned(cap, v) for k, v in sizes.items()}

        def views(n):
            return {k: a[:n] for k, a in host.items()}
        ids = gpu.leaves()
        state = gpu.download_fields(ids, out=views(len(ids)))
        _, _, u0 = gpu.profile_read(0)
        h2d = d2h = 0
        barrier()
        t_e2e = 0.0
        for _ in range(args.steps):
            t = time.perf_counter()
            gpu.upload_fields(ids, state)
            h2d += sum(a.nbytes for a in state.values()) + ids.nbytes
            gpu.main_loop(inner)
            ids = gpu.leaves()
            state = gpu.download_fields(ids, out=views(len(ids)))
            diag = gpu.output()
            d2h += sum(a.nbytes for a in state.values()) + ids.nbytes + 8 * len(diag)
            t_e2e += time.perf_counter() - t
            check_state(diag, "end-to-end step")
        barrier()
        _, _, u1 = gpu.profile_read(0)
        t_max = allreduce([t_e2e], _op("max"), world, dev)[0]
        u_all = allreduce([float(u1 - u0)], _op("sum"), world, dev)[0]
        e2e = {"value": u_all / t_max / 1e6, "unit": "MLUPS",
               "h2d_bytes_per_step": int(h2d / args.steps),
               "d2h_bytes_per_step": int(d2h / args.steps)}

    # ---- the same workload with mixed-precision storage (the state goes on)
    mixed = {}
    if not args.no_mixed:
        for prec in ("fp16", "bf16"):
            gpu.set_precision(prec)
            for _ in range(2):
                gpu.main_loop(inner)
            v = amrlbm.time_intervals(gpu, args.steps, inner)
            # compulsory traffic with 16-bit populations and FP32 fields: 2 (18 x 2 + 4 x 4) B
            mixed[prec] = {"mlups": v, "hbm_gbs": v * 1e6 * BYTES_PER_UPDATE_MIXED / 1e9}
            check_state(gpu.output(), f"{prec} leg")
        gpu.set_precision("fp64")
        mixed["fp64_mlups"] = value
    diag = gpu.output()
    if rank != 0:
        gpu.close()
        _finish(world)
        return 0

    # ---- roofline of the dominant kernel
    peak, peak_kind = measured_peak()
    dom = max((k for k in kern if kern[k][1]), key=lambda k: kern[k][2])
    name, bpc, ms, n = kern[dom]
    cells_per_launch = updates / (args.steps * inner)  # every kernel visits every leaf
    avg_s = ms / max(n, 1) / 1e3
    achieved = cells_per_launch * bpc / avg_s / 1e9
    traffic = profile_traffic(name)
    roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                               if peak_kind == "measured" else "fallback 6650 GB/s",
                "algorithmic_bytes_per_cell": bpc, "cells_per_launch": cells_per_launch,
                "avg_launch_us": avg_s * 1e6}
    total_prof = sum(v[2] for v in kern.values()) or 1.0
    kernels = {v[0]: {"launches": v[3], "total_ms": round(v[2], 4),
                      "avg_us": round(v[2] / max(v[3], 1) * 1e3, 2),
                      "share": round(v[2] / total_prof, 4)} for v in kern.values()}

    cpu = cpu4 = None
    if orc is not None:
        def same_as_device(d):
            for k, v in diag_timed.items():
                if d[k] != v:
                    raise RuntimeError(f"oracle differs from the device over the timed "
                                       f"window: {k} {d[k]} != {v}")
        threads = os.cpu_count() or 1
        v, chunks, el = cpu_leg(orc, p, inner, args.cpu_seconds, min_chunks=args.steps,
                                check_after=(args.steps, same_as_device))
        cpu = {"value": v, "unit": "MLUPS", "cores": threads, "kind": "port",
               "sample": f"{chunks} x {inner} time steps from the state the timed region "
                         f"started from ({el:.1f} s); after the first {args.steps} "
                         f"intervals its diagnostics equalled the device's bit for bit",
               "parity_over_timed_window": "bit-exact",
               "phase_share": cpu_leg.phase_share}
        orc.set_threads(4)
        v4, chunks4, el4 = cpu_leg(orc, p, inner, args.cpu_seconds / 2)
        cpu4 = {"value": v4, "unit": "MLUPS", "cores": 4, "kind": "port",
                "sample": f"the next {chunks4} x {inner} time steps ({el4:.1f} s) at 4 threads, "
                          f"the reference's OMP_NUM_THREADS",
                "phase_share": cpu_leg.phase_share}
        orc.close()
    mixed_err = batched = learned = None
    # the single-GPU legs (minutes of rank 0 alone) only at N = 1: in a
    # scaling run the other ranks' GPUs would wait for them
    long_run = None if (args.no_long or world > 1) else long_run_leg()
    if not args.no_mixed and world == 1:
        mixed_err = mixed_error_report()
        learned, net = learned_leg()
        net.close()
        batched = batched_leg()
    line = {"metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (analytic rising bubble of the reference start-up)",
            "config": config_dict(p, inner), "hbm_gbs": value * 1e6 * BYTES_PER_UPDATE / 1e9,
            "roofline": roofline, "cpu_baseline": cpu, "cpu_baseline_4_threads": cpu4,
            "e2e": e2e, "clocks": clk,
            "gpu_launches": int(launches), "kernels": kernels,
            "mixed_precision": mixed or None, "mixed_precision_error": mixed_err,
            "batched": batched, "learned_regrid": learned,
            "long_run": long_run,
            "leaf_cells_per_step": updates / (args.steps * inner),
            "diagnostics": {k: diag[k] for k in ("mass", "y_centroid", "rise_velocity")}}
    print(json.dumps(line), flush=True)
    gpu.close()
    _finish(world)
    return 0


def _op(name):
    try:
        import torch.distributed as dist
        return dist.ReduceOp.MAX if name == "max" else dist.ReduceOp.SUM
    except Exception:
        return None


def _finish(world):
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_profile(args):
    """The workload in one storage precision, warm-up and timed intervals
    only, for profiler captures of its kernels."""
    import amrlbm
    p = workload()
    if args.max_blks:
        p.max_blks = args.max_blks
    g = amrlbm.AmrLbm(p)
    g.initialize_rising_bubble()
    g.set_precision(args.profile_precision)
    for _ in range(args.warmup):
        g.main_loop(p.regrid_every)
    g.sync()
    v = amrlbm.time_intervals(g, args.steps, p.regrid_every)
    check_state(g.output(), "profile run")
    print(json.dumps({"profile_precision": args.profile_precision, "mlups": v}), flush=True)
    g.close()
    return 0


def run_profile_forecast(args):
    """The forecast kernel on the learned workload reduced to a 256x512 base
    (4 bubbles R 32 to 128, 3 levels): a seeded net, regrids every 32 steps,
    warm-up and timed intervals."""
    import amrlbm
    p, b = amrlbm.learned_workload(256, 512, 3, 4, regrid_every=32)
    if args.max_blks:
        p.max_blks = args.max_blks
    g = amrlbm.AmrLbm(p)
    g.set_bubbles(b)
    g.initialize_rising_bubble()
    net = amrlbm.Net(seed=7, max_batch=64)
    g.set_regrid_net(net, horizon=16.0, threshold=0.5)
    g.main_loop(32 * args.warmup)
    v = amrlbm.time_intervals(g, args.steps, 32)
    check_state(g.output(), "forecast profile run")
    print(json.dumps({"profile_forecast": True, "leaves": g.counts()["nleaf"], "mlups": v,
                      "regrid_stats": g.regrid_stats()}), flush=True)
    g.close()
    net.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_forecast:
        return run_profile_forecast(args)
    if args.profile_precision:
        return run_profile(args)
    return run_own(args)


if __name__ == "__main__":
    sys.exit(main())
