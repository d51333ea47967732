#!/usr/bin/env python
"""Benchmark of the B200 pressure projection.

Metric: ms per projection (and PCG iterations) to 1e-6 relative residual
(infinity norm, the reference's stopping rule) on the 256^3 sloshing-tank
workload: free surface y = 0.5 + 0.1 sin(2 pi x) cos(2 pi z), eight seeded
solid boxes, Gaussian face velocities (sigma 0.5), dt = 0.005.

A step is one full projection (labelling, tile pool, weights/rhs, MIC(0)
factor, FP32 PCG with FP64 reductions and refinement, velocity update), on
inputs already resident in HBM, preceded by a device copy that restores the
input velocity (the projection updates it in place). ``e2e`` is the same
projection through the host-buffer C-ABI call with pinned host arrays, so the
host-device copies are inside its timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU runs are independent replicas (the projection does not shard):
each rank projects its own copy; the time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DEFAULT_MODEL = os.path.join(ROOT, "shiokaze_b200", "models", "shkz_net.bin")
METRIC = "ms/projection & PCG iters to 1e-6 rel. residual at 256³: learned vs plain, 1 B200"
UNIT = "ms/projection"

# Algorithmic bytes per pool cell (cells of 8^3 tiles holding >= 1 unknown)
# for each kernel, FP32 data: reads + writes of the arrays it must touch once.
# The MIC(0)-PCG iteration on 16^3 macro tiles runs as two passes:
ALGO_BYTES = {
    # stencil with the direction update: read p_old, z, diag, 3 lower
    # weights; write p_new, q
    "spmv": 32,
    # forward sweep with the x/r update: read r q p x d + 3 w, write r x t
    # (44); backward sweep: read t d 3 w r, write z (28)
    "mic_sweeps": 72,
    # the unfused kernels (8^3-tile sweeps, learned preconditioner path)
    "spmv_plain": 24,        # x, diag, 3 lower weights, y
    "mic_sweeps_plain": 52,  # forward 24, backward 28
    "update_xr": 24,         # read p, q, x, r; write x, r
    "update_p": 12,          # read z, p; write p
}

# One fused MIC(0)-PCG iteration: stencil pass 32 + sweep pair 72.
ITER_BYTES = 104

# library kernels one splat call launches: bin, tile scan, three scan passes,
# scatter, sort, three face compactions, three work counts, work scan, three
# face sorts, three gathers, clear
SPLAT_LAUNCHES = 21

# FLIP splat workload (--workload flip_splat): the splat and combined grid
# velocity before a projection, on the 256^3 sloshing tank with particles in
# the 3-cell narrow band at 8 per cell. Algorithmic bytes: every particle's
# record fields read once (p 12, c 36, velocity 12, mass 4, bullet 1) and
# every splatted face's velocity and mask read and written (4 + 1 + 4 + 1).
SPLAT_METRIC = "ms/splat (FLIP splat + combined grid velocity) at 256³, 3-cell narrow band, 8 particles/cell"
SPLAT_UNIT = "ms/splat"
SPLAT_BYTES_PARTICLE = 65
SPLAT_BYTES_FACE = 10


def job_ms_per_projection(elapsed_ms: float, steps: int, world: int, device=None) -> float:
    """Whole-job ms per projection: the slowest rank's timed region (max over
    ranks, all_reduce MAX) over the projections all ranks ran. Replicas run
    independent projections, so per-rank work is fixed as ranks are added."""
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([elapsed_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    return elapsed_ms / (steps * world)


def measured_bf16_peak():
    """Dense BF16 tensor peak for a kernel timed alone (burst figure)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        if "bf16_tflops" in d:
            return float(d["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes of the stencil kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    # where the samples go: --clock-log DIR, else the system temp directory
    LOG_DIR = None

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join(self.LOG_DIR or tempfile.gettempdir(), f"clocks_bench_{os.getpid()}_{device}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sms, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                maxes.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        if not sms:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": max(maxes), "reasons": sorted(reasons),
                "samples": len(sms)}


def cpu_reference_sample(n: int = 128):
    """The compiled reference (oracle/_ref) on a bounded sample of the workload:
    the same scene at n^3, timed with the reference's own projection path."""
    from shiokaze_b200 import scenes
    from oracle import ref_runner
    sc = scenes.sloshing_tank(n=n, seed=0, tol=1e-6)
    if ref_runner.ref_available("float"):
        # no system dump: the reference's solver would write it inside project()
        r = ref_runner.run_reference(sc, mode="mic0", dump_system=False)
        its = r.console_solves[-1][0] if r.console_solves else None
        return {"value": r.projection_ms, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                "sample": f"sloshing tank {n}^3 (1/{(256 // n) ** 3} of the 256^3 cells), reference "
                          f"macpressuresolver3 + MIC(0)-PCG to 1e-6, Threads={os.cpu_count()} (its PCG is "
                          f"single-threaded), {its} iterations, 1 projection"}
    from oracle import oracle
    t = time.perf_counter()
    o = oracle.project(sc, mic0=True)
    ms = (time.perf_counter() - t) * 1e3
    return {"value": ms, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"sloshing tank {n}^3, C restatement of the reference, MIC(0)-PCG to 1e-6, "
                      f"{o.iterations} iterations, 1 projection"}


def splat_workload(n: int):
    from shiokaze_b200 import scenes
    sc = scenes.sloshing_tank(n=n, seed=0, tol=1e-6)
    P = scenes.flip_particles(sc, per_cell=8, seed=0, band=3.0)
    return sc, P


def splat_reference_sample(n: int):
    """The compiled reference splat (oracle/_ref shkz_ref_splat: pointgridhash3
    hash, macnbflip3::splat, combined velocity) on the splat workload at n^3;
    its own timers, file I/O excluded."""
    from oracle import ref_runner
    sc, P = splat_workload(n)
    r = ref_runner.run_reference_splat(sc.nx, sc.ny, sc.nz, sc.dx, P, sc.velocity_effective(),
                                       [m.astype(np.uint8) for m in sc.velocity_active])
    return sc, P, r["hash_ms"] + r["splat_ms"] + r["combine_ms"]


def run_splat_reference_arm(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    from oracle import ref_runner
    if not ref_runner.ref_available("float"):
        print(json.dumps({"impl": "reference", "unavailable": "compiled reference splat (oracle/_ref) not built"}))
        return 0
    budget_s = float(os.environ.get("SHKZ_REF_BUDGET_S", "240"))
    times, t_start = [], time.perf_counter()
    while len(times) < max(1, args.steps):
        sc, P, ms = splat_reference_sample(args.n)
        times.append(ms)
        if time.perf_counter() - t_start > budget_s:
            break
    value = float(np.mean(times))
    sample = (f"sloshing tank {args.n}^3, {len(P)} particles, reference pointgridhash3 + macnbflip3::splat + "
              f"combined velocity, {len(times)} of {args.steps} requested splats within {budget_s:.0f} s")
    line = {"metric": SPLAT_METRIC, "value": value, "unit": SPLAT_UNIT, "n_gpus": args.gpus, "steps": len(times),
            "warmup": 0, "ms_per_step": value, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 weights into f32 sums", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"flip_splat sloshing_tank {args.n}^3, 3-cell band, 8 particles/cell, APIC"},
            "cpu_baseline": {"value": value, "unit": SPLAT_UNIT, "cores": os.cpu_count(), "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": SPLAT_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_splat(args):
    """The FLIP splat workload on the device: particles and grids resident in
    HBM; a step restores the input velocity (device copy) and runs
    shkz_b200_splat_device. e2e: shkz_b200_splat_host with pinned host arrays."""
    import torch
    import torch.distributed as dist
    from shiokaze_b200 import native

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    sc, P = splat_workload(args.n)
    nx, ny, nz = sc.nx, sc.ny, sc.nz
    cfg = native.default_config()
    cfg.device = local
    ctx = native.Context(cfg)
    L = native.load()
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    T = lambda arr: torch.from_numpy(np.ascontiguousarray(arr)).to(dev)
    rec = T(P.view(np.uint8))
    vel0 = [T(v) for v in sc.velocity_effective()]
    act0 = [T(m.astype(np.uint8)) for m in sc.velocity_active]
    vel = [v.clone() for v in vel0]
    act = [m.clone() for m in act0]
    sact = [torch.zeros_like(m) for m in act0]
    mass = [torch.zeros_like(v) for v in vel0]
    mom = [torch.zeros_like(v) for v in vel0]
    torch.cuda.synchronize(dev)
    a = native.splat_args(nx, ny, nz, sc.dx, rec.data_ptr(), len(P), P.dtype, apic=True)
    for d in range(3):
        a.velocity[d], a.velocity_active[d] = vel[d].data_ptr(), act[d].data_ptr()

    def step():
        with torch.cuda.stream(stream):
            for d in range(3):
                vel[d].copy_(vel0[d], non_blocking=True)
                act[d].copy_(act0[d], non_blocking=True)
        ctx.check(L.shkz_b200_splat_device(ctx.handle, ctypes.byref(a)), "shkz_b200_splat_device")

    # untimed: the splat grid, for the count of splatted faces
    b = native.splat_args(nx, ny, nz, sc.dx, rec.data_ptr(), len(P), P.dtype, apic=True)
    for d in range(3):
        b.velocity[d], b.velocity_active[d] = vel[d].data_ptr(), act[d].data_ptr()
        b.mass[d], b.momentum[d], b.splat_active[d] = mass[d].data_ptr(), mom[d].data_ptr(), sact[d].data_ptr()
    ctx.check(L.shkz_b200_splat_device(ctx.handle, ctypes.byref(b)), "shkz_b200_splat_device")
    faces = int(sum(int(x.sum()) for x in sact))
    for _ in range(args.warmup):
        step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    value = job_ms_per_projection(ev0.elapsed_time(ev1), args.steps, world, dev)
    # the splat call alone (no restore copies) for the roofline
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ctx.check(L.shkz_b200_splat_device(ctx.handle, ctypes.byref(a)), "shkz_b200_splat_device")
    e1.record(stream)
    torch.cuda.synchronize(dev)
    call_ms = e0.elapsed_time(e1) / args.steps
    algo = SPLAT_BYTES_PARTICLE * len(P) + SPLAT_BYTES_FACE * faces
    peak, peak_kind = measured_peaks()
    achieved = algo / (call_ms * 1e-3) / 1e9
    t0 = (ncu_traffic() or {}).get("splat_call")
    traffic = t0["dram_bytes_per_launch"] * len(P) / t0["particles"] if t0 else None
    roofline = {"kernel": "shkz_b200_splat_device (bin, scan, bucket sort, face lists, k_splat_gather x3)",
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "ms": call_ms, "algo_bytes_per_launch": algo, "traffic": traffic,
                "note": ("not HBM-bound: the gather (about 3/5 of the call) is bound by FP64 issue and latency, "
                         "each face summing its particles serially in the reference's order; traffic is 9.5x the "
                         "algorithmic bytes because of the hash (packed and bucket-ordered particle copies, the "
                         "gather's L2 re-reads)")}
    # end to end through the host-buffer entry point, pinned host arrays
    pin = lambda arr: torch.from_numpy(np.ascontiguousarray(arr)).pin_memory()
    h_rec = pin(P.view(np.uint8))
    h_vel0 = [v.copy() for v in sc.velocity_effective()]
    h_act0 = [m.astype(np.uint8) for m in sc.velocity_active]
    h_vel = [pin(v) for v in h_vel0]
    h_act = [pin(m) for m in h_act0]
    ha = native.splat_args(nx, ny, nz, sc.dx, h_rec.data_ptr(), len(P), P.dtype, apic=True)
    for d in range(3):
        ha.velocity[d], ha.velocity_active[d] = h_vel[d].data_ptr(), h_act[d].data_ptr()
    tot = 0.0
    for i in range(args.steps + 1):
        for d in range(3):
            h_vel[d].numpy()[...] = h_vel0[d]
            h_act[d].numpy()[...] = h_act0[d]
        t0 = time.perf_counter()
        ctx.check(L.shkz_b200_splat_host(ctx.handle, ctypes.byref(ha)), "shkz_b200_splat_host")
        if i > 0:
            tot += (time.perf_counter() - t0) * 1e3
    nfaces = sum(v.numel() for v in h_vel)
    e2e = {"value": job_ms_per_projection(tot, args.steps, world, dev), "unit": SPLAT_UNIT,
           "h2d_bytes_per_step": int(h_rec.numel() + 5 * nfaces),
           "d2h_bytes_per_step": int(5 * nfaces), "steps": args.steps, "timer": "host wall clock around the call"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import ref_runner
            if ref_runner.ref_available("float"):
                _, Ps, ms = splat_reference_sample(128)
                cpu = {"value": ms, "unit": SPLAT_UNIT, "cores": os.cpu_count(), "kind": "reference",
                       "sample": f"sloshing tank 128^3 (1/8 of the cells), {len(Ps)} particles: reference "
                                 f"pointgridhash3 hash + macnbflip3::splat + combined velocity, its own timers"}
        except Exception as exc:
            cpu = {"error": str(exc)}
    if rank == 0:
        line = {"metric": SPLAT_METRIC, "value": value, "unit": SPLAT_UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64 weights into f32 sums", "data": "synthetic",
                "config": {"workload": f"flip_splat sloshing_tank {nx}^3, 3-cell band, 8 particles/cell, APIC",
                           "particles": len(P), "splatted_faces": faces,
                           "l2": "particle records 0.2 GB + face grids 0.25 GB > 126 MB L2 (no flush needed)",
                           "step": "device velocity restore + one splat"},
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk.summary(),
                "gpu_launches": args.steps * SPLAT_LAUNCHES}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_liquid_step(args):
    """The projection with its timestep neighbours on the device: FLIP splat ->
    projection -> velocity extension (width 3 + constraint) on device arrays,
    against the same three steps through the host-buffer entry points, each of
    which moves its grids across PCIe/C2C. The first is what the liquid solver
    gets from keeping the velocity resident between the steps."""
    import torch
    from shiokaze_b200 import native
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    sc, P = splat_workload(args.n)
    nx, ny, nz = sc.nx, sc.ny, sc.nz
    cfg = native.default_config()
    cfg.residual = sc.tol
    ctx = native.Context(cfg)
    L = native.load()
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    T = lambda arr: torch.from_numpy(np.ascontiguousarray(arr)).to(dev)
    host = {"rec": P.view(np.uint8), "fluid": sc.fluid_effective(), "fact": sc.fluid_active.astype(np.uint8),
            "solid": sc.solid_effective(), "sact": sc.solid_active.astype(np.uint8)}
    hvel = [np.ascontiguousarray(v) for v in sc.velocity_effective()]
    hact = [m.astype(np.uint8) for m in sc.velocity_active]
    pinned = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in host.items()}
    pvel = [torch.from_numpy(v).pin_memory() for v in hvel]
    pact = [torch.from_numpy(m).pin_memory() for m in hact]
    out_vel = [torch.empty_like(v) for v in pvel]
    out_act = [torch.empty_like(m) for m in pact]
    d = {k: torch.empty(v.shape, dtype=v.dtype, device=dev) for k, v in pinned.items()}
    vel = [torch.empty(v.shape, dtype=v.dtype, device=dev) for v in pvel]
    act = [torch.empty(m.shape, dtype=m.dtype, device=dev) for m in pact]
    pres = torch.empty((nz, ny, nx), dtype=torch.float32, device=dev)
    pres_a = torch.empty((nz, ny, nx), dtype=torch.uint8, device=dev)
    sp = native.splat_args(nx, ny, nz, sc.dx, d["rec"].data_ptr(), len(P), P.dtype, apic=True)
    pa = native.ProjectArgs()
    pa.nx, pa.ny, pa.nz, pa.dx, pa.dt = nx, ny, nz, sc.dx, sc.dt
    pa.fluid, pa.fluid_active = d["fluid"].data_ptr(), d["fact"].data_ptr()
    pa.solid, pa.solid_active = d["solid"].data_ptr(), d["sact"].data_ptr()
    pa.pressure, pa.pressure_active = pres.data_ptr(), pres_a.data_ptr()
    ea = native.ExtendArgs()
    ea.nx, ea.ny, ea.nz, ea.dx, ea.width, ea.constrain = nx, ny, nz, sc.dx, 3, 1
    ea.solid, ea.solid_active = d["solid"].data_ptr(), d["sact"].data_ptr()
    for k in range(3):
        sp.velocity[k], sp.velocity_active[k] = vel[k].data_ptr(), act[k].data_ptr()
        pa.velocity[k], pa.velocity_active[k], pa.solid_velocity[k] = vel[k].data_ptr(), act[k].data_ptr(), None
        ea.velocity[k], ea.velocity_active[k] = vel[k].data_ptr(), act[k].data_ptr()
    res = native.Result()
    h2d = sum(t.numel() * t.element_size() for t in list(pinned.values()) + pvel + pact)
    d2h = sum(t.numel() * t.element_size() for t in pvel + pact)

    def chain():
        ctx.check(L.shkz_b200_splat_device(ctx.handle, ctypes.byref(sp)), "splat_device")
        ctx.check(L.shkz_b200_project_device(ctx.handle, ctypes.byref(pa), ctypes.byref(res)), "project_device")
        ctx.check(L.shkz_b200_extend_velocity_device(ctx.handle, ctypes.byref(ea)), "extend_velocity_device")

    def upload():
        with torch.cuda.stream(stream):
            for k in pinned:
                d[k].copy_(pinned[k], non_blocking=True)
            for k in range(3):
                vel[k].copy_(pvel[k], non_blocking=True)
                act[k].copy_(pact[k], non_blocking=True)

    def download():
        with torch.cuda.stream(stream):
            for k in range(3):
                out_vel[k].copy_(vel[k], non_blocking=True)
                out_act[k].copy_(act[k], non_blocking=True)
        stream.synchronize()

    for _ in range(args.warmup):
        upload(); chain(); download()
    # device: inputs resident, a step restores the velocity on the device and runs the chain
    dvel0 = [v.clone() for v in vel]
    dact0 = [m.clone() for m in act]
    upload()
    torch.cuda.synchronize(dev)
    for k in range(3):
        dvel0[k].copy_(vel[k]); dact0[k].copy_(act[k])
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                for k in range(3):
                    vel[k].copy_(dvel0[k], non_blocking=True)
                    act[k].copy_(dact0[k], non_blocking=True)
            chain()
        e1.record(stream)
        torch.cuda.synchronize(dev)
    value = e0.elapsed_time(e1) / args.steps
    iters = res.iterations
    # chained e2e: upload once, three device steps, download once
    t = 0.0
    for _ in range(args.steps):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        upload(); chain(); download()
        t += time.perf_counter() - t0
    chained = t / args.steps * 1e3
    # the same three steps through the host-buffer entry points
    hp = native.ProjectArgs()
    hp.nx, hp.ny, hp.nz, hp.dx, hp.dt = nx, ny, nz, sc.dx, sc.dt
    hp.fluid, hp.fluid_active = pinned["fluid"].data_ptr(), pinned["fact"].data_ptr()
    hp.solid, hp.solid_active = pinned["solid"].data_ptr(), pinned["sact"].data_ptr()
    hpres = torch.empty((nz, ny, nx), dtype=torch.float32).pin_memory()
    hpres_a = torch.empty((nz, ny, nx), dtype=torch.uint8).pin_memory()
    hp.pressure, hp.pressure_active = hpres.data_ptr(), hpres_a.data_ptr()
    hs = native.splat_args(nx, ny, nz, sc.dx, pinned["rec"].data_ptr(), len(P), P.dtype, apic=True)
    he = native.ExtendArgs()
    he.nx, he.ny, he.nz, he.dx, he.width, he.constrain = nx, ny, nz, sc.dx, 3, 1
    he.solid, he.solid_active = pinned["solid"].data_ptr(), pinned["sact"].data_ptr()
    for k in range(3):
        for a_ in (hs, hp, he):
            a_.velocity[k], a_.velocity_active[k] = out_vel[k].data_ptr(), out_act[k].data_ptr()
        hp.solid_velocity[k] = None
    hres = native.Result()
    t = 0.0
    for i in range(args.steps + 1):
        for k in range(3):
            out_vel[k].copy_(pvel[k]); out_act[k].copy_(pact[k])
        t0 = time.perf_counter()
        ctx.check(L.shkz_b200_splat_host(ctx.handle, ctypes.byref(hs)), "splat_host")
        ctx.check(L.shkz_b200_project_host(ctx.handle, ctypes.byref(hp), ctypes.byref(hres)), "project_host")
        ctx.check(L.shkz_b200_extend_velocity_host(ctx.handle, ctypes.byref(he)), "extend_velocity_host")
        if i > 0:
            t += time.perf_counter() - t0
    separate = t / args.steps * 1e3
    line = {"metric": "ms per liquid step's projection neighbourhood (FLIP splat + projection + velocity extension) "
                      "at 256³", "value": value, "unit": "ms/step", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (f64 reductions, refinement, assembly and splat weights)",
            "data": "synthetic",
            "config": {"workload": f"liquid_step sloshing_tank {nx}^3: splat of {len(P)} particles, MIC(0)-PCG "
                                   f"projection to 1e-6 ({iters} iterations), extension width 3 + constraint",
                       "step": "device velocity restore + the three device entry points"},
            "e2e": {"value": chained, "unit": "ms/step", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "timer": "host wall clock: pinned upload once, three device steps, download once"},
            "separate_host_calls": {"value": separate, "unit": "ms/step",
                                    "what": "shkz_b200_splat_host + shkz_b200_project_host + "
                                            "shkz_b200_extend_velocity_host, each copying its grids both ways"},
            "clocks": clk.summary(), "gpu_launches": None}
    print(json.dumps(line), flush=True)
    # torch's copies ran on the context's stream: free their tensors (and the
    # events torch keeps for them) before that stream is destroyed
    torch.cuda.synchronize(dev)
    del pinned, pvel, pact, out_vel, out_act, d, vel, act, dvel0, dact0, pres, pres_a, hpres, hpres_a
    import gc
    gc.collect()
    torch.cuda.synchronize(dev)
    ctx.close()
    return 0


def time_neighbours(ctx, L, sc, stream, dev, vel, vact, solid, sact, reps: int = 20):
    """Device time of the FLIP splat (3-cell band, 8 particles per cell) and
    of the velocity extension (3 passes + constraint) on the headline grid,
    CUDA events on the context stream, after one warm-up call each."""
    import torch
    from shiokaze_b200 import native, scenes
    P = scenes.flip_particles(sc, per_cell=8, seed=0, band=3.0)
    rec = torch.from_numpy(np.ascontiguousarray(P.view(np.uint8))).to(dev)
    sp = native.splat_args(sc.nx, sc.ny, sc.nz, sc.dx, rec.data_ptr(), len(P), P.dtype, apic=True)
    ea = native.ExtendArgs()
    ea.nx, ea.ny, ea.nz, ea.dx, ea.width, ea.constrain = sc.nx, sc.ny, sc.nz, sc.dx, 3, 1
    ea.solid, ea.solid_active = solid.data_ptr(), sact.data_ptr()
    for d in range(3):
        sp.velocity[d], sp.velocity_active[d] = vel[d].data_ptr(), vact[d].data_ptr()
        ea.velocity[d], ea.velocity_active[d] = vel[d].data_ptr(), vact[d].data_ptr()
    out = {"particles": len(P)}
    for name, fn, a_ in (("splat", L.shkz_b200_splat_device, sp), ("extend", L.shkz_b200_extend_velocity_device, ea)):
        ctx.check(fn(ctx.handle, ctypes.byref(a_)), name)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            ctx.check(fn(ctx.handle, ctypes.byref(a_)), name)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        out[f"{name}_ms"] = e0.elapsed_time(e1) / reps
    out["what"] = ("splat: shkz_b200_splat_device (macnbflip3::splat + combined velocity); extend: "
                   "shkz_b200_extend_velocity_device (3 passes + constrain_velocity); both repeated on the "
                   "projected velocity, untimed in the headline value")
    del rec
    return out


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from shiokaze_b200 import scenes
    from oracle import ref_runner
    n = args.n
    sc = scenes.sloshing_tank(n=n, seed=0, tol=1e-6)
    budget_s = float(os.environ.get("SHKZ_REF_BUDGET_S", "240"))
    times, iters = [], None
    kind = "reference" if ref_runner.ref_available("float") else "port"
    t_start = time.perf_counter()
    while len(times) < max(1, args.steps):
        if kind == "reference":
            # no system dump: the reference's solver would write it inside project()
            r = ref_runner.run_reference(sc, mode="mic0", dump_system=False)
            times.append(r.projection_ms)
            iters = r.console_solves[-1][0] if r.console_solves else None
        else:
            from oracle import oracle
            t = time.perf_counter()
            o = oracle.project(sc, mic0=True)
            times.append((time.perf_counter() - t) * 1e3)
            iters = o.iterations
        if time.perf_counter() - t_start > budget_s:
            break
    value = float(np.mean(times))
    cores = os.cpu_count() if kind == "reference" else 1
    sample = (f"sloshing tank {n}^3, reference macpressuresolver3 with MIC(0)-PCG to 1e-6 "
              f"({iters} iterations), {len(times)} of {args.steps} requested projections within a "
              f"{budget_s:.0f} s budget, no warm-up (CPU path has no warm state)")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": len(times),
            "warmup": 0, "ms_per_step": value, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 system, f32 grids", "data": "synthetic",
            "impl": "reference", "iterations": iters,
            "config": {"workload": f"sloshing_tank {n}^3, plain MIC(0)-PCG projection to 1e-6 (inf-norm)",
                       "seed": 0},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--precond", default="mic0", choices=["mic0", "none", "learned"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--mic-block", type=int, default=16, choices=[8, 16],
                    help="MIC(0) sweep block edge (16: 2x2x2 tiles per CTA)")
    ap.add_argument("--model", default=None, help="trained network for the learned preconditioner")
    ap.add_argument("--scene", default="sloshing_tank",
                    choices=["sloshing_tank", "splash", "dambreak_rain", "dambreak_sphere"],
                    help="sloshing_tank 256^3 (headline), splash 384^3, dambreak_rain 512^3, dambreak_sphere 64^3")
    ap.add_argument("--learned-steps", type=int, default=2,
                    help="timed projections of the learned-preconditioner arm (0: skip)")
    ap.add_argument("--no-neighbours", dest="neighbours", action="store_false",
                    help="skip the splat and extension timings added to the headline line")
    ap.add_argument("--clock-log", default=None,
                    help="directory for the nvidia-smi clock samples of the timed region (default: temp dir)")
    ap.add_argument("--workload", default="projection", choices=["projection", "flip_splat", "liquid_step"],
                    help="projection (headline), the FLIP splat before it, or splat + projection + extension")
    args = ap.parse_args()
    if args.clock_log:
        os.makedirs(args.clock_log, exist_ok=True)
        ClockSampler.LOG_DIR = args.clock_log
    if args.workload == "liquid_step":
        args.warmup = max(args.warmup, 3)
        return run_liquid_step(args)
    if args.workload == "flip_splat":
        if args.impl == "reference":
            return run_splat_reference_arm(args)
        args.warmup = max(args.warmup, 3)
        return run_splat(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    args.warmup = max(args.warmup, 3)

    import torch
    import torch.distributed as dist
    from shiokaze_b200 import native, scenes

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    if args.scene == "sloshing_tank":
        sc = scenes.sloshing_tank(n=args.n, seed=0, tol=1e-6)
    elif args.scene == "splash":
        sc = scenes.splash(n=args.n if args.n != 256 else 384, seed=0, tol=1e-6)
    elif args.scene == "dambreak_rain":
        sc = scenes.dambreak_rain(n=args.n if args.n != 256 else 512, seed=0, tol=1e-6)
    else:
        # the CPU-runnable configuration: 64^3 dam break + sphere, tolerance 1e-4
        sc = scenes.dambreak_sphere(n=args.n if args.n != 256 else 64, seed=0)
    nx, ny, nz = sc.nx, sc.ny, sc.nz

    cfg = native.default_config()
    cfg.residual = sc.tol
    cfg.preconditioner = {"mic0": native.PRECOND_MIC0, "none": native.PRECOND_NONE,
                          "learned": native.PRECOND_LEARNED}[args.precond]
    cfg.device = local
    cfg.mic_block = args.mic_block
    ctx = native.Context(cfg)
    L = native.load()
    if args.precond == "learned":
        model = args.model or DEFAULT_MODEL
        ctx.check(L.shkz_b200_learned_load(ctx.handle, model.encode()), "shkz_b200_learned_load")
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)

    # device-resident inputs
    def dev_t(a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    fluid = dev_t(sc.fluid_effective(), np.float32)
    fact = dev_t(sc.fluid_active.astype(np.uint8), np.uint8)
    has_solid = sc.solid_phi is not None
    solid = dev_t(sc.solid_effective(), np.float32) if has_solid else None
    sact = dev_t(sc.solid_active.astype(np.uint8), np.uint8) if has_solid else None
    vel0 = [dev_t(v, np.float32) for v in sc.velocity_effective()]
    vact0 = [dev_t(m.astype(np.uint8), np.uint8) for m in sc.velocity_active]
    vel = [v.clone() for v in vel0]
    vact = [m.clone() for m in vact0]
    pressure = torch.zeros((nz, ny, nx), dtype=torch.float32, device=dev)
    pact = torch.zeros((nz, ny, nx), dtype=torch.uint8, device=dev)
    torch.cuda.synchronize(dev)

    a = native.ProjectArgs()
    a.nx, a.ny, a.nz, a.dx, a.dt = nx, ny, nz, sc.dx, sc.dt
    a.fluid, a.fluid_active = fluid.data_ptr(), fact.data_ptr()
    if has_solid:
        a.solid, a.solid_active = solid.data_ptr(), sact.data_ptr()
    for d in range(3):
        a.velocity[d] = vel[d].data_ptr()
        a.velocity_active[d] = vact[d].data_ptr()
        a.solid_velocity[d] = None
    a.pressure, a.pressure_active = pressure.data_ptr(), pact.data_ptr()
    res = native.Result()

    def step():
        with torch.cuda.stream(stream):
            for d in range(3):
                vel[d].copy_(vel0[d], non_blocking=True)
                vact[d].copy_(vact0[d], non_blocking=True)
        rc = L.shkz_b200_project_device(ctx.handle, ctypes.byref(a), ctypes.byref(res))
        if rc != 0:
            raise native.ShkzError(rc, "shkz_b200_project_device", ctx.last_error())
        return res.as_dict()

    for _ in range(args.warmup):
        step()
    results = []
    launches = 0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            r = step()
            results.append(r)
            launches += r["kernel_launches"]  # the restore copies are torch copies, not counted
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    value = job_ms_per_projection(ev0.elapsed_time(ev1), args.steps, world, dev)
    clocks = clk.summary()
    last = results[-1]

    # kernel timings on the last system (CUDA events on the context stream)
    kern = {}
    ms = ctypes.c_double()
    cells = ctypes.c_longlong()
    fused_kernels = (("spmv", 9), ("mic_sweeps", 10))
    plain_kernels = (("spmv_plain", 0), ("mic_sweeps_plain", 1), ("update_xr", 3), ("update_p", 4))
    for name, which in fused_kernels + (("label", 5), ("coeff", 6), ("mic_factor", 7)):
        # each timing loop in an NVTX range "time_kernel_<name>", so that a
        # profiler can select its launches (ncu --nvtx --nvtx-include ...)
        torch.cuda.nvtx.range_push(f"time_kernel_{name}")
        rc = L.shkz_b200_time_kernel(ctx.handle, which, 30 if which != 7 else 5, ctypes.byref(ms), ctypes.byref(cells))
        torch.cuda.nvtx.range_pop()
        if rc != 0:
            kern[name] = {"error": rc}
            continue
        entry = {"ms": ms.value, "cells": cells.value}
        if name in ALGO_BYTES:
            gbs = ALGO_BYTES[name] * cells.value / (ms.value * 1e-3) / 1e9
            entry["algo_bytes_per_cell"] = ALGO_BYTES[name]
            entry["achieved_gbs"] = gbs
        kern[name] = entry
    if any("error" in kern.get(k, {"error": 1}) for k, _ in fused_kernels):
        # no macro tiles (8^3 sweeps): the iteration runs the unfused kernels
        for name, which in plain_kernels:
            if L.shkz_b200_time_kernel(ctx.handle, which, 30, ctypes.byref(ms), ctypes.byref(cells)) == 0:
                kern[name] = {"ms": ms.value, "cells": cells.value, "algo_bytes_per_cell": ALGO_BYTES[name],
                              "achieved_gbs": ALGO_BYTES[name] * cells.value / (ms.value * 1e-3) / 1e9}
    peak, peak_kind = measured_peaks()
    traffic = ncu_traffic() or {}
    names = {"spmv": "k_spmv (stencil q = A p, p = z + beta p formed on the fly, fused p.q)",
             "mic_sweeps": "k_mic_forward16 + k_mic_backward16 (MIC(0) wavefront sweeps; x/r update and norms "
                           "in the forward staging, fused z.r)",
             "spmv_plain": "k_spmv (stencil q = A p with fused p.q)",
             "mic_sweeps_plain": "k_mic_forward16 + k_mic_backward16 (plain MIC(0) apply)",
             "update_xr": "k_update_xr (x, r update with inf/2-norms)", "update_p": "k_update_p"}
    rooflines = {}
    for kname, entry in kern.items():
        if "achieved_gbs" not in entry:
            continue
        tb = None
        if kname in traffic and entry.get("cells"):
            t0 = traffic[kname]
            tb = t0["dram_bytes_per_launch"] * entry["cells"] / t0["cells"]
        rooflines[kname] = {"kernel": names.get(kname, kname), "bound": "hbm", "achieved": entry["achieved_gbs"],
                            "peak": peak, "unit": "GB/s", "frac": entry["achieved_gbs"] / peak,
                            "peak_kind": peak_kind, "ms": entry["ms"],
                            "algo_bytes_per_launch": ALGO_BYTES[kname] * entry["cells"], "traffic": tb}
    # the dominant kernel of an iteration by device time
    roofline = None
    if rooflines:
        dom = max(rooflines, key=lambda k: rooflines[k]["ms"])
        roofline = dict(rooflines[dom])
        if dom.startswith("mic_sweeps"):
            roofline["note"] = ("wavefront-latency bound: each sweep is a chain of dependent macro-tile levels "
                                "(38 in the 256^3 tank) of 46 diagonal steps each; the HBM fraction shows how far "
                                "the dependency chain keeps it from streaming")
    ms_it = last["ms_solve"] / max(1, last["iterations"])
    fused = "spmv" in rooflines and "mic_sweeps" in rooflines
    it_cells = kern.get("spmv" if fused else "spmv_plain", {}).get("cells", 0)
    it_per_cell = ITER_BYTES if fused else (ALGO_BYTES["spmv_plain"] + ALGO_BYTES["mic_sweeps_plain"] +
                                            ALGO_BYTES["update_xr"] + ALGO_BYTES["update_p"])
    it_bytes = it_per_cell * it_cells
    iteration_roofline = {"bytes_per_iteration": it_bytes, "ms_per_iteration": ms_it,
                          "achieved": it_bytes / (ms_it * 1e-3) / 1e9 if ms_it else None, "peak": peak,
                          "unit": "GB/s", "frac": (it_bytes / (ms_it * 1e-3) / 1e9) / peak if ms_it else None,
                          "algo_bytes_per_cell": it_per_cell}

    # end to end through the host-buffer C-ABI call with pinned host memory
    e2e = None
    if rank == 0 or world > 1:
        pin = lambda arr: torch.from_numpy(np.ascontiguousarray(arr)).pin_memory()
        h_fluid, h_fact = pin(sc.fluid_effective()), pin(sc.fluid_active.astype(np.uint8))
        h_solid = pin(sc.solid_effective()) if has_solid else None
        h_sact = pin(sc.solid_active.astype(np.uint8)) if has_solid else None
        h_vel0 = [v.copy() for v in sc.velocity_effective()]
        h_vact0 = [m.astype(np.uint8).copy() for m in sc.velocity_active]
        h_vel = [pin(v) for v in h_vel0]
        h_vact = [pin(m) for m in h_vact0]
        h_p = torch.zeros((nz, ny, nx), dtype=torch.float32).pin_memory()
        h_pa = torch.zeros((nz, ny, nx), dtype=torch.uint8).pin_memory()
        ha = native.ProjectArgs()
        ha.nx, ha.ny, ha.nz, ha.dx, ha.dt = nx, ny, nz, sc.dx, sc.dt
        ha.fluid, ha.fluid_active = h_fluid.data_ptr(), h_fact.data_ptr()
        if has_solid:
            ha.solid, ha.solid_active = h_solid.data_ptr(), h_sact.data_ptr()
        for d in range(3):
            ha.velocity[d] = h_vel[d].data_ptr()
            ha.velocity_active[d] = h_vact[d].data_ptr()
            ha.solid_velocity[d] = None
        ha.pressure, ha.pressure_active = h_p.data_ptr(), h_pa.data_ptr()
        h2d = (h_fluid.numel() * 4 + h_fact.numel() + (h_solid.numel() * 5 if has_solid else 0)
               + sum(v.numel() * 5 for v in h_vel))
        d2h = sum(v.numel() * 5 for v in h_vel) + h_p.numel() * 5
        e2e_steps = args.e2e_steps or args.steps
        tot = 0.0
        hres = native.Result()
        for i in range(e2e_steps + 1):
            for d in range(3):
                h_vel[d].numpy()[...] = h_vel0[d]
                h_vact[d].numpy()[...] = h_vact0[d]
            rc = L.shkz_b200_project_host(ctx.handle, ctypes.byref(ha), ctypes.byref(hres))
            if rc != 0:
                raise native.ShkzError(rc, "shkz_b200_project_host", ctx.last_error())
            if i > 0:  # first call is the warm-up
                tot += hres.ms_total
        # whole-job figure like `value`: the slowest rank's time over all ranks' projections
        e2e = {"value": job_ms_per_projection(tot, e2e_steps, world, dev), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
               "h2d_ms": hres.ms_h2d, "d2h_ms": hres.ms_d2h}

    # error against the FP64 tight-tolerance solve on the device (untimed)
    fp64 = None
    if rank == 0:
        cfg.fp64_reference = 1
        ctx.set_config(cfg)
        r64 = step()
        fp64 = {"err_inf_vs_fp64": r64["err_fp64_inf"], "fp64_reresid": r64["fp64_reresid"]}
        cfg.fp64_reference = 0
        ctx.set_config(cfg)

    # learned-preconditioner arm on the same device inputs: flexible PCG with
    # the trained network, MIC(0) fallback on stall
    learned = None
    model = args.model or DEFAULT_MODEL
    if rank == 0 and args.precond == "mic0" and args.learned_steps > 0 and os.path.exists(model):
        try:
            ctx.check(L.shkz_b200_learned_load(ctx.handle, model.encode()), "shkz_b200_learned_load")
            cfg.preconditioner = native.PRECOND_LEARNED
            ctx.set_config(cfg)
            step()  # warm-up (network block activity of this system)
            torch.cuda.synchronize(dev)
            la, lb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            lres = []
            la.record(stream)
            for _ in range(args.learned_steps):
                lres.append(step())
            lb.record(stream)
            torch.cuda.synchronize(dev)
            lms = la.elapsed_time(lb) / args.learned_steps
            ll = lres[-1]
            learned = {"ms_per_projection": lms, "iterations": ll["iterations"], "fallbacks": ll["fallbacks"],
                       "reresid_inf": ll["reresid"], "ms_solve": ll["ms_solve"], "status": ll["status"],
                       "model": os.path.relpath(model, ROOT), "steps": args.learned_steps,
                       "plain_ms_per_projection": value, "plain_iterations": last["iterations"],
                       "speedup_vs_plain": value / lms if lms else None}
            # the network application on the tensor cores: time and FLOP rate
            nms = ctypes.c_double()
            ncells = ctypes.c_longlong()
            if L.shkz_b200_time_kernel(ctx.handle, 8, 5, ctypes.byref(nms), ctypes.byref(ncells)) == 0:
                flops = L.shkz_b200_learned_flops(ctx.handle)
                tf = flops / (nms.value * 1e-3) / 1e12
                bf16_peak, bf16_kind = measured_bf16_peak()
                learned["network"] = {"ms_per_application": nms.value, "tflop_per_application": flops / 1e12,
                                      "achieved_tflops": tf, "peak_tflops": bf16_peak, "peak_kind": bf16_kind,
                                      "frac": tf / bf16_peak, "bound": "tensor",
                                      "kernel": "k_conv_tc (tcgen05 implicit-GEMM 3^3 convolutions, BF16)"}
        except native.ShkzError as exc:  # reported in the line, not hidden
            learned = {"error": str(exc), "model": os.path.relpath(model, ROOT)}
        cfg.preconditioner = native.PRECOND_MIC0
        ctx.set_config(cfg)

    # the projection's timestep neighbours on the same grid (untimed in the
    # headline): the FLIP splat before it and the velocity extension after it
    neighbours = None
    if rank == 0 and args.scene == "sloshing_tank" and args.neighbours:
        try:
            neighbours = time_neighbours(ctx, L, sc, stream, dev, vel, vact, solid, sact)
        except Exception as exc:  # reported in the line, not hidden
            neighbours = {"error": str(exc)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_reference_sample(128)
        except Exception as exc:  # reported, not hidden
            cpu = {"error": str(exc)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (f64 reductions, refinement and assembly)", "data": "synthetic",
            "config": {"workload": f"{args.scene} {nx}^3, {'plain MIC(0)' if args.precond == 'mic0' else args.precond}"
                                   f"-PCG projection to {sc.tol:g} (inf-norm), FP64 refinement, seed 0",
                       "preconditioner": args.precond,
                       "unknowns": last["unknowns"], "pool_tiles": last["tiles"],
                       "l2": "inputs (0.42 GB at 256^3) and pool arrays > 126 MB L2 (no flush needed)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "step": "device velocity restore + one projection"},
            "iterations": last["iterations"], "outer_steps": last["outer_steps"],
            "reresid_inf": last["reresid"], "reresid_l2": last["reresid_l2"],
            "phase_ms": {"assemble": last["ms_assemble"], "solve": last["ms_solve"], "update": last["ms_update"]},
            "ms_per_iteration": last["ms_solve"] / max(1, last["iterations"]),
            "e2e": e2e, "roofline": roofline, "roofline_kernels": rooflines, "roofline_iteration": iteration_roofline,
            "error_vs_fp64": fp64, "learned": learned, "neighbours": neighbours,
            "kernels": kern, "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
