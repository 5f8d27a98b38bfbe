#!/usr/bin/env python
"""Benchmark of the hot path on the batched 3-D configuration.

Workload (seeded synthetic, no dataset): 64 independent 3-D simulations,
grid side U{40..120} voxels at dx = 20 um, 2 substrates, 1k-100k cells each
(physicell-mac-metal_b200/workloads.py: batched_3d).  One bench step is one
mechanics period of the main loop (src/main.mm:341-391): 10 diffusion
sub-steps (x/y/z Thomas sweeps, Dirichlet reset, secretion) and one
mechanics step (binning, cell-start table, forces, AB2, then every cell's
voxel index recomputed from its new position and the secretion order
rebuilt), over all instances, one CUDA graph launch per period.

Reports (one JSON line on rank 0):
  value            aggregate voxel-steps/s of the batched path, inputs resident
  e2e              the same through the C ABI with host buffers: every step
                   uploads the 16 cell fields the host owns (radius,
                   volumes, strengths, phenotype: every field the steps do
                   not write) from pinned memory and reads back the density
                   arena and the 12 cell fields the steps write
  roofline         the Thomas sweeps: 8 B per voxel-substrate per sweep
                   launch / average launch time (CUDA events), vs measured HBM
  cpu_baseline     the multi-threaded FP32 CPU port on a bounded sample
  plain            the same instances advanced one at a time through the
                   single-simulation API (Microenvironment / CellMechanics)
  serving          config 4 on a bounded horizon: Poisson request arrivals
                   served by continuous batching; p50/p99 time-to-result
                   and aggregate voxel-steps/s, cell-steps/s
Multi-GPU: one process per GPU; 64 x N instances are split across the N
ranks by predicted bytes (greedy packing, computed identically on every
rank) and each rank runs its shard as one batch, with no collective on the
data path: weak scaling.
--impl reference times the CPU port alone (the reference's shaders exist
only for Apple Metal, which this machine does not have).
"""
import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "physicell-mac-metal_b200")
SUB_STEPS = 10          # diffusion sub-steps per mechanics period (0.1 / 0.01 min)


def load_pcg():
    spec = importlib.util.spec_from_file_location("pcg", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pcg"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_summary():
    """Per-launch DRAM bytes of the sweep kernels from the committed ncu
    summary (profiles/sweeps_traffic.json), scaled to this workload."""
    try:
        with open(os.path.join(ROOT, "profiles", "sweeps_traffic.json")) as f:
            return json.load(f)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi samples (50 ms) taken by a reader thread, each stamped on
    arrival; only the samples inside [begin(), end()] are summarised."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self.t0 = self.t1 = None

    def start(self):
        import threading
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        def reader():
            for line in self.proc.stdout:
                self.lines.append((time.monotonic(), line))
        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()
        deadline = time.monotonic() + 10.0   # wait until the sampler is producing
        while not self.lines and time.monotonic() < deadline and self.proc.poll() is None:
            time.sleep(0.02)

    def begin(self):
        self.t0 = time.monotonic()

    def end(self):
        self.t1 = time.monotonic()

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        t0 = self.t0 if self.t0 is not None else float("-inf")
        t1 = self.t1 if self.t1 is not None else float("inf")
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for t, line in list(self.lines):
            if not (t0 <= t <= t1):
                continue
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def setup_dist(gpus, backend="nccl"):
    """One process per GPU (torchrun): rank, world size, local rank and the
    process group (None when alone).  The group only carries the barrier and
    the max / sum of timings; no simulation data crosses GPUs."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as td
        if backend == "nccl":
            torch.cuda.set_device(local)
        td.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        dist = td
    return rank, world, local, dist


def _reduce(dist, local, x, op):
    if dist is None:
        return x
    import torch
    dev = f"cuda:{local}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def dist_max(dist, local, x):
    return _reduce(dist, local, x, dist.ReduceOp.MAX if dist is not None else None)


def dist_sum(dist, local, x):
    return _reduce(dist, local, x, dist.ReduceOp.SUM if dist is not None else None)


def rank_shard(n_per_gpu, rank, world, seed=1237):
    """Weak scaling: world * n_per_gpu batched 3-D instances, split across
    ranks by predicted bytes (physicell-mac-metal_b200/sharding.py); rank
    'rank' gets its shard's indices."""
    from pcg import sharding, workloads
    work = workloads.batched_3d_work(n_instances=n_per_gpu * world, seed=seed)
    return sharding.partition(work, world)[rank]


def barrier(dist):
    if dist is not None:
        dist.barrier()


def cpu_prepare(inst):
    """Oracle-side arrays for one instance (the CPU port's inputs)."""
    import pyoracle as po
    g = inst.grid
    og = po.make_grid(g.nx, g.ny, g.nz, g.n_substrates, dx=g.dx, dt=g.dt, x_min=g.x_min, y_min=g.y_min,
                      z_min=g.z_min)
    S = g.n_substrates
    osubs = po.make_subs([(s.diffusion_coefficient, s.decay_rate, bool(s.dirichlet_enabled), s.target_value)
                          for s in inst.substrates[:S]])
    m = inst.mech
    om = po.Mech(m.dt, m.cell_cell_repulsion, m.cell_cell_adhesion, m.max_interaction_distance,
                 m.mechanics_voxel_size, m.mech_grid_nx, m.mech_grid_ny, m.mech_grid_nz)
    dens = np.repeat(inst.initial_values, g.nx * g.ny * g.nz).astype(np.float32)
    n = inst.n_cells
    soa = inst.soa.copy()
    vox_idx = soa[26 * n:27 * n].view(np.uint32).copy()
    vol = soa[11 * n:12 * n].copy()
    return (og, osubs, om, dens, soa, n, vox_idx, vol, inst.rates, (g.x_min, g.y_min, g.z_min),
            g.nx * g.ny * g.nz, bool(inst.flags & 1))


def cpu_period(prepared):
    """One mechanics period of the CPU port over the prepared instances."""
    import pyoracle as po
    for og, osubs, om, dens, soa, n, vox_idx, vol, rates, origin, _, refresh in prepared:
        for _ in range(SUB_STEPS):
            po.port_sweeps(dens, og, osubs)
            po.port_dirichlet(dens, og, osubs)
            po.port_secretion(dens, og, vox_idx, vol, *rates, None, 0.01)
        po.port_mech_step(soa, n, n, om, origin, 0.1)
        if refresh:   # voxel indices from the new positions, as the device does
            po.voxel_refresh(soa, n, n, og)
            vox_idx[:] = soa[26 * n:27 * n].view(np.uint32)


def cpu_baseline(instances, budget_s):
    """The multi-threaded FP32 CPU port on a bounded sample: instances are
    added in order, each timed for one mechanics period, until budget_s of
    CPU work (at least one instance)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    cores = po.port_threads(os.cpu_count() or 1)
    prepared, secs = [], 0.0
    for inst in instances:
        p = cpu_prepare(inst)
        t0 = time.perf_counter()
        cpu_period([p])
        secs += time.perf_counter() - t0
        prepared.append(p)
        if secs >= budget_s:
            break
    vox = sum(p[10] for p in prepared)
    cells = sum(p[5] for p in prepared)
    return {"voxels": vox, "cells": cells, "seconds": secs, "cores": cores, "instances": len(prepared),
            "prepared": prepared}


def one_thread_baseline(prepared, cores):
    """The same port on one sample, one host thread against all of them:
    one mechanics period of one (the smallest sampled) instance each way;
    the all-thread count is restored afterwards."""
    import pyoracle as po
    vox, cells = prepared[10], prepared[5]
    out = {}
    for n_thr in (1, cores):
        po.port_threads(n_thr)
        try:
            t0 = time.perf_counter()
            cpu_period([prepared])
            secs = time.perf_counter() - t0
        finally:
            po.port_threads(cores)
        out[n_thr] = secs
    sample = f"one instance ({vox} voxels, {cells} cells), one mechanics period"
    return {"value": vox * SUB_STEPS / out[1], "unit": "voxel-steps/s", "cores": 1, "sample": sample,
            "cell_steps_per_s": cells / out[1],
            "all_threads_same_sample": {"value": vox * SUB_STEPS / out[cores], "cores": cores,
                                        "cell_steps_per_s": cells / out[cores]}}


def run_reference_arm(args, rank, world):
    """--impl reference: the CPU path only, rank 0 only."""
    if rank != 0:
        return
    load_pcg()
    from pcg import workloads
    insts = workloads.batched_3d(seed=1237)
    per_step = max(0.5, 150.0 / (args.steps + args.warmup))
    cb = cpu_baseline(insts, per_step)
    prepared = cb["prepared"]
    for _ in range(args.warmup):
        cpu_period(prepared)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu_period(prepared)
    dt = time.perf_counter() - t0
    value = cb["voxels"] * SUB_STEPS * args.steps / dt
    sample = (f"first {cb['instances']} of 64 batched_3d instances ({cb['voxels']} voxels, {cb['cells']} cells), "
              f"one mechanics period (10 diffusion sub-steps + 1 mechanics step) per step")
    line = {
        "impl": "reference", "metric": "voxel-steps/s", "value": value, "unit": "voxel-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)", "config": {"workload": "batched_3d (CPU sample)", "sample": sample},
        "cpu_baseline": {"value": value, "unit": "voxel-steps/s", "cores": cb["cores"], "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "voxel-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cell_steps_per_s": cb["cells"] * args.steps / dt,
    }
    print(json.dumps(line), flush=True)


def time_steps(ctx, fn, k):
    """CUDA events on the library's stream, synchronised on both sides; the
    closing event also follows the library's host copies (pcg_join)."""
    import torch
    st = torch.cuda.ExternalStream(ctx.stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ctx.sync()
    e0.record(st)
    for _ in range(k):
        fn()
    ctx.join()
    e1.record(st)
    ctx.sync()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1000.0


def plain_path(pcg, ctx, insts, periods):
    """Each instance alone through the single-simulation API."""
    objs = []
    for inst in insts:
        me = pcg.Microenvironment(ctx, inst.grid, inst.substrates)
        me.fill(inst.initial_values)
        c = pcg.Cells(ctx, max(inst.n_cells, 1), inst.grid.n_substrates)
        c.upload(inst.soa, inst.n_cells, inst.soa_max)
        c.set_secretion(*inst.rates)
        if inst.flags & pcg.INST_REFRESH_VOXELS:
            c.set_voxel_refresh(me)
        g = inst.grid
        m = pcg.CellMechanics(ctx, inst.mech, (g.x_min, g.y_min, g.z_min), max(inst.n_cells, 1))
        objs.append((me, c, m))

    def period():
        for me, c, m in objs:
            me.step(c, SUB_STEPS)
            m.update(c, 0.1)
    period()
    secs = time_steps(ctx, period, periods)
    for o in objs:
        for x in o:
            x.close()
    return secs


def serving_leg(pcg, ctx, horizon_s):
    """Config 4 on a bounded horizon: Poisson arrivals (20 req/s, seeded) of
    mixed 2-D / 3-D parameter-sweep requests submitted in real time to the
    continuous-batching server (150 GB budget); runs until every request is
    done.  Time-to-result = submit -> results on the host."""
    from pcg import workloads
    reqs = workloads.serving_requests(horizon_s=horizon_s)
    srv = pcg.Server(ctx, budget_bytes=150e9, steps_per_tick=100)
    ids = []
    i = 0
    t0 = time.perf_counter()
    peak_running = 0
    while True:
        now = time.perf_counter() - t0
        while i < len(reqs) and reqs[i][0] <= now:
            ids.append(srv.submit(reqs[i][1], reqs[i][2]))
            i += 1
        running, queued, _ = srv.tick()
        peak_running = max(peak_running, running)
        if running == 0 and queued == 0:
            if i == len(reqs):
                break
            time.sleep(max(0.0, min(0.01, reqs[i][0] - (time.perf_counter() - t0))))
    wall = time.perf_counter() - t0
    lat = np.array([srv.times(r)[0] for r in ids])
    vox, cells, _ = srv.totals()
    srv.close()
    return {"requests": len(ids), "horizon_s": horizon_s, "arrival_rate_per_s": 20.0, "wall_s": wall,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "voxel_steps_per_s": vox / wall, "cell_steps_per_s": cells / wall, "peak_running": peak_running,
            "budget_bytes": 150e9}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-refresh", action="store_true",
                    help="skip the leg with the reference's stale voxel indices (no refresh after mechanics)")
    ap.add_argument("--tune-cache", default=None, help="JSON file of autotuned launch shapes (read and updated)")
    ap.add_argument("--pin-x", type=int, default=0,
                    help="x-sweep launch shape warps*16 + stages instead of the tuned one")
    ap.add_argument("--pin-cols", type=int, default=0, help="the same for the y and z sweeps")
    ap.add_argument("--serve-horizon", type=float, default=10.0,
                    help="seconds of request arrivals for the serving leg (0 = skip)")
    args = ap.parse_args()
    if args.impl == "reference":
        # the CPU port on rank 0's host cores: no GPU, no process group (the
        # other ranks of a torchrun launch exit without work)
        run_reference_arm(args, int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")))
        return
    rank, world, local, dist = setup_dist(args.gpus)

    import torch
    pcg = load_pcg()
    from pcg import workloads
    torch.cuda.set_device(local)
    ctx = pcg.Context(local)
    shard = rank_shard(args.instances, rank, world)
    insts = workloads.batched_3d(n_instances=args.instances * world, seed=1237, only=shard)
    batch = pcg.Batch(ctx, insts, tune_cache=args.tune_cache, pin_x=args.pin_x, pin_cols=args.pin_cols)
    voxels, voxel_subs, cells = batch.totals()

    def period():
        batch.step(SUB_STEPS)

    for _ in range(args.warmup):
        period()
    barrier(dist)
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = ctx.launches
    clocks.begin()
    secs = time_steps(ctx, period, args.steps)
    clocks.end()
    launches = ctx.launches - launches0
    clk = clocks.stop()
    secs_max = dist_max(dist, local, secs)
    total_vox = dist_sum(dist, local, float(voxels))
    total_cells = dist_sum(dist, local, float(cells))
    total_vox_sub = dist_sum(dist, local, float(voxel_subs))
    value = total_vox * SUB_STEPS * args.steps / secs_max
    vox_sub_rate = total_vox_sub * SUB_STEPS * args.steps / secs_max
    cell_rate = total_cells * args.steps / secs_max

    # end to end through the C ABI with pinned host buffers
    n_soa = 28 * cells
    arena = batch.layout(0)[3]
    soa_h = pcg.PinnedArray((n_soa,))
    soa_out = pcg.PinnedArray((n_soa,))
    dens_out = pcg.PinnedArray((arena,))
    batch.download_all_cells(soa_h.array)
    ctx.sync()

    # the host owns the fields the steps do not write (radius, volumes,
    # strengths, phenotype) and sends them up every period; the device owns
    # the kinematic state; the density and the 12 fields the steps write come
    # back every period
    written = pcg.STEP_WRITTEN_FIELDS
    host_owned = pcg.HOST_OWNED_FIELDS

    def e2e_period():
        batch.upload_cell_fields(soa_h.array, host_owned)
        batch.step(SUB_STEPS)
        batch.download_cell_fields(soa_out.array, written)
        batch.download_all_density(dens_out.array)

    e2e_period()
    barrier(dist)
    t0 = time.perf_counter()
    e2e_secs = time_steps(ctx, e2e_period, args.steps)
    wall = time.perf_counter() - t0
    e2e_secs = dist_max(dist, local, max(e2e_secs, 0.0))
    e2e_value = total_vox * SUB_STEPS * args.steps / e2e_secs
    h2d = bin(host_owned).count("1") * cells * 4
    d2h = bin(written).count("1") * cells * 4 + arena * 4

    # roofline: phase events on the same kernels (profile mode launches directly)
    batch.set_profile(True)
    batch.phase_times(reset=True)
    batch.step(SUB_STEPS * 2)
    ctx.sync()
    ph, nst = batch.phase_times(reset=True)
    batch.set_profile(False)
    # dominant kernel: the plane kernel when every sweep launch of a sub-step
    # is a plane pass (x + y planes, x-z planes; 8 bytes per voxel-substrate
    # each covers), else all the sweep launches together
    plane_units, all_units = batch.sweep_units()
    launch_shapes = batch.describe()
    sweep_ms = (ph["x_sweep"] + ph["y_sweep"] + ph["z_sweep"]) / max(nst, 1)
    if plane_units and plane_units == all_units:
        kname = "k_sweep_planes (x+y plane pass and z plane pass)"
        kbytes = 8 * plane_units
        kms = sweep_ms
    else:
        kname = "Thomas sweeps (x/y/z)"
        kbytes = 8 * all_units
        kms = sweep_ms
    achieved = kbytes / (kms / 1000.0) / 1e9
    sweeps_gbs = 8 * all_units / (sweep_ms / 1000.0) / 1e9
    peak, peak_kind = measured_hbm()
    tr = traffic_summary()
    traffic = None
    if tr and tr.get("plane_bytes_per_voxel_substrate") and plane_units:
        traffic = tr["plane_bytes_per_voxel_substrate"] * plane_units

    # the same workload with the reference's stale voxel indices (never
    # refreshed within the run, so the secretion order is never rebuilt)
    refresh = None
    if not args.no_refresh:
        batch.close()
        rinsts = workloads.batched_3d(n_instances=args.instances * world, seed=1237, only=shard, flags=0)
        rb = pcg.Batch(ctx, rinsts, tune_cache=args.tune_cache)
        for _ in range(2):
            rb.step(SUB_STEPS)
        barrier(dist)
        rk = max(3, args.steps // 2)
        rsecs = dist_max(dist, local, time_steps(ctx, lambda: rb.step(SUB_STEPS), rk))
        refresh = {"value": total_vox * SUB_STEPS * rk / rsecs, "unit": "voxel-steps/s",
                   "cell_steps_per_s": total_cells * rk / rsecs, "ms_per_step": 1000 * rsecs / rk, "steps": rk}
        rb.close()
        batch = None

    plain_rate = None
    if not args.no_plain and rank == 0:
        psecs = plain_path(pcg, ctx, insts, 2)
        plain_rate = voxels * SUB_STEPS * 2 / psecs

    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        cb = cpu_baseline(insts, 15.0)
        cpu = {"value": cb["voxels"] * SUB_STEPS / cb["seconds"], "unit": "voxel-steps/s", "cores": cb["cores"],
               "kind": "port",
               "sample": f"first {cb['instances']} of {len(insts)} instances ({cb['voxels']} voxels, "
                         f"{cb['cells']} cells), one mechanics period each",
               "cell_steps_per_s": cb["cells"] / cb["seconds"],
               "one_thread": one_thread_baseline(min(cb["prepared"], key=lambda q: q[10]), cb["cores"])}

    serving = None
    if args.serve_horizon > 0 and rank == 0 and world == 1:
        serving = serving_leg(pcg, ctx, args.serve_horizon)

    if rank == 0:
        line = {
            "metric": "voxel-steps/s", "value": value, "unit": "voxel-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * secs_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": f"batched_3d: {args.instances} instances per GPU ({args.instances * world} in all, "
                                   f"sharded by predicted bytes), side U{{40..120}}, S=2, 1k-100k cells; "
                                   f"step = 10 diffusion sub-steps + 1 mechanics step, voxel indices "
                                   f"refreshed after it",
                       "voxels_per_gpu": voxels, "voxel_substrates_per_gpu": voxel_subs, "cells_per_gpu": cells,
                       "l2": f"inputs larger than L2 ({voxel_subs * 4 / 1e6:.0f} MB density per GPU)",
                       "launch_shapes": launch_shapes},
            "cell_steps_per_s": cell_rate, "voxel_substrate_steps_per_s": vox_sub_rate,
            "plain_voxel_steps_per_s": plain_rate,
            "batched_over_plain": (value / world / plain_rate) if plain_rate else None,
            "e2e": {"value": e2e_value, "unit": "voxel-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "wall_s": wall},
            "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "algorithmic_bytes_per_substep": kbytes, "ms_per_substep": kms,
                         "sweeps": {"achieved": sweeps_gbs, "frac": sweeps_gbs / peak,
                                    "algorithmic_bytes_per_substep": 8 * all_units, "ms_per_substep": sweep_ms},
                         "phase_ms_per_substep": {k: v / max(nst, 1) for k, v in ph.items()}},
            "reference_stale_voxels": refresh,
            "cpu_baseline": cpu,
            "serving": serving,
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    for a in (soa_h, soa_out, dens_out):
        a.free()
    if batch is not None:
        batch.close()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
