#!/usr/bin/env python
"""Benchmark of the FLIP step on the MSBG (metric: P2G+G2P Mparticles/s; Poisson time to a
relative residual, mixed vs FP32 V-cycle).

Workload (one process per GPU; the path does not shard, so N GPUs run N replicas):
  step     = one FLIP step of dam_drop_128 (128^3 effective, 3 levels, 4.14M particles) on
             library-owned particles already resident in HBM.
  value    = particles * steps / sum over steps of (P2G kernel + G2P kernel) device time.
  e2e      = the same metric through the drop-in C-ABI calls with host buffers: per step a pinned
             host->device copy of positions and velocities, aw_p2g (sort + P2G), backup, aw_g2p,
             and a device->host copy of the velocities; copies run on their own streams so that the
             next step's upload and this step's read-back overlap this step's kernels.
  poisson  = poisson_256 (256^3 effective, 4 levels) projection to 1e-6 and 1e-9 relative residual,
             FP32 V-cycle vs mixed precision.
  flip_256 = dam_drop2_256 (256^3 effective, 4 levels, 34.7M particles) FLIP steps/s with the mixed
             and the plain FP32 projection.
  --impl reference: the FP64 OpenMP CPU restatement (oracle) of the same P2G+G2P workload, timed on
             the host cores.

Inputs are larger than L2 (cfg particles 4.14M x 24 B = 99 MB SoA + grid); the timed steps also
re-sort and re-scatter the particle arrays, so consecutive steps do not reuse a warm L2 copy.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Poisson ms to 1e-6 rel. resid (mixed vs FP32 V-cycle); P2G+G2P Mparticles/s"
UNIT = "Mparticles/s"
WORKLOAD = "dam_drop_128"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index=0):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, pw, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
                pw.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        # "under load": samples drawing well above idle power (host-side scene set-up sits between the
        # timed regions)
        load = [c for c, w in zip(sm, pw) if w > 250.0] or sm
        return {"sm_mhz": float(np.median(load)) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm), "samples_under_load": len(load),
                "power_w_max": max(pw) if pw else None}


def dist_init(backend="nccl"):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v):
    """The largest of the ranks' values (device time of the slowest replica)."""
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------------------------------------
# CPU baseline: FP64 OpenMP oracle on the host cores
# --------------------------------------------------------------------------------------------
def old_field(u):
    """A u_old distinct from u_new for the timed FLIP blend (the GPU step blends two different
    fields too): the P2G field scaled by one half."""
    return [0.5 * x for x in u]


def cpu_p2g_g2p(S, budget_s=12.0, max_reps=6):
    from oracle import pyoracle as po
    lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, S.pos, S.thresholds)
    lv, _ = po.enforce_grading(S.dims, S.num_levels, lv)
    O = po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)
    _, perm = O.particle_keys(S.pos)
    pos, vel = S.pos[perm], S.vel[perm]
    times = []
    t0 = time.perf_counter()
    while len(times) < max_reps and (time.perf_counter() - t0 < budget_s or not times):
        t = time.perf_counter()
        u, m, _ = O.p2g(pos, vel)
        O.g2p(pos, u, old_field(u), S.alpha, vel)
        times.append(time.perf_counter() - t)
    return S.n / np.mean(times) / 1e6, po.num_threads(), len(times), times


# --------------------------------------------------------------------------------------------
def run_reference(args, ws, rank):
    from anitowave_adaptive_b200 import scenes
    if rank != 0:
        return
    S = scenes.config(WORKLOAD)
    from oracle import pyoracle as po
    po.set_threads(os.cpu_count() or 1)
    lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, S.pos, S.thresholds)
    lv, _ = po.enforce_grading(S.dims, S.num_levels, lv)
    O = po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)
    _, perm = O.particle_keys(S.pos)
    pos, vel = S.pos[perm], S.vel[perm]
    for _ in range(args.warmup):
        u, m, _ = O.p2g(pos, vel)
        O.g2p(pos, u, old_field(u), S.alpha, vel)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        u, m, _ = O.p2g(pos, vel)
        O.g2p(pos, u, old_field(u), S.alpha, vel)
    dt = time.perf_counter() - t0
    value = S.n * args.steps / dt / 1e6
    cores = po.num_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "particles": S.n, "grid": "128^3 effective, 8^3-cell blocks, 3 levels",
                   "l2": "inputs > L2 (99 MB particles + grid)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"full {WORKLOAD} P2G+G2P per step ({S.n} particles), FP64 OpenMP restatement; "
                                   "the reference has no CPU implementation"},
        "note": "measured on rank 0's host cores only (no GPU); other ranks exit without work",
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, ws, rank, local):
    import torch
    import anitowave_adaptive_b200 as aw
    from anitowave_adaptive_b200 import scenes

    torch.cuda.set_device(local)
    S = scenes.config(WORKLOAD)
    g = aw.build_grid(S)
    F = aw.Flip(g, S.pos, S.vel, S.dt, S.alpha, (0, S.gravity, 0), precision=aw.PRECISION_MIXED, tolerance=1e-6,
                max_cycles=100)
    for _ in range(args.warmup):
        F.step()
    torch.cuda.synchronize()
    barrier(ws)
    clk = Clocks(local) if rank == 0 else None
    l0 = aw.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record()
    ms_p2g = ms_g2p = 0.0
    stats = []
    for _ in range(args.steps):
        F.step()
        st = F.stats()
        stats.append(st)
        ms_p2g += st["ms_p2g"]
        ms_g2p += st["ms_g2p"]
    ev1.record()
    torch.cuda.synchronize()
    launches = aw.launch_count() - l0
    barrier(ws)
    ms_total = max_over_ranks(ws, ev0.elapsed_time(ev1))
    kern_ms = max_over_ranks(ws, ms_p2g + ms_g2p)
    value = ws * S.n * args.steps / (kern_ms / 1e3) / 1e6

    # roofline of the P2G kernel (algorithmic bytes: particles 24 B, faces u + m 8 B)
    tot = g.totals()
    faces = sum(tot[1:])
    p2g_bytes = S.n * 24 + faces * 8
    g2p_bytes = S.n * 36 + faces * 8
    hbm, peak_kind = peaks()
    # DRAM bytes per launch measured by one ncu capture of each kernel on this workload
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic_dam_drop_128.json")) as f:
            traffic = json.load(f)
    except Exception:
        traffic = {}
    p2g_ms = ms_p2g / args.steps
    g2p_ms = ms_g2p / args.steps
    p2g_gbs = p2g_bytes / (p2g_ms / 1e3) / 1e9
    g2p_gbs = g2p_bytes / (g2p_ms / 1e3) / 1e9

    resample = None if args.skip_resample else resample_bench(g, aw)

    # e2e through the drop-in C ABI with host buffers: every step uploads its positions and
    # velocities from pinned host memory, runs aw_p2g (sort + P2G), the backup and aw_g2p, and reads
    # the velocities back.  Two device buffer sets and two copy streams let step k+1's upload and
    # step k's read-back run while step k computes.
    pos_h = torch.from_numpy(S.pos).pin_memory()
    vel_h = torch.from_numpy(S.vel).pin_memory()
    vel_out = [torch.empty_like(vel_h).pin_memory() for _ in range(2)]
    pos_d = [torch.empty_like(pos_h, device="cuda") for _ in range(2)]
    vel_d = [torch.empty_like(vel_h, device="cuda") for _ in range(2)]
    comp = torch.cuda.current_stream()
    cin, cout = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_done = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]

    def upload(k):
        with torch.cuda.stream(cin):
            cin.wait_event(ev_out[k])  # the previous read-back of buffer set k has finished
            pos_d[k].copy_(pos_h, non_blocking=True)
            vel_d[k].copy_(vel_h, non_blocking=True)
            ev_in[k].record(cin)

    def run(nsteps):
        upload(0)
        for it in range(nsteps):
            k = it & 1
            comp.wait_event(ev_in[k])
            if it + 1 < nsteps:
                upload(k ^ 1)
            g.p2g(pos_d[k], vel_d[k])
            g.backup_grid_velocity()
            g.g2p(vel_d[k], pos_d[k], S.alpha)
            ev_done[k].record(comp)
            with torch.cuda.stream(cout):
                cout.wait_event(ev_done[k])
                vel_out[k].copy_(vel_d[k], non_blocking=True)
                ev_out[k].record(cout)
        comp.wait_event(ev_out[(nsteps - 1) & 1])
        comp.wait_event(ev_out[nsteps & 1])

    e2e_steps = max(3, args.steps)
    run(args.warmup)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(comp)
    cin.wait_event(e0)
    run(e2e_steps)
    e1.record(comp)
    torch.cuda.synchronize()
    assert torch.equal(vel_out[(e2e_steps - 1) & 1], vel_d[(e2e_steps - 1) & 1].cpu())
    e2e_ms = max_over_ranks(ws, e0.elapsed_time(e1))
    e2e_value = ws * S.n * e2e_steps / (e2e_ms / 1e3) / 1e6
    dropin = dropin_bench(g, S, pos_d[0], vel_d[0], pos_h, vel_h)

    poisson = None
    if not args.skip_poisson:
        poisson = poisson_bench(args)
    flip256 = None
    if not args.skip_flip256:
        flip256 = flip256_bench()
    two_phase = None
    if not args.skip_two_phase:
        two_phase = two_phase_bench()
    rebuild = None
    if not args.skip_rebuild:
        rebuild = rebuild_bench()
    # clocks sampled from the first timed FLIP step through the last timed region of this run
    clocks = clk.stop() if clk else None

    if rank != 0:
        return
    cpu = None
    if ws == 1 and not args.skip_cpu:
        v, cores, reps, times = cpu_p2g_g2p(S)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"P2G+G2P of the full {WORKLOAD} particle set ({S.n}), FP64 OpenMP restatement, "
                         f"{reps} repetitions ({sum(times):.1f} s)"}
    last = stats[-1]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_total / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded dam break + falling sphere)",
        "config": {"workload": WORKLOAD, "particles": S.n, "grid": "128^3 effective, 8^3-cell blocks, 3 levels",
                   "cells": tot[0], "faces": faces, "parallelism": f"replicas x{ws}",
                   "l2": "inputs larger than L2 (particles 99 MB + grid); particles re-sorted every step"},
        "roofline": {"kernel": "k_p2g_own (+ k_p2g_normalize)", "bound": "hbm", "achieved": p2g_gbs, "peak": hbm,
                     "unit": "GB/s", "frac": p2g_gbs / hbm, "peak_kind": peak_kind,
                     "traffic": traffic.get("k_p2g_own"), "bytes_per_launch": p2g_bytes, "ms_per_launch": p2g_ms,
                     "note": "HBM is the roofline; the kernel runs below it, limited by instruction issue and "
                             "particle-load latency in the per-cell register deposits (own and coarse tiles), "
                             "see profiles/k_p2g_own_dam_drop_128.md"},
        "roofline_g2p": {"kernel": "k_g2p_fused (+ k_g2p_inactive)", "bound": "hbm", "achieved": g2p_gbs, "peak": hbm,
                         "unit": "GB/s", "frac": g2p_gbs / hbm, "traffic": traffic.get("k_g2p_fused"),
                         "bytes_per_launch": g2p_bytes, "ms_per_launch": g2p_ms},
        "step_breakdown_ms": {k: last[k] for k in ("ms_sort", "ms_p2g", "ms_solve", "ms_g2p", "ms_advect", "ms_other")},
        "solver": {"cycles": last["cycles"], "residual": last["residual"], "div_before": last["div_before"],
                   "div_after": last["div_after"]},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": S.n * 24, "d2h_bytes_per_step": S.n * 12},
        "dropin_ms": dropin,
        "gpu_launches": int(launches),
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if poisson is not None:
        line["poisson"] = poisson
    if flip256 is not None:
        line["flip_256"] = flip256
    if two_phase is not None:
        line["two_phase_128"] = two_phase
    if rebuild is not None:
        line["rebuild_128"] = rebuild
    if resample is not None:
        line["resample_256"] = resample
    print(json.dumps(line), flush=True)


def dropin_bench(g, S, pos, vel, pos_h, vel_h, reps=5):
    """Device time of the drop-in calls alone on resident AoS arrays: aw_p2g (sort + P2G), then
    aw_g2p, and aw_advect after another aw_p2g (each reuses the sort of the aw_p2g before it)."""
    import torch
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    tot = {"p2g": 0.0, "g2p": 0.0, "advect": 0.0}
    for it in range(reps + 1):
        pos.copy_(pos_h)
        vel.copy_(vel_h)
        ev[0].record()
        g.p2g(pos, vel)
        ev[1].record()
        g.backup_grid_velocity()
        ev[2].record()
        g.g2p(vel, pos, S.alpha)
        ev[3].record()
        g.p2g(pos, vel)
        ev[4].record()
        g.advect(pos, S.dt)
        ev[5].record()
        torch.cuda.synchronize()
        if it:  # the first round warms up
            tot["p2g"] += ev[0].elapsed_time(ev[1])
            tot["g2p"] += ev[2].elapsed_time(ev[3])
            tot["advect"] += ev[4].elapsed_time(ev[5])
    return {k: v / reps for k, v in tot.items()}


def poisson_bench(args):
    """poisson_256: closed box, level map from 32 spheres, blob divergence.  Three forms: the plain
    FP32 V-cycle iteration, conjugate gradients preconditioned by the same V-cycle with every vector
    and scalar in FP32 (fp32_pcg), and the mixed form (the same CG with FP64 residual, direction and
    accumulation, FP16-stored coarse corrections).  fp32_pcg vs mixed isolates the precision."""
    import torch
    import anitowave_adaptive_b200 as aw
    from anitowave_adaptive_b200 import poisson as pz
    prob = pz.build_problem(256)
    out = {"workload": "poisson_256", "cells": int(prob.b.numel())}
    for name, prec in (("fp32", aw.PRECISION_FP32), ("fp32_pcg", aw.PRECISION_FP32_PCG),
                       ("mixed", aw.PRECISION_MIXED)):
        for tol in (1e-5, 1e-6, 1e-9):
            sv = aw.Solver(prob.grid, precision=prec, tolerance=tol, max_cycles=60)
            sv.setup(None)
            p = torch.zeros(prob.b.numel(), dtype=torch.float64 if prec == aw.PRECISION_MIXED else torch.float32,
                            device="cuda")
            sv.solve(prob.b, p, raise_on_error=False)  # warm
            times = []
            for _ in range(3):
                p.zero_()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                cyc, rel, st = sv.solve(prob.b, p, raise_on_error=False)
                torch.cuda.synchronize()
                times.append(1e3 * (time.perf_counter() - t0))
            div = prob.divergence_after(sv, p)
            div64 = prob.divergence_after(sv, p, fp64=True)
            out[f"{name}_{tol:.0e}"] = {"ms": min(times), "cycles": cyc, "rel_residual": rel,
                                        "converged": st == 0, "div_after": div, "div_after_fp64": div64}
            sv.close()
    for base in ("fp32", "fp32_pcg"):
        for tol in ("1e-05", "1e-06", "1e-09"):
            a, b = out.get(f"{base}_{tol}"), out.get(f"mixed_{tol}")
            if a and b and a["converged"] and b["converged"]:
                out[f"speedup_mixed_vs_{base}_{tol}"] = a["ms"] / b["ms"]
    return out


def poisson_solve_once():
    import torch
    import anitowave_adaptive_b200 as aw
    from anitowave_adaptive_b200 import poisson as pz
    prob = pz.build_problem(256)
    sv = aw.Solver(prob.grid, precision=aw.PRECISION_MIXED, tolerance=1e-6, max_cycles=60)
    sv.setup(None)
    p = torch.zeros(prob.b.numel(), dtype=torch.float64, device="cuda")
    sv.solve(prob.b, p, raise_on_error=False)
    p.zero_()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    cyc, rel, st = sv.solve(prob.b, p, raise_on_error=False)
    torch.cuda.synchronize()
    return {"workload": "poisson_256", "ms": 1e3 * (time.perf_counter() - t0), "cycles": cyc, "rel_residual": rel}


def flip256_bench(steps=5, warmup=2):
    """dam_drop2_256 (256^3 effective, 4 levels, 34.7M particles): FLIP steps/s, mixed vs plain FP32
    projection.  Plain FP32 stalls above 1e-6 relative residual at this size, so it runs to 1e-5."""
    import torch
    import anitowave_adaptive_b200 as aw
    from anitowave_adaptive_b200 import scenes
    S = scenes.config("dam_drop2_256")
    g = aw.build_grid(S)
    tot = g.totals()
    out = {"workload": "dam_drop2_256", "particles": S.n, "cells": tot[0], "faces": sum(tot[1:]), "steps": steps}
    for name, prec, tol in (("mixed", aw.PRECISION_MIXED, 1e-6), ("fp32_pcg", aw.PRECISION_FP32_PCG, 1e-5),
                            ("fp32", aw.PRECISION_FP32, 1e-5)):
        F = aw.Flip(g, S.pos, S.vel, S.dt, S.alpha, (0, S.gravity, 0), precision=prec, tolerance=tol, max_cycles=60)
        try:
            for _ in range(warmup):
                F.step()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            st = []
            for _ in range(steps):
                F.step()
                st.append(F.stats())
            e1.record()
            torch.cuda.synchronize()
        except aw.AWError as err:  # a form that does not reach its tolerance is reported as such
            torch.cuda.synchronize()
            out[name] = {"tolerance": tol, "converged": False, "error": str(err), "cycles": F.stats()["cycles"],
                         "residual": F.stats()["residual"]}
            F.close()
            continue
        ms = e0.elapsed_time(e1) / steps
        out[name] = {"tolerance": tol, "converged": True, "ms_per_step": ms, "steps_per_s": 1e3 / ms,
                     "cycles": [x["cycles"] for x in st], "residual": st[-1]["residual"],
                     "div_before": st[-1]["div_before"], "div_after": st[-1]["div_after"],
                     "ms_solve": float(np.mean([x["ms_solve"] for x in st])),
                     "ms_p2g": float(np.mean([x["ms_p2g"] for x in st])),
                     "ms_g2p": float(np.mean([x["ms_g2p"] for x in st]))}
        F.close()
    g.close()
    return out


def resample_bench(g, aw, dims=(256, 256, 256), reps=10, warmup=3):
    """Dense resampling for inspection on the workload's grid after its FLIP steps: PRESSURE (nearest
    cell) and the MAC velocity (trilinear) on a 256^3 lattice.  Bytes counted: the lattice written
    (4 or 12 B per point) plus the grid channel read once (cells 4 B; velocity faces 4 B each)."""
    import torch
    tot = g.totals()
    npts = dims[0] * dims[1] * dims[2]
    out = {"lattice": list(dims), "points": npts}
    for name, fn, wbytes, rbytes in (
            ("pressure", lambda: g.resample_cells(aw.PRESSURE, dims), 4, tot[0] * 4),
            ("velocity", lambda: g.resample_velocity(dims), 12, sum(tot[1:]) * 4)):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        gbs = (npts * wbytes + rbytes) / (ms / 1e3) / 1e9
        out[name] = {"ms": ms, "GBps": gbs, "frac_of_hbm": gbs / peaks()[0]}
    return out


def rebuild_bench(steps=20, warmup=3):
    """dam_drop_128 with the level map re-derived from the particles after every FLIP step
    (aw_flip_rebuild_levels): host wall time of the rebuild when the map is unchanged (map, grading
    and comparison on the device, one read-back) and when it changed (new layout; channels, tiles
    and solver hierarchy rebuilt in the storage they hold), and of the FLIP step that follows each."""
    import torch
    import anitowave_adaptive_b200 as aw
    from anitowave_adaptive_b200 import scenes
    S = scenes.config(WORKLOAD)
    g = aw.build_grid(S)
    F = aw.Flip(g, S.pos, S.vel, S.dt, S.alpha, (0, S.gravity, 0), precision=aw.PRECISION_MIXED, tolerance=1e-6,
                max_cycles=100)
    for _ in range(warmup):
        F.step()
    same, new, step_same, step_new = [], [], [], []
    changed = False
    for _ in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        F.step()
        torch.cuda.synchronize()
        (step_new if changed else step_same).append(1e3 * (time.perf_counter() - t0))
        t0 = time.perf_counter()
        changed = F.rebuild_levels(S.thresholds)
        dt = 1e3 * (time.perf_counter() - t0)
        (new if changed else same).append(dt)
    F.close()
    g.close()
    med = lambda v: float(np.median(v)) if v else None  # noqa: E731
    return {"workload": WORKLOAD, "steps": steps, "layout_changes": len(new),
            "ms_unchanged": med(same), "ms_changed": med(new),
            "ms_step_after_unchanged": med(step_same), "ms_step_after_changed": med(step_new)}


def two_phase_bench(steps=10, warmup=3, rho=(1.0, 3.0)):
    """dam_drop_128 with the falling sphere as a second, heavier liquid (rho 3 vs 1): FLIP steps with
    beta = 1/rho from the P2G phase field (coefficients rebuilt every step), beside the one-phase step
    on the same layout.  Mixed projection to 1e-6."""
    import torch
    import anitowave_adaptive_b200 as aw
    from anitowave_adaptive_b200 import scenes
    S = scenes.config(WORKLOAD)
    ph = scenes.phase_sphere(S.pos, (0.7, 0.8, 0.5), 0.12)
    out = {"workload": WORKLOAD, "particles": S.n, "heavy_particles": int(ph.sum()), "rho": list(rho),
           "steps": steps}
    for name in ("one_phase", "two_phase"):
        g = aw.build_grid(S)
        F = aw.Flip(g, S.pos, S.vel, S.dt, S.alpha, (0, S.gravity, 0), precision=aw.PRECISION_MIXED, tolerance=1e-6,
                    max_cycles=100)
        if name == "two_phase":
            F.set_phase(ph, *rho)
        for _ in range(warmup):
            F.step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = []
        for _ in range(steps):
            F.step()
            st.append(F.stats())
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[name] = {"ms_per_step": ms, "cycles": [x["cycles"] for x in st], "div_after": st[-1]["div_after"],
                     "ms_p2g": float(np.mean([x["ms_p2g"] for x in st])),
                     "ms_solve": float(np.mean([x["ms_solve"] for x in st]))}
        F.close()
        g.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-poisson", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-flip256", action="store_true", help="skip the dam_drop2_256 FLIP steps/s section")
    ap.add_argument("--skip-two-phase", action="store_true", help="skip the two-phase dam_drop_128 section")
    ap.add_argument("--skip-resample", action="store_true", help="skip the 256^3 resampling section")
    ap.add_argument("--skip-rebuild", action="store_true", help="skip the level-map rebuild section")
    ap.add_argument("--poisson-only", action="store_true",
                    help="only the poisson_256 projection comparison (for profiling the solver)")
    ap.add_argument("--poisson-solve-once", action="store_true",
                    help="one mixed-precision poisson_256 solve to 1e-6 after one warm-up solve (small ncu captures)")
    args = ap.parse_args()
    # the reference arm runs on the host cores only and takes no collective: a gloo group suffices
    ws, rank, local = dist_init("gloo" if args.impl == "reference" else "nccl")
    try:
        if args.poisson_only:
            import torch
            torch.cuda.set_device(local)
            print(json.dumps(poisson_bench(args)), flush=True)
        elif args.poisson_solve_once:
            import torch
            torch.cuda.set_device(local)
            print(json.dumps(poisson_solve_once()), flush=True)
        elif args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
