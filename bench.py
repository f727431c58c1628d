#!/usr/bin/env python
"""Benchmark of the B200 Tsunami-HySEA time stepper.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: one 4096 x 4096 scenario, Gaussian-random-field
bathymetry with a shelf and ~10 % dry cells, four contiguous Okada
subfaults, 3600 s simulated; seeded synthetic inputs (no dataset exists).

A "step" is one time step of the whole grid (16.8 M cell-updates: the five
stepping launches - deep-water and general kernels of each phase and the
step controller).  `value` = cell-updates/s over K steps with the state
resident in HBM, timed with CUDA events on the stepping stream (the 268 MB
state exceeds the 126 MB L2, so no flush is needed between steps).
`e2e` = the same metric through the public C ABI (thy_run) on host
buffers: upload of the dimensionless problem, Okada, the full 3600 s loop and
the download of the output fields, per full run.

--impl reference: the reference's own time stepper compiled for the host
(oracle/_ref, OpenMP on all host cores) on a bounded band of the same
workload (all 4096 columns x 256 rows around the source), same metric.
Under torchrun each rank runs an independent replica of the scenario
(weak scaling, no collective on the data path); only the reference arm's
rank 0 works.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tsunami-hysea_b200"))

METRIC = "cell-updates/s"
BYTES_PHASE1 = 36   # eta, dep, qx, qy read (16) + eta written (4) + max-height/arrival/initial eta read, max written (16)
BYTES_PHASE2 = 24   # eta, dep, qx, qy read (16) + qx, qy written (8)
UNIT_CELLS = 112 * 16   # cells of a work unit (half tile, kTileX x kHalfRows)


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


class Dist:
    """torch.distributed plumbing of the replicas: barrier, max and sum over
    ranks (NCCL on GPUs, gloo for CPU tests)."""

    def __init__(self, backend: str = "nccl"):
        self.world = env_int("WORLD_SIZE", 1)
        self.rank = env_int("RANK", 0)
        self.local = env_int("LOCAL_RANK", 0)
        self.pg = None
        self.device = "cuda" if backend == "nccl" else "cpu"
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "step_kernels_4096.md")
    try:
        for line in open(path):
            if line.startswith(f"traffic_bytes_per_launch {kernel}:"):
                return float(line.split(":")[1].split()[0])
    except OSError:
        pass
    return None


def band_problem(p, rows: int):
    """A band of `rows` rows around the source (all columns) of problem p."""
    import copy

    import numpy as np

    ny = p.ny
    lat_c = p.faults[0].lat if p.faults else float(p.lat[ny // 2])
    j0 = int(np.clip(np.searchsorted(p.lat, lat_c) - rows // 2, 0, ny - rows))
    q = copy.copy(p)
    q.lat = p.lat[j0:j0 + rows].copy()
    q.z = p.z[j0:j0 + rows].copy()
    q.name = f"{p.name}_band{rows}"
    return q


def cpu_reference_rate(p, warmup: int, steps: int, rows: int = 256):
    """The reference's own stepper (oracle/_ref) on a band of the workload,
    all host threads; returns (cell-updates/s, cores, sample text)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from thysea import synth

    q = band_problem(p, rows)
    d = tempfile.mkdtemp(prefix="thy_ref_")
    txt = synth.write_problem(q, d)
    cores = os.cpu_count() or 1
    s = oracle.RefemuSession(txt, threads=cores)
    if warmup:
        s.steps(warmup)
    sec = s.steps(steps)
    cells = s.cells
    s.close()
    return cells * steps / sec, cores, f"{q.nx}x{q.ny} band of the 4096x4096 workload, {steps} steps after {warmup}"


def run_ours(a, dist: Dist):
    import numpy as np

    import thysea
    from thysea import synth

    if thysea.device_count() == 0:
        raise SystemExit("bench: no CUDA device")
    thysea._ffi.lib().thy_set_device(dist.local)
    p = synth.single_large(n=a.n, sim_time=3600.0)
    prep = thysea.Prepared(p)
    cells = p.nx * p.ny
    sess = thysea.Session(prep)
    sess.steps(a.warmup)
    l0 = sess.launches()
    clk = ClockSampler(dist.local)
    clk.start()
    dist.barrier()
    t0 = time.perf_counter()
    dev_ms, done = sess.steps(a.steps)
    wall = time.perf_counter() - t0
    dist.barrier()
    clocks = clk.stop()
    launches = sess.launches() - l0
    if done != a.steps:
        raise SystemExit(f"bench: only {done} of {a.steps} steps (simulation time reached); lower --steps")
    dev_s = dist.max(dev_ms / 1e3)
    total_cells = dist.sum(float(cells * a.steps))
    value = total_cells / dev_s
    # per-kernel device time for the roofline (individually launched steps);
    # each kernel's algorithmic bytes count the cells it steps: deep units are
    # interior units of UNIT_CELLS cells, dry land units are skipped, the
    # general kernels step the rest
    t0_units, t0_deep, t0_dry = sess.tiles()
    prof_steps = 32
    ms6 = sess.profile_launches(prof_steps)
    t1_units, t1_deep, t1_dry = sess.tiles()
    sess.close()
    nunits = max(1, t1_units - t0_units)
    deep_frac = (t1_deep - t0_deep) / nunits
    dry_frac = (t1_dry - t0_dry) / nunits
    cells_deep = (t1_deep - t0_deep) / prof_steps * UNIT_CELLS
    cells_gen = max(0.0, cells - cells_deep - (t1_dry - t0_dry) / prof_steps * UNIT_CELLS)
    peak, peak_kind = measured_peak()
    kern = {"deep_phase1": (ms6[0], BYTES_PHASE1, cells_deep), "general_phase1": (ms6[1], BYTES_PHASE1, cells_gen),
            "deep_phase2": (ms6[3], BYTES_PHASE2, cells_deep), "general_phase2": (ms6[4], BYTES_PHASE2, cells_gen)}
    dom = max(kern, key=lambda k: kern[k][0])
    ms, bpc, kcells = kern[dom]
    achieved = bpc * kcells / (ms * 1e-3) / 1e9
    traffic = ncu_traffic(dom)
    step_ms = sum(ms6)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_kind,
                "algorithmic_bytes_per_cell": bpc, "cells_per_launch": int(kcells),
                "per_kernel_ms": {**{k: round(v[0], 5) for k, v in kern.items()}, "classify": round(ms6[2], 5),
                                  "controller": round(ms6[5], 5)},
                "deep_unit_fraction": round(deep_frac, 4), "dry_unit_fraction": round(dry_frac, 4),
                "units": int(nunits // prof_steps),
                "step_frac_of_peak": round((BYTES_PHASE1 + BYTES_PHASE2) * cells / (step_ms * 1e-3) / 1e9 / peak, 4)}
    # end to end through the public API on host buffers: full 3600 s runs,
    # inputs (the FP64 problem arrays) and outputs (six float fields) in
    # page-locked host memory that every run reuses
    e2e = None
    if not a.skip_e2e:
        prep.pin()
        outs = thysea.PinnedOutputs(prep)
        thysea.run(prep, snapshots=False, series=False, out=outs.fields)  # warm-up run
        times, steps_run, parts = [], 0, []
        for _ in range(a.e2e_runs):
            dist.barrier()
            t0 = time.perf_counter()
            out = thysea.run(prep, snapshots=False, series=False, out=outs.fields)
            times.append(time.perf_counter() - t0)
            steps_run = out["iterations"]
            parts.append((out["setup_seconds"], out["loop_seconds"], out["device_ms"] / 1e3, out["output_seconds"],
                          out["total_seconds"]))
        t = dist.max(statistics.mean(times))
        e2e = {"value": round(dist.sum(float(cells * steps_run)) / t, 1), "unit": METRIC,
               "h2d_bytes_per_step": int(32 * cells + 4 * (5 * p.ny + 1) + 80 * len(p.faults)),
               "d2h_bytes_per_step": int(6 * 4 * cells),
               "step": "one full 3600 s run through thy_run, pinned host inputs and outputs",
               "run_seconds": round(t, 4), "steps_per_run": int(steps_run),
               "setup_s": round(statistics.mean(x[0] for x in parts), 4),
               "loop_s": round(statistics.mean(x[1] for x in parts), 4),
               "loop_device_s": round(statistics.mean(x[2] for x in parts), 4),
               "output_s": round(statistics.mean(x[3] for x in parts), 4),
               "library_call_s": round(statistics.mean(x[4] for x in parts), 4)}
    cpu = None
    if dist.rank == 0 and dist.world == 1 and not a.skip_cpu:
        try:
            rate, cores, sample = cpu_reference_rate(p, 2, a.cpu_steps)
            cpu = {"value": round(rate, 1), "unit": METRIC, "cores": cores, "kind": "reference", "sample": sample}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": METRIC, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {e}"}
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": dist.world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": round(dev_s * 1e3 / a.steps, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": f"single_large {p.nx}x{p.ny} cells, 4 Okada subfaults, 3600 s simulated (BASELINE config 2)",
                   "cells": cells, "parallelism": f"replicas x{dist.world}" if dist.world > 1 else "single GPU",
                   "l2": "state 268 MB > 126 MB L2, no flush", "simulated_s_per_step": None},
        "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": int(launches),
        "wall_s_timed": round(wall, 4),
    }
    return line


def run_reference(a, dist: Dist):
    from thysea import synth

    if dist.rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    if not oracle.refemu_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/librefemu.so not built (reference tree absent at build)"}
    p = synth.single_large(n=a.n, sim_time=3600.0)
    q = band_problem(p, 256)
    d = tempfile.mkdtemp(prefix="thy_ref_")
    txt = synth.write_problem(q, d)
    cores = os.cpu_count() or 1
    s = oracle.RefemuSession(txt, threads=cores)
    s.steps(a.warmup)
    k = min(a.steps, a.ref_steps)
    sec = s.steps(k)
    cells = s.cells
    s.close()
    value = cells * k / sec
    sample = f"{q.nx}x{q.ny} band of the 4096x4096 workload, {k} steps after {a.warmup}"
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": dist.world,
        "steps": k, "warmup": a.warmup, "ms_per_step": round(sec * 1e3 / k, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": f"single_large {p.nx}x{p.ny} cells, 4 Okada subfaults, 3600 s simulated (BASELINE config 2)",
                   "sample": sample},
        "cpu_baseline": {"value": round(value, 1), "unit": METRIC, "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": round(value, 1), "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=960, help="timed time steps (multiple of 16)")
    ap.add_argument("--warmup", type=int, default=32)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=4096, help="grid side")
    ap.add_argument("--e2e-runs", type=int, default=2)
    ap.add_argument("--cpu-steps", type=int, default=60)
    ap.add_argument("--ref-steps", type=int, default=400)
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)
    dist = Dist()
    try:
        line = run_reference(a, dist) if a.impl == "reference" else run_ours(a, dist)
        if line is not None and dist.rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
