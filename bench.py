#!/usr/bin/env python
"""Benchmark of the B200 Tsunami-HySEA time stepper.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: one 4096 x 4096 scenario, Gaussian-random-field
bathymetry with a shelf and ~10 % dry cells, four contiguous Okada
subfaults, 3600 s simulated; seeded synthetic inputs (no dataset exists).

A "step" is one time step of the whole grid (16.8 M cell-updates: the six
stepping launches - deep-water and general kernels of each phase, the
work-unit classification and the step controller).  `value` = cell-updates/s over K steps with the state
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
    """SM clock and clock-event (throttle) reasons of this rank's GPU, read
    through NVML by a background thread every `period` seconds while the
    timed work runs (the library's calls release the GIL).  The NVML device
    is the one CUDA_VISIBLE_DEVICES maps this rank's device to."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, device: int, period: float = 0.0005):
        self.device = device
        self.period = period
        self.thread = None
        self.samples = []
        self.error = None

    def _handle(self, nv):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").strip()
        ids = [x.strip() for x in vis.split(",") if x.strip()] if vis else []
        if self.device < len(ids):
            x = ids[self.device]
            if x.isdigit():
                return nv.nvmlDeviceGetHandleByIndex(int(x))
            return nv.nvmlDeviceGetHandleByUUID(x)
        return nv.nvmlDeviceGetHandleByIndex(self.device)

    def start(self):
        import threading

        try:
            import pynvml as nv

            nv.nvmlInit()
            h = self._handle(nv)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        except Exception as e:  # noqa: BLE001
            self.error = f"NVML unavailable: {e}"
            return
        self.stop_flag = threading.Event()

        def loop():
            while not self.stop_flag.is_set():
                try:
                    self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                         int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))))
                except Exception as e:  # noqa: BLE001
                    self.error = str(e)
                    return
                self.stop_flag.wait(self.period)

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def stop(self) -> dict:
        if self.thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.error or "not sampled"], "samples": 0}
        self.stop_flag.set()
        self.thread.join(timeout=5)
        sm = [s for s, _ in self.samples]
        reasons = sorted({n for _, r in self.samples for n, bit in self.REASONS if r & bit})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(sm), "period_ms": self.period * 1e3, "source": "NVML"}


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
    # one full untimed run first: its chunks are the autotuner's samples for
    # every work mix the run passes through (keys of deep and general units
    # per step), so that the timed steps and the end-to-end runs below use
    # decided tilings (with THY_TILING or THY_TUNE=0 set the tuner is off)
    tuning_run = None
    if not os.environ.get("THY_TILING") and os.environ.get("THY_TUNE", "1") != "0":
        r = thysea.run(prep, snapshots=False, series=False)
        tuning_run = {"steps": int(r["iterations"]), "tune_samples": int(r["tune_samples"])}
    sess = thysea.Session(prep)
    tune_steps = sess.tune()
    sess.steps(a.warmup)
    tiling = sess.tiling()
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
    # general kernels step the rest (a dry unit counts as UNIT_CELLS cells;
    # boundary units can be narrower, so the general count is a lower bound)
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
        clk_e2e = ClockSampler(dist.local)
        clk_e2e.start()
        for _ in range(a.e2e_runs):
            dist.barrier()
            t0 = time.perf_counter()
            out = thysea.run(prep, snapshots=False, series=False, out=outs.fields)
            times.append(time.perf_counter() - t0)
            steps_run = out["iterations"]
            parts.append((out["setup_seconds"], out["loop_seconds"], out["device_ms"] / 1e3, out["output_seconds"],
                          out["total_seconds"], out["release_seconds"]))
        clocks_e2e = clk_e2e.stop()
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
               "library_call_s": round(statistics.mean(x[4] for x in parts), 4),
               "release_s": round(statistics.mean(x[5] for x in parts), 4), "clocks": clocks_e2e}
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
        "config": {"workload": f"single_large {p.nx}x{p.ny} cells, 4 Okada subfaults, 3600 s simulated",
                   "cells": cells, "parallelism": f"replicas x{dist.world}" if dist.world > 1 else "single GPU",
                   "l2": "state 268 MB > 126 MB L2, no flush", "simulated_s_per_step": None,
                   "tiling": {k: thysea.TILING_GROUPS[k][v] for k, v in zip(("deep1", "deep2", "general"), tiling)},
                   "tiling_note": "row groups per work unit at the start of the timed steps, picked by the autotuner",
                   "tuning_run": tuning_run, "tune_steps": int(tune_steps)},
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
        "config": {"workload": f"single_large {p.nx}x{p.ny} cells, 4 Okada subfaults, 3600 s simulated",
                   "sample": sample},
        "cpu_baseline": {"value": round(value, 1), "unit": METRIC, "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": round(value, 1), "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def _pct(xs, q):
    import numpy as np

    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else None


def _plain_service(preps, out_fields, keep=None):
    """One-at-a-time path: thy_run per scenario (an iterable of Prepared,
    made lazily by the caller if it likes), back to back; returns the service
    time of each (s), the cell updates and the step counts.  keep(k): whether
    to keep a copy of scenario k's max-height field (copied after its timing)
    for the comparison with the reference CUDA build."""
    import thysea

    times, cu, steps, kept = [], 0.0, [], {}
    for k, prep in enumerate(preps):
        out = out_fields(prep)   # (page-locked once per grid size, outside the timing)
        t0 = time.perf_counter()
        r = thysea.run(prep, snapshots=False, series=False, out=out)
        times.append(time.perf_counter() - t0)
        cu += float(prep.c.nx) * float(prep.c.ny) * float(r["iterations"])
        steps.append(int(r["iterations"]))
        if keep is not None and keep(k):
            kept[k] = out["max_height"].copy()
    return times, cu, steps, kept


REFGPU = os.path.join(ROOT, "oracle", "_ref", "TsunamiHySEA_refgpu")


def _rel_l2_wet(a, b):
    """relative L2 of max-height a against b over the cells wet in both (-9999: never wet)"""
    import numpy as np

    m = (a != -9999.0) & (b != -9999.0)
    ref = b[m].astype(np.float64)
    den = float(np.sqrt((ref ** 2).sum()))
    num = float(np.sqrt(((a[m].astype(np.float64) - ref) ** 2).sum()))
    return num / den if den > 0 else num


def _ref_cuda_service(probs, ours, sample=1, tol=1e-4):
    """The reference CUDA build one scenario per process, back to back: the
    reference's own path, whose main() runs one shallowWater() per run
    (src/ShallowWater.cxx:146-151).  Each problem's files are written before
    its clock starts; the service time is the process's wall time (CUDA
    start-up, file input, Okada, the loop, the NetCDF output).  Every
    `sample`-th scenario runs; each result's
    maximum height is compared with this library's result for the same
    scenario (ours[k]).  The reference writes its output file only when
    saving is on (src/GPU/ShallowWater.cu:313,456), so it runs with a saving
    interval of twice the simulated time: one snapshot at t = 0, then the
    maximum height and arrival times at the end.  Returns per sampled
    scenario: index, service time, the reference's own loop time,
    iterations, max-height relative L2."""
    import copy
    import shutil

    from scipy.io import netcdf_file

    from thysea import synth

    out = []
    for k, p in enumerate(probs):
        if k % sample:
            continue
        d = tempfile.mkdtemp(prefix="thy_refcuda_")
        try:
            q = copy.copy(p)
            q.save_time = 2.0 * p.sim_time
            txt = synth.write_problem(q, d)
            t0 = time.perf_counter()
            r = subprocess.run([REFGPU, txt], cwd=d, capture_output=True, text=True, timeout=1800)
            wall = time.perf_counter() - t0
            if r.returncode != 0:
                raise RuntimeError(f"reference CUDA build failed on {p.name}: {r.stdout[-500:]} {r.stderr[-500:]}")
            import re

            runtime = float(re.findall(r"Runtime: ([0-9.eE+-]+) sec", r.stdout)[-1])
            its = re.findall(r"Iteration\s+(\d+),", r.stdout)
            with netcdf_file(os.path.join(d, p.name + ".nc"), "r", mmap=False) as f:
                maxh = f.variables["max_height"][:].copy()
            err = _rel_l2_wet(ours[k], maxh) if k in ours else None
            out.append({"k": k, "service_s": wall, "runtime_s": runtime, "iterations": int(its[-1]) if its else None,
                        "max_height_rel_l2": err, "ok": (err is not None and err <= tol)})
        finally:
            shutil.rmtree(d, ignore_errors=True)
    return out


def _fifo(arrivals, service):
    """Time-to-result of a single FIFO server with the given arrivals and
    service times (the plain path serving the same stream)."""
    free, ttr, last = 0.0, [], 0.0
    for t_a, t_s in zip(arrivals, service):
        start = max(t_a, free)
        free = start + t_s
        ttr.append(free - t_a)
        last = free
    return ttr, last


def run_batched(a, dist):
    """The many-scenario workloads (batch: 64 scenarios of 2048^2 on one
    bathymetry; mixed: 32 scenarios of sides 256-4096; serving: a Poisson
    request stream) through the multi-scenario runtime (thy_server),
    next to the plain path (one thy_run per scenario) on the same inputs.

      batch:   64 scenarios on one shared 2048^2 bathymetry, one seeded
               Okada fault each, 1800 s, all submitted at once;
      mixed:   32 scenarios, sides log-uniform 256-4096, own bathymetry and
               fault, 600-7200 s, all submitted at once;
      serving: Poisson arrivals (--rate req/s for --duration s) of config-4
               requests under a 150 GB HBM budget; time-to-result = arrival
               -> outputs on the host.  Grid sides are drawn log-uniformly
               from 24 log-spaced sides (multiples of 64) so that one seeded
               bathymetry per side, generated before the clock starts, serves
               all its requests (each request keeps its own seeded fault and
               duration); background threads prepare each request ahead of
               its arrival, and the stepping loop never waits for them (the
               plain path's preparation is outside its timing as well).
    """
    import concurrent.futures as cf
    import math

    import numpy as np

    import thysea
    from thysea import synth

    thysea._ffi.lib().thy_set_device(dist.local)
    pinned_cache = {}

    def out_fields(prep):
        key = (int(prep.c.ny), int(prep.c.nx))
        if key not in pinned_cache:
            pinned_cache[key] = thysea.PinnedOutputs(shape=key)
        return pinned_cache[key].fields

    budget = int(a.budget_gb * 1e9)
    if a.workload in ("batch", "mixed"):
        probs = synth.batch_uniform(count=a.count or 64) if a.workload == "batch" else synth.mixed(count=a.count or 32)
        preps = [thysea.Prepared(p).pin() for p in probs]
        cells = [float(p.nx) * float(p.ny) for p in probs]
        for pr in preps:
            out_fields(pr)   # page-locked output buffers exist before either clock starts
        # batched: everything submitted at t = 0
        srv = thysea.Server(hbm_budget_bytes=budget)
        dist.barrier()
        t0 = time.perf_counter()
        ids = [srv.submit(pr, out=out_fields(pr)) for pr in preps]
        srv.drain()
        wall = time.perf_counter() - t0
        st = srv.stats()
        res = [srv.results[i] for i in ids]
        srv.close()
        ok = all(r["status"] == 0 for r in res)
        ttr = [r["done_at"] - t0 for r in res]
        cu = sum(c * r["stats"]["steps"] for c, r in zip(cells, res))
        # plain: one thy_run per scenario
        p_times, p_cu, p_steps, ours = _plain_service(preps, out_fields, keep=lambda k: a.ref_arm)
        p_wall = sum(p_times)
        p_ttr = list(np.cumsum(p_times))
        ref = None
        if a.ref_arm:
            if not os.path.exists(REFGPU):
                ref = {"unavailable": "oracle/_ref/TsunamiHySEA_refgpu not built (reference tree absent at build)"}
            else:
                rr = _ref_cuda_service(probs, ours, sample=1)
                r_wall = sum(x["service_s"] for x in rr)
                r_ttr = list(np.cumsum([x["service_s"] for x in rr]))
                errs = [x["max_height_rel_l2"] for x in rr if x["max_height_rel_l2"] is not None]
                ref = {"path": "reference CUDA build, one process per scenario, back to back (one snapshot at t = 0)",
                       "scenarios_per_hour": round(len(rr) / r_wall * 3600.0, 1), "wall_s": round(r_wall, 3),
                       "loop_s_total": round(sum(x["runtime_s"] for x in rr), 3),
                       "cell_updates_per_s": round(sum(c * (x["iterations"] or 0) for c, x in zip(cells, rr)) / r_wall, 1),
                       "time_to_result_p50_s": round(_pct(r_ttr, 50), 3),
                       "time_to_result_p99_s": round(_pct(r_ttr, 99), 3),
                       "max_height_rel_l2_max": max(errs) if errs else None,
                       "results_within_1e-4": sum(1 for x in rr if x["ok"]), "results": len(rr),
                       "iterations_equal": sum(1 for x, st in zip(rr, p_steps) if x["iterations"] == st)}
        del ours
        line = {
            "metric": "scenarios/hour", "value": round(len(probs) / wall * 3600.0, 1), "unit": "scenarios/h",
            "n_gpus": dist.world, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": a.workload, "scenarios": len(probs),
                       "cells_total": int(sum(cells)), "hbm_budget_gb": a.budget_gb},
            "all_ok": ok, "wall_s": round(wall, 3), "cell_updates_per_s": round(cu / wall, 1),
            "device_s": round(st["device_ms"] / 1e3, 3), "chunks": st["chunks"],
            "time_to_result_p50_s": round(_pct(ttr, 50), 3), "time_to_result_p99_s": round(_pct(ttr, 99), 3),
            "plain": {"scenarios_per_hour": round(len(probs) / p_wall * 3600.0, 1), "wall_s": round(p_wall, 3),
                      "cell_updates_per_s": round(p_cu / p_wall, 1),
                      "time_to_result_p50_s": round(_pct(p_ttr, 50), 3),
                      "time_to_result_p99_s": round(_pct(p_ttr, 99), 3)},
            "reference_cuda": ref,
        }
        if ref and "scenarios_per_hour" in ref:
            line["batched_over_reference_cuda"] = round(line["value"] / ref["scenarios_per_hour"], 2)
            line["batched_over_plain"] = round(line["value"] / line["plain"]["scenarios_per_hour"], 2)
        return line

    # ---- serving ----
    rng = np.random.default_rng(5)
    arrivals = synth.poisson_arrivals(rate=a.rate, duration=a.duration, seed=5)
    side_set = sorted({int(64 * round(v / 64)) for v in np.exp(np.linspace(math.log(256), math.log(4096), 24))})
    sides = [side_set[int(rng.integers(len(side_set)))] for _ in arrivals]
    seeds = rng.integers(1 << 30, size=len(arrivals))
    t_sim = rng.uniform(600.0, 7200.0, size=len(arrivals))
    bathy = {}

    def gen(n):
        r0 = np.random.default_rng(1000 + n)
        lon, lat = synth.lonlat_grid(n, n)
        return n, (lon, lat, synth.shelf_bathymetry(n, n, r0))

    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        bathy.update(dict(ex.map(gen, sorted(set(sides)))))
    for n in set(sides):
        pinned_cache[(n, n)] = thysea.PinnedOutputs(shape=(n, n))   # before the clock

    def make_problem(k):
        n = sides[k]
        lon, lat, z = bathy[n]
        rr = np.random.default_rng(int(seeds[k]))
        return synth.Problem(name=f"req{k:04d}", lon=lon, lat=lat, z=z, faults=[synth.random_fault(lon, lat, z, rr)],
                             sim_time=float(t_sim[k]))

    def make(k):
        # not page-locked: registering hundreds of MB from the preparing
        # threads would hold the driver while the stepping loop issues work
        return thysea.Prepared(make_problem(k))

    lead = 4.0   # seconds of look-ahead for the preparing threads
    pool = cf.ThreadPoolExecutor(max_workers=4)
    futs = {}
    srv = thysea.Server(hbm_budget_bytes=budget)
    t0 = time.perf_counter()
    nxt, submitted, rid_to_k = 0, 0, {}
    while True:
        now = time.perf_counter() - t0
        while nxt < len(arrivals) and arrivals[nxt] <= now + lead:
            futs[nxt] = pool.submit(make, nxt)
            nxt += 1
        while submitted < len(arrivals) and arrivals[submitted] <= now and futs[submitted].done():
            prep = futs.pop(submitted).result()
            rid_to_k[srv.submit(prep, out=out_fields(prep))] = submitted
            submitted += 1
        active = srv.progress()
        if submitted == len(arrivals) and active == 0:
            break
        if active == 0 and submitted < len(arrivals):
            time.sleep(max(0.0, min(0.005, arrivals[submitted] - (time.perf_counter() - t0))))
    wall = time.perf_counter() - t0
    st = srv.stats()
    res = {k: srv.results[r] for r, k in rid_to_k.items()}
    srv.close()
    pool.shutdown()
    ok = all(r["status"] == 0 for r in res.values())
    ttr = [res[k]["done_at"] - t0 - arrivals[k] for k in sorted(res)]
    by_side = {}
    for k in sorted(res):
        by_side.setdefault(sides[k], []).append(res[k]["done_at"] - t0 - arrivals[k])
    cu = sum(float(sides[k]) ** 2 * res[k]["stats"]["steps"] for k in res)
    # plain path: measured service times of the same requests, FIFO over the same arrivals
    ref_every = max(1, a.ref_sample)
    p_times, p_cu, p_steps, ours = _plain_service((make(k) for k in range(len(arrivals))), out_fields,
                                                  keep=lambda k: a.ref_arm and k % ref_every == 0)
    p_ttr, p_end = _fifo(list(arrivals), p_times)
    ref = None
    if a.ref_arm:
        if not os.path.exists(REFGPU):
            ref = {"unavailable": "oracle/_ref/TsunamiHySEA_refgpu not built (reference tree absent at build)"}
        else:
            # the reference CUDA build on every ref_every-th request (all of
            # them with --ref-sample 1); the others' service times are
            # modelled from those, as a + b x cell-updates (least squares; the
            # step counts are this library's, equal to the reference's where
            # both ran), and the stream is served FIFO over the same arrivals
            rr = _ref_cuda_service([make_problem(k) if k % ref_every == 0 else None for k in range(len(arrivals))],
                                   ours, sample=ref_every)
            cu_k = [float(sides[k]) ** 2 * p_steps[k] for k in range(len(arrivals))]
            xs = np.array([cu_k[x["k"]] for x in rr])
            ys = np.array([x["service_s"] for x in rr])
            A = np.stack([np.ones_like(xs), xs], axis=1)
            coef = np.linalg.lstsq(A, ys, rcond=None)[0] if len(rr) >= 2 else np.array([ys.mean(), 0.0])
            measured = {x["k"]: x["service_s"] for x in rr}
            r_times = [measured.get(k, float(coef[0] + coef[1] * cu_k[k])) for k in range(len(arrivals))]
            r_ttr, r_end = _fifo(list(arrivals), r_times)
            errs = [x["max_height_rel_l2"] for x in rr if x["max_height_rel_l2"] is not None]
            ref = {"path": "reference CUDA build, one process per request, FIFO (one snapshot at t = 0)",
                   "measured_requests": len(rr), "modelled_requests": len(arrivals) - len(rr),
                   "service_model_s": [round(float(coef[0]), 4), float(coef[1])],
                   "scenarios_per_hour": round(len(arrivals) / r_end * 3600.0, 1),
                   "time_to_result_p50_s": round(_pct(r_ttr, 50), 3),
                   "time_to_result_p99_s": round(_pct(r_ttr, 99), 3),
                   "service_s_total": round(sum(r_times), 3),
                   "max_height_rel_l2_max": max(errs) if errs else None,
                   "results_within_1e-4": sum(1 for x in rr if x["ok"]), "results": len(rr)}
    del ours
    line = {
        "metric": "scenarios/hour", "value": round(len(res) / wall * 3600.0, 1), "unit": "scenarios/h",
        "n_gpus": dist.world, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": "serving", "rate_per_s": a.rate, "duration_s": a.duration, "requests": len(arrivals),
                   "hbm_budget_gb": a.budget_gb, "sides": "log-uniform 256-4096 (multiples of 64)",
                   "sim_time_s": "uniform 600-7200"},
        "all_ok": ok, "wall_s": round(wall, 3), "cell_updates": cu, "cell_updates_per_s": round(cu / wall, 1),
        "device_busy_s": round(st["device_ms"] / 1e3, 3),
        "time_to_result_p50_s": round(_pct(ttr, 50), 3), "time_to_result_p99_s": round(_pct(ttr, 99), 3),
        "time_to_result_max_by_side_s": {str(n): round(max(v), 3) for n, v in sorted(by_side.items())},
        "plain": {"scenarios_per_hour": round(len(arrivals) / p_end * 3600.0, 1),
                  "time_to_result_p50_s": round(_pct(p_ttr, 50), 3),
                  "time_to_result_p99_s": round(_pct(p_ttr, 99), 3),
                  "service_s_total": round(sum(p_times), 3), "cell_updates_per_s": round(p_cu / sum(p_times), 1)},
        "reference_cuda": ref,
    }
    if ref and "scenarios_per_hour" in ref:
        line["batched_over_reference_cuda_p99"] = round(ref["time_to_result_p99_s"] / line["time_to_result_p99_s"], 2)
    return line


def run_tilings(a, dist):
    """Per-tiling device times of the single-scenario workload (side --n), at
    one stage of the run: the autotuner first decides from a fresh search
    (real steps), then every tiling that differs from the default in one
    kernel, and the tuner's pick, run one 16-step chunk each, round robin for
    --tiling-rounds rounds (so that all see the same work mix), with two
    individually launched steps each per round for the per-launch times.
    Not the headline line: it shows what the autotuner chooses between."""
    import thysea
    from thysea import synth

    if thysea.device_count() == 0:
        raise SystemExit("bench: no CUDA device")
    thysea._ffi.lib().thy_set_device(dist.local)
    p = synth.single_large(n=a.n, sim_time=3600.0)
    sess = thysea.Session(thysea.Prepared(p))
    sess.steps(a.warmup)
    thysea.force_tiling(None)
    thysea.clear_tuner()
    t0 = sess.time()
    tune_steps = sess.tune()
    decided, pick = sess.tuned()
    names = ("deep_phase1", "general_phase1", "classify", "deep_phase2", "general_phase2", "controller")
    tilings = [(0, 0, 0), (1, 0, 0), (2, 0, 0), (0, 1, 0), (0, 2, 0), (0, 0, 1), (0, 0, 2)]
    if tuple(pick) not in tilings:
        tilings.append(tuple(pick))
    chunk = {t: [] for t in tilings}
    launch = {t: [] for t in tilings}
    t1 = sess.time()
    try:
        for _ in range(a.tiling_rounds):
            for t in tilings:
                thysea.force_tiling(t)
                dms, k = sess.steps(16)
                chunk[t].append(dms / max(k, 1))
                launch[t].append(sess.profile_launches(2))
    finally:
        thysea.force_tiling(None)
    t2 = sess.time()
    sess.close()
    rows = []
    for t in tilings:
        groups = {n: thysea.TILING_GROUPS[n][v] for n, v in zip(("deep1", "deep2", "general"), t)}
        per = [statistics.mean(x[i] for x in launch[t]) for i in range(6)]
        rows.append({"tiling": t, "row_groups": groups, "ms_per_step_min": round(min(chunk[t]), 5),
                     "ms_per_step_median": round(statistics.median(chunk[t]), 5),
                     "launch_ms": {n: round(v, 5) for n, v in zip(names, per)}})
    return {"metric": "ms per step by warp tiling", "unit": "ms", "n_gpus": 1, "workload": "tilings",
            "config": {"workload": f"single_large {p.nx}x{p.ny}", "warmup": a.warmup, "rounds": a.tiling_rounds,
                       "simulated_s": [round(t0, 1), round(t1, 1), round(t2, 1)]},
            "tilings": rows, "autotuner": {"pick": list(pick), "decided": decided, "tune_steps": tune_steps}}


def run_launches(a, dist):
    """Per-launch device times of the single-scenario workload (side --n):
    --warmup steps in graphs, then --steps individually launched steps, each
    launch timed with CUDA events.  The command the ncu summaries under
    profiles/ capture (the launches of the individually launched steps come
    after a known number of graph launches).  Not the headline line."""
    import thysea
    from thysea import synth

    if thysea.device_count() == 0:
        raise SystemExit("bench: no CUDA device")
    thysea._ffi.lib().thy_set_device(dist.local)
    p = synth.single_large(n=a.n, sim_time=3600.0)
    sess = thysea.Session(thysea.Prepared(p))
    sess.steps(a.warmup)
    ms = sess.profile_launches(a.steps)
    total, deep, dry = sess.tiles()
    tiling = sess.tiling()
    sess.close()
    names = ("deep_phase1", "general_phase1", "classify", "deep_phase2", "general_phase2", "controller")
    return {"metric": "ms per launch", "unit": "ms", "n_gpus": 1, "workload": "launches",
            "config": {"workload": f"single_large {p.nx}x{p.ny}", "graph_steps": a.warmup, "launched_steps": a.steps,
                       "tiling": {n: thysea.TILING_GROUPS[n][v] for n, v in zip(("deep1", "deep2", "general"), tiling)}},
            "launch_ms": {n: round(v, 5) for n, v in zip(names, ms)},
            "units": {"stepped": total, "deep": deep, "dry": dry}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=960, help="timed time steps")
    ap.add_argument("--warmup", type=int, default=32)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=4096, help="grid side")
    ap.add_argument("--e2e-runs", type=int, default=2)
    ap.add_argument("--cpu-steps", type=int, default=60)
    ap.add_argument("--ref-steps", type=int, default=400)
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--workload", choices=["single", "batch", "mixed", "serving", "tilings", "launches"],
                    default="single",
                    help="single: one 4096^2 scenario (the headline line); batch: 64 x 2048^2 on one "
                         "bathymetry; mixed: 32 scenarios of sides 256-4096; serving: Poisson requests; "
                         "tilings: device time of each warp tiling (side --n); launches: per-launch times of "
                         "--steps individually launched steps after --warmup steps in graphs (side --n)")
    ap.add_argument("--count", type=int, default=0, help="batch / mixed: number of scenarios (0: 64 / 32)")
    ap.add_argument("--rate", type=float, default=2.0, help="serving: requests per second")
    ap.add_argument("--duration", type=float, default=60.0, help="serving: seconds of arrivals")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="batch / mixed / serving: HBM budget")
    ap.add_argument("--tiling-rounds", type=int, default=4, help="tilings: round-robin rounds")
    ap.add_argument("--ref-arm", type=int, default=1,
                    help="batch / mixed / serving: also run the reference CUDA build one scenario per process (1) or not (0)")
    ap.add_argument("--ref-sample", type=int, default=10,
                    help="serving: the reference CUDA build runs every n-th request (1: all), the rest modelled")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)
    dist = Dist()
    try:
        if a.impl == "reference":
            line = run_reference(a, dist)
        elif a.workload == "tilings":
            line = run_tilings(a, dist) if dist.rank == 0 else None
        elif a.workload == "launches":
            line = run_launches(a, dist) if dist.rank == 0 else None
        elif a.workload != "single":
            line = run_batched(a, dist)
        else:
            line = run_ours(a, dist)
        if line is not None and dist.rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
