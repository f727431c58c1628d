"""thysea — Python host layer over libthysea.so, the B200 Tsunami-HySEA
time stepper.

The product is the C ABI in include/thysea.h; this module only marshals
numpy arrays into it (ctypes), the way a Python caller of the reference
would drive its shallowWater() through a small FFI stub.

    from thysea import synth, run
    p = synth.plain_small()
    out = run(p)                      # max_height, arrival, eta, ... (numpy)
"""
from __future__ import annotations

import ctypes
import time
from typing import Dict, Optional

import numpy as np

from . import _ffi, synth  # noqa: F401

THY_OK = 0
THY_ERR_GPU_MEMORY, THY_ERR_HOST, THY_ERR_INVALID, THY_ERR_CUDA, THY_ERR_NO_DEVICE = 1, 2, 3, 4, 5
THY_ERR_NONFINITE, THY_ERR_BUDGET, THY_ERR_CANCELLED, THY_ERR_TOO_LARGE, THY_ERR_TIMEOUT = 6, 7, 8, 9, 10


class ThyError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        msg = _ffi.lib().thy_strerror(code)
        super().__init__(f"{what} failed: {code} ({msg.decode() if msg else ''})")


def _check(code: int, what: str) -> None:
    if code != THY_OK:
        raise ThyError(code, what)


def _p(a, t):
    return ctypes.cast(None, t) if a is None else a.ctypes.data_as(t)


def device_count() -> int:
    return int(_ffi.lib().thy_device_count())


class Prepared:
    """A dimensionless problem (thy_problem) owned by the library."""

    def __init__(self, problem: "synth.Problem"):
        L = _ffi.lib()
        self.problem = problem
        self._keep = []
        raw = _ffi.Raw()
        raw.nx, raw.ny = problem.nx, problem.ny
        lon = np.ascontiguousarray(problem.lon, np.float64)
        lat = np.ascontiguousarray(problem.lat, np.float64)
        z = np.ascontiguousarray(problem.z, np.float32)
        self._keep += [lon, lat, z]
        raw.lon, raw.lat, raw.z = _p(lon, _ffi.f64p), _p(lat, _ffi.f64p), _p(z, _ffi.f32p)
        if problem.faults:
            f = np.ascontiguousarray(problem.fault_array(), np.float64)
            self._keep.append(f)
            raw.nfaults, raw.faults = len(problem.faults), _p(f, _ffi.f64p)
            raw.eta_file = _p(None, _ffi.f32p)
        else:
            e = np.ascontiguousarray(np.zeros_like(z) if problem.eta_init is None else problem.eta_init, np.float32)
            self._keep.append(e)
            raw.eta_file = _p(e, _ffi.f32p)
            raw.nfaults, raw.faults = 0, _p(None, _ffi.f64p)
        raw.crop_flag, raw.crop_value = int(problem.crop_flag), float(problem.crop_value)
        for i in range(4):
            raw.borders[i] = float(problem.borders[i])
        raw.sim_time, raw.save_time = float(problem.sim_time), float(problem.save_time)
        if problem.points is not None and len(problem.points) > 0:
            pts = np.ascontiguousarray(problem.points, np.float64)
            self._keep.append(pts)
            raw.npoints, raw.points, raw.series_time = len(pts), _p(pts, _ffi.f64p), float(problem.series_time)
        else:
            raw.npoints, raw.points, raw.series_time = 0, _p(None, _ffi.f64p), -1.0
        raw.cfl, raw.eps_h, raw.hpos, raw.stability = problem.cfl, problem.eps_h, problem.hpos, problem.stability
        raw.manning, raw.vmax, raw.L, raw.H, raw.dif_at = (problem.manning, problem.vmax, problem.L, problem.H,
                                                           problem.dif_at)
        self._raw = raw
        h = ctypes.c_void_p()
        _check(L.thy_prepare(ctypes.byref(raw), ctypes.byref(h)), "thy_prepare")
        self._h = h
        self.view = L.thy_problem_view(h)

    @property
    def c(self) -> "_ffi.ProblemC":
        return self.view.contents

    @property
    def npoints(self) -> int:
        return int(self.c.npoints)

    def pin(self):
        """Page-locks the problem's FP64 cell arrays (h, Hs, qx, qy) so that
        every thy_run uploads them at full link speed."""
        if getattr(self, "_pinned", None):
            return self
        L, c = _ffi.lib(), self.c
        n = int(c.nx) * int(c.ny)
        self._pinned = []
        for name in ("h", "Hs", "qx", "qy"):
            ptr = ctypes.cast(getattr(c, name), ctypes.c_void_p)
            if ptr.value:
                _check(L.thy_host_register(ptr, n * 8), "thy_host_register")
                self._pinned.append(ptr)
        return self

    def __del__(self):
        try:
            for ptr in getattr(self, "_pinned", None) or []:
                _ffi.lib().thy_host_unregister(ptr)
            if getattr(self, "_h", None):
                _ffi.lib().thy_problem_free(self._h)
        except Exception:
            pass


OUTPUT_FIELDS = ("max_height", "arrival", "deformed_bathy", "eta", "ux", "uy")


class PinnedOutputs:
    """Page-locked output fields for repeated runs of one grid (thysea.run's
    `out`): allocated and registered once, reused by every run."""

    def __init__(self, prep: Optional["Prepared"] = None, shape: Optional[tuple] = None):
        ny, nx = (int(prep.c.ny), int(prep.c.nx)) if prep is not None else (int(shape[0]), int(shape[1]))
        self.fields = {k: np.empty((ny, nx), np.float32) for k in OUTPUT_FIELDS}
        L = _ffi.lib()
        self._reg = []
        for v in self.fields.values():
            v.fill(0)   # touch the pages before locking them
            ptr = ctypes.c_void_p(v.ctypes.data)
            _check(L.thy_host_register(ptr, v.nbytes), "thy_host_register")
            self._reg.append(ptr)

    def release(self):
        for ptr in self._reg:
            _ffi.lib().thy_host_unregister(ptr)
        self._reg = []

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def run(problem, max_steps: int = -1, snapshots: bool = True, series: bool = True,
        out: Optional[Dict[str, np.ndarray]] = None) -> Dict:
    """Runs one scenario end to end on the GPU through thy_run().  `out`:
    caller-owned (ny, nx) float32 output fields to fill (e.g.
    PinnedOutputs.fields); new arrays otherwise."""
    L = _ffi.lib()
    prep = problem if isinstance(problem, Prepared) else Prepared(problem)
    pc = prep.c
    pc.max_steps = max_steps
    ny, nx = pc.ny, pc.nx
    if out is not None:
        fields = {k: out[k] for k in OUTPUT_FIELDS}
        for v in fields.values():
            if v.shape != (ny, nx) or v.dtype != np.float32 or not v.flags.c_contiguous:
                raise ValueError("output fields must be C-contiguous float32 arrays of shape (ny, nx)")
    else:
        fields = {k: np.empty((ny, nx), np.float32) for k in OUTPUT_FIELDS}
    npts = max(pc.npoints, 1)
    pts = {k: np.empty(npts, np.float32) for k in ("series_min", "series_max", "series_bathy")}
    snaps = {"time": [], "eta": [], "ux": [], "uy": []}
    ser = {"time": [], "eta": [], "ux": [], "uy": []}

    def on_snap(user, idx, t, e, u, v):
        n = nx * ny
        snaps["time"].append(t)
        snaps["eta"].append(np.ctypeslib.as_array(e, (n,)).reshape(ny, nx).copy())
        snaps["ux"].append(np.ctypeslib.as_array(u, (n,)).reshape(ny, nx).copy())
        snaps["uy"].append(np.ctypeslib.as_array(v, (n,)).reshape(ny, nx).copy())

    def on_ser(user, idx, t, e, u, v):
        n = pc.npoints
        ser["time"].append(t)
        ser["eta"].append(np.ctypeslib.as_array(e, (n,)).copy())
        ser["ux"].append(np.ctypeslib.as_array(u, (n,)).copy())
        ser["uy"].append(np.ctypeslib.as_array(v, (n,)).copy())

    o = _ffi.Outputs()
    for k, v in fields.items():
        setattr(o, k, _p(v, _ffi.f32p))
    for k, v in pts.items():
        setattr(o, k, _p(v, _ffi.f32p))
    cb_snap = _ffi.FieldFn(on_snap) if snapshots else _ffi.FieldFn()
    cb_ser = _ffi.FieldFn(on_ser) if series else _ffi.FieldFn()
    o.on_snapshot, o.on_series, o.user = cb_snap, cb_ser, None
    st = _ffi.Stats()
    _check(L.thy_run(prep.view, ctypes.byref(o), ctypes.byref(st)), "thy_run")
    res: Dict = dict(fields)
    res["snapshots"] = {k: (np.asarray(v) if v else np.empty((0,))) for k, v in snaps.items()}
    res["series"] = {k: (np.asarray(v) if v else np.empty((0,))) for k, v in ser.items()}
    res["series"].update(min=pts["series_min"][:pc.npoints], max=pts["series_max"][:pc.npoints],
                         bathy=pts["series_bathy"][:pc.npoints])
    res.update(iterations=st.steps, final_time=st.final_time_s, first_dt=st.first_dt_s,
               loop_seconds=st.loop_seconds, device_ms=st.device_loop_ms, kernel_launches=st.kernel_launches,
               nsnaps=st.snapshots, nseries=st.series_samples, tiles=st.tiles, deep_tiles=st.deep_tiles,
               dry_tiles=st.dry_tiles, setup_seconds=st.setup_seconds, output_seconds=st.output_seconds,
               total_seconds=st.total_seconds, tiling=(st.tiling.deep1, st.tiling.deep2, st.tiling.general),
               tune_samples=st.tune_samples, release_seconds=st.release_seconds, chunks=st.chunks,
               graph_captures=st.graph_captures, capture_seconds=st.capture_seconds,
               event_seconds=st.event_seconds, initial_seconds=st.initial_seconds)
    return res


# Warp tilings of the stepping kernels (thy_tiling): row groups per work unit
# of each variant index, per kernel.  Results never depend on the tiling.
TILING_GROUPS = {"deep1": (3, 2, 4), "deep2": (4, 2, 8), "general": (2, 1, 8)}


def force_tiling(tiling=None):
    """Run every later chunk with tiling (deep1, deep2, general) variant
    indices; None: autotune again (thy_tiling_force)."""
    if tiling is None:
        _check(_ffi.lib().thy_tiling_force(None), "thy_tiling_force")
        return
    t = _ffi.Tiling(*tiling)
    _check(_ffi.lib().thy_tiling_force(ctypes.byref(t)), "thy_tiling_force")


def tuned_tiling(deep_units: float, general_units: float):
    """(decided, (deep1, deep2, general)) of the autotuner for steps of
    deep_units deep and general_units general work units on the current
    device (thy_tiling_tuned)."""
    t = _ffi.Tiling()
    done = _ffi.lib().thy_tiling_tuned(float(deep_units), float(general_units), ctypes.byref(t))
    return bool(done), (t.deep1, t.deep2, t.general)


def clear_tuner():
    """Forget every tiling the autotuner decided in this process."""
    _ffi.lib().thy_tuner_clear()


class Session:
    """Step-level access (thy_session_*): the problem is set up on the device
    (faults at t=0 applied), then any number of time steps can be timed."""

    def __init__(self, problem):
        L = _ffi.lib()
        self.prep = problem if isinstance(problem, Prepared) else Prepared(problem)
        h = ctypes.c_void_p()
        _check(L.thy_session_open(self.prep.view, ctypes.byref(h)), "thy_session_open")
        self._h = h
        self.cells = self.prep.c.nx * self.prep.c.ny

    def steps(self, k: int):
        """Runs k steps; returns (device milliseconds, steps done)."""
        ms = ctypes.c_double()
        done = ctypes.c_longlong()
        _check(_ffi.lib().thy_session_steps(self._h, k, ctypes.byref(ms), ctypes.byref(done)), "thy_session_steps")
        return ms.value, done.value

    def time(self) -> float:
        return float(_ffi.lib().thy_session_time(self._h))

    def tune(self, max_steps: int = 1 << 30) -> int:
        """Steps (real steps of the run) until the autotuner has decided the
        tiling for this problem's work size; returns the steps taken."""
        k = ctypes.c_longlong()
        _check(_ffi.lib().thy_session_tune(self._h, max_steps, ctypes.byref(k)), "thy_session_tune")
        return k.value

    def inject(self, what: int):
        """Test hook (thy_session_inject): 1 = the deep-water kernels issue
        none of this session's staging copies, so their bounded waits run out
        and the next steps fail with THY_ERR_TIMEOUT; 0 = off."""
        _check(_ffi.lib().thy_session_inject(self._h, what), "thy_session_inject")

    def tuned(self):
        """(decided, (deep1, deep2, general)) for the session's current work"""
        t = _ffi.Tiling()
        done = _ffi.lib().thy_session_tuned(self._h, ctypes.byref(t))
        return bool(done == 1), (t.deep1, t.deep2, t.general)

    def tiling(self):
        """(deep1, deep2, general) variant indices of the last chunk"""
        t = _ffi.Tiling()
        _check(_ffi.lib().thy_session_tiling(self._h, ctypes.byref(t)), "thy_session_tiling")
        return t.deep1, t.deep2, t.general

    def profile(self, k: int):
        """k individually launched steps; returns the average (phase-1 ms, phase-2 ms)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(_ffi.lib().thy_session_profile(self._h, k, ctypes.byref(a), ctypes.byref(b)), "thy_session_profile")
        return a.value, b.value

    def profile_launches(self, k: int):
        """k individually launched steps; average ms of each launch of a step
        (deep phase 1, general phase 1, classification, deep phase 2, general
        phase 2, controller)."""
        t = (ctypes.c_double * 6)()
        _check(_ffi.lib().thy_session_profile_launches(self._h, k, t), "thy_session_profile_launches")
        return list(t)

    def launches(self) -> int:
        return int(_ffi.lib().thy_session_launches(self._h))

    def tiles(self):
        """(work units x steps so far, of which deep-water, of which skipped dry land)"""
        t, d, r = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        _check(_ffi.lib().thy_session_tiles(self._h, ctypes.byref(t), ctypes.byref(d), ctypes.byref(r)),
               "thy_session_tiles")
        return t.value, d.value, r.value

    def fetch(self):
        c = self.prep.c
        out = {k: np.empty((c.ny, c.nx), np.float32) for k in ("max_height", "eta", "ux", "uy")}
        _check(_ffi.lib().thy_session_fetch(self._h, *(_p(out[k], _ffi.f32p) for k in ("max_height", "eta", "ux", "uy"))),
               "thy_session_fetch")
        return out

    def close(self):
        if getattr(self, "_h", None):
            _ffi.lib().thy_session_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Multi-scenario runtime (thy_server_*): requests are admitted under an
    HBM budget and stepped together in one batch; results arrive through
    completion callbacks, collected in `results` (request id -> dict with
    status, stats and the output fields)."""

    def __init__(self, hbm_budget_bytes: int = 0, max_scenarios: int = 0, device: int = 0, chunk_cells: int = 0):
        L = _ffi.lib()
        o = _ffi.ServerOpts(int(hbm_budget_bytes), int(max_scenarios), int(device), int(chunk_cells))
        h = ctypes.c_void_p()
        _check(L.thy_server_open(ctypes.byref(o), ctypes.byref(h)), "thy_server_open")
        self._h = h
        self._live = {}
        self.results: Dict[int, Dict] = {}
        self._cb = _ffi.DoneFn(self._done)

    def _done(self, user, request, status, stats_ptr):
        keep = self._live.pop(int(request), None)
        res = {"status": int(status), "outputs": keep["fields"] if keep else None, "stats": None,
               "done_at": time.perf_counter()}
        if stats_ptr:
            st = ctypes.cast(stats_ptr, ctypes.POINTER(_ffi.Stats)).contents
            res["stats"] = {k: getattr(st, k) for k, _ in _ffi.Stats._fields_ if k != "tiling"}
            res["stats"]["tiling"] = (st.tiling.deep1, st.tiling.deep2, st.tiling.general)
        self.results[int(request)] = res

    def submit(self, problem, out: Optional[Dict[str, np.ndarray]] = None) -> int:
        """Queues a scenario (a synth.Problem or a Prepared); returns the request id."""
        prep = problem if isinstance(problem, Prepared) else Prepared(problem)
        ny, nx = int(prep.c.ny), int(prep.c.nx)
        fields = out if out is not None else {k: np.empty((ny, nx), np.float32) for k in OUTPUT_FIELDS}
        o = _ffi.Outputs()
        for k in OUTPUT_FIELDS:
            setattr(o, k, _p(fields[k], _ffi.f32p))
        rid = ctypes.c_longlong()
        _check(_ffi.lib().thy_server_submit(self._h, prep.view, ctypes.byref(o), self._cb, None, ctypes.byref(rid)),
               "thy_server_submit")
        self._live[rid.value] = {"prep": prep, "fields": fields, "outputs": o}
        return rid.value

    def cancel(self, request: int):
        _check(_ffi.lib().thy_server_cancel(self._h, int(request)), "thy_server_cancel")

    def progress(self) -> int:
        """One round (admit, events, one chunk of steps, retire); returns queued + running."""
        active = ctypes.c_int()
        _check(_ffi.lib().thy_server_progress(self._h, ctypes.byref(active)), "thy_server_progress")
        return active.value

    def drain(self):
        _check(_ffi.lib().thy_server_drain(self._h), "thy_server_drain")

    def stats(self) -> Dict:
        st = _ffi.ServerStats()
        _check(_ffi.lib().thy_server_get_stats(self._h, ctypes.byref(st)), "thy_server_get_stats")
        return {k: getattr(st, k) for k, _ in _ffi.ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            _ffi.lib().thy_server_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
