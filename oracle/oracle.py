"""ctypes bindings of the two CPU oracles.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs, never by the product.

* :func:`run_oracle`  — oracle/build/libthy_oracle.so, the FP64 restatement
  of the time stepper (thy_oracle.c), fed with in-memory inputs.
* :func:`run_refemu`  — oracle/_ref/librefemu.so, the reference's own
  kernels, loader and NetCDF writers compiled for the host; it reads the
  problem files from disk exactly as the reference's main() does.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "build", "libthy_oracle.so")
REFEMU_SO = os.path.join(HERE, "_ref", "librefemu.so")

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)


class _Problem(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("lon", _f64p), ("lat", _f64p), ("z", _f32p), ("eta_file", _f32p),
        ("nfaults", ctypes.c_int), ("faults", _f64p),
        ("crop_flag", ctypes.c_int), ("crop_value", ctypes.c_double),
        ("borders", ctypes.c_double * 4),
        ("sim_time", ctypes.c_double), ("save_time", ctypes.c_double), ("series_time", ctypes.c_double),
        ("npoints", ctypes.c_int), ("points", _f64p),
        ("cfl", ctypes.c_double), ("eps_h", ctypes.c_double), ("hpos", ctypes.c_double),
        ("stability", ctypes.c_double), ("manning", ctypes.c_double), ("vmax", ctypes.c_double),
        ("L", ctypes.c_double), ("H", ctypes.c_double), ("dif_at", ctypes.c_double),
        ("max_iterations", ctypes.c_longlong), ("threads", ctypes.c_int),
    ]


class _Result(ctypes.Structure):
    _fields_ = [
        ("max_height", _f32p), ("arrival", _f32p), ("deformed_bathy", _f32p),
        ("eta", _f32p), ("ux", _f32p), ("uy", _f32p),
        ("max_snaps", ctypes.c_int), ("snap_eta", _f32p), ("snap_ux", _f32p), ("snap_uy", _f32p),
        ("snap_time", _f64p), ("nsnaps", ctypes.c_int),
        ("max_series", ctypes.c_int), ("ts_eta", _f32p), ("ts_ux", _f32p), ("ts_uy", _f32p),
        ("ts_time", _f64p), ("ts_min", _f32p), ("ts_max", _f32p), ("ts_bathy", _f32p),
        ("nseries", ctypes.c_int), ("npoints_unique", ctypes.c_int),
        ("iterations", ctypes.c_longlong), ("final_time", ctypes.c_double),
        ("first_dt", ctypes.c_double), ("loop_seconds", ctypes.c_double),
    ]


_lib = None
_ref = None


def oracle_lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"oracle library missing: {ORACLE_SO} (run `make -C oracle`)")
        _lib = ctypes.CDLL(ORACLE_SO)
        _lib.thy_oracle_run.argtypes = [ctypes.POINTER(_Problem), ctypes.POINTER(_Result)]
        _lib.thy_oracle_run.restype = ctypes.c_int
        _lib.thy_oracle_okada_points.argtypes = [ctypes.c_int, _f64p, _f64p, _f64p, _f64p]
        _lib.thy_oracle_slab_open.argtypes = [ctypes.POINTER(_Problem), ctypes.c_int, ctypes.c_int]
        _lib.thy_oracle_slab_open.restype = ctypes.c_void_p
        _lib.thy_oracle_slab_initial_dt.argtypes = [ctypes.c_void_p]
        _lib.thy_oracle_slab_initial_dt.restype = ctypes.c_double
        _lib.thy_oracle_slab_apply_fault.argtypes = [ctypes.c_void_p, ctypes.c_int]
        _lib.thy_oracle_slab_phase1.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        _lib.thy_oracle_slab_phase2.argtypes = [ctypes.c_void_p, ctypes.c_double]
        _lib.thy_oracle_slab_phase2.restype = ctypes.c_double
        _lib.thy_oracle_slab_field.argtypes = [ctypes.c_void_p, ctypes.c_int]
        _lib.thy_oracle_slab_field.restype = _f64p
        _lib.thy_oracle_slab_scales.argtypes = [ctypes.c_void_p, _f64p]
        _lib.thy_oracle_slab_close.argtypes = [ctypes.c_void_p]
    return _lib


def refemu_available() -> bool:
    return os.path.exists(REFEMU_SO)


def refemu_lib():
    global _ref
    if _ref is None:
        if not refemu_available():
            raise RuntimeError(f"ref-emu library missing: {REFEMU_SO} (run `make -C oracle ref`)")
        _ref = ctypes.CDLL(REFEMU_SO)
        _ref.refemu_run.argtypes = [ctypes.c_char_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, _f64p]
        _ref.refemu_run.restype = ctypes.c_int
        _ref.refemu_okada_points.argtypes = [ctypes.c_int, _f64p, _f64p, _f64p, _f64p]
        _ref.refemu_open.argtypes = [ctypes.c_char_p, ctypes.c_int]
        _ref.refemu_open.restype = ctypes.c_void_p
        _ref.refemu_steps.argtypes = [ctypes.c_void_p, ctypes.c_longlong]
        _ref.refemu_steps.restype = ctypes.c_double
        _ref.refemu_cells.argtypes = [ctypes.c_void_p]
        _ref.refemu_cells.restype = ctypes.c_longlong
        _ref.refemu_close.argtypes = [ctypes.c_void_p]
    return _ref


class RefemuSession:
    """The reference's own loop body on the host, step by step (for timing)."""

    def __init__(self, txt_path: str, threads: int = 0):
        self.lib = refemu_lib()
        self.h = self.lib.refemu_open(txt_path.encode(), threads)
        if not self.h:
            raise RuntimeError(f"refemu_open failed for {txt_path}")
        self.cells = int(self.lib.refemu_cells(self.h))

    def steps(self, k: int) -> float:
        s = float(self.lib.refemu_steps(self.h, k))
        if s < 0:
            raise RuntimeError("refemu_steps failed")
        return s

    def close(self):
        if self.h:
            self.lib.refemu_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ptr(a: Optional[np.ndarray], ctype):
    if a is None:
        return ctypes.cast(None, ctype)
    return a.ctypes.data_as(ctype)


def _problem_struct(p, max_iterations: int = -1, threads: int = 0):
    """The oracle's problem struct for a thysea.synth.Problem, and the arrays
    it points to (keep them alive while it is used)."""
    nx, ny = p.nx, p.ny
    lon = np.ascontiguousarray(p.lon, dtype=np.float64)
    lat = np.ascontiguousarray(p.lat, dtype=np.float64)
    z = np.ascontiguousarray(p.z, dtype=np.float32)
    eta_file = None if p.faults else np.ascontiguousarray(
        np.zeros_like(z) if p.eta_init is None else p.eta_init, dtype=np.float32)
    faults = np.ascontiguousarray(p.fault_array(), dtype=np.float64) if p.faults else None
    pts = None if p.points is None else np.ascontiguousarray(p.points, dtype=np.float64)
    pr = _Problem()
    pr.nx, pr.ny = nx, ny
    pr.lon, pr.lat, pr.z = _ptr(lon, _f64p), _ptr(lat, _f64p), _ptr(z, _f32p)
    pr.eta_file = _ptr(eta_file, _f32p)
    pr.nfaults = len(p.faults)
    pr.faults = _ptr(faults, _f64p)
    pr.crop_flag, pr.crop_value = int(p.crop_flag), float(p.crop_value)
    for i in range(4):
        pr.borders[i] = float(p.borders[i])
    pr.sim_time, pr.save_time = float(p.sim_time), float(p.save_time)
    pr.series_time = float(p.series_time) if pts is not None else -1.0
    pr.npoints = 0 if pts is None else len(pts)
    pr.points = _ptr(pts, _f64p)
    pr.cfl, pr.eps_h, pr.hpos, pr.stability = p.cfl, p.eps_h, p.hpos, p.stability
    pr.manning, pr.vmax, pr.L, pr.H, pr.dif_at = p.manning, p.vmax, p.L, p.H, p.dif_at
    pr.max_iterations = max_iterations
    pr.threads = threads
    return pr, [lon, lat, z, eta_file, faults, pts]


class OracleSlab:
    """The oracle stepping only rows [row_lo, row_hi) of its copy of the grid
    (thy_oracle_slab_*): the building block of the row-slab decomposition
    test.  The caller exchanges the two halo rows above and below after each
    phase and takes the minimum next dt over all slabs."""

    FIELDS = ("h", "qx", "qy", "eta_max", "t_arr", "dep")

    def __init__(self, p, row_lo: int, row_hi: int, threads: int = 1):
        lib = oracle_lib()
        self.p = p
        self.pr, self._keep = _problem_struct(p, threads=threads)
        self.h = lib.thy_oracle_slab_open(ctypes.byref(self.pr), row_lo, row_hi)
        if not self.h:
            raise RuntimeError("thy_oracle_slab_open failed")
        self.row_lo, self.row_hi = row_lo, row_hi
        sc = (ctypes.c_double * 3)()
        lib.thy_oracle_slab_scales(self.h, sc)
        self.Ts, self.Hs, self.Hmin = sc[0], sc[1], sc[2]

    def field(self, name: str) -> np.ndarray:
        """the whole-grid array (ny, nx), a view of the oracle's memory"""
        ptr = oracle_lib().thy_oracle_slab_field(self.h, self.FIELDS.index(name))
        return np.ctypeslib.as_array(ptr, (self.p.ny, self.p.nx))

    def initial_dt(self) -> float:
        return float(oracle_lib().thy_oracle_slab_initial_dt(self.h))

    def apply_fault(self, k: int):
        oracle_lib().thy_oracle_slab_apply_fault(self.h, k)

    def phase1(self, t: float, dt: float):
        oracle_lib().thy_oracle_slab_phase1(self.h, t, dt)

    def phase2(self, dt: float) -> float:
        return float(oracle_lib().thy_oracle_slab_phase2(self.h, dt))

    def close(self):
        if self.h:
            oracle_lib().thy_oracle_slab_close(self.h)
            self.h = None


def slab_rows(ny: int, rank: int, world: int):
    """rows [lo, hi) of rank `rank` in an even row-slab split of ny rows"""
    return ny * rank // world, ny * (rank + 1) // world


def run_slabs(p, rank: int, world: int, steps: int, exchange, allreduce_min, threads: int = 1):
    """Steps problem p for `steps` steps as rank `rank` of `world` row slabs.
    exchange(name, arr, lo, hi): makes rows lo-2, lo-1 and hi, hi+1 of the
    whole-grid array `arr` (those that exist) the neighbouring ranks' values;
    allreduce_min(v): the minimum over ranks.  Faults are applied at their
    times as the single-process loop does (all of them at t = 0 here: no dt
    truncation to later fault times).  Returns the slab object."""
    lo, hi = slab_rows(p.ny, rank, world)
    s = OracleSlab(p, lo, hi, threads=threads)
    tf = [f.time for f in p.faults]
    if any(t > 0.0 for t in tf):
        raise ValueError("run_slabs: faults at t = 0 only")
    dt = allreduce_min(s.initial_dt())
    t = 0.0
    fidx = 0
    for _ in range(steps):
        while fidx < len(tf) and t * s.Ts >= tf[fidx]:
            s.apply_fault(fidx)
            fidx += 1
        s.phase1(t, dt)
        exchange("h", s.field("h"), lo, hi)
        local = s.phase2(dt)
        exchange("qx", s.field("qx"), lo, hi)
        exchange("qy", s.field("qy"), lo, hi)
        nxt = allreduce_min(local)
        t += dt
        dt = nxt
    s.t = t
    return s


def run_oracle(p, max_iterations: int = -1, threads: int = 0, max_snaps: int = 0, max_series: int = 0) -> Dict:
    """Runs the FP64 oracle on a thysea.synth.Problem; returns numpy fields."""
    lib = oracle_lib()
    nx, ny = p.nx, p.ny
    lon = np.ascontiguousarray(p.lon, dtype=np.float64)
    lat = np.ascontiguousarray(p.lat, dtype=np.float64)
    z = np.ascontiguousarray(p.z, dtype=np.float32)
    eta_file = None if p.faults else np.ascontiguousarray(
        np.zeros_like(z) if p.eta_init is None else p.eta_init, dtype=np.float32)
    faults = np.ascontiguousarray(p.fault_array(), dtype=np.float64) if p.faults else None
    pts = None if p.points is None else np.ascontiguousarray(p.points, dtype=np.float64)
    pr = _Problem()
    pr.nx, pr.ny = nx, ny
    pr.lon, pr.lat, pr.z = _ptr(lon, _f64p), _ptr(lat, _f64p), _ptr(z, _f32p)
    pr.eta_file = _ptr(eta_file, _f32p)
    pr.nfaults = len(p.faults)
    pr.faults = _ptr(faults, _f64p)
    pr.crop_flag, pr.crop_value = int(p.crop_flag), float(p.crop_value)
    for i in range(4):
        pr.borders[i] = float(p.borders[i])
    pr.sim_time, pr.save_time = float(p.sim_time), float(p.save_time)
    pr.series_time = float(p.series_time) if pts is not None else -1.0
    pr.npoints = 0 if pts is None else len(pts)
    pr.points = _ptr(pts, _f64p)
    pr.cfl, pr.eps_h, pr.hpos, pr.stability = p.cfl, p.eps_h, p.hpos, p.stability
    pr.manning, pr.vmax, pr.L, pr.H, pr.dif_at = p.manning, p.vmax, p.L, p.H, p.dif_at
    pr.max_iterations = max_iterations
    pr.threads = threads
    out = {k: np.empty((ny, nx), np.float32) for k in ("max_height", "arrival", "deformed_bathy", "eta", "ux", "uy")}
    npts = 0 if pts is None else len(pts)
    snaps = {k: np.empty((max(max_snaps, 1), ny, nx), np.float32) for k in ("snap_eta", "snap_ux", "snap_uy")}
    snap_time = np.empty(max(max_snaps, 1), np.float64)
    ser = {k: np.empty((max(max_series, 1), max(npts, 1)), np.float32) for k in ("ts_eta", "ts_ux", "ts_uy")}
    ts_time = np.empty(max(max_series, 1), np.float64)
    ts_pts = {k: np.empty(max(npts, 1), np.float32) for k in ("ts_min", "ts_max", "ts_bathy")}
    r = _Result()
    for k, v in out.items():
        setattr(r, k, _ptr(v, _f32p))
    r.max_snaps = max_snaps
    for k, v in snaps.items():
        setattr(r, k, _ptr(v, _f32p))
    r.snap_time = _ptr(snap_time, _f64p)
    r.max_series = max_series
    for k, v in ser.items():
        setattr(r, k, _ptr(v, _f32p))
    r.ts_time = _ptr(ts_time, _f64p)
    for k, v in ts_pts.items():
        setattr(r, k, _ptr(v, _f32p))
    rc = lib.thy_oracle_run(ctypes.byref(pr), ctypes.byref(r))
    if rc != 0:
        raise RuntimeError(f"thy_oracle_run failed: {rc}")
    res = dict(out)
    ns = min(r.nsnaps, max_snaps)
    res["snapshots"] = {"eta": snaps["snap_eta"][:ns], "ux": snaps["snap_ux"][:ns], "uy": snaps["snap_uy"][:ns],
                        "time": snap_time[:ns]}
    nt, nu = min(r.nseries, max_series), r.npoints_unique
    res["series"] = {"eta": ser["ts_eta"][:nt, :nu], "ux": ser["ts_ux"][:nt, :nu], "uy": ser["ts_uy"][:nt, :nu],
                     "time": ts_time[:nt], "min": ts_pts["ts_min"][:nu], "max": ts_pts["ts_max"][:nu],
                     "bathy": ts_pts["ts_bathy"][:nu]}
    res.update(iterations=r.iterations, final_time=r.final_time, first_dt=r.first_dt,
               loop_seconds=r.loop_seconds, nsnaps=r.nsnaps, nseries=r.nseries)
    return res


def oracle_okada_points(lon, lat, fault_row) -> np.ndarray:
    lib = oracle_lib()
    lon = np.ascontiguousarray(lon, np.float64)
    lat = np.ascontiguousarray(lat, np.float64)
    f = np.ascontiguousarray(fault_row, np.float64)
    out = np.empty_like(lon)
    lib.thy_oracle_okada_points(len(lon), _ptr(lon, _f64p), _ptr(lat, _f64p), _ptr(f, _f64p), _ptr(out, _f64p))
    return out


def refemu_okada_points(lon, lat, fault_row) -> np.ndarray:
    lib = refemu_lib()
    lon = np.ascontiguousarray(lon, np.float64)
    lat = np.ascontiguousarray(lat, np.float64)
    f = np.ascontiguousarray(fault_row, np.float64)
    out = np.empty_like(lon)
    lib.refemu_okada_points(len(lon), _ptr(lon, _f64p), _ptr(lat, _f64p), _ptr(f, _f64p), _ptr(out, _f64p))
    return out


def run_refemu(txt_path: str, max_iterations: int = -1, threads: int = 0, quiet: bool = True) -> Dict:
    """Runs the reference's own code (compiled for the host) on a problem
    file; the outputs are the NetCDF files named by the file's prefix."""
    lib = refemu_lib()
    info = (ctypes.c_double * 4)()
    rc = lib.refemu_run(txt_path.encode(), max_iterations, threads, 1 if quiet else 0, info)
    if rc != 0:
        raise RuntimeError(f"refemu_run failed: {rc}")
    return {"iterations": int(info[0]), "final_time": info[1], "loop_seconds": info[2], "first_dt": info[3]}
