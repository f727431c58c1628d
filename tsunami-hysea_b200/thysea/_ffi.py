"""ctypes declarations of the C ABI in include/thysea.h (libthysea.so)."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "lib", "libthysea.so")

f32p = ctypes.POINTER(ctypes.c_float)
f64p = ctypes.POINTER(ctypes.c_double)
i32p = ctypes.POINTER(ctypes.c_int)


class Raw(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("lon", f64p), ("lat", f64p), ("z", f32p), ("eta_file", f32p),
        ("nfaults", ctypes.c_int), ("faults", f64p),
        ("crop_flag", ctypes.c_int), ("crop_value", ctypes.c_double),
        ("borders", ctypes.c_double * 4),
        ("sim_time", ctypes.c_double), ("save_time", ctypes.c_double), ("series_time", ctypes.c_double),
        ("npoints", ctypes.c_int), ("points", f64p),
        ("cfl", ctypes.c_double), ("eps_h", ctypes.c_double), ("hpos", ctypes.c_double),
        ("stability", ctypes.c_double), ("manning", ctypes.c_double), ("vmax", ctypes.c_double),
        ("L", ctypes.c_double), ("H", ctypes.c_double), ("dif_at", ctypes.c_double),
    ]


class ProblemC(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("h", f64p), ("Hs", f64p), ("qx", f64p), ("qy", f64p),
        ("area_cos", f64p), ("dlon", f64p), ("dlat", f64p), ("lon", f64p), ("lat", f64p),
        ("Hmin", ctypes.c_double),
        ("border_up", ctypes.c_double), ("border_low", ctypes.c_double),
        ("border_left", ctypes.c_double), ("border_right", ctypes.c_double),
        ("sponge_up", ctypes.c_int), ("sponge_low", ctypes.c_int),
        ("sponge_left", ctypes.c_int), ("sponge_right", ctypes.c_int),
        ("t_end", ctypes.c_double), ("save_nc", ctypes.c_double), ("save_ts", ctypes.c_double),
        ("cfl", ctypes.c_double), ("mf0", ctypes.c_double), ("vmax", ctypes.c_double),
        ("eps_h", ctypes.c_double), ("hpos", ctypes.c_double), ("cvis", ctypes.c_double),
        ("dif_at", ctypes.c_double),
        ("L", ctypes.c_double), ("H", ctypes.c_double), ("Q", ctypes.c_double), ("T", ctypes.c_double),
        ("okada_flag", ctypes.c_int), ("nfaults", ctypes.c_int), ("faults", f64p),
        ("crop_flag", ctypes.c_int), ("crop_value", ctypes.c_double),
        ("npoints", ctypes.c_int), ("point_cell", i32p), ("point_lon", f64p), ("point_lat", f64p),
        ("max_steps", ctypes.c_longlong),
    ]


FieldFn = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int, ctypes.c_double, f32p, f32p, f32p)


class Outputs(ctypes.Structure):
    _fields_ = [
        ("max_height", f32p), ("arrival", f32p), ("deformed_bathy", f32p),
        ("eta", f32p), ("ux", f32p), ("uy", f32p),
        ("series_min", f32p), ("series_max", f32p), ("series_bathy", f32p),
        ("on_snapshot", FieldFn), ("on_series", FieldFn), ("user", ctypes.c_void_p),
    ]


class Tiling(ctypes.Structure):
    _fields_ = [("deep1", ctypes.c_int), ("deep2", ctypes.c_int), ("general", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_longlong), ("final_time_s", ctypes.c_double), ("first_dt_s", ctypes.c_double),
        ("loop_seconds", ctypes.c_double), ("device_loop_ms", ctypes.c_double),
        ("kernel_launches", ctypes.c_longlong), ("snapshots", ctypes.c_int), ("series_samples", ctypes.c_int),
        ("tiles", ctypes.c_longlong), ("deep_tiles", ctypes.c_longlong), ("dry_tiles", ctypes.c_longlong),
        ("setup_seconds", ctypes.c_double), ("output_seconds", ctypes.c_double), ("total_seconds", ctypes.c_double),
        ("tiling", Tiling), ("tune_samples", ctypes.c_longlong), ("release_seconds", ctypes.c_double),
        ("chunks", ctypes.c_longlong), ("graph_captures", ctypes.c_longlong), ("capture_seconds", ctypes.c_double),
        ("event_seconds", ctypes.c_double), ("initial_seconds", ctypes.c_double),
    ]


class ServerOpts(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_longlong), ("max_scenarios", ctypes.c_int), ("device", ctypes.c_int),
                ("chunk_cells", ctypes.c_longlong)]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_longlong), ("admitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
        ("failed", ctypes.c_longlong), ("cancelled", ctypes.c_longlong), ("rejected", ctypes.c_longlong),
        ("chunks", ctypes.c_longlong), ("queued", ctypes.c_int), ("running", ctypes.c_int),
        ("hbm_in_use", ctypes.c_longlong), ("hbm_budget", ctypes.c_longlong),
        ("device_ms", ctypes.c_double), ("cell_updates", ctypes.c_double),
    ]


DoneFn = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_void_p)

# names and signatures of every function include/thysea.h declares
SIGNATURES = {
    "thy_version": ([], ctypes.c_char_p),
    "thy_strerror": ([ctypes.c_int], ctypes.c_char_p),
    "thy_device_count": ([], ctypes.c_int),
    "thy_set_device": ([ctypes.c_int], ctypes.c_int),
    "thy_host_register": ([ctypes.c_void_p, ctypes.c_size_t], ctypes.c_int),
    "thy_host_unregister": ([ctypes.c_void_p], ctypes.c_int),
    "thy_load_problem_file": ([ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "thy_raw_view": ([ctypes.c_void_p], ctypes.POINTER(Raw)),
    "thy_raw_name": ([ctypes.c_void_p], ctypes.c_char_p),
    "thy_raw_bathy_file": ([ctypes.c_void_p], ctypes.c_char_p),
    "thy_raw_prefix": ([ctypes.c_void_p], ctypes.c_char_p),
    "thy_raw_free": ([ctypes.c_void_p], None),
    "thy_prepare": ([ctypes.POINTER(Raw), ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "thy_problem_view": ([ctypes.c_void_p], ctypes.POINTER(ProblemC)),
    "thy_problem_free": ([ctypes.c_void_p], None),
    "thy_run": ([ctypes.POINTER(ProblemC), ctypes.POINTER(Outputs), ctypes.POINTER(Stats)], ctypes.c_int),
    "thy_run_netcdf": ([ctypes.POINTER(ProblemC), ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(Stats)],
                       ctypes.c_int),
    "thy_apply_okada": ([ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                         ctypes.c_double, f64p, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                         ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "thy_apply_okada_noalloc": ([ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, f64p, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "thy_session_open": ([ctypes.POINTER(ProblemC), ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "thy_session_steps": ([ctypes.c_void_p, ctypes.c_longlong, f64p, ctypes.POINTER(ctypes.c_longlong)],
                          ctypes.c_int),
    "thy_session_fetch": ([ctypes.c_void_p, f32p, f32p, f32p, f32p], ctypes.c_int),
    "thy_session_time": ([ctypes.c_void_p], ctypes.c_double),
    "thy_session_profile": ([ctypes.c_void_p, ctypes.c_longlong, f64p, f64p], ctypes.c_int),
    "thy_session_profile_launches": ([ctypes.c_void_p, ctypes.c_longlong, f64p], ctypes.c_int),
    "thy_session_launches": ([ctypes.c_void_p], ctypes.c_longlong),
    "thy_session_tiles": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                           ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
    "thy_session_close": ([ctypes.c_void_p], None),
    "thy_session_tune": ([ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
    "thy_session_inject": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "thy_session_tiling": ([ctypes.c_void_p, ctypes.POINTER(Tiling)], ctypes.c_int),
    "thy_tiling_force": ([ctypes.POINTER(Tiling)], ctypes.c_int),
    "thy_tiling_tuned": ([ctypes.c_double, ctypes.c_double, ctypes.POINTER(Tiling)], ctypes.c_int),
    "thy_session_tuned": ([ctypes.c_void_p, ctypes.POINTER(Tiling)], ctypes.c_int),
    "thy_tuner_clear": ([], None),
    "thy_server_open": ([ctypes.POINTER(ServerOpts), ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "thy_server_submit": ([ctypes.c_void_p, ctypes.POINTER(ProblemC), ctypes.POINTER(Outputs), DoneFn,
                           ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
    "thy_server_cancel": ([ctypes.c_void_p, ctypes.c_longlong], ctypes.c_int),
    "thy_server_progress": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "thy_server_drain": ([ctypes.c_void_p], ctypes.c_int),
    "thy_server_get_stats": ([ctypes.c_void_p, ctypes.POINTER(ServerStats)], ctypes.c_int),
    "thy_server_close": ([ctypes.c_void_p], None),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Loads libthysea.so; raises if it has not been built (there is no
    fallback implementation)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libthysea.so not built: {LIB_PATH} (run `python tsunami-hysea_b200/build.py`)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


_nclite = None


def nclite() -> ctypes.CDLL:
    """Loads libnclite.so, the library's NetCDF classic reader / writer with
    the NetCDF C API (nc_*) exported; libthysea.so keeps its own copy private."""
    global _nclite
    if _nclite is None:
        path = os.path.join(os.path.dirname(LIB_PATH), "libnclite.so")
        if not os.path.exists(path):
            raise RuntimeError(f"libnclite.so not built: {path} (run `python tsunami-hysea_b200/build.py`)")
        _nclite = ctypes.CDLL(path)
    return _nclite
