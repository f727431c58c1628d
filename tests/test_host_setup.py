"""Host side of the boundary on the CPU: the C++ problem loader and
nondimensionalisation (thy_load_problem_file, thy_prepare), the NetCDF
library, and the C ABI's behaviour without a GPU."""
import ctypes
import math
import os
import re
import subprocess
import tempfile

import numpy as np

from thysea import Prepared, _ffi, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _load(txt):
    L = _ffi.lib()
    h = ctypes.c_void_p()
    rc = L.thy_load_problem_file(txt.encode(), ctypes.byref(h))
    return rc, h


def test_header_symbols_are_exported():
    """every function declared in include/*.h is exported by libthysea.so"""
    L = _ffi.lib()
    names = set()
    for hdr in ("thysea.h", "thysea_dropin.h"):
        src = open(os.path.join(ROOT, "include", hdr)).read()
        names |= set(re.findall(r"\b(thy_\w+|shallowWater)\s*\(", src))
    names = {n for n in names if not n.endswith("_fn")}
    assert "shallowWater" in names and "thy_run" in names and "thy_apply_okada_noalloc" in names
    for n in sorted(names):
        assert hasattr(L, n), n
    assert set(_ffi.SIGNATURES) <= names


def test_only_the_c_abi_is_exported():
    """libthysea.so exports the C ABI and shallowWater and nothing else: in
    particular not the nc_* functions of its built-in NetCDF code, so that a
    program that also links a real libnetcdf keeps that library's calls"""
    so = os.path.join(ROOT, "tsunami-hysea_b200", "lib", "libthysea.so")
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    syms = [ln.split()[-1] for ln in out.splitlines() if ln.split() and ln.split()[-2] in ("T", "D", "B", "W", "V")]
    assert "shallowWater" in syms and "thy_run" in syms
    assert [s for s in syms if not (s.startswith("thy_") or s == "shallowWater")] == []
    assert not [s for s in syms if s.startswith("nc_")]


def test_no_device_fails_loudly():
    L = _ffi.lib()
    if L.thy_device_count() > 0:
        return
    p = Prepared(synth.plain_small(nx=32, ny=32, sim_time=10.0, npoints=0))
    st = _ffi.Stats()
    assert L.thy_run(p.view, None, ctypes.byref(st)) == 5        # THY_ERR_NO_DEVICE
    h = ctypes.c_void_p()
    assert L.thy_session_open(p.view, ctypes.byref(h)) == 5
    assert b"no CUDA device" in L.thy_strerror(5)


def test_loader_reads_what_synth_writes():
    p = synth.plain_small(nx=70, ny=50, sim_time=123.0, save_time=40.0, series_time=10.0, npoints=5)
    p.borders = (1.0, -1.0, 2.0, 2.0)
    p.crop_flag, p.crop_value = 2, 0.25
    d = tempfile.mkdtemp()
    txt = synth.write_problem(p, d)
    rc, h = _load(txt)
    assert rc == 0
    L = _ffi.lib()
    r = L.thy_raw_view(h).contents
    assert (r.nx, r.ny) == (70, 50)
    assert np.allclose(np.ctypeslib.as_array(r.lon, (70,)), p.lon)
    assert np.array_equal(np.ctypeslib.as_array(r.z, (50 * 70,)).reshape(50, 70), p.z)
    assert r.nfaults == 1 and r.crop_flag == 2 and r.crop_value == 0.25
    assert list(r.borders) == [1.0, -1.0, 2.0, 2.0]
    assert (r.sim_time, r.save_time, r.series_time) == (123.0, 40.0, 10.0)
    assert r.npoints == 5 and r.dif_at == 1e-6
    assert L.thy_raw_name(h) == b"plain_small"
    L.thy_raw_free(h)


def test_loader_rejects_bad_files():
    d = tempfile.mkdtemp()
    assert _load(os.path.join(d, "missing.txt"))[0] != 0
    p = synth.plain_small(nx=16, ny=16, npoints=0)
    txt = synth.write_problem(p, d)
    lines = open(txt).read().splitlines()
    # upper border periodic is rejected (src/Problema.cxx:293-298)
    bad = [ln.replace("1.0    # Upper border", "2.0    # Upper border") for ln in lines]
    open(txt, "w").write("\n".join(bad) + "\n")
    assert _load(txt)[0] != 0
    # wrong number of levels
    bad = [ln.replace("1    # Number of levels", "2    # Number of levels") for ln in lines]
    open(txt, "w").write("\n".join(bad) + "\n")
    assert _load(txt)[0] != 0


def test_prepare_nondimensionalisation():
    """thy_prepare against the loader formulas of src/Problema.cxx:319-456"""
    p = synth.plain_small(nx=40, ny=30, sim_time=600.0, save_time=60.0, series_time=30.0, npoints=4)
    pr = Prepared(p)
    c = pr.c
    H, L_ = p.H, p.L
    Q = math.sqrt(9.81 * H ** 3)
    T = L_ * H / Q
    assert math.isclose(c.Q, Q) and math.isclose(c.T, T)
    assert math.isclose(c.t_end, 600.0 / T) and math.isclose(c.save_nc, 60.0 / T)
    assert math.isclose(c.mf0, p.manning * (9.81 * p.manning * L_ / H ** (4.0 / 3.0)))
    assert math.isclose(c.vmax, p.vmax / (Q / H)) and math.isclose(c.cvis, 1.0 - p.stability)
    assert (c.sponge_up, c.sponge_low, c.sponge_left, c.sponge_right) == (4, 4, 4, 4)
    n = p.nx * p.ny
    depth = -p.z.astype(np.float64).ravel() / H
    Hmin = min(depth.min(), 0.0)
    assert c.Hmin == Hmin
    Hs = np.ctypeslib.as_array(c.Hs, (n,))
    hh = np.ctypeslib.as_array(c.h, (n,))
    assert np.array_equal(Hs, depth - Hmin)
    assert np.array_equal(hh, np.maximum(depth, 0.0))
    ac = np.ctypeslib.as_array(c.area_cos, (2 * p.ny,)).reshape(p.ny, 2)
    dlat = np.abs(np.diff(p.lat))
    area = 6378136.6 / L_ * abs(p.lon[1] - p.lon[0]) * dlat * (math.pi / 180.0)
    assert np.allclose(ac[:-1, 0], area, rtol=1e-15) and ac[-1, 0] == ac[-2, 0]
    assert np.allclose(ac[:, 1], np.cos(p.lat * math.pi / 180.0))
    cells = np.ctypeslib.as_array(c.point_cell, (c.npoints,))
    for k, (lo, la) in enumerate(p.points):
        i, j = int(np.argmin(np.abs(p.lon - lo))), int(np.argmin(np.abs(p.lat - la)))
        assert cells[k] == j * p.nx + i


def test_faults_sorted_by_time():
    p = synth.plain_small(nx=20, ny=20, npoints=0)
    f0 = p.faults[0]
    p.faults = [synth.Fault(t, f0.lon, f0.lat, 10.0, 50.0, 25.0, 0.0, 15.0, 90.0, float(t))
                for t in (300.0, 0.0, 120.0, 0.0)]
    pr = Prepared(p)   # keeps the library-owned problem alive
    f = np.ctypeslib.as_array(pr.c.faults, (40,)).reshape(4, 10)
    assert list(f[:, 0]) == [0.0, 0.0, 120.0, 300.0]


def test_nclite_roundtrip_with_scipy():
    """files written through the library's NetCDF API read back with scipy and vice versa"""
    from scipy.io import netcdf_file

    L = _ffi.nclite()
    d = tempfile.mkdtemp()
    path = os.path.join(d, "t.nc").encode()
    nc, dx, dt, vx, vt = (ctypes.c_int() for _ in range(5))
    assert L.nc_create(path, 0x1000, ctypes.byref(nc)) == 0
    L.nc_def_dim(nc, b"lon", ctypes.c_size_t(7), ctypes.byref(dx))
    L.nc_def_dim(nc, b"time", ctypes.c_size_t(0), ctypes.byref(dt))
    dims = (ctypes.c_int * 2)(dt.value, dx.value)
    L.nc_def_var(nc, b"lon", 6, 1, ctypes.byref(dx), ctypes.byref(vx))
    L.nc_def_var(nc, b"eta", 5, 2, dims, ctypes.byref(vt))
    L.nc_put_att_text(nc, vt, b"units", ctypes.c_size_t(6), b"meters")
    assert L.nc_enddef(nc) == 0
    lon = np.arange(7, dtype=np.float64)
    L.nc_put_var_double(nc, vx, lon.ctypes.data_as(_ffi.f64p))
    for r in range(3):
        e = (np.arange(7) + 10 * r).astype(np.float32)
        start = (ctypes.c_size_t * 2)(r, 0)
        count = (ctypes.c_size_t * 2)(1, 7)
        assert L.nc_put_vara_float(nc, vt, start, count, e.ctypes.data_as(_ffi.f32p)) == 0
    assert L.nc_close(nc) == 0
    with netcdf_file(path.decode(), "r", mmap=False) as f:
        assert f.variables["eta"].shape == (3, 7)
        assert f.variables["eta"][2, 3] == 23.0
        assert f.variables["eta"].units == b"meters"


def test_cli_usage_and_missing_file():
    exe = os.path.join(ROOT, "tsunami-hysea_b200", "bin", "TsunamiHySEA")
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode != 0 and "dataFile format" in r.stderr
    r = subprocess.run([exe, "/nonexistent/problem.txt"], capture_output=True, text=True)
    assert r.returncode != 0 and "not found" in r.stderr
