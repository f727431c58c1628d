"""Failures made on the host, without a GPU: damaged or missing input files
are refused with an error code (never a crash), the multi-scenario runtime
refuses to start without a device, and NetCDF files written from several
threads at once come out intact."""
import ctypes
import os
import tempfile
import threading

import numpy as np
import pytest

import thysea
from thysea import _ffi, synth


def _load(txt):
    h = ctypes.c_void_p()
    rc = _ffi.lib().thy_load_problem_file(txt.encode(), ctypes.byref(h))
    if rc == 0:
        _ffi.lib().thy_raw_free(h)
    return rc


def _problem_dir(points=0):
    d = tempfile.mkdtemp()
    p = synth.plain_small(nx=24, ny=20, npoints=points)
    p.name = "faulty"
    return d, synth.write_problem(p, d)


def test_valid_problem_loads():
    d, txt = _problem_dir(points=3)
    assert _load(txt) == 0


def test_truncated_bathymetry_file_is_refused():
    d, txt = _problem_dir()
    grd = os.path.join(d, "faulty.grd")
    data = open(grd, "rb").read()
    for cut in (len(data) // 2, 64, 3):
        open(grd, "wb").write(data[:cut])
        assert _load(txt) != 0, cut


def test_garbage_bathymetry_file_is_refused():
    d, txt = _problem_dir()
    open(os.path.join(d, "faulty.grd"), "wb").write(os.urandom(4096))
    assert _load(txt) != 0


def test_missing_bathymetry_and_points_files_are_refused():
    d, txt = _problem_dir(points=3)
    os.remove(os.path.join(d, "faulty_points.txt"))
    assert _load(txt) != 0
    d, txt = _problem_dir()
    os.remove(os.path.join(d, "faulty.grd"))
    assert _load(txt) != 0


def test_truncated_problem_file_is_refused():
    """every value up to H is required; only the arrival threshold, the last
    line, is optional (it defaults to epsilon h, src/Problema.cxx:327)"""
    d, txt = _problem_dir()
    lines = open(txt).read().splitlines()
    for keep in range(1, len(lines) - 1):
        open(txt, "w").write("\n".join(lines[:keep]) + "\n")
        assert _load(txt) != 0, keep
    open(txt, "w").write("\n".join(lines[:-1]) + "\n")
    assert _load(txt) == 0


def test_server_needs_a_device():
    if thysea.device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(thysea.ThyError) as e:
        thysea.Server()
    assert e.value.code == thysea.THY_ERR_NO_DEVICE


def test_netcdf_files_written_from_many_threads():
    """one NetCDF file per thread, created, written and closed concurrently
    (the snapshot writers of several scenarios do this)"""
    from scipy.io import netcdf_file

    L = _ffi.nclite()
    d = tempfile.mkdtemp()
    errors = []

    def writer(k):
        try:
            for rep in range(20):
                path = os.path.join(d, f"t{k}_{rep}.nc").encode()
                nc, dx, vx = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
                assert L.nc_create(path, 0x1000, ctypes.byref(nc)) == 0
                assert L.nc_def_dim(nc, b"x", ctypes.c_size_t(64), ctypes.byref(dx)) == 0
                assert L.nc_def_var(nc, b"v", 5, 1, ctypes.byref(dx), ctypes.byref(vx)) == 0
                assert L.nc_enddef(nc) == 0
                v = np.full(64, k * 1000 + rep, np.float32)
                assert L.nc_put_var_float(nc, vx, v.ctypes.data_as(_ffi.f32p)) == 0
                assert L.nc_close(nc) == 0
        except AssertionError as e:  # pragma: no cover - reported below
            errors.append((k, e))

    threads = [threading.Thread(target=writer, args=(k,)) for k in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors
    for k in range(8):
        for rep in range(20):
            with netcdf_file(os.path.join(d, f"t{k}_{rep}.nc"), "r", mmap=False) as f:
                assert np.all(f.variables["v"][:] == k * 1000 + rep)
