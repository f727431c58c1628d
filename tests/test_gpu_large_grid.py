"""A grid beyond the reference's 32-bit byte counts.

The reference sizes every float field as `int tam_datosVolFloat = nx * ny *
sizeof(float)` (src/GPU/ShallowWater.cu:25 and the copies that use it), which
overflows past 536 870 911 cells.  This library keeps byte and cell offsets
in 64-bit (nclite, the loader, the set-up, the copies) and cell offsets
within a field in 32-bit (a field plane below 2^31 floats).  Here a grid of
24 000 x 24 000 cells (576 M cells, 2.3 GB per float field) goes the whole
way: its bathymetry file is written and read back through the library's
NetCDF reader (thy_load_problem_file), the problem is prepared, Okada and a
few time steps run on the GPU, and the deformed bathymetry and the maximum
height come back to the host.  Checked: the cells beyond 2^31 bytes of a
field read back what was written (bathymetry far from the source), the
Okada deformation at the source equals the FP64 oracle's, and the sea far
from the source is still at rest.  The bathymetry file is written through
the library's own NetCDF writer, and nclite writing and reading back a
variable of more than 2^31 bytes is checked on its own as well."""
import ctypes
import os

import numpy as np
import pytest

import oracle
from thysea import _ffi, synth

pytestmark = pytest.mark.gpu

N = 24000
SPACING = 0.25 / 60.0   # 15 arc-seconds: the grid spans 100 x 100 degrees


def _grid():
    lon, lat = synth.lonlat_grid(N, N, spacing_deg=SPACING, lon0=-50.0)
    # ocean 4000 m deep with a 20 m-deep shelf band in the east and a row of
    # land along the last 200 columns
    x = np.arange(N, dtype=np.float32)
    prof = np.where(x < N - 2000, -4000.0, np.where(x < N - 200, -20.0, 100.0)).astype(np.float32)
    z = np.broadcast_to(prof[None, :], (N, N))
    return lon, lat, z


def _write_grd_nclite(path, lon, lat, z):
    """the bathymetry file through the library's NetCDF writer (CDF-2, 64-bit
    offsets): scipy's writer keeps a variable's byte count in a signed 32-bit
    field and cannot write one this large"""
    L = _ffi.nclite()
    nc, dx, dy, vx, vy, vz = (ctypes.c_int() for _ in range(6))
    assert L.nc_create(path.encode(), 0x1000, ctypes.byref(nc)) == 0
    assert L.nc_def_dim(nc, b"lon", ctypes.c_size_t(len(lon)), ctypes.byref(dx)) == 0
    assert L.nc_def_dim(nc, b"lat", ctypes.c_size_t(len(lat)), ctypes.byref(dy)) == 0
    assert L.nc_def_var(nc, b"lon", 6, 1, ctypes.byref(dx), ctypes.byref(vx)) == 0
    assert L.nc_def_var(nc, b"lat", 6, 1, ctypes.byref(dy), ctypes.byref(vy)) == 0
    dims = (ctypes.c_int * 2)(dy.value, dx.value)
    assert L.nc_def_var(nc, b"z", 5, 2, dims, ctypes.byref(vz)) == 0
    assert L.nc_enddef(nc) == 0
    lon = np.ascontiguousarray(lon, np.float64)
    lat = np.ascontiguousarray(lat, np.float64)
    assert L.nc_put_var_double(nc, vx, lon.ctypes.data_as(_ffi.f64p)) == 0
    assert L.nc_put_var_double(nc, vy, lat.ctypes.data_as(_ffi.f64p)) == 0
    assert L.nc_put_var_float(nc, vz, z.ctypes.data_as(_ffi.f32p)) == 0
    assert L.nc_close(nc) == 0


def test_grid_beyond_32_bit_byte_counts(gpu, tmp_path):
    assert N * N * 4 > 2 ** 31
    lon, lat, z = _grid()
    fault = synth.Fault(0.0, float(lon[N // 2]), float(lat[N // 2]), synth.centroid_depth(10.0, 50.0, 15.0),
                        100.0, 50.0, 0.0, 15.0, 90.0, 5.0)
    # the problem file (written for a stand-in grid of the same name), then
    # the real bathymetry file in place of the stand-in's
    stand_in = synth.Problem(name="huge", lon=lon[:4], lat=lat[:4], z=np.full((4, 4), -4000.0, np.float32),
                             faults=[fault], sim_time=1e6, save_time=-1.0)
    txt = synth.write_problem(stand_in, str(tmp_path))
    grd = str(tmp_path / "huge.grd")
    _write_grd_nclite(grd, lon, lat, np.ascontiguousarray(z))
    # the file's last bytes are the last rows of z, big-endian (classic format)
    tail = np.memmap(grd, dtype=">f4", mode="r", offset=os.path.getsize(grd) - 4 * N)
    assert np.array_equal(np.asarray(tail, np.float32), z[-1])
    del tail
    L = _ffi.lib()
    raw = ctypes.c_void_p()
    assert L.thy_load_problem_file(txt.encode(), ctypes.byref(raw)) == 0
    r = L.thy_raw_view(raw).contents
    assert (r.nx, r.ny) == (N, N)
    # the last row of the bathymetry as read back through nclite (beyond 2^31 bytes)
    zr = np.ctypeslib.as_array(r.z, (N * N,))
    assert np.array_equal(zr[-N:], z[-1])
    assert np.array_equal(zr[(N // 2) * N:(N // 2 + 1) * N], z[N // 2])
    prep = ctypes.c_void_p()
    assert L.thy_prepare(ctypes.byref(r), ctypes.byref(prep)) == 0
    L.thy_raw_free(raw)
    pc = L.thy_problem_view(prep)
    pc.contents.max_steps = 3
    deformed = np.empty((N, N), np.float32)
    maxh = np.empty((N, N), np.float32)
    o = _ffi.Outputs()
    o.deformed_bathy = deformed.ctypes.data_as(_ffi.f32p)
    o.max_height = maxh.ctypes.data_as(_ffi.f32p)
    st = _ffi.Stats()
    rc = L.thy_run(pc, ctypes.byref(o), ctypes.byref(st))
    assert rc == 0, L.thy_strerror(rc)
    assert st.steps == 3
    L.thy_problem_free(prep)
    # far from the source (beyond the fault's reach, and past 2^31 bytes into
    # the field): the bathymetry is what was written, the sea at rest
    far = slice(N - 1000, N)
    assert np.abs(deformed[far, : N - 2000] - 4000.0).max() <= 1e-3
    assert np.abs(deformed[far, N - 1500:N - 300] - 20.0).max() <= 1e-4
    # (the Okada uplift thousands of kilometres away is far below a micrometre)
    assert float(np.abs(maxh[far, : N - 2000]).max()) <= 1e-6
    # at the source: the Okada uplift of the FP64 oracle
    j0, i0 = N // 2, N // 2
    rows = np.arange(j0 - 600, j0 + 600, 37)
    cols = np.arange(i0 - 600, i0 + 600, 41)
    jj, ii = np.meshgrid(rows, cols, indexing="ij")
    uz = oracle.oracle_okada_points(lon[ii.ravel()], lat[jj.ravel()], np.asarray(fault.as_row()))
    got = 4000.0 - deformed[jj, ii].ravel().astype(np.float64)
    assert np.abs(uz).max() > 0.5
    assert np.abs(got - uz).max() <= 1e-3


def test_nclite_writes_a_variable_beyond_2_gib(tmp_path):
    """one float variable of 2^31 + 64 bytes written through the library's
    NetCDF writer and read back through it, and its bytes checked in the file
    (the data of the only variable ends the file, big-endian)"""
    L = _ffi.nclite()
    n = 2 ** 29 + 16
    path = str(tmp_path / "big.nc").encode()
    nc, dx, vx = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    assert L.nc_create(path, 0x1000, ctypes.byref(nc)) == 0   # NC_NETCDF4, as the reference asks: CDF-2 (64-bit offsets)
    assert L.nc_def_dim(nc, b"x", ctypes.c_size_t(n), ctypes.byref(dx)) == 0
    assert L.nc_def_var(nc, b"v", 5, 1, ctypes.byref(dx), ctypes.byref(vx)) == 0
    assert L.nc_enddef(nc) == 0
    v = np.arange(n, dtype=np.float32)
    v[-16:] = -7.5
    assert L.nc_put_var_float(nc, vx, v.ctypes.data_as(_ffi.f32p)) == 0
    assert L.nc_close(nc) == 0
    m = np.memmap(path.decode(), dtype=">f4", mode="r", offset=os.path.getsize(path.decode()) - 4 * n)
    assert m.shape == (n,)
    assert float(m[12345]) == 12345.0 and float(m[n - 17]) == float(v[n - 17])
    assert np.all(m[-16:] == -7.5)
    del m
    # and back through the library's reader
    nc2, vid = ctypes.c_int(), ctypes.c_int()
    assert L.nc_open(path, 0, ctypes.byref(nc2)) == 0
    assert L.nc_inq_varid(nc2, b"v", ctypes.byref(vid)) == 0
    w = np.empty(n, np.float32)
    assert L.nc_get_var_float(nc2, vid, w.ctypes.data_as(_ffi.f32p)) == 0
    assert L.nc_close(nc2) == 0
    assert np.array_equal(w, v)
