"""GPU path (FP32 states, FP64 Okada / metrics / time) against the FP64
oracle on the same seeded inputs: surface elevation within 1e-3 m, maximum
height within 1e-4 relative L2, same number of steps and final time.

Every case runs end to end through the C ABI (thy_prepare + thy_run).
"""
import numpy as np
import pytest

import oracle
from parity import ETA_TOL_M, MAXH_REL_L2, compare, max_abs_eta
from thysea import synth

pytestmark = pytest.mark.gpu


def _both(gpu, p, max_snaps=16, max_series=256):
    g = gpu.run(p)
    r = oracle.run_oracle(p, max_snaps=max_snaps, max_series=max_series)
    c = compare(g, r, p.name)
    print(c)
    return g, r, c


def _assert_parity(c, snaps=True):
    assert c["iterations"][0] == c["iterations"][1]
    assert abs(c["final_time"][0] - c["final_time"][1]) < 1e-3 * max(1.0, c["final_time"][1])
    assert c["maxh_rel_l2"] <= MAXH_REL_L2
    assert c["eta_final_max_abs"] <= ETA_TOL_M
    if snaps and "eta_snap_max_abs" in c:
        assert c["eta_snap_max_abs"] <= ETA_TOL_M


def test_plain_small_quarter(gpu):
    """the plain small problem's shape at 256^2: open borders, one fault, 600 s, 16 gauges"""
    p = synth.plain_small(nx=256, ny=256, sim_time=600.0, save_time=200.0, series_time=60.0, npoints=16)
    g, r, c = _both(gpu, p)
    _assert_parity(c)
    assert len(g["snapshots"]["time"]) == r["nsnaps"]
    # gauges: same sample count, eta within tolerance
    assert g["nseries"] == r["nseries"]
    ge, re_ = np.asarray(g["series"]["eta"]), r["series"]["eta"]
    assert np.abs(ge - re_).max() <= ETA_TOL_M
    # arrival times: identical except where the threshold is met within a step of each other
    arr_g, arr_r = g["arrival"], r["arrival"]
    agree = np.mean(np.abs(arr_g - arr_r) <= 5.0)
    assert agree > 0.999


def test_shelf_wet_dry(gpu):
    """random-field shelf with ~10% dry cells: coastal wet/dry, WAF branch"""
    p = synth.single_large(n=192, sim_time=1200.0, save_time=400.0)
    p.name = "shelf192"
    g, r, c = _both(gpu, p)
    _assert_parity(c)


def test_walls_and_relative_crop(gpu):
    p = synth.single_large(n=160, seed=9, sim_time=600.0, save_time=300.0)
    p.name = "walls"
    p.borders = (-1.0, -1.0, -1.0, -1.0)
    p.crop_flag, p.crop_value = 1, 5e-3
    g, r, c = _both(gpu, p)
    _assert_parity(c)


def test_periodic_absolute_crop(gpu):
    p = synth.single_large(n=160, seed=11, sim_time=600.0, save_time=200.0)
    p.name = "periodic"
    p.borders = (1.0, -1.0, 2.0, 2.0)
    p.crop_flag, p.crop_value = 2, 0.05
    g, r, c = _both(gpu, p)
    _assert_parity(c)


def test_faults_at_two_times(gpu):
    p = synth.plain_small(nx=128, ny=96, sim_time=400.0, save_time=100.0, npoints=4)
    p.name = "twofault"
    f0 = p.faults[0]
    f1 = synth.Fault(150.0, f0.lon + 0.2, f0.lat + 0.1, 12.0, 60.0, 30.0, 45.0, 20.0, 80.0, 3.0)
    p.faults = [f1, f0]
    g, r, c = _both(gpu, p)
    _assert_parity(c)


def test_initial_state_from_file(gpu):
    p = synth.plain_small(nx=128, ny=112, sim_time=300.0, save_time=100.0, npoints=0)
    p.name = "fromfile"
    p.faults = []
    yy, xx = np.mgrid[0:112, 0:128]
    p.eta_init = (2.0 * np.exp(-((xx - 40) ** 2 + (yy - 50) ** 2) / 60.0)).astype(np.float32)
    g, r, c = _both(gpu, p)
    _assert_parity(c)


def test_lake_at_rest(gpu):
    """no source: the surface stays exactly at rest over any bathymetry"""
    p = synth.single_large(n=128, seed=3, sim_time=300.0, save_time=-1.0)
    p.faults = []
    p.eta_init = np.zeros_like(p.z)
    g = gpu.run(p)
    wet = g["eta"] != -9999.0
    assert np.abs(g["eta"][wet]).max() == 0.0
    assert np.abs(g["ux"]).max() == 0.0 and np.abs(g["uy"]).max() == 0.0


def test_okada_deformation_matches_oracle(gpu):
    """deformed bathymetry after the first step (Okada in FP64 on the GPU)"""
    p = synth.single_large(n=192, seed=5, sim_time=1.0)
    g = gpu.run(p, max_steps=1)
    r = oracle.run_oracle(p, max_iterations=1)
    d = np.abs(g["deformed_bathy"].astype(np.float64) - r["deformed_bathy"])
    # FP32 storage of the depth: about one float ulp of a 7 km depth (~0.5 mm)
    assert d.max() <= 2e-3


@pytest.mark.parametrize("borders", [(1.0, 1.0, 1.0, 1.0), (1.0, -1.0, 2.0, 2.0)], ids=["open", "periodic"])
def test_deep_and_coastal_tiles(gpu, borders):
    """1024^2 shelf: interior open-ocean tiles take the deep-water kernels,
    coastal, border and sponge tiles the general ones; one result"""
    p = synth.single_large(n=1024, seed=5, sim_time=900.0, save_time=300.0)
    p.name = "deep1024"
    p.borders = borders
    g, r, c = _both(gpu, p)
    _assert_parity(c)
    assert 0 < g["deep_tiles"] < g["tiles"]
    assert g["deep_tiles"] > g["tiles"] // 2


def test_deep_tiles_fault_mid_run(gpu):
    """a second fault at t = 300 s deforms the state between two steps: the
    tile depth minima are re-measured before any tile is stepped as deep"""
    import dataclasses

    p = synth.single_large(n=512, seed=6, sim_time=900.0, save_time=150.0)
    p.name = "deep512_twofault"
    f0 = p.faults[0]
    p.faults = [f0, dataclasses.replace(p.faults[2], time=300.0, slip=6.0)]
    g, r, c = _both(gpu, p)
    _assert_parity(c)
    assert g["deep_tiles"] > 0


def test_async_snapshots_and_gauges_in_order(gpu):
    """snapshots every 20 s and gauges every 10 s are delivered by the writer
    thread while the GPU steps on: all of them, in order, each the state of
    its own step (against the oracle's snapshots and gauges)"""
    p = synth.plain_small(nx=256, ny=192, sim_time=400.0, save_time=20.0, series_time=10.0, npoints=8)
    p.name = "async_out"
    g, r, c = _both(gpu, p, max_snaps=32, max_series=64)
    _assert_parity(c)
    t = np.asarray(g["snapshots"]["time"])
    assert len(t) == g["nsnaps"] == r["nsnaps"] and np.all(np.diff(t) > 0)
    for i in range(len(t)):
        assert abs(t[i] - r["snapshots"]["time"][i]) < 1e-3
        assert max_abs_eta(g["snapshots"]["eta"][i], r["snapshots"]["eta"][i]) <= ETA_TOL_M
    ts = np.asarray(g["series"]["time"])
    assert len(ts) == g["nseries"] == r["nseries"] and np.all(np.diff(ts) > 0)
    assert np.abs(np.asarray(g["series"]["eta"]) - r["series"]["eta"]).max() <= ETA_TOL_M


def test_gauges_sampled_on_the_device_do_not_stop_the_run(gpu):
    """gauge times are handled by the step controller on the device: a run
    with gauges every 10 s takes exactly the graph launches of the same run
    without gauges, its samples are those of the oracle at the same times, and
    the extremes of eta folded on the device are the oracle's"""
    base = dict(nx=256, ny=192, sim_time=400.0, save_time=-1.0, npoints=8)
    with_g = synth.plain_small(series_time=10.0, **base)
    with_g.name = "gauges_device"
    without = synth.plain_small(series_time=-1.0, **base)
    without.name = "gauges_none"
    g, r, c = _both(gpu, with_g, max_snaps=4, max_series=64)
    _assert_parity(c, snaps=False)
    g0 = gpu.run(without)
    assert g["iterations"] == g0["iterations"]
    assert g["chunks"] == g0["chunks"], (g["chunks"], g0["chunks"])
    assert g["nseries"] == r["nseries"] and g["nseries"] >= 40
    ts = np.asarray(g["series"]["time"])
    assert np.all(np.diff(ts) > 0)
    assert np.abs(ts - r["series"]["time"][:len(ts)]).max() < 1e-3
    assert np.abs(np.asarray(g["series"]["eta"]) - r["series"]["eta"]).max() <= ETA_TOL_M
    nu = len(r["series"]["min"])
    assert np.abs(g["series"]["min"][:nu] - r["series"]["min"]).max() <= ETA_TOL_M
    assert np.abs(g["series"]["max"][:nu] - r["series"]["max"]).max() <= ETA_TOL_M


@pytest.mark.parametrize("lat_centre", [70.0, -80.0])
def test_high_latitude_metric_terms(gpu, lat_centre):
    """far from the equator (cos(lat) 0.34 at 70 degrees, 0.17 at 80): the
    spherical metric terms (cos(lat), dlat / cos(lat), the cell area, dlon)
    are formed in FP64 on the host once and kept in FP32 row tables; the
    surface, the maximum height and the gauges stay within the tolerances of
    the FP64 oracle, which keeps them in FP64 throughout"""
    p = synth.plain_small(nx=256, ny=224, sim_time=600.0, save_time=200.0, series_time=60.0, npoints=8)
    p.name = f"lat{int(lat_centre)}"
    p.lat = p.lat + lat_centre
    p.faults[0].lat += lat_centre
    p.points = p.points.copy()
    p.points[:, 1] += lat_centre
    g, r, c = _both(gpu, p)
    _assert_parity(c)
    assert g["nseries"] == r["nseries"]
    assert np.abs(np.asarray(g["series"]["eta"]) - r["series"]["eta"]).max() <= ETA_TOL_M
    # the wave is there: the fault deformed the surface by more than the tolerance
    assert float(np.abs(r["max_height"][r["max_height"] != -9999.0]).max()) > 100 * ETA_TOL_M
