"""The oracle restatement against the reference's own code compiled for the
host (oracle/_ref), on fresh seeded problems (skipped where that build is
absent)."""
import os
import tempfile

import numpy as np
import pytest

import oracle
from thysea import synth

pytestmark = pytest.mark.skipif(not oracle.refemu_available(), reason="oracle/_ref not built")


def test_okada_closed_form_matches_reference_dc3d():
    rng = np.random.default_rng(11)
    lon = 10.0 + rng.uniform(-3, 3, 4000)
    lat = 5.0 + rng.uniform(-3, 3, 4000)
    faults = [
        [0.0, 10.0, 5.0, 16.47, 100.0, 50.0, 33.0, 15.0, 90.0, 5.0],
        [0.0, 10.0, 5.0, 12.0, 80.0, 40.0, 200.0, 60.0, 30.0, 2.0],
        [0.0, 10.0, 5.0, 8.0, 50.0, 25.0, 10.0, 90.0, 90.0, 2.0],     # vertical fault
        [0.0, 10.0, 5.0, 30.0, 300.0, 150.0, 300.0, 10.0, 120.0, 9.0],
    ]
    for f in faults:
        a = oracle.oracle_okada_points(lon, lat, f)
        b = oracle.refemu_okada_points(lon, lat, f)
        assert np.abs(a - b).max() < 1e-12
        assert np.abs(b).max() > 0.1


def test_step_session_matches_full_run():
    """refemu_steps (bench.py's reference arm) runs the same loop body"""
    p = synth.plain_small(nx=96, ny=96, sim_time=100.0, save_time=-1.0, npoints=0)
    d = tempfile.mkdtemp()
    txt = synth.write_problem(p, d)
    s = oracle.RefemuSession(txt, threads=2)
    assert s.cells == 96 * 96
    assert s.steps(5) > 0
    s.close()


def test_random_problem_to_the_last_float_ulp():
    rng = np.random.default_rng(5)
    p = synth.single_large(n=72, seed=int(rng.integers(1000)), sim_time=300.0, save_time=150.0, npoints=4)
    p.name = "rand"
    d = tempfile.mkdtemp()
    txt = synth.write_problem(p, d)
    info = oracle.run_refemu(txt)
    r = oracle.run_oracle(p, max_snaps=8)
    from scipy.io import netcdf_file

    with netcdf_file(os.path.join(d, "rand.nc"), "r", mmap=False) as f:
        assert info["iterations"] == r["iterations"]
        assert np.abs(f.variables["max_height"][:] - r["max_height"]).max() <= 4e-9
        assert np.abs(f.variables["eta"][-1] - r["snapshots"]["eta"][-1]).max() <= 1e-9
