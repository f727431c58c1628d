"""The GPU path against the golden fixtures of the reference's own code
(tests/golden/): same step count, surface within 1e-3 m, maximum height
within 1e-4 relative L2, gauges within 1e-3 m."""
import os

import numpy as np
import pytest

from golden import cases
from parity import ETA_TOL_M, MAXH_REL_L2, max_abs_eta, rel_l2

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", list(cases.CASES))
def test_gpu_matches_reference_fixture(gpu, name):
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    p = cases.CASES[name]()
    r = gpu.run(p)
    assert r["iterations"] == int(g["iterations"])
    assert abs(r["final_time"] - float(g["final_time"])) < 1e-3
    assert rel_l2(r["max_height"], g["max_height"]) <= MAXH_REL_L2
    snaps = r["snapshots"]
    assert len(snaps["time"]) == len(g["snap_time"])
    assert np.abs(np.asarray(snaps["time"]) - g["snap_time"]).max() < 1e-3
    assert max_abs_eta(snaps["eta"][-1], g["eta_last"]) <= ETA_TOL_M
    arr_ok = np.abs(r["arrival"] - g["arrival_times"]) <= 30.0
    assert arr_ok.mean() > 0.99
    if "ts_eta" in g:
        assert np.abs(np.asarray(r["series"]["eta"]) - g["ts_eta"]).max() <= ETA_TOL_M
        assert np.abs(r["series"]["max"] - g["ts_max"]).max() <= ETA_TOL_M
