"""Failure detection on the GPU without a fault: every wait of the deep-water
kernels is bounded (four seconds of global time), so a staging copy that does not
land stops the step with THY_ERR_TIMEOUT instead of hanging.  The test hook
thy_session_inject makes the kernels issue none of a session's copies (a
flag that nothing sets); afterwards the context still runs other work, with
the same results as before."""
import numpy as np
import pytest

import thysea
from thysea import synth

pytestmark = pytest.mark.gpu


def _small():
    p = synth.plain_small(nx=256, ny=224, seed=5, sim_time=200.0, save_time=-1.0, npoints=0)
    p.name = "after_timeout"
    return p


def test_copy_timeout_is_reported_and_the_context_survives(gpu):
    before = thysea.run(_small(), snapshots=False, series=False)
    s = thysea.Session(synth.single_large(n=640, seed=33, sim_time=3600.0))
    _, k = s.steps(32)
    assert k == 32
    t0, d0, _ = s.tiles()
    _, k = s.steps(16)
    t1, d1, _ = s.tiles()
    assert d1 > d0   # the deep-water kernels step this problem
    s.inject(1)
    with pytest.raises(thysea.ThyError) as e:
        s.steps(16)
    assert e.value.code == thysea.THY_ERR_TIMEOUT
    s.close()
    after = thysea.run(_small(), snapshots=False, series=False)
    assert after["iterations"] == before["iterations"]
    for key in ("max_height", "arrival", "eta", "ux", "uy"):
        assert np.array_equal(after[key], before[key], equal_nan=True), key
