"""The multi-scenario runtime (thy_server_*): scenarios stepped together in
one batch give bitwise the results they give alone (thy_run); admission
under an HBM budget queues what does not fit; cancelled, rejected and failing
requests are retired without disturbing the others."""
import numpy as np
import pytest

import thysea
from thysea import synth

pytestmark = pytest.mark.gpu

FIELDS = ("max_height", "arrival", "eta", "ux", "uy", "deformed_bathy")


def _mix():
    """Three scenarios of different sizes, sources and borders, with deep,
    coastal and dry units."""
    a = synth.single_large(n=320, seed=21, sim_time=600.0)
    a.name = "mix_a"
    b = synth.plain_small(nx=256, ny=192, seed=22, sim_time=450.0, save_time=-1.0, npoints=0)
    b.name = "mix_b"
    c = synth.single_large(n=288, seed=23, sim_time=700.0)
    c.name = "mix_c"
    c.borders = (1.0, -1.0, 2.0, 2.0)
    return [a, b, c]


def _alone(p):
    r = thysea.run(p, snapshots=False, series=False)
    return {k: r[k] for k in FIELDS}, r["iterations"]


def _assert_same(got, ref):
    for k in FIELDS:
        assert np.array_equal(got[k], ref[k], equal_nan=True), k


def test_batch_matches_alone_bitwise(gpu):
    probs = _mix()
    alone = [_alone(p) for p in probs]
    srv = thysea.Server()
    ids = [srv.submit(p) for p in probs]
    srv.drain()
    st = srv.stats()
    srv.close()
    assert st["completed"] == 3 and st["failed"] == 0
    for rid, (ref, steps) in zip(ids, alone):
        res = srv.results[rid]
        assert res["status"] == 0
        assert res["stats"]["steps"] == steps
        _assert_same(res["outputs"], ref)


def test_budget_queues_and_results_stay_identical(gpu):
    probs = _mix()
    alone = [_alone(p) for p in probs]
    # room for one scenario at a time (~60 B per cell): the others wait in the queue
    budget = max(p.nx * p.ny for p in probs) * 64
    srv = thysea.Server(hbm_budget_bytes=budget)
    ids = [srv.submit(p) for p in probs]
    max_running = 0
    while srv.progress() > 0:
        max_running = max(max_running, srv.stats()["running"])
    srv.close()
    assert max_running == 1
    for rid, (ref, steps) in zip(ids, alone):
        assert srv.results[rid]["status"] == 0
        assert srv.results[rid]["stats"]["setup_seconds"] >= 0.0
        _assert_same(srv.results[rid]["outputs"], ref)


def test_cancel_and_reject(gpu):
    probs = _mix()
    srv = thysea.Server(hbm_budget_bytes=int(1.2 * 320 * 320 * 64))
    keep = srv.submit(probs[0])
    dropped = srv.submit(probs[1])          # queued behind the first
    srv.cancel(dropped)
    assert srv.results[dropped]["status"] == thysea.THY_ERR_CANCELLED
    big = synth.single_large(n=1024, seed=3, sim_time=60.0)
    with pytest.raises(thysea.ThyError) as e:
        srv.submit(big)                      # can never fit this budget
    assert e.value.code == thysea.THY_ERR_BUDGET
    running = srv.submit(probs[2])
    srv.progress()
    srv.cancel(keep)                         # cancelled between chunks while running
    srv.drain()
    st = srv.stats()
    srv.close()
    assert srv.results[keep]["status"] == thysea.THY_ERR_CANCELLED
    assert srv.results[running]["status"] == 0
    assert st["rejected"] == 1 and st["cancelled"] == 2 and st["completed"] == 1


def test_nonfinite_scenario_retires_alone(gpu):
    """a scenario whose state is not finite fails with THY_ERR_NONFINITE; the
    batch it shares keeps stepping and its other results are unchanged"""
    probs = _mix()
    ref, steps = _alone(probs[0])
    bad = synth.plain_small(nx=192, ny=160, seed=5, sim_time=300.0, save_time=-1.0, npoints=0)
    bad.faults = []
    e0 = np.zeros((bad.ny, bad.nx), np.float32)
    e0[80, 60] = 1e30    # finite input whose fluxes overflow in the first step
    bad.eta_init = e0
    srv = thysea.Server()
    good = srv.submit(probs[0])
    fail = srv.submit(bad)
    srv.drain()
    srv.close()
    assert srv.results[fail]["status"] == thysea.THY_ERR_NONFINITE
    assert srv.results[good]["status"] == 0
    assert srv.results[good]["stats"]["steps"] == steps
    _assert_same(srv.results[good]["outputs"], ref)
