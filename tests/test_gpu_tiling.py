"""Warp tilings and their autotuner on the GPU: every tiling of the stepping
kernels gives bitwise the same results (a tiling only changes which warp
computes which cells), a run whose chunks the autotuner switches between
tilings gives the default tiling's results, and the tuner reaches a decision
on a session."""
import numpy as np
import pytest

import thysea
from thysea import synth

pytestmark = pytest.mark.gpu

FIELDS = ("max_height", "arrival", "eta", "ux", "uy")
TILINGS = [(0, 0, 0), (1, 0, 0), (2, 0, 0), (0, 1, 0), (0, 2, 0), (0, 0, 1), (0, 0, 2), (2, 1, 2), (1, 2, 1)]


def _problem():
    # deep ocean, shelf, coast and land (deep, general and dry units), with a
    # partial last tile in both directions
    p = synth.single_large(n=352, seed=31, sim_time=900.0)
    p.name = "tiling"
    return p


def _run(prep):
    r = thysea.run(prep, snapshots=False, series=False)
    return {k: r[k].copy() for k in FIELDS}, r


@pytest.fixture
def untuned():
    thysea.clear_tuner()
    yield
    thysea.force_tiling(None)
    thysea.clear_tuner()


def test_every_tiling_gives_the_same_results(gpu, untuned):
    prep = thysea.Prepared(_problem())
    thysea.force_tiling((0, 0, 0))
    ref, r0 = _run(prep)
    assert r0["iterations"] > 100 and r0["tiling"] == (0, 0, 0) and r0["tune_samples"] == 0
    assert r0["deep_tiles"] > 0 and r0["dry_tiles"] > 0
    for t in TILINGS[1:]:
        thysea.force_tiling(t)
        got, r = _run(prep)
        assert r["tiling"] == t and r["iterations"] == r0["iterations"]
        for k in FIELDS:
            assert np.array_equal(got[k], ref[k], equal_nan=True), (t, k)


def _tuned_problem():
    # enough work per step (640 units) for the autotuner, which leaves steps
    # of at most 512 units at the default tiling
    p = synth.single_large(n=1024, seed=31, sim_time=600.0)
    p.name = "tiling_tuned"
    return p


def test_small_steps_run_the_short_chain_tiling_untuned(gpu, untuned):
    r = thysea.run(thysea.Prepared(_problem()), snapshots=False, series=False)
    assert r["tune_samples"] == 0 and r["tiling"] == (0, 2, 2)


def test_autotuned_run_gives_the_default_results(gpu, untuned):
    prep = thysea.Prepared(_tuned_problem())
    thysea.force_tiling((0, 0, 0))
    ref, r0 = _run(prep)
    thysea.force_tiling(None)
    got, r = _run(prep)   # its chunks switch tilings while the tuner samples
    assert r["tune_samples"] > 0
    for k in FIELDS:
        assert np.array_equal(got[k], ref[k], equal_nan=True), k


def test_session_tune_decides(gpu, untuned):
    p = synth.single_large(n=1024, seed=32, sim_time=3600.0)
    s = thysea.Session(p)
    steps = s.tune()
    # 3 kernels x 3 candidates x 2 samples of one 16-step chunk each, after a
    # first chunk that measures the work mix (more when the mix moves into
    # another key meanwhile)
    assert 19 * 16 <= steps <= 80 * 16
    # decided for the session's current work (deep and general units per step)
    decided, best = s.tuned()
    assert decided and all(0 <= v < 3 for v in best)
    s.steps(16)
    decided, best = s.tuned()
    if decided:   # (the work may have moved into a new bucket meanwhile)
        assert s.tiling() == best
    s.close()
