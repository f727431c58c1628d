"""A mixed-size batch (log-uniform sides, each scenario with its own
random-field bathymetry, seeded fault and duration, as the mixed workload
draws them, scaled down so that the FP64 oracle finishes in seconds) stepped
together by the multi-scenario runtime: each result's error against the
FP64 host oracle is reported and held to the parity tolerances (surface
within 1e-3 m, maximum height within 1e-4 relative L2, same steps)."""
import pytest

import oracle
from parity import ETA_TOL_M, MAXH_REL_L2, compare
from thysea import synth

pytestmark = pytest.mark.gpu


def test_mixed_batch_each_result_against_the_oracle(gpu):
    probs = synth.mixed(count=5, seed=41, side_range=(128, 384), time_range=(300.0, 900.0))
    srv = gpu.Server()
    ids = [srv.submit(p) for p in probs]
    srv.drain()
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(probs) and st["failed"] == 0
    rows = []
    for rid, p in zip(ids, probs):
        res = srv.results[rid]
        assert res["status"] == 0
        got = dict(res["outputs"])
        got["iterations"] = res["stats"]["steps"]
        got["final_time"] = res["stats"]["final_time_s"]
        c = compare(got, oracle.run_oracle(p), p.name)
        rows.append((p.name, p.nx, c["iterations"][0], c["eta_final_max_abs"], c["maxh_rel_l2"]))
        assert c["iterations"][0] == c["iterations"][1], p.name
        assert abs(c["final_time"][0] - c["final_time"][1]) < 1e-3 * max(1.0, c["final_time"][1])
        assert c["eta_final_max_abs"] <= ETA_TOL_M, p.name
        assert c["maxh_rel_l2"] <= MAXH_REL_L2, p.name
    for name, side, steps, e, m in rows:
        print(f"{name}: {side}^2, {steps} steps, max |d eta| {e:.2e} m, max-height rel L2 {m:.2e}")
