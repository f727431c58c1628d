"""The reference CUDA build against this library, on the same problem files.

oracle/_ref/TsunamiHySEA_refgpu is the reference's own program (main, loader
and NetCDF writers) with its own GPU stepper (src/GPU/ShallowWater.cu and the
edge, cell, reduction, Okada and metrics kernels it includes), compiled by
nvcc for sm_100a as its Release build does, NetCDF through nclite.  It is
FP64 throughout.  Beside it runs this library's TsunamiHySEA program, which
has the reference's command line and output files.

* parity: snapshots (after asserting equal snapshot times) within 1e-3 m,
  gauges within 1e-3 m, maximum height within 1e-4 relative L2.  The grids
  have at least 65 536 cells: below that the reference's min-reduction of
  the time step (src/GPU/Reduccion_kernel.cu:130-160) skips its second pass
  whenever the first pass's block count is not a power of two, and its dt is
  then the minimum over a subset of the cells;
* head to head on the plain small workload (512 x 512 cells, one Okada
  fault, 600 s simulated, snapshots every 300 s) and the single large one
  (4096 x 4096 cells, four Okada subfaults, 3600 s, snapshots every 1800 s):
  both programs print their loop wall time ("Runtime: ... sec", the
  reference's *tiempo), which includes Okada and the snapshot writes in both;
  cell-updates/s = cells x iterations / runtime, printed for both.  On the
  4096 x 4096 grid this library must step the same problem faster; at
  512 x 512 both loop times are mostly fixed per-run and per-step work
  (0.15 ms a step for 0.26 M cells), so only parity is asserted there.
"""
import json
import os
import re
import subprocess

import numpy as np
import pytest
from scipy.io import netcdf_file

from parity import ETA_TOL_M, MAXH_REL_L2, max_abs_eta, rel_l2
from thysea import synth

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFGPU = os.path.join(ROOT, "oracle", "_ref", "TsunamiHySEA_refgpu")
CLI = os.path.join(ROOT, "tsunami-hysea_b200", "bin", "TsunamiHySEA")


def _vars(path):
    f = netcdf_file(path, "r", mmap=False)
    out = {k: np.array(v.data) for k, v in f.variables.items()}
    f.close()
    return out


def _run(exe, p, d):
    os.makedirs(d, exist_ok=True)
    txt = synth.write_problem(p, d)
    r = subprocess.run([exe, txt], cwd=d, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    runtime = float(re.findall(r"Runtime: ([0-9.eE+-]+) sec", r.stdout)[-1])
    its = re.findall(r"Iteration\s+(\d+),", r.stdout)          # the reference: one line per step
    if its:
        iterations = int(its[-1])
    else:
        iterations = int(re.findall(r"Iterations: (\d+),", r.stdout)[-1])
    return os.path.join(d, p.name), runtime, iterations


def _compare(prefix, ref_prefix, gauges=True, same_times=True):
    """same_times=False: FP32 and FP64 time steps may drift apart by a step
    over a long run, which moves a snapshot by one step; then only snapshots
    whose recorded times agree are compared (t = 0 always does)"""
    got, ref = _vars(prefix + ".nc"), _vars(ref_prefix + ".nc")
    assert len(got["time"]) == len(ref["time"])
    same = np.abs(got["time"] - ref["time"]) <= 1e-3
    assert same.all() if same_times else same[0]
    assert rel_l2(got["max_height"], ref["max_height"]) <= MAXH_REL_L2
    errs = [max_abs_eta(got["eta"][i], ref["eta"][i]) for i in range(len(ref["time"])) if same[i]]
    assert max(errs) <= ETA_TOL_M, errs
    if gauges:
        gts, rts = _vars(prefix + "_ts.nc"), _vars(ref_prefix + "_ts.nc")
        assert np.allclose(gts["time"], rts["time"], rtol=0, atol=1e-3)
        assert np.abs(gts["eta"] - rts["eta"]).max() <= ETA_TOL_M
    return max(errs), rel_l2(got["max_height"], ref["max_height"])


@pytest.fixture(scope="module")
def refgpu():
    if not os.path.exists(REFGPU):
        pytest.fail("oracle/_ref/TsunamiHySEA_refgpu is not built (make -C oracle ref)")
    return REFGPU


def test_parity_with_reference_cuda_build(refgpu, tmp_path):
    p = synth.plain_small(nx=288, ny=256, seed=7, sim_time=500.0, save_time=150.0, series_time=50.0, npoints=6)
    p.name = "refgpu_small"
    ref, _, ref_it = _run(refgpu, p, str(tmp_path / "ref"))
    got, _, got_it = _run(CLI, p, str(tmp_path / "got"))
    assert got_it == ref_it
    _compare(got, ref)


HEAD_TO_HEAD = {
    "plain_small_512": ("plain_small 512x512, 1 Okada fault, 600 s, snapshots every 300 s",
                        lambda: synth.plain_small(nx=512, ny=512, sim_time=600.0, save_time=300.0, npoints=16)),
    "single_large_4096": ("single_large 4096x4096, 4 Okada subfaults, 3600 s, snapshots every 1800 s",
                          lambda: synth.single_large(n=4096, sim_time=3600.0, save_time=1800.0)),
}


@pytest.mark.parametrize("workload", sorted(HEAD_TO_HEAD))
def test_head_to_head(refgpu, tmp_path, workload):
    name, make = HEAD_TO_HEAD[workload]
    p = make()
    p.name = "refgpu_" + workload
    ref, ref_s, ref_it = _run(refgpu, p, str(tmp_path / "ref"))
    got, got_s, got_it = _run(CLI, p, str(tmp_path / "got"))
    cells = p.nx * p.ny
    eta_err, maxh_err = _compare(got, ref, gauges=False, same_times=False)
    rec = {"workload": name,
           "reference_cuda": {"runtime_s": ref_s, "iterations": ref_it, "cell_updates_per_s": cells * ref_it / ref_s},
           "thysea": {"runtime_s": got_s, "iterations": got_it, "cell_updates_per_s": cells * got_it / got_s},
           "max_abs_eta_m": eta_err, "max_height_rel_l2": maxh_err}
    print("REFGPU " + json.dumps(rec))
    assert abs(got_it - ref_it) <= 2
    if workload == "single_large_4096":
        assert cells * got_it / got_s > cells * ref_it / ref_s
    else:
        # the small grid: fixed per-run and per-step costs dominate both loops
        # (graphs captured before the loop, short-chain tiling); at least 3x
        assert got_s * 3.0 <= ref_s, (got_s, ref_s)
