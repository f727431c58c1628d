"""Generates the golden fixtures in this directory by running the
reference's own time stepper compiled for the host (oracle/_ref/librefemu.so,
built by `make -C oracle ref` from the reference tree) on small seeded
problems, through its own loader and NetCDF writers.

    python tests/golden/make_golden.py

Each case writes <case>.npz: max_height, arrival_times, the last eta / ux / uy
snapshot and its time, gauge eta series, iteration count and final time.
The reference ships no tests or golden data of its own, so these runs of its
code are the pin for the FP64 oracle (tests/test_oracle_golden.py) and the
GPU path (tests/test_gpu_golden.py).
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tsunami-hysea_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

import cases  # noqa: E402
import oracle  # noqa: E402
from thysea import synth  # noqa: E402


def run_case(name, p):
    from scipy.io import netcdf_file

    d = tempfile.mkdtemp(prefix="golden_")
    txt = synth.write_problem(p, d)
    info = oracle.run_refemu(txt)
    out = {"iterations": np.int64(info["iterations"]), "final_time": np.float64(info["final_time"]),
           "first_dt": np.float64(info["first_dt"])}
    with netcdf_file(os.path.join(d, p.name + ".nc"), "r", mmap=False) as f:
        out["max_height"] = f.variables["max_height"][:].copy()
        out["arrival_times"] = f.variables["arrival_times"][:].copy()
        out["snap_time"] = f.variables["time"][:].copy()
        for k in ("eta", "ux", "uy"):
            out[k + "_last"] = f.variables[k][-1].copy()
        if "deformed_bathy" in f.variables:
            out["deformed_bathy"] = f.variables["deformed_bathy"][:].copy()
    ts = os.path.join(d, p.name + "_ts.nc")
    if os.path.exists(ts):
        with netcdf_file(ts, "r", mmap=False) as f:
            out["ts_eta"] = f.variables["eta"][:].copy()
            out["ts_time"] = f.variables["time"][:].copy()
            out["ts_min"] = f.variables["min_height"][:].copy()
            out["ts_max"] = f.variables["max_height"][:].copy()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, p.nx, p.ny, "iterations", info["iterations"], "final time", info["final_time"])


def main():
    if not oracle.refemu_available():
        raise SystemExit("oracle/_ref/librefemu.so missing: run `make -C oracle ref` with the reference tree present")
    for name, make in cases.CASES.items():
        run_case(name, make())


if __name__ == "__main__":
    main()
