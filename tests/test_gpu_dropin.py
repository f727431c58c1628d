"""The drop-in, end to end on problem files: the reference's own program
(src/ShallowWater.cxx with its loader and NetCDF writers, relinked against
libthysea.so in place of its GPU code; oracle/_ref/TsunamiHySEA_refmain) and
this library's TsunamiHySEA program each run a problem file and write
<prefix>.nc and <prefix>_ts.nc.  Against the files the reference's own code
writes for the same problem (ref-emu): the same dimensions, variables and
attributes, the same snapshot and gauge times, surfaces within 1e-3 m and
maximum height within 1e-4 relative L2."""
import os
import subprocess

import numpy as np
import pytest
from scipy.io import netcdf_file

import oracle
from parity import ETA_TOL_M, MAXH_REL_L2, max_abs_eta, rel_l2
from thysea import synth

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFMAIN = os.path.join(ROOT, "oracle", "_ref", "TsunamiHySEA_refmain")
CLI = os.path.join(ROOT, "tsunami-hysea_b200", "bin", "TsunamiHySEA")


def _problem():
    p = synth.plain_small(nx=256, ny=224, seed=7, sim_time=500.0, save_time=150.0, series_time=50.0, npoints=6)
    p.name = "dropin"
    return p


def _read(path):
    f = netcdf_file(path, "r", mmap=False)
    out = {"dims": dict(f.dimensions), "attrs": sorted(f._attributes.keys()), "vars": {}}
    for k, v in f.variables.items():
        out["vars"][k] = (v.dimensions, sorted(v._attributes.keys()), np.array(v.data))
    f.close()
    return out


def _run_program(exe, tmp_path, sub):
    d = tmp_path / sub
    d.mkdir()
    txt = synth.write_problem(_problem(), str(d))
    r = subprocess.run([exe, txt], cwd=str(d), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return str(d / "dropin")


@pytest.fixture(scope="module")
def reference_files(tmp_path_factory):
    if not oracle.refemu_available():
        pytest.fail("oracle/_ref/librefemu.so is not built")
    d = tmp_path_factory.mktemp("refemu")
    txt = synth.write_problem(_problem(), str(d))
    oracle.run_refemu(txt)
    return str(d / "dropin")


def _compare(prefix, ref_prefix):
    got, ref = _read(prefix + ".nc"), _read(ref_prefix + ".nc")
    assert got["dims"] == ref["dims"]
    assert got["attrs"] == ref["attrs"]
    assert sorted(got["vars"]) == sorted(ref["vars"])
    for k, (dims, attrs, _) in ref["vars"].items():
        assert got["vars"][k][0] == dims and got["vars"][k][1] == attrs, k
    for k in ("lon", "lat", "time", "original_bathy"):
        assert np.allclose(got["vars"][k][2], ref["vars"][k][2], rtol=0, atol=1e-3), k
    assert rel_l2(got["vars"]["max_height"][2], ref["vars"]["max_height"][2]) <= MAXH_REL_L2
    for i in range(len(ref["vars"]["time"][2])):
        assert max_abs_eta(got["vars"]["eta"][2][i], ref["vars"]["eta"][2][i]) <= ETA_TOL_M
    gts, rts = _read(prefix + "_ts.nc"), _read(ref_prefix + "_ts.nc")
    assert gts["dims"] == rts["dims"] and sorted(gts["vars"]) == sorted(rts["vars"])
    assert np.allclose(gts["vars"]["time"][2], rts["vars"]["time"][2], rtol=0, atol=1e-3)
    assert np.abs(gts["vars"]["eta"][2] - rts["vars"]["eta"][2]).max() <= ETA_TOL_M


def test_reference_main_relinked_against_libthysea(reference_files, tmp_path):
    if not os.path.exists(REFMAIN):
        pytest.fail("oracle/_ref/TsunamiHySEA_refmain is not built (make -C oracle ref)")
    _compare(_run_program(REFMAIN, tmp_path, "refmain"), reference_files)


def test_library_program_on_the_problem_file(reference_files, tmp_path):
    _compare(_run_program(CLI, tmp_path, "cli"), reference_files)
