"""The tiling autotuner's search (runtime/tuner.cu) on the host: the tuner is
compiled with tests/native/tuner_driver.cpp, which feeds it synthetic chunk
times the way the batch loop does; plus the C ABI's argument checks."""
import ctypes
import os
import subprocess

import pytest

import thysea
from thysea import _ffi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "tsunami-hysea_b200", "csrc")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("tuner") / "tuner_driver")
    cmd = ["g++", "-std=c++17", "-O1", "-I" + CSRC, "-I" + os.path.join(CUDA, "include"), "-x", "c++",
           os.path.join(CSRC, "runtime", "tuner.cu"), "-x", "c++", os.path.join(ROOT, "tests", "native", "tuner_driver.cpp"),
           "-L" + os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _run(exe, scenario, env=None):
    e = dict(os.environ)
    for k in ("THY_TILING", "THY_TUNE", "THY_TUNE_CACHE"):
        e.pop(k, None)
    e.update(env or {})
    r = subprocess.run([exe, scenario], capture_output=True, text=True, env=e, timeout=60)
    assert r.returncode == 0, r.stderr
    return r.stdout.split("\n")


def _field(line, key):
    return dict(kv.split("=") for kv in line.split()[1:])[key]


def test_coordinate_descent_finds_the_best_per_kernel(driver):
    out = _run(driver, "descent")
    # 3 kernels x 3 candidates x 2 rounds = 18 timed chunks
    assert _field(out[0], "done") == "1" and _field(out[0], "tiling") == "2,1,0" and _field(out[0], "chunks") == "18"


def test_an_alternative_must_be_one_percent_faster(driver):
    assert _field(_run(driver, "margin")[0], "tiling") == "0,0,0"


def test_stale_samples_are_ignored(driver):
    out = _run(driver, "stale")
    assert _field(out[0], "first") == "0,0,0"
    assert _field(out[1], "tiling") == "1,0,0" and _field(out[1], "chunks") == "18"


def test_minimum_over_noisy_samples(driver):
    assert _field(_run(driver, "noisy")[0], "tiling") == "2,1,0"


def test_size_buckets_are_independent(driver):
    out = _run(driver, "keys")
    assert _field(out[0], "tiling") == "1,0,0"
    assert _field(out[1], "tiling") == "0,0,2"
    assert out[2] == "bucket 1=0 2=1 3=2 1024=10 1025=11"


def test_small_steps_are_not_tuned(driver):
    out = _run(driver, "small")
    assert _field(out[0], "pick") == "0,2,2" and _field(out[0], "sampling") == "0"
    assert _field(out[0], "done") == "1" and _field(out[0], "best") == "0,2,2"
    assert _field(out[1], "sampling") == "1"


def test_forced_tiling_and_environment(driver):
    out = _run(driver, "force")
    assert _field(out[0], "pick") == "2,1,2" and _field(out[0], "sampling") == "0"
    assert _field(out[1], "pick") == "0,0,0" and _field(out[1], "sampling") == "1"
    # THY_TILING forces; THY_TUNE=0 keeps the default without sampling
    out = _run(driver, "descent", {"THY_TILING": "1,2,1"})
    assert _field(out[0], "tiling") == "1,2,1" and _field(out[0], "chunks") == "0"
    out = _run(driver, "descent", {"THY_TUNE": "0"})
    assert _field(out[0], "tiling") == "0,0,0" and _field(out[0], "chunks") == "0"


def test_cache_file_round_trip(driver, tmp_path):
    path = str(tmp_path / "tune.txt")
    out = _run(driver, "cache", {"THY_TUNE_CACHE": path})
    assert _field(out[0], "tiling") == "1,2,0" and _field(out[0], "chunks") == "18"
    # read back after the in-process state is cleared: decided without samples
    assert _field(out[1], "done") == "1" and _field(out[1], "tiling") == "1,2,0"
    lines = open(path).read().split("\n")
    assert lines[0].split()[2:] == ["13", "10", "1", "2", "0"]   # deep and general buckets, tiling
    # a second process starts decided from the file
    out = _run(driver, "cache", {"THY_TUNE_CACHE": path})
    assert _field(out[0], "chunks") == "0" and _field(out[0], "tiling") == "1,2,0"


def test_abi_checks_tiling_arguments():
    L = _ffi.lib()
    assert L.thy_tiling_force(ctypes.byref(_ffi.Tiling(3, 0, 0))) == thysea.THY_ERR_INVALID
    assert L.thy_tiling_force(ctypes.byref(_ffi.Tiling(0, -1, 0))) == thysea.THY_ERR_INVALID
    assert L.thy_tiling_force(ctypes.byref(_ffi.Tiling(2, 2, 2))) == 0
    assert L.thy_tiling_force(None) == 0
    assert L.thy_session_tune(None, 10, None) == thysea.THY_ERR_INVALID
    assert L.thy_session_tiling(None, None) == thysea.THY_ERR_INVALID
    assert L.thy_session_tuned(None, None) == thysea.THY_ERR_INVALID
    assert L.thy_session_inject(None, 1) == thysea.THY_ERR_INVALID
    assert set(thysea.TILING_GROUPS) == {"deep1", "deep2", "general"}
