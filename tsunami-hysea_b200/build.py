"""Builds libthysea.so (kernels for sm_100a + host runtime + C ABI) and the
drop-in command-line program in this package directory.

    python tsunami-hysea_b200/build.py            # incremental
    python tsunami-hysea_b200/build.py --clean

nvcc cross-compiles without a GPU.  Objects go to _build/, the library to
lib/, the program to bin/.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib")
BIN = os.path.join(HERE, "bin")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = ["-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(CSRC, "nclite")]

CUDA_SOURCES = [
    "kernels/step.cu",
    "kernels/init_extract.cu",
    "kernels/okada.cu",
    "runtime/engine.cu",
    "runtime/server.cu",
    "runtime/tuner.cu",
    "runtime/okada_api.cu",
    "host/netcdf_out.cpp",
    "host/dropin.cpp",
    "host/problem.cpp",
]
C_SOURCES = ["nclite/nclite.c"]
# the library's exported symbols: the C ABI and shallowWater only
EXPORTS = os.path.join(CSRC, "exports.map")
# FP32 stepping kernels: approximate division / sqrt / exp (<= 2 ulp); the FP64
# Okada and set-up kernels keep IEEE arithmetic
FAST_MATH = {"kernels/step.cu"}


def _obj(src: str) -> str:
    return os.path.join(BUILD, src.replace("/", "_") + ".o")


def _deps_newer(src: str, obj: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    if os.path.getmtime(src) > t:
        return True
    for d in ("kernels", "runtime", "host", "nclite"):
        for f in os.listdir(os.path.join(CSRC, d)):
            if f.endswith((".h", ".cuh")) and os.path.getmtime(os.path.join(CSRC, d, f)) > t:
                return True
    hdr = os.path.join(ROOT, "include")
    for f in os.listdir(hdr):
        if os.path.getmtime(os.path.join(hdr, f)) > t:
            return True
    return False


def _compile(src: str, verbose: bool) -> str:
    path = os.path.join(CSRC, src)
    obj = _obj(src)
    if not _deps_newer(path, obj):
        return obj
    if src.endswith(".c"):
        cmd = ["gcc", "-O2", "-fPIC", "-std=c11", "-Wall", *INCLUDES, "-c", path, "-o", obj]
    else:
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-Wall",
               "--expt-relaxed-constexpr", *INCLUDES, "-c", path, "-o", obj]
        if src.endswith(".cpp"):
            cmd.insert(1, "-x")
            cmd.insert(2, "cu")
        if src in FAST_MATH:
            cmd.insert(1, "-use_fast_math")
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    sources = [s for s in CUDA_SOURCES + C_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), sources))
    so = os.path.join(LIB, "libthysea.so")
    if not os.path.exists(so) or any(os.path.getmtime(o) > os.path.getmtime(so) for o in objs + [EXPORTS]):
        cmd = [NVCC, *ARCH, "-shared", "-o", so, *objs, "-Xlinker", "--version-script=" + EXPORTS]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    # nclite on its own, with the NetCDF C API exported: for programs that
    # call nc_* themselves (the reference's own writers relinked against this
    # library, the tests of the NetCDF code); libthysea.so keeps its copy private
    nclite_so = os.path.join(LIB, "libnclite.so")
    nclite_src = os.path.join(CSRC, "nclite", "nclite.c")
    if not os.path.exists(nclite_so) or os.path.getmtime(nclite_src) > os.path.getmtime(nclite_so):
        cmd = ["gcc", "-O2", "-fPIC", "-shared", "-std=c11", "-Wall", *INCLUDES, nclite_src, "-o", nclite_so]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    main_src = os.path.join(CSRC, "host", "main.cpp")
    exe = os.path.join(BIN, "TsunamiHySEA")
    if os.path.exists(main_src) and (not os.path.exists(exe) or os.path.getmtime(so) > os.path.getmtime(exe)
                                     or os.path.getmtime(main_src) > os.path.getmtime(exe)):
        cmd = ["g++", "-O2", "-std=c++17", *INCLUDES, "-I/usr/local/cuda/include", main_src, "-o", exe,
               "-L" + LIB, "-lthysea", "-Wl,-rpath,$ORIGIN/../lib"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return so


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true", help="print ptxas register / spill report")
    a = ap.parse_args()
    if a.clean:
        for d in (BUILD, LIB, BIN):
            shutil.rmtree(d, ignore_errors=True)
    print(build(verbose=a.verbose))


if __name__ == "__main__":
    main()
