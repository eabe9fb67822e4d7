"""Builds ``lib/libnecsim_b200.so`` in place with nvcc for sm_100a.

The kernels are compiled with ``--fmad=false`` (no multiply-add
contraction) and the host code with ``-ffp-contract=off``: every f64
operation rounds once, in source order, like the reference's.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libnecsim_b200.so")
DRIVER = os.path.join(LIB_DIR, "necsim-b200")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["kernels.cu", "noalloc.cu", "learned.cu"]
CPP_SOURCES = ["host.cpp", "tables.cpp", "event_log.cpp", "maps.cpp"]
DRIVER_SOURCES = ["driver.cpp", "ron.cpp"]


def _sources():
    out = []
    for name in os.listdir(CSRC):
        if name.endswith((".cu", ".cuh", ".cpp", ".h")):
            out.append(os.path.join(CSRC, name))
    out.append(os.path.join(HERE, "..", "include", "necsim_b200.h"))
    return out


def up_to_date():
    if not os.path.exists(LIB) or not os.path.exists(DRIVER):
        return False
    t = min(os.path.getmtime(LIB), os.path.getmtime(DRIVER))
    return all(os.path.getmtime(s) <= t for s in _sources())


def build(force=False, verbose=False):
    """Compile every CUDA/C++ source and link the shared library."""
    if not force and up_to_date():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
              "-I", CSRC]
    for src in CU_SOURCES:
        obj = os.path.join(obj_dir, src + ".o")
        cmd = [NVCC] + ARCH + common + ["-lineinfo", "--fmad=false", "-Xptxas", "-v",
                                        "-c", os.path.join(CSRC, src), "-o", obj]
        _run(cmd, verbose)
        objs.append(obj)
    for src in CPP_SOURCES:
        obj = os.path.join(obj_dir, src + ".o")
        cmd = [NVCC] + common + ["-x", "c++", "-c", os.path.join(CSRC, src), "-o", obj]
        _run(cmd, verbose)
        objs.append(obj)
    tmp = LIB + ".tmp"
    _run([NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lpthread", "-lz"], verbose)
    os.replace(tmp, LIB)
    # the rustcoalescence-style front end, linked against the library
    drv_objs = []
    for src in DRIVER_SOURCES:
        obj = os.path.join(obj_dir, src + ".o")
        _run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-c", os.path.join(CSRC, src), "-o", obj], verbose)
        drv_objs.append(obj)
    tmp = DRIVER + ".tmp"
    _run(["g++", "-o", tmp] + drv_objs + ["-L" + LIB_DIR, "-lnecsim_b200", "-Wl,-rpath,$ORIGIN"], verbose)
    os.replace(tmp, DRIVER)
    return LIB


def _run(cmd, verbose):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("build step failed: " + " ".join(cmd[:4]))


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
