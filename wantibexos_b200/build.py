"""Build recipe for libwtbgpu.so (sm_100a) and the wtb_bse driver, in-tree.

Usage: python -m wantibexos_b200.build  (or call build()).  nvcc cross-compiles for
sm_100a without a GPU; the outputs land next to this file so they travel with the tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libwtbgpu.so")
SOURCES = ["api.cu", "bands.cu", "bse_build.cu", "tridiag.cu", "tridiag2.cu", "tdeig.cu", "spectrum.cu", "davidson.cu", "haydock.cu", "fastprod.cu", "learned.cu", "temperature.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
              "-I" + os.path.join(ROOT, "include")]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _newer(target: str, deps: list) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + \
        [os.path.join(ROOT, "include", "wtbgpu.h")]
    if not force and _newer(LIB, deps):
        build_driver(verbose=verbose)
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = [os.path.join(objdir, os.path.basename(s) + ".o") for s in srcs]

    def compile_one(pair):
        src, obj = pair
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)

    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        list(ex.map(compile_one, zip(srcs, objs)))
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB + ".tmp"] + objs
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    build_driver(force=True, verbose=verbose)
    return LIB


DRIVER_LIB = os.path.join(HERE, "libwtbdriver.so")
DRIVER_EXE = os.path.join(HERE, "wtb_bse")


def build_driver(force: bool = False, verbose: bool = False) -> str:
    """Compile the C++ host driver (libwtbdriver.so + the wtb_bse executable) against libwtbgpu.so."""
    src = os.path.join(HERE, "driver", "wtb_driver.cpp")
    main = os.path.join(HERE, "driver", "wtb_main.cpp")
    hdrs = [os.path.join(ROOT, "include", "wtb_driver.h"), os.path.join(ROOT, "include", "wtbgpu.h")]
    if not force and _newer(DRIVER_LIB, [src] + hdrs + [LIB]) and _newer(DRIVER_EXE, [main, DRIVER_LIB]):
        return DRIVER_LIB
    gxx = shutil.which("g++") or "g++"
    rpath = "-Wl,-rpath,$ORIGIN"
    cmd = [gxx, "-O2", "-std=c++17", "-pthread", "-fPIC", "-shared", "-I" + os.path.join(ROOT, "include"), src,
           "-o", DRIVER_LIB + ".tmp", "-L" + HERE, "-lwtbgpu", rpath]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(DRIVER_LIB + ".tmp", DRIVER_LIB)
    cmd = [gxx, "-O2", "-std=c++17", "-pthread", "-I" + os.path.join(ROOT, "include"), main, "-o", DRIVER_EXE + ".tmp",
           "-L" + HERE, "-lwtbdriver", "-lwtbgpu", rpath]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(DRIVER_EXE + ".tmp", DRIVER_EXE)
    return DRIVER_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
