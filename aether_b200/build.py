"""Builds the CUDA library aether_b200/libaefdtd.so for sm_100a, in-tree.

    python -m aether_b200.build [--force]

FP64 kernels are compiled with --fmad=false (the reference's x86-64 build
rounds every multiply and add separately); FP32 kernels may contract.
Objects go to aether_b200/_build/; the library lands next to this file."""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libaefdtd.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++20", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
           "--expt-relaxed-constexpr"] + ARCH
CXXFLAGS = ["-std=c++20", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
            f"-I{CUDA_HOME}/include"]

# (source, extra flags)
UNITS = [
    ("yee_f64.cu", ["--fmad=false"]),
    ("yee_f32.cu", []),
    ("leapfrog_f64.cu", ["--fmad=false"]),
    ("leapfrog_f32.cu", []),
    ("sensors.cu", []),
    ("dft_tc.cu", []),
    ("voxel.cu", ["--fmad=false"]),
    ("plane_static.cu", []),
    ("probe.cu", []),
    ("oblique.cu", ["--fmad=false"]),
    ("runtime.cpp", None),
    ("fused.cpp", None),
    ("tma.cpp", None),
    ("oblique_driver.cpp", None),
    ("batch.cpp", None),
    ("server.cpp", None),
]
HEADERS = ["aefdtd_dev.hpp", "kernels.hpp", "sensors.cuh", "yee.cuh", "leapfrog.cuh", "sim.hpp", "mbar.cuh",
           "interior_tma.cuh", "batch_persist.cuh", "pulse.cuh"]


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, extra):
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    deps = [path, __file__, os.path.join(ROOT, "include", "aefdtd.h")] + [os.path.join(CSRC, h) for h in HEADERS]
    if not _stale(obj, deps):
        return obj, None
    if extra is None:
        cmd = ["g++"] + CXXFLAGS + ["-c", path, "-o", obj]
    else:
        cmd = [NVCC] + NVFLAGS + extra + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    return obj, None


def build(force: bool = False, verbose: bool = False) -> str:
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    if force and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        res = list(ex.map(lambda u: _compile(*u), UNITS))
    errs = [e for _, e in res if e]
    if errs:
        raise RuntimeError("build failed:\n" + "\n".join(errs))
    objs = [o for o, _ in res]
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
