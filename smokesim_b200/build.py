"""Build libsmokesim.so in-tree with nvcc for sm_100a.

    python -m smokesim_b200.build [--force]

The kernels are compiled with -fmad=false (no multiply-add contraction) and
the default IEEE division / square root, so every cell rounds exactly like the
CPU oracle's FP32 build.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG_DIR, "csrc")
OUT = os.path.join(PKG_DIR, "libsmokesim.so")
BUILD_DIR = os.path.join(PKG_DIR, "_build")

SOURCES = ["api.cpp", "k_fluid.cu", "k_mg.cu", "k_rbgs.cu", "k_rbgs_tma.cu", "k_rb.cu", "k_scene.cu", "k_mixed.cu", "k_adjoint.cu", "adjoint.cpp", "k_render.cu", "state_io.cpp", "k_noalloc.cu"]
HEADERS = ["common.cuh", "ss_internal.h", "tma.cuh"]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr"]


def _stale(force):
    if force or not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(os.path.dirname(PKG_DIR), "include", "smokesim.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not _stale(force):
        return OUT
    os.makedirs(BUILD_DIR, exist_ok=True)
    env = dict(os.environ)
    # the image's CC/CXX wrappers lack libgomp; nvcc drives the system g++
    env.pop("CC", None)
    env.pop("CXX", None)
    def compile_one(src):
        obj = os.path.join(BUILD_DIR, os.path.splitext(src)[0] + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        return src, obj, r

    # the translation units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor
    jobs = max(1, min(len(SOURCES), os.cpu_count() or 1))
    with ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(compile_one, SOURCES))
    objs = []
    for src, obj, r in results:
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}")
        if verbose and r.stdout:
            print(r.stdout)
        objs.append(obj)
    tmp = OUT + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    r = subprocess.run(cmd, env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stdout}")
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
