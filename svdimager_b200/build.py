"""Build the in-tree sm_100a library and command-line tools.

    python -m svdimager_b200.build            # incremental
    python -m svdimager_b200.build --force

Outputs (git-ignored, shipped with the tree):
    svdimager_b200/lib/libsvdimager_b200.so   C ABI of include/svdimager_b200.h
    svdimager_b200/bin/sharedlibrary_gpu       archive CLI (archive/pipe_interface.cpp argv)
    svdimager_b200/bin/svd_integrated_imager_gpu  main CLI (SVDIntegratedImager.cu argv)
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "lib")
BIN_DIR = os.path.join(HERE, "bin")
LIB = os.path.join(LIB_DIR, "libsvdimager_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
           "--expt-relaxed-constexpr", "-I", INCLUDE] + ARCH
CU_SOURCES = ["preprocess.cu", "binning.cu", "gridder.cu", "gridder_tc.cu", "gridder_i8.cu", "fft_cols.cu", "image.cu", "engine.cu", "server.cu",
              "noalloc.cu", "accuracy.cu", "host_stage.cu", "sii_entry.cpp"]
# diagnostics built beside the CLIs: tcgen05 MMA issue rates and operand-layout check, shared-memory
# reduction rates (the measurements behind the gridders' design)
PROBE_SOURCES = {"probe_tcgen05_mma": "probe_tcgen05_mma.cu", "probe_shared_red": "probe_shared_red.cu"}
CLI_SOURCES = {"sharedlibrary_gpu": ["fits.cpp", "cli_sharedlibrary_gpu.cpp"],
               "svd_integrated_imager_gpu": ["fits.cpp", "bundle.cpp", "cli_svd_integrated_imager_gpu.cpp"]}


def _deps(src):
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    return [src] + headers + [os.path.join(INCLUDE, h) for h in os.listdir(INCLUDE)]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(BIN_DIR, exist_ok=True)
    objs, jobs = [], []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, _deps(s)):
            jobs.append([NVCC] + NVFLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", "-o", o, s])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        logs = list(ex.map(_run, jobs))
    if verbose:
        for l in logs:
            sys.stdout.write(l)
    if force or jobs or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcufft", "-lcudart"])
    for name, srcs in CLI_SOURCES.items():
        paths = [os.path.join(CSRC, s) for s in srcs]
        out = os.path.join(BIN_DIR, name)
        if all(os.path.exists(p) for p in paths) and (force or _stale(out, paths + [LIB])):
            _run(["g++", "-O2", "-std=c++17", "-I", INCLUDE, "-o", out] + paths +
                 ["-L", LIB_DIR, "-lsvdimager_b200", "-Wl,-rpath,$ORIGIN/../lib",
                  "-L/usr/local/cuda/lib64", "-lcudart"])
    for name, src in PROBE_SOURCES.items():
        path = os.path.join(CSRC, src)
        out = os.path.join(BIN_DIR, name)
        if os.path.exists(path) and (force or _stale(out, [path])):
            _run([NVCC, "-O3", "-std=c++17", "-lineinfo"] + ARCH + ["-o", out, path])
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
