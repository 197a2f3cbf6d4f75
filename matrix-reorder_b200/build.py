"""Builds the in-tree shared libraries of the package.

  libmr.so      CUDA kernels for sm_100a + host C++ + the C-ABI of include/mr.h
  libmr_gen.so  seeded synthetic workload generators (host C++, OpenMP)

Every CUDA source is compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; the CUDA
runtime is linked statically so the library does not depend on which
libcudart another component of the process (e.g. torch) loaded first.
Rebuilds only what is out of date. Usage: ``python build.py [--force] [-v]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(REPO, "include")
OBJ = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I" + INCLUDE, "-I" + CSRC] + ARCH
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-ffp-contract=off",
             "-I" + INCLUDE, "-I" + CSRC, "-I/usr/local/cuda/include"]

CU_SOURCES = ["abi.cu", "merbit.cu", "csr.cu", "permute.cu", "rd_exact.cu", "rd_hll.cu", "graph.cu",
              "batch.cu", "serve.cu", "noalloc.cu", "probe.cu", "producers.cu", "pgorder_gpu.cu"]
CXX_SOURCES = ["pgorder.cpp", "predictor.cpp"]
HEADERS = ["common.cuh", "internal.hpp", "merbit_tile.cuh"]

LIBMR = os.path.join(HERE, "libmr.so")
LIBGEN = os.path.join(HERE, "libmr_gen.so")


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    # the system g++ (an environment CXX may point at a wrapper without OpenMP)
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout.strip() or r.stderr.strip()):
        print(r.stdout, r.stderr, flush=True)


def build(force: bool = False, verbose: bool = False, extra_nvcc: list[str] | None = None) -> list[str]:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "mr.h")]
    jobs = []
    objs = []
    for src in CU_SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(OBJ, src + ".o")
        objs.append(obj)
        if force or _newer(obj, [path] + headers):
            jobs.append([_nvcc()] + NVCC_FLAGS + (extra_nvcc or []) + ["-c", path, "-o", obj])
    for src in CXX_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        objs.append(obj)
        if force or _newer(obj, [path] + headers):
            jobs.append([_cxx()] + CXX_FLAGS + ["-c", path, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    built = []
    if force or jobs or _newer(LIBMR, objs):
        _run([_nvcc()] + ARCH + ["-shared", "-o", LIBMR + ".tmp"] + objs +
             ["-Xcompiler", "-fopenmp", "-lgomp", "-lpthread"], verbose)
        os.replace(LIBMR + ".tmp", LIBMR)
        built.append(LIBMR)
    gen_src = os.path.join(CSRC, "gen.cpp")
    if force or _newer(LIBGEN, [gen_src, os.path.join(CSRC, "gen.h")]):
        _run([_cxx(), "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-shared", "-Wall", gen_src, "-o", LIBGEN + ".tmp"],
             verbose)
        os.replace(LIBGEN + ".tmp", LIBGEN)
        built.append(LIBGEN)
    return built


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    out = build(force=a.force, verbose=a.verbose)
    print("built:", ", ".join(os.path.basename(o) for o in out) if out else "up to date")
    return 0


if __name__ == "__main__":
    sys.exit(main())
