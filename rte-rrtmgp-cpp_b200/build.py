"""Builds the rrtmgp_b200 CUDA library in-tree for sm_100a.

    python rte-rrtmgp-cpp_b200/build.py [--force]

Compiles every csrc/*.cu with nvcc (-gencode arch=compute_100a,code=sm_100a) and links
rrtmgp_b200/_lib/librrtmgp_b200.so.  Object files are rebuilt only when a source or header is
newer than them.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
CSRC = HERE / "csrc"
OBJ = HERE / "_build"
LIBDIR = HERE / "rrtmgp_b200" / "_lib"
LIB = LIBDIR / "librrtmgp_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I", str(REPO / "include"), "-I", str(CSRC)]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return list(CSRC.glob("*.cuh")) + list((REPO / "include").glob("*.h"))


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    LIBDIR.mkdir(parents=True, exist_ok=True)
    hdr_mtime = max((p.stat().st_mtime for p in _headers()), default=0.0)
    srcs = sorted(CSRC.glob("*.cu"))
    jobs = []
    for s in srcs:
        o = OBJ / (s.stem + ".o")
        if force or not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, hdr_mtime):
            jobs.append((s, o))
    cc = nvcc()

    def compile_one(job):
        s, o = job
        cmd = [cc, *ARCH, *NVCC_FLAGS, "-c", str(s), "-o", str(o)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {s.name}:\n{r.stderr}")
        return r.stderr

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for msg in ex.map(compile_one, jobs):
            if msg and verbose:
                print(msg)
    objs = [OBJ / (s.stem + ".o") for s in srcs]
    if force or jobs or not LIB.exists():
        cmd = [cc, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
