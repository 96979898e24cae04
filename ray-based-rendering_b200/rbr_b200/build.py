"""Builds librbr_b200.so (CUDA for sm_100a + host C++) in-tree.

    python -m rbr_b200.build            (from ray-based-rendering_b200/)

Objects go to ray-based-rendering_b200/_build/, the library to rbr_b200/librbr_b200.so. The
CUDA runtime is linked statically so the library only needs the driver at run time.
Set RBR_PTXAS_VERBOSE=1 to print per-kernel register and shared-memory use.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent          # .../ray-based-rendering_b200/rbr_b200
ROOT = PKG_DIR.parent                               # .../ray-based-rendering_b200
REPO = ROOT.parent
CSRC = ROOT / "csrc"
INCLUDE = REPO / "include"
BUILD = ROOT / "_build"
LIB = PKG_DIR / "librbr_b200.so"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXX = shutil.which("g++") or "g++"

COMMON = ["-O3", "-std=c++17", f"-I{INCLUDE}", f"-I{CSRC}"]
HOST_FLAGS = ["-fPIC", "-ffp-contract=off", "-Wall", "-Wextra", "-Wno-unused-parameter"]


def _sources():
    cu = sorted(CSRC.glob("*.cu"))
    cpp = sorted(CSRC.glob("*.cpp"))
    headers = sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))
    return cu, cpp, headers


def _stale(obj: Path, src: Path, headers) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in headers)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")
    if r.stderr.strip() and (verbose or os.environ.get("RBR_PTXAS_VERBOSE")):
        sys.stderr.write(r.stderr)
    return r


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    cu, cpp, headers = _sources()
    objs = []
    jobs = []
    ptxas = ["-Xptxas", "-v"] if os.environ.get("RBR_PTXAS_VERBOSE") else []
    for src in cu:
        obj = BUILD / (src.stem + ".cu.o")
        objs.append(obj)
        if force or _stale(obj, src, headers):
            jobs.append([NVCC, *ARCH, "-lineinfo", *COMMON, *ptxas, "-Xcompiler", ",".join(HOST_FLAGS),
                         "-c", src, "-o", obj])
    for src in cpp:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src, headers):
            jobs.append([CXX, *COMMON, *HOST_FLAGS, f"-I{CUDA_HOME / 'include'}", "-c", src, "-o", obj])
    procs = []
    for cmd in jobs:  # compile in parallel
        if verbose:
            print(" ".join(str(c) for c in cmd), flush=True)
        procs.append((cmd, subprocess.Popen([str(c) for c in cmd], stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                            text=True)))
    failed = False
    for cmd, p in procs:
        out, err = p.communicate()
        if p.returncode != 0:
            failed = True
            sys.stderr.write(f"--- {cmd[-3]}\n{out}{err}")
        elif err.strip() and (verbose or ptxas):
            sys.stderr.write(err)
    if failed:
        raise RuntimeError("librbr_b200 compilation failed")
    if force or jobs or not LIB.exists():
        _run([NVCC, *ARCH, "-shared", "--cudart", "static", "-o", LIB, *objs, "-lpthread", "-ldl", "-lrt"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
