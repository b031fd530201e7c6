"""Build the sm_100a CUDA library and the drop-in libraries in-tree.

Outputs (next to this file):
  libhh.so      C ABI of include/hh.h (all kernels)
  libhh2d.so    drop-in for the reference 2D program: solver(System), forwardDST, reverseDST
  libhh3d.so    drop-in for the reference 3D program: solver(System), DST
  hh_direct_solver   Direct_Solver-compatible command line driver

Run `python -m hackathon_b200.build` (or __graft_entry__.build()).  Incremental: a target is
rebuilt when any source is newer.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"] + ARCH
CC_FLAGS = ["-O2", "-fPIC", "-std=gnu11", "-Wall"]

CU_SOURCES = ["hh_api.cu", "hh_dst.cu", "hh_tridiag.cu", "hh_server.cu", "hh_refine.cu", "hh_rhs.cu"]
C_SOURCES = ["hh_coef.c"]
HEADERS = ["hh_internal.cuh", "hh_tma.cuh"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cc() -> str:
    for cand in ("/usr/bin/gcc", shutil.which("gcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("gcc not found")


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
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout.strip() or r.stderr.strip()):
        print(r.stdout + r.stderr, flush=True)


def build(verbose: bool = False, ptxas_info: bool = False) -> dict:
    os.makedirs(OBJ, exist_ok=True)
    nvcc, cc = _nvcc(), _cc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "hh.h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if _newer(o, [s] + hdrs) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            _run([nvcc, *NVCC_FLAGS, *extra, "-I", INCLUDE, "-c", s, "-o", o], verbose or ptxas_info)
        objs.append(o)
    for src in C_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if _newer(o, [s] + hdrs):
            _run([cc, *CC_FLAGS, "-I", INCLUDE, "-c", s, "-o", o], verbose)
        objs.append(o)
    out = {}
    lib = os.path.join(HERE, "libhh.so")
    if _newer(lib, objs):
        _run([nvcc, "-shared", *ARCH, "-o", lib, *objs, "-lm"], verbose)
    out["libhh"] = lib

    # drop-in libraries and CLI (plain C over the C ABI)
    for name, src in (("libhh2d.so", "hh_dropin2d.c"), ("libhh3d.so", "hh_dropin3d.c")):
        s = os.path.join(CSRC, src)
        if not os.path.exists(s):
            continue
        target = os.path.join(HERE, name)
        if _newer(target, [s, lib] + hdrs + [os.path.join(INCLUDE, "hh_dropin2d.h"),
                                             os.path.join(INCLUDE, "hh_dropin3d.h")]):
            _run([cc, *CC_FLAGS, "-shared", "-I", INCLUDE, "-o", target, s, "-L", HERE, "-lhh",
                  "-Wl,-rpath,$ORIGIN", "-lm"], verbose)
        out[name] = target
    cli_src = os.path.join(CSRC, "hh_direct_solver.c")
    if os.path.exists(cli_src):
        cli = os.path.join(HERE, "hh_direct_solver")
        if _newer(cli, [cli_src, lib]):
            _run([cc, *CC_FLAGS, "-I", INCLUDE, "-o", cli, cli_src, "-L", HERE, "-lhh", "-Wl,-rpath,$ORIGIN", "-lm"],
                 verbose)
        out["cli"] = cli
    return out


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
