"""Builds the sm_100a shared library ``libpt_b200.so`` in-tree with nvcc.

The library is the product: C ABI in include/pt_b200.h, CUDA kernels in
csrc/.  It links the CUDA runtime statically so that it does not depend on the
runtime version that torch ships.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from typing import List, Optional

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libpt_b200.so")
SOURCES = ["pt_bvh.cu", "pt_render.cu", "pt_scene.cu", "pt_output.cu", "pt_adjoint.cu", "pt_api.cu", "pt_noalloc.cu", "pt_spectral.cu", "pt_l2probe.cu",
           "pt_sort.cu"]
HEADERS = ["pt_common.cuh", "pt_bvh.cuh", "pt_render.cuh", "pt_trace.cuh", "pt_bsdf.cuh", "pt_scene.cuh", "pt_output.cuh", "pt_path.cuh", "pt_adjoint.cuh", "pt_spectral.cuh",
           "pt_select.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--cudart", "static",
              "-Xcompiler", "-ffp-contract=off"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _inputs() -> List[str]:
    return [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(INCLUDE, "pt_b200.h")]


def needs_build(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    return any(os.path.getmtime(p) > t for p in _inputs())


def build(force: bool = False, verbose: bool = False, extra: Optional[List[str]] = None, lib: str = LIB) -> str:
    """Compiles every .cu for sm_100a and links libpt_b200.so; returns its path."""
    if not force and not needs_build(lib):
        return lib
    nvcc = nvcc_path()
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, *(extra or []), "-I", INCLUDE, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.append("-Xptxas=-v")
            print(" ".join(cmd), file=sys.stderr)
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT), src))
        objs.append(obj)
    for p, src in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{out.decode(errors='replace')}")
        if verbose:
            sys.stderr.write(out.decode(errors="replace"))
    tmp = lib + ".tmp"
    cmd = [nvcc, *ARCH, "--cudart", "static", "-shared", "-o", tmp, *objs]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout.decode(errors='replace')}")
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
