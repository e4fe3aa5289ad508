"""Build the engine in-tree: libgst_b200.so (CUDA kernels for sm_100a + host engine +
C ABI + reference IO) and the reference-compatible command-line drivers.

    python gpu4gst-sigmod-fullexp_b200/build.py [--force]

nvcc cross-compiles for sm_100a without a GPU.  Outputs land next to this file so
that they travel with the source tree.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX_HOST", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["gst_engine.cu", "gst_probe.cu"]
CPP_SOURCES = ["gst_io.cpp", "gst_synth.cpp"]
# every device header of csrc/ (a kernel edited in any of them rebuilds its sources)
HEADERS = sorted(f for f in os.listdir(os.path.join(HERE, "csrc")) if f.endswith((".cuh", ".h")))
LIB = os.path.join(HERE, "libgst_b200.so")
CLI = {"gst_nonhop": "gst_cli.cpp", "gst_hop": "gst_cli.cpp"}


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose_ptxas: bool = False, checked: bool = False) -> str:
    """checked=True builds libgst_b200_checked.so: every kernel bounds-checks its
    table / edge / worklist indices and reports ERR_BOUNDS instead of faulting."""
    if checked:
        return _build_checked(force)
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(INC, "gst.h"), os.path.join(INC, "gst_io.h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + hdrs):
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-Xcompiler", "-fopenmp", "-I", INC, "-I", CSRC, "-c", s, "-o", o]
            if verbose_ptxas:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd)
        objs.append(o)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + hdrs):
            _run([CXX, "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-I", INC, "-c", s, "-o", o])
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-Xcompiler", "-fopenmp", "-lgomp"])
    cli_src = os.path.join(CSRC, "gst_cli.cpp")
    if os.path.exists(cli_src):
        exe = os.path.join(HERE, "gst_cli")
        if force or _stale(exe, [cli_src, LIB] + hdrs):
            _run([CXX, "-O2", "-std=c++17", "-I", INC, cli_src, "-o", exe, "-L", HERE,
                  "-lgst_b200", f"-Wl,-rpath,{HERE}", "-Wl,-rpath,$ORIGIN"])
    gen_srcs = [os.path.join(CSRC, f) for f in ("gst_gen.cpp", "gst_synth.cpp", "gst_io.cpp")]
    gen = os.path.join(HERE, "gst_gen")
    if all(os.path.exists(f) for f in gen_srcs) and (force or _stale(gen, gen_srcs + hdrs)):
        # standalone: the generator and IO sources only, no engine library
        _run([CXX, "-O3", "-std=c++17", "-fopenmp", "-I", INC, *gen_srcs, "-o", gen])
    return LIB


def _build_checked(force: bool) -> str:
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(HERE, "libgst_b200_checked.so")
    objs = []
    for src in CU_SOURCES:
        o = os.path.join(BUILD, src + ".checked.o")
        _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-DGST_CHECKED", "-Xcompiler",
              "-fPIC", "-Xcompiler", "-fopenmp", "-I", INC, "-I", CSRC, "-c",
              os.path.join(CSRC, src), "-o", o])
        objs.append(o)
    build(force)
    objs += [os.path.join(BUILD, s + ".o") for s in CPP_SOURCES]
    _run([NVCC, *ARCH, "-shared", "-o", out, *objs, "-Xcompiler", "-fopenmp", "-lgomp"])
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register / smem usage")
    ap.add_argument("--checked", action="store_true", help="also build the bounds-checked library")
    a = ap.parse_args()
    build(a.force, a.ptxas)
    if a.checked:
        build(a.force, checked=True)
    sys.exit(0)
