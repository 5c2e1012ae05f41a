"""Build libtopx.so (the sm_100a engine behind include/topx.h) in-tree with nvcc.

Usage:  python -m top3d_xl_b200.build [--force] [--debug]

Objects go to top3d_xl_b200/_build/, the library to top3d_xl_b200/libtopx.so.
A source is recompiled when it (or a header) is newer than its object.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtopx.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

CUDA_SOURCES = ["topx_fem.cu", "topx_coarse.cu", "topx_nd.cu", "topx_opt.cu", "topx_engine.cu", "topx_noalloc.cu"]
CXX_SOURCES = ["topx_mesh.cpp", "topx_nd_plan.cpp", "topx_api.cpp", "topx_server.cpp", "topx_export.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "topx.h"))
    return hs


def build(force: bool = False, debug: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    newest_header = max(os.path.getmtime(h) for h in _headers())
    opt = ["-O0", "-g", "-G"] if debug else ["-O3"]
    objs = []
    for src in CUDA_SOURCES + CXX_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(path), newest_header):
            continue
        cmd = [NVCC, "-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo", *opt, *ARCH, "-c", path, "-o", obj,
               "-I", CSRC, "-I", os.path.join(ROOT, "include")]
        if src.endswith(".cu"):
            cmd += ["--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
            if verbose:
                cmd += ["-Xptxas", "-v"]
        elif src in ("topx_api.cpp", "topx_server.cpp"):
            cmd += ["-x", "cu"]  # includes the engine's device headers
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    cmd = [NVCC, "-shared", *ARCH, "-o", LIB, *objs, "-lcudart", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.debug, a.verbose))


if __name__ == "__main__":
    sys.exit(main())
