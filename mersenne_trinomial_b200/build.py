"""Build libgf2e.so (all CUDA sources, sm_100a) in-tree.

    python -m mersenne_trinomial_b200.build          # library only
    python -m mersenne_trinomial_b200.build --tools  # also the C++ CLIs

Objects are cached per source file under _build/ (git-ignored) so a change
to one .cu recompiles only that file.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
TOOLS = os.path.join(CSRC, "tools")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libgf2e.so")
BIN = os.path.join(PKG, "bin")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                  "-I" + os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:6]) + " ...")
    return r


def _newer(src_list, dst):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(s) > t for s in src_list)


def build_lib(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    objs = []
    for cu in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(cu) + ".o")
        if _newer([cu] + headers, obj):
            if verbose:
                print("nvcc", os.path.basename(cu), flush=True)
            _run([NVCC] + NVFLAGS + ["-dc", "-o", obj, cu])
        objs.append(obj)
    for cpp in sorted(glob.glob(os.path.join(CSRC, "*.cpp"))):
        obj = os.path.join(BUILD, os.path.basename(cpp) + ".o")
        if _newer([cpp] + headers + glob.glob(os.path.join(CSRC, "*.h")), obj):
            if verbose:
                print("g++", os.path.basename(cpp), flush=True)
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-c", "-o", obj, cpp])
        objs.append(obj)
    if _newer(objs, LIB):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    return LIB


def build_tools(verbose: bool = False) -> list:
    """C++ command-line drop-ins for the reference tools, linked to libgf2e.so."""
    os.makedirs(BIN, exist_ok=True)
    out = []
    srcs = sorted(glob.glob(os.path.join(TOOLS, "*.cpp")))
    hdrs = glob.glob(os.path.join(ROOT, "include", "*")) + glob.glob(os.path.join(TOOLS, "*.h"))
    for src in srcs:
        exe = os.path.join(BIN, os.path.splitext(os.path.basename(src))[0])
        if _newer([src, LIB] + hdrs, exe):
            if verbose:
                print("g++", os.path.basename(src), flush=True)
            _run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
                  "-I/usr/local/cuda/include", "-o", exe, src,
                  "-L" + PKG, "-lgf2e", "-Wl,-rpath,$ORIGIN/..",
                  "-L/usr/local/cuda/lib64", "-lcudart", "-pthread"])
        out.append(exe)
    return out


if __name__ == "__main__":
    build_lib(verbose=True)
    if "--tools" in sys.argv:
        build_tools(verbose=True)
    print(LIB)
