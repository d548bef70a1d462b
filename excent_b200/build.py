"""Build libexcent_b200.so and the `excent` CLI in-tree for sm_100a.

    python -m excent_b200.build [--force] [-v]

CUDA sources are compiled with nvcc for `-gencode arch=compute_100a,code=sm_100a`
(cross-compiles without a GPU); host C++ with g++ and OpenMP. Objects go to
excent_b200/_build/, the library to excent_b200/libexcent_b200.so and the tools to
excent_b200/bin/ (excent, excent_params, excent_reference; rpath $ORIGIN/..).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libexcent_b200.so")
CLI = os.path.join(PKG, "bin", "excent")
TOOLS = {"cli_main": CLI, "cli_params": os.path.join(PKG, "bin", "excent_params"),
         "cli_reference": os.path.join(PKG, "bin", "excent_reference"),
         "cli_convert": os.path.join(PKG, "bin", "excent_convert"),
         "cli_info": os.path.join(PKG, "bin", "excent_info"),
         "cli_evict": os.path.join(PKG, "bin", "excent_evict")}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def nvcc():
    p = shutil.which("nvcc") or os.path.join(CUDA_HOME, "bin", "nvcc")
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build excent_b200")
    return p


def _deps():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INC, "*.h"))


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _compile(src, verbose):
    base = os.path.splitext(os.path.basename(src))[0]
    obj = os.path.join(OBJ, base + (".cu.o" if src.endswith(".cu") else ".o"))
    if not _stale(obj, [src] + _deps()):
        return obj
    if src.endswith(".cu"):
        cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp", "-I" + INC,
               "-I" + CSRC, "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
    else:
        cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-I" + INC, "-I" + CSRC,
               "-I" + os.path.join(CUDA_HOME, "include"), "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0 or verbose:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    if force:
        for o in glob.glob(os.path.join(OBJ, "*.o")):
            os.remove(o)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    lib_srcs = [s for s in srcs if not os.path.basename(s).startswith("cli_")]
    cli_srcs = [s for s in srcs if os.path.basename(s).startswith("cli_")]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), lib_srcs + cli_srcs))
    lib_objs = objs[:len(lib_srcs)]
    cli_objs = objs[len(lib_srcs):]
    if force or _stale(LIB, lib_objs):
        # cudart linked statically: the library never binds to another runtime loaded in the process
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-Xcompiler", "-fopenmp", "-o", LIB, *lib_objs,
               "-lgomp"]
        subprocess.run(cmd, check=True)
    for obj in cli_objs:   # one binary per cli_*.cpp
        out = TOOLS[os.path.basename(obj).rsplit(".", 1)[0]]
        if force or _stale(out, [obj, LIB]):
            cmd = ["g++", "-o", out, obj, "-L" + PKG, "-lexcent_b200", "-Wl,-rpath,$ORIGIN/..", "-fopenmp"]
            subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.v))
