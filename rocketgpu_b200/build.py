"""Builds the CUDA extension in-tree: rocketgpu_b200/_lib/librocketgpu_b200.so (sm_100a only).

    python -m rocketgpu_b200.build

nvcc compiles the device code for sm_100a with --fmad=false and IEEE division / square root (the defaults without
--use_fast_math), so every float32 operation rounds exactly like the reference's CPU build (-ffp-contract=off).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
LIB_NAME = "librocketgpu_b200.so"
LIB_PATH = os.path.join(LIB_DIR, LIB_NAME)

CU_SOURCES = ["rg_batch.cu"]
CPP_SOURCES = ["rg_mesh.cpp"]  # py_module.cpp builds separately (build_py_module)
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
    "-Xptxas", "-warn-spills",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "rocketgpu_b200.h")]
    if not force and _newer(LIB_PATH, deps):
        return LIB_PATH
    objs = []
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    for src in CU_SOURCES + CPP_SOURCES:
        obj = os.path.join(LIB_DIR, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc()] + NVCC_FLAGS + inc + ["-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cpp"):
            cmd = [nvcc(), "-x", "c++", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden"] \
                + inc + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs + ["-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    build_py_module(verbose)
    return LIB_PATH


def build_py_module(verbose: bool = False) -> str:
    """The pybind11 module rocketgpu_py_b200 (csrc/py_module.cpp) over the C ABI, next to the library it links."""
    import sysconfig

    import pybind11
    out = os.path.join(LIB_DIR, "rocketgpu_py_b200" + sysconfig.get_config_var("EXT_SUFFIX"))
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
           "-I", os.path.join(ROOT, "include"), "-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"],
           os.path.join(CSRC, "py_module.cpp"), "-L", LIB_DIR, "-lrocketgpu_b200", "-Wl,-rpath,$ORIGIN", "-o", out]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
