"""Build the CUDA library and the pybind11 facade in-tree.

    python ai-phyiscs_b200/build.py [--force]

Outputs (next to the Python package, so they ship with the tree):
    chysx/libchysx_cloth.so          C-ABI library: kernels + host orchestration
    chysx/_chysx_native<ext>.so      pybind11 facade over the C ABI

Kernels are compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a); nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
PKG = os.path.join(HERE, "chysx")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

LIB = os.path.join(PKG, "libchysx_cloth.so")
CU_SOURCES = [os.path.join(CSRC, f) for f in ("cloth_sim.cu", "topology.cpp")]
CU_DEPS = CU_SOURCES + [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
                        if f.endswith((".cuh", ".h"))] + [os.path.join(INCLUDE, f) for f in ("chysx_cloth.h",
                                                                                          "chysx_vbd.h")]


def _ext_suffix() -> str:
    return sysconfig.get_config_var("EXT_SUFFIX") or ".so"


NATIVE = os.path.join(PKG, "_chysx_native" + _ext_suffix())
PY_SOURCES = [os.path.join(CSRC, "pybind_module.cpp"), os.path.join(INCLUDE, "chysx_cloth.h"),
              os.path.join(INCLUDE, "chysx_vbd.h")]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build_library(force: bool = False, verbose_ptxas: bool = False) -> str:
    if force or _stale(LIB, CU_DEPS):
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
               "-Xcompiler", "-fPIC", "-shared", "-I", INCLUDE, "-o", LIB, *CU_SOURCES, "-lcudart"]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        _run(cmd)
    return LIB


def build_native(force: bool = False) -> str:
    build_library(force)
    if force or _stale(NATIVE, PY_SOURCES + [LIB]):
        import pybind11

        py_inc = sysconfig.get_paths()["include"]
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden",
               "-I", pybind11.get_include(), "-I", py_inc, "-I", INCLUDE,
               PY_SOURCES[0], "-o", NATIVE, "-L", PKG, "-lchysx_cloth", "-Wl,-rpath,$ORIGIN"]
        _run(cmd)
    return NATIVE


def build(force: bool = False) -> None:
    build_native(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
