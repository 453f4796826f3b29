"""Builds libpyrocmc.so in-tree with nvcc for sm_100a (no JIT, no torch)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpyrocmc.so")
SOURCES = ["system.cu", "sweep.cu", "sweep_lifted.cu", "sweep_staged.cu", "sweep_cluster.cu", "grad.cu", "ssf.cu",
           "pt.cu", "pt_persistent.cu", "noalloc.cu", "lt.cu", "merge.cu", "energy_cell.cu",
           "hostio.cu"]
HEADERS = ["common.cuh", "kernels.h", "pyro_struct.cuh", "struct_field.cuh", "moves.cuh", "dft.cuh", "pt.cuh",
           "energy_cell.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
]
OBJ_DIR = os.path.join(HERE, "_build")


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(REPO, "include", "pyrocmc.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, force: bool, verbose: bool) -> str:
    """One translation unit to an object; skipped when the object is newer
    than the source and every header (no device symbol crosses units, so
    whole-program device compilation is not needed)."""
    obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS] + \
        [os.path.join(REPO, "include", "pyrocmc.h")]
    if not force and os.path.exists(obj) and all(os.path.getmtime(d) <= os.path.getmtime(obj) for d in deps):
        return obj
    cmd = [_nvcc(), *NVCC_FLAGS, "-I", os.path.join(REPO, "include"), "-c", os.path.join(CSRC, src),
           "-o", obj + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(obj + ".tmp", obj)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    if force or needs_build():
        from concurrent.futures import ThreadPoolExecutor

        os.makedirs(OBJ_DIR, exist_ok=True)
        with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as ex:
            objs = list(ex.map(lambda f: _compile(f, force, verbose), SOURCES))
        cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB + ".tmp", *objs,
               "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        os.replace(LIB + ".tmp", LIB)
    build_host(force=force, verbose=verbose)
    return LIB


HOST = os.path.join(HERE, "host")
BIN = os.path.join(HERE, "bin")
HOST_LIB_SOURCES = ["MC.cpp", "managers.cpp", "h5out.cpp", "h5file.cpp"]
HOST_HEADERS = ["MC.hpp", "managers.hpp", "h5out.hpp", "h5file.hpp", "cli_bits.hpp", "vec3.hpp"]
DRIVERS = ["anneal", "fieldcool", "temper", "spiral_byhand", "ltgs"]


def build_host(force: bool = False, verbose: bool = False) -> None:
    """The C++ drivers (the reference's executables) over libpyrocmc.so,
    built with g++ into pyro_cmc_b200/bin/."""
    os.makedirs(BIN, exist_ok=True)
    deps = [os.path.join(HOST, f) for f in HOST_LIB_SOURCES + HOST_HEADERS] + [LIB]
    for d in DRIVERS:
        exe = os.path.join(BIN, d)
        src = os.path.join(HOST, d + ".cpp")
        if not force and os.path.exists(exe) and all(os.path.getmtime(x) <= os.path.getmtime(exe) for x in deps + [src]):
            continue
        cmd = ["g++", "-O2", "-std=c++20", "-Wall", "-I", os.path.join(REPO, "include"), "-o", exe, src,
               *[os.path.join(HOST, f) for f in HOST_LIB_SOURCES], "-L", HERE, "-lpyrocmc",
               "-Wl,-rpath,$ORIGIN/.."]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    print(build(force=True, verbose=True))
