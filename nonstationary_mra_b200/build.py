"""Builds the in-tree shared library ``libmra_b200.so`` for sm_100a with nvcc.

    python -m nonstationary_mra_b200.build [--verbose]

The library holds the CUDA kernels and the C ABI declared in include/mra_b200.h.
It is built in place (next to this file) so that it travels with the source
tree; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmra_b200.so")

CU_SOURCES = ["mra_kernels.cu", "mra_api.cu", "mra_static.cu", "mra_mlp.cu", "mra_opt.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def sources() -> list:
    return [os.path.join(CSRC, s) for s in CU_SOURCES]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + \
        [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


HOST_SOURCES = ["host/mra_host.cpp"]
HOST_MAIN = "host/mra_main.cpp"
HOST_LIB = os.path.join(HERE, "libmra_host.so")
HOST_EXE = os.path.join(HERE, "mra_b200")


def build_host(force: bool = False) -> str:
    """The C++ host (include/mra_host.hpp): libmra_host.so and the drop-in
    executable ``mra_b200``, both linked against libmra_b200.so (rpath $ORIGIN)."""
    build()
    srcs = [os.path.join(HERE, s) for s in HOST_SOURCES]
    deps = srcs + [os.path.join(HERE, HOST_MAIN), LIB] + \
        [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    if not force and os.path.exists(HOST_EXE) and os.path.exists(HOST_LIB) and \
            all(os.path.getmtime(d) <= min(os.path.getmtime(HOST_EXE), os.path.getmtime(HOST_LIB)) for d in deps):
        return HOST_EXE
    cxx = shutil.which("g++") or "/usr/bin/g++"
    common = ["-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), "-L", HERE, "-lmra_b200",
              "-Wl,-rpath,$ORIGIN"]
    for cmd in ([cxx, "-shared", "-fPIC", "-o", HOST_LIB] + srcs + common,
                [cxx, "-o", HOST_EXE, os.path.join(HERE, HOST_MAIN)] + srcs + common):
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"host build failed:\n{res.stderr}")
    return HOST_EXE


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                    "-I", os.path.join(ROOT, "include")]
    if verbose:
        flags += ["-Xptxas", "-v"]
    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [nvcc()] + flags + ["-c", src, "-o", obj]
        return obj, subprocess.run(cmd, capture_output=True, text=True)

    # the translation units compile independently: one nvcc per source at once
    with ThreadPoolExecutor(max_workers=len(CU_SOURCES)) as pool:
        results = list(pool.map(compile_one, sources()))
    for src, (obj, res) in zip(sources(), results):
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{res.stderr}")
        if verbose and res.stderr:
            print(res.stderr, file=sys.stderr)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))
    print(build_host(force=True))
