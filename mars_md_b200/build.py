"""Build libmarsb200.so in-tree with nvcc for sm_100a.

    python -m mars_md_b200.build          # or: from mars_md_b200.build import build; build()

The library is plain CUDA C++ behind a C ABI (include/marsb200.h); no torch
headers are involved. Objects are cached under mars_md_b200/_build/ and only
rebuilt when a source or header changed.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmarsb200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
                     "-I" + os.path.join(ROOT, "include")]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(ROOT, "include", "marsb200.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD_DIR, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = _headers()
    objs = []
    for src in sources:
        obj = os.path.join(BUILD_DIR, os.path.basename(src).replace(".cu", ".o"))
        objs.append(obj)
        if _stale(obj, [src] + headers):
            cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


HOST_DIR = os.path.join(HERE, "host")
CPP_TEST_SRC = os.path.join(ROOT, "tests", "cpp", "pairlist_mirror_test.cpp")
CPP_TEST_BIN = os.path.join(ROOT, "tests", "cpp", "_build", "pairlist_mirror_test")


def build_cpp_mirror_test(verbose: bool = False) -> str:
    """Compile the C++ host-mirror test program (g++ against libmarsb200.so)."""
    lib = build(verbose)
    deps = [CPP_TEST_SRC, lib, os.path.join(ROOT, "include", "marsb200.h")] + \
        glob.glob(os.path.join(HOST_DIR, "*.hpp"))
    if _stale(CPP_TEST_BIN, deps):
        os.makedirs(os.path.dirname(CPP_TEST_BIN), exist_ok=True)
        cuda = os.path.dirname(os.path.dirname(NVCC))
        cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-Wall", "-Wextra",
               "-I" + os.path.join(ROOT, "include"), "-I" + HOST_DIR,
               "-I" + os.path.join(cuda, "include"), CPP_TEST_SRC, "-o", CPP_TEST_BIN,
               "-L" + HERE, "-lmarsb200", "-L" + os.path.join(cuda, "lib64"), "-lcudart",
               "-Wl,-rpath,$ORIGIN/../../../mars_md_b200",
               "-Wl,-rpath," + os.path.join(cuda, "lib64")]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return CPP_TEST_BIN


REF_ADAPTER_SRC = os.path.join(ROOT, "tests", "cpp", "ref_adapter", "ref_adapter_test.cpp")
REF_ADAPTER_BIN = os.path.join(ROOT, "tests", "cpp", "_build", "ref_adapter_test")


def reference_checkout():
    """The reference source tree: the MARS_MD_REFERENCE environment variable,
    else a directory named "reference" beside this repository; None if absent."""
    path = os.environ.get("MARS_MD_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")
    return path if os.path.isdir(os.path.join(path, "src", "PatchOperation")) else None


def build_ref_adapter_test(reference=None, verbose: bool = False):
    """Compile the test program of the adapter that derives from the
    reference's own MARS::Pairlist (host/b200_ref_adapter.hpp) against the
    reference's headers, with tests/cpp/ref_adapter/inc standing in for the
    reference's Backend layer (CUDA device memory) and the oracle harness's fmt
    stand-in. Returns the binary, or None when no reference checkout is here
    and no binary was built earlier."""
    reference = reference or reference_checkout()
    if reference is None:
        return REF_ADAPTER_BIN if os.path.exists(REF_ADAPTER_BIN) else None
    lib = build(verbose)
    shim = os.path.join(ROOT, "tests", "cpp", "ref_adapter", "inc")
    deps = [REF_ADAPTER_SRC, lib, os.path.join(ROOT, "include", "marsb200.h"),
            os.path.join(HOST_DIR, "b200_ref_adapter.hpp")] + \
        glob.glob(os.path.join(shim, "Backend", "*.h"))
    if _stale(REF_ADAPTER_BIN, deps):
        os.makedirs(os.path.dirname(REF_ADAPTER_BIN), exist_ok=True)
        cuda = os.path.dirname(os.path.dirname(NVCC))
        cmd = ["g++", "-std=c++20", "-O2", "-ffp-contract=off", "-Wall",
               "-I" + shim, "-I" + os.path.join(ROOT, "oracle", "ref_harness", "shim", "inc"),
               "-I" + os.path.join(reference, "src"), "-I" + os.path.join(ROOT, "include"),
               "-I" + HOST_DIR, "-I" + os.path.join(cuda, "include"), REF_ADAPTER_SRC,
               "-o", REF_ADAPTER_BIN, "-L" + HERE, "-lmarsb200",
               "-L" + os.path.join(cuda, "lib64"), "-lcudart",
               "-Wl,-rpath,$ORIGIN/../../../mars_md_b200",
               "-Wl,-rpath," + os.path.join(cuda, "lib64")]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return REF_ADAPTER_BIN


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
