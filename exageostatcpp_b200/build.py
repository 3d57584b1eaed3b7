"""Build the sm_100a shared library ``libexageostat_b200.so`` in-tree.

Usage: ``python -m exageostatcpp_b200.build`` (or ``python exageostatcpp_b200/build.py``).
Each ``csrc/*.cu`` is compiled separately with nvcc for ``sm_100a`` and linked
into one shared object next to this file; the C ABI is ``include/exageostat_b200.h``.
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
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libexageostat_b200.so")

SOURCES = ["matern.cu", "potrf.cu", "dst.cu", "dgemm_tma.cu", "split_gemm.cu", "ozaki_band.cu", "mixed.cu", "fisher.cu", "capi.cu", "batch.cu", "host_data.cpp", "host_bobyqa.cpp", "host_server.cpp"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-I", os.path.join(ROOT, "include"),
]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    cmd = [nvcc(), *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    if verbose:
        sys.stderr.write(res.stderr)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs,
           "-Xcompiler", "-fPIC", "-lcudart_static", "-ldl", "-lpthread", "-lrt"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


HOST_INCLUDE = os.path.join(HERE, "host", "include")
HOST_SOURCES = [os.path.join(HERE, "host", "src", "Configurations.cpp")]
API_TEST_SRC = os.path.join(ROOT, "tests", "cpp", "test_exageostat_api.cpp")
API_TEST_BIN = os.path.join(ROOT, "tests", "cpp", "_build", "test_exageostat_api")
EXAMPLE_SRC = os.path.join(HERE, "host", "examples", "end_to_end.cpp")
EXAMPLE_BIN = os.path.join(HERE, "host", "examples", "_build", "end_to_end")


def build_host_tests() -> str:
    """Compile the C++ API test driver against the host headers and the library."""
    os.makedirs(os.path.dirname(API_TEST_BIN), exist_ok=True)
    cmd = [nvcc(), "-std=c++17", "-O2", "-x", "c++", "-I", HOST_INCLUDE, "-I", os.path.join(ROOT, "include"),
           *HOST_SOURCES, API_TEST_SRC, "-L", HERE, "-lexageostat_b200",
           "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN/../../../exageostatcpp_b200", "-o", API_TEST_BIN]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"host API test build failed:\n{res.stdout}\n{res.stderr}")
    build_example()
    return API_TEST_BIN


def build_example() -> str:
    """Compile the end-to-end example program of the C++ API (host/examples)."""
    os.makedirs(os.path.dirname(EXAMPLE_BIN), exist_ok=True)
    cmd = [nvcc(), "-std=c++17", "-O2", "-x", "c++", "-I", HOST_INCLUDE, "-I", os.path.join(ROOT, "include"),
           *HOST_SOURCES, EXAMPLE_SRC, "-L", HERE, "-lexageostat_b200",
           "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN/../../..", "-o", EXAMPLE_BIN]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"example build failed:\n{res.stdout}\n{res.stderr}")
    return EXAMPLE_BIN


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
    print(build_host_tests())
