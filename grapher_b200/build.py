"""Builds libgvizcuda.so (sm_100a) in-tree with nvcc.

    python -m grapher_b200.build        # or grapher_b200.build.build()

Objects go to grapher_b200/_build/, the library to grapher_b200/lib/.
precise.cu, noalloc.cu and grip.cu are compiled with --fmad=false (their FP64
paths keep the reference's rounding); everything else with fused
multiply-add.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libgvizcuda.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                 "-I" + INCLUDE, "-I" + CSRC, "--expt-relaxed-constexpr"]

SOURCES = {
    "sort.cu": [],
    "tree.cu": [],
    "forces.cu": [],
    "precise.cu": ["--fmad=false"],
    "noalloc.cu": ["--fmad=false"],
    "grip.cu": ["--fmad=false"],
    "mlp.cu": [],
    "api.cu": [],
    "host_graphs.cpp": [],
    "loaders.cpp": [],
}


def _headers_mtime() -> float:
    m = os.path.getmtime(os.path.join(INCLUDE, "gvizcuda.h"))
    for f in os.listdir(CSRC):
        if f.endswith((".cuh", ".h")):
            m = max(m, os.path.getmtime(os.path.join(CSRC, f)))
    return m


def _compile(src: str, extra: list[str], hdr: float, verbose: bool) -> str:
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(path), hdr):
        return obj
    if src.endswith(".cpp"):
        cmd = ["g++", "-O3", "-fPIC", "-std=c++17", "-I" + INCLUDE, "-I" + CSRC,
               "-I/usr/local/cuda/include", "-c", path, "-o", obj]
    else:
        cmd = [NVCC] + COMMON + extra + ["-c", path, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{out.stdout}{out.stderr}")
    if verbose and (out.stdout or out.stderr):
        sys.stderr.write(out.stdout + out.stderr)
    return obj


WORKLOADS_SRC = os.path.join(CSRC, "workloads.cpp")
WORKLOADS_LIB = os.path.join(LIBDIR, "libgvizworkloads.so")


def build_workloads() -> str:
    """The synthetic-graph library, host C++ only (no CUDA)."""
    hdr = os.path.join(INCLUDE, "gvizworkloads.h")
    if os.path.exists(WORKLOADS_LIB) and os.path.getmtime(WORKLOADS_LIB) >= max(
            os.path.getmtime(WORKLOADS_SRC), os.path.getmtime(hdr)):
        return WORKLOADS_LIB
    cmd = ["g++", "-O3", "-fPIC", "-shared", "-std=c++17", "-I" + INCLUDE, WORKLOADS_SRC,
           "-o", WORKLOADS_LIB]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"workloads build failed: {' '.join(cmd)}\n{out.stdout}{out.stderr}")
    return WORKLOADS_LIB


ADAPTER_SRC = os.path.join(HERE, "gviz", "gvizCudaForceEmbedder.c")
GRIP_ADAPTER_SRC = os.path.join(HERE, "gviz", "gvizCudaGripEmbedder.c")
ADAPTER_LIB = os.path.join(LIBDIR, "libgvizcuda_gviz.so")


def build_gviz_adapter(gviz_include: str | None = None) -> str | None:
    """Compiles the gviz-side glue against gviz's headers. The gviz symbols
    stay undefined: the program that loads it (gviz itself) provides them."""
    inc = gviz_include or os.environ.get("GVIZ_INCLUDE")
    if not inc or not os.path.isdir(inc):
        return None
    if os.path.exists(ADAPTER_LIB) and os.path.getmtime(ADAPTER_LIB) >= max(
            os.path.getmtime(ADAPTER_SRC), os.path.getmtime(GRIP_ADAPTER_SRC),
            os.path.getmtime(LIB),
            os.path.getmtime(os.path.join(INCLUDE, "gvizCudaForceEmbedder.h")),
            os.path.getmtime(os.path.join(INCLUDE, "gvizCudaGripEmbedder.h"))):
        return ADAPTER_LIB
    cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-include", "stdint.h",
           "-I" + INCLUDE, "-I" + inc, ADAPTER_SRC, GRIP_ADAPTER_SRC, "-o", ADAPTER_LIB,
           "-L" + LIBDIR, "-lgvizcuda", "-Wl,-rpath,$ORIGIN"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"adapter build failed: {' '.join(cmd)}\n{out.stdout}{out.stderr}")
    return ADAPTER_LIB


def build(verbose: bool = False, gviz_include: str | None = None) -> str:
    """Compiles libgvizcuda and libgvizworkloads; the gviz glue as well when
    gviz's headers are given (gviz_include or $GVIZ_INCLUDE)."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdr = _headers_mtime()
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        futs = [ex.submit(_compile, s, e, hdr, verbose) for s, e in SOURCES.items()]
        objs = [f.result() for f in futs]
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static"]
        out = subprocess.run(cmd, capture_output=True, text=True)
        if out.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{out.stdout}{out.stderr}")
    build_workloads()
    build_gviz_adapter(gviz_include)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
