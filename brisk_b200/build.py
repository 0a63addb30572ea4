"""Build of the in-tree CUDA library brisk_b200/libbrisk.so (sm_100a only).

One shared library holds the kernels, the host-side interior-point loop and both C ABIs
(include/brisk.h: the reference's brisk_* interface; include/bgpu.h: the step kernels).  It is
compiled with nvcc for ``-gencode arch=compute_100a,code=sm_100a`` and links only the CUDA
runtime.  Objects are cached by content hash under brisk_b200/_build/.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbrisk.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]

SOURCES = ["gemm_f64.cu", "dense.cu", "schur.cu", "elementwise.cu", "tf32x3.cu", "small.cu", "sparse.cu", "lockstep.cu", "nt.cu", "ozaki.cu", "lowrank.cu", "lanczos.cu", "solver.cu",
           "bgpu.cu", "capi.cpp", "sdpa.cpp"]


def _digest(path: str, extra: str) -> str:
    h = hashlib.sha256(extra.encode())
    with open(path, "rb") as f:
        h.update(f.read())
    for name in sorted(os.listdir(CSRC)):          # headers change every object
        if name.endswith((".h", ".cuh")):
            with open(os.path.join(CSRC, name), "rb") as f:
                h.update(f.read())
    for name in sorted(os.listdir(os.path.join(ROOT, "include"))):
        with open(os.path.join(ROOT, "include", name), "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def _compile(src: str, verbose: bool) -> str:
    path = os.path.join(CSRC, src)
    flags = ARCH + FLAGS
    obj = os.path.join(BUILD, f"{src}.{_digest(path, ' '.join(flags))}.o")
    if os.path.exists(obj):
        return obj
    cmd = [NVCC] + flags + (["-x", "cu"] if src.endswith(".cpp") else []) + ["-c", path, "-o", obj + ".tmp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    os.replace(obj + ".tmp", obj)
    return obj


def build(verbose: bool = False) -> str:
    """Compile every source for sm_100a and link brisk_b200/libbrisk.so; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, len(SOURCES))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    key = hashlib.sha256("".join(objs).encode()).hexdigest()[:16]
    stamp = os.path.join(BUILD, "link.stamp")
    if os.path.exists(LIB) and os.path.exists(stamp) and open(stamp).read() == key:
        return LIB
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    with open(stamp, "w") as f:
        f.write(key)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
