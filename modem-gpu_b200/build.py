"""Build libmt3d.so (the CUDA solver and its C ABI) for sm_100a with nvcc.

Run ``python modem-gpu_b200/build.py``; the library is written next to this
file, in ``modem-gpu_b200/lib/``, so it travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libmt3d.so")
SOURCES = ["kernels.cu", "colkernels.cu", "stagekernels.cu", "tmakernels.cu", "setupkernels.cu", "bc2d.cu", "datafunc.cu", "solnio.cu", "solver.cu",
           "noalloc.cu", "capi.cu"]
# the operator set-up reproduces the host's operation order bit for bit: no contraction to FMA
FILE_FLAGS = {"setupkernels.cu": ["-fmad=false"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "mt3d.h")]
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d)):
            return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
                    "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include")]
    if verbose:
        flags += ["-Xptxas", "-v"]
    for src in SOURCES:
        obj = os.path.join(objdir, src + ".o")
        cmd = [nvcc(), "-c", os.path.join(CSRC, src), "-o", obj] + flags + FILE_FLAGS.get(src, [])
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-shared", "-o", tmp] + objs + ARCH + ["-Xcompiler", "-fPIC", "-lcudart_static", "-lrt", "-ldl",
                                                          "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
