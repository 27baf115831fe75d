"""Build libmt3d.so (the CUDA solver and its C ABI) for sm_100a with nvcc.

Run ``python modem-gpu_b200/build.py``; the library is written next to this
file, in ``modem-gpu_b200/lib/``, so it travels with the source tree.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libmt3d.so")
SOURCES = ["kernels.cu", "colkernels.cu", "stagekernels.cu", "tmakernels.cu", "hatkernels.cu", "setupkernels.cu", "bc2d.cu", "datafunc.cu", "solnio.cu", "solver.cu", "sens.cu", "multi.cu",
           "noalloc.cu", "capi.cu"]
# the operator set-up reproduces the host's operation order bit for bit: no contraction to FMA
FILE_FLAGS = {"setupkernels.cu": ["-fmad=false"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def source_hash(flags: list) -> str:
    """SHA-256 (first 16 hex digits) of every source and header the library is
    built from, this script and the compiler flags; mt3d_version() reports it,
    so a library whose sources changed is rebuilt whatever the file times."""
    h = hashlib.sha256()
    files = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC))
    files += [os.path.join(HERE, "..", "include", "mt3d.h"), os.path.abspath(__file__)]
    for f in files:
        h.update(os.path.basename(f).encode())
        with open(f, "rb") as fh:
            h.update(fh.read())
    h.update(" ".join(flags).encode())
    return h.hexdigest()[:16]


def built_hash(path: str = LIB):
    """The source hash the library at `path` was built from (None if absent)."""
    if not os.path.exists(path):
        return None
    with open(path, "rb") as fh:
        data = fh.read()
    k = data.find(b"mt3d-src-")
    return data[k + 9:k + 25].decode() if k >= 0 else None


def compile_flags() -> list:
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
                   "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include")]


def expected_hash() -> str:
    """The source hash a library built from the current sources reports.
    Paths in the flags are hashed relative to this directory, so a tree
    copied elsewhere (the library travels with it) keeps its hash."""
    flags = [os.path.relpath(f, HERE) if os.path.isabs(f) else f for f in compile_flags()]
    return source_hash(flags + [f"{k}={v}" for k, v in sorted(FILE_FLAGS.items())])


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    flags = compile_flags()
    digest = expected_hash()
    if not force and built_hash() == digest:
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    if verbose:
        flags = flags + ["-Xptxas", "-v"]
    def compile_one(src):
        obj = os.path.join(objdir, src + ".o")
        extra = [f'-DMT3D_SRC_HASH="{digest}"'] if src == "capi.cu" else []
        cmd = [nvcc(), "-c", os.path.join(CSRC, src), "-o", obj] + flags + FILE_FLAGS.get(src, []) + extra
        return src, obj, subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as pool:
        results = list(pool.map(compile_one, SOURCES))
    for src, obj, r in results:
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
