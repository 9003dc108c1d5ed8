"""Build the sm_100a shared library in-tree: astr_gpu_b200/libastr_b200.so, and its strict-parity
variant astr_gpu_b200/libastr_b200_strict.so (the same sources with -fmad=false: no multiply-add
contraction, as the reference's gfortran build without -march emits none), used to attribute any
difference from the oracle above rounding to the algorithm rather than to contraction.

    python -m astr_gpu_b200.build [--force] [--verbose] [--strict]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libastr_b200.so")
LIB_STRICT = os.path.join(HERE, "libastr_b200_strict.so")
SOURCES = ["capi.cu", "tgv.cu", "lines.cu", "schemes.cu", "tgv_l3_1.cu", "tgv_l5_1.cu", "tgv_l9_1.cu", "tgv_l9_2.cu",
           "tgv_l9_4.cu", "tgv_l5_2.cu", "tgv_l5_4.cu", "tgv_l17_1.cu", "noalloc.cu", "fullsolver.cu", "adjoint.cu", "adj_l3_1.cu", "adj_l5_1.cu",
           "adj_l9_1.cu", "adj_l9_2.cu", "adj_l9_4.cu", "adj_l5_2.cu", "adj_l5_4.cu", "checkpoint.cu", "h5file.cpp"]
HEADERS = ["ops.cuh", "internal.h", "tgv.cuh", "tgv_kernels.cuh", "adjoint.cuh", "adj_kernels.cuh", "h5file.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(lib: str) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "astr_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None, strict: bool = False) -> str:
    """Compile each translation unit in parallel, then link the shared library (the strict-parity
    variant with `strict`)."""
    lib = LIB_STRICT if strict else LIB
    if not force and not _stale(lib):
        return lib
    objdir = os.path.join(HERE, "_build_strict" if strict else "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]
    if verbose:
        flags.append("-Xptxas=-v")
    if strict:
        flags.append("-fmad=false")
    if extra:
        flags.extend(extra)
    procs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        procs.append(subprocess.Popen([nvcc(), *flags, "-c", os.path.join(CSRC, src), "-o", obj],
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    logs, failed = [], False
    for p in procs:
        out, _ = p.communicate()
        logs.append(out)
        failed |= p.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed:\n" + "".join(logs))
    res = subprocess.run([nvcc(), *ARCH, "-shared", "-o", lib, *objs], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("link failed:\n" + res.stdout + res.stderr)
    if verbose:
        sys.stdout.write("".join(logs))
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv, strict="--strict" in sys.argv))
