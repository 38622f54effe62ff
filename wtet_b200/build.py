"""Build recipe for libwtet.so (sm_100a).

``python -m wtet_b200.build`` compiles the CUDA sources in ``csrc/`` with
nvcc for ``arch=compute_100a,code=sm_100a`` into ``wtet_b200/libwtet.so``
(in-tree, so the library travels with the repository).  Each source is its
own object, compiled in parallel, with the compiler's default contraction of
multiplies and adds: the exact predicates (exact.cuh, the FP32 stage of the
round kernels and the normalisation) spell every operation whose rounding
matters as a separately rounded intrinsic.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libwtet.so")
SOURCES = ["engine.cu", "capi.cu", "noalloc.cu", "learned.cu", "verify.cu"]
HEADERS = ["exact.cuh", "engine.cuh", "learned.cuh", "order.cuh", "devbuf.cuh"]

EXACT_SOURCES: set = set()  # sources that would need -fmad=false (none)

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC",
    "-diag-suppress",
    "177,550",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the wtet_b200 CUDA library cannot be built")


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, h) for h in HEADERS if os.path.exists(os.path.join(CSRC, h))]
    deps.append(os.path.join(HERE, "..", "include", "wtet.h"))
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    import concurrent.futures as cf
    import tempfile

    tmp = tempfile.mkdtemp(prefix="wtet_build_")

    def compile_one(src):
        obj = os.path.join(tmp, os.path.basename(src) + ".o")
        flags = NVCC_FLAGS + (["-fmad=false"] if os.path.basename(src) in EXACT_SOURCES else [])
        cmd = [nvcc()] + flags + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj]
        return obj, subprocess.run(cmd, capture_output=True, text=True)

    try:
        with cf.ThreadPoolExecutor(len(sources())) as ex:
            results = list(ex.map(compile_one, sources()))
        failed = False
        for obj, r in results:
            if r.returncode != 0 or verbose:
                sys.stderr.write(r.stdout + r.stderr)
            failed = failed or r.returncode != 0
        if failed:
            raise RuntimeError("nvcc failed building libwtet.so")
        link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB + ".tmp"]
        r = subprocess.run(link + [o for o, _ in results], capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed linking libwtet.so")
        os.replace(LIB + ".tmp", LIB)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
