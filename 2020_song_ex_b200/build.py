"""Build the sm_100a shared library ``libsong_b200.so`` in-tree with nvcc.

Usage: ``python 2020_song_ex_b200/build.py [--verbose]``.  The library is
written next to this file so that it travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsong_b200.so")
SOURCES = ["song_search.cu", "song_build.cu", "song_learn.cu", "song_capi.cu", "song_serve.cu",
           "song_noalloc.cu", "song_bithash.cu", "song_entry.cu",
           "song_graphsearch.cu", "song_gt.cu"]
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
]


def sources() -> list[str]:
    return [os.path.join(CSRC, s) for s in SOURCES]


def _deps() -> list[str]:
    out = sources()
    for d in (CSRC, os.path.join(ROOT, "include")):
        out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh", ".hpp"))]
    return out


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every source to an object in parallel (one nvcc per file), then
    link the shared library."""
    if not force and not stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]

    def compile_one(src: str) -> str:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC, *FLAGS, *inc, "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        return obj

    with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = LIB + ".tmp"
    subprocess.check_call([NVCC, *FLAGS, "-shared", *objs, "-o", tmp])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose="--verbose" in sys.argv)
    print(LIB)
