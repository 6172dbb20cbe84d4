"""Build recipe for ``oracle/_ref``: the reference's own sources, compiled here.

TEST INFRASTRUCTURE ONLY.  Nothing in the product links or loads what this
script builds; tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of
``bench.py`` use it as a checker and as the timed reference CPU path.

The reference (lrlorry/2020_song_ex) fixes its search parameters at compile
time in ``config.h`` (config.h:9-58).  Each *variant* here is one choice of
those constants: the reference headers are copied into the git-ignored
``oracle/_ref/<variant>/src`` directory, ``config.h`` is rewritten with the
variant's constants, and two shared libraries are compiled against them:

* ``libref_cpu.so`` from ``oracle/ref_cpu.cpp`` (g++ -O3, the reference
  Makefile's CXXFLAGS): ``build_graph`` (graph.h:190-199) and the CPU search
  ``Graph::search`` (graph.h:33-115), single- or multi-threaded.
* ``libref_gpu.so`` from ``oracle/ref_gpu.cu`` (nvcc -O3 for sm_100a, the
  reference Makefile's NVCCFLAGS with ``ARCH=sm_100a``): the NSW builders of
  kernalGraph.h:140-149 / hashKernelGraph.h:196-207, ``BitHash``
  (bitHash.h:17-56) and the reference GPU search ``gpu_search``
  (kernalGraph.h:307-382, hashKernelGraph.h:360-435).  Its kernels only run on
  a GPU host; its builders run anywhere.

The reference sources are read from ``$SONG_REF_DIR``, or else from a
``reference`` checkout beside this repository (``../reference`` relative to
the repository root); nothing of them is committed.  Usage::

    python oracle/build_ref.py                 # the default variant set
    python oracle/build_ref.py --bs 16 --bfw 16 --pq 256
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys
from dataclasses import dataclass, asdict

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.environ.get("SONG_REF_DIR") or os.path.normpath(
    os.path.join(HERE, os.pardir, os.pardir, "reference"))
OUT_DIR = os.path.join(HERE, "_ref")
HEADERS = [
    "config.h", "distance.h", "telemetry.h", "graph.h", "kernalGraph.h",
    "hashKernelGraph.h", "bitHash.h", "gpuHeap.h", "bloomFilter.h", "parser.h",
]
NVCC = os.environ.get("NVCC", "nvcc")
CXX = os.environ.get("CXX", "g++")


@dataclass(frozen=True)
class RefVariant:
    """One compile-time configuration of the reference (config.h:9-58)."""
    block_size: int = 32       # BLOCK_SIZE
    fixed_degree: int = 31     # FIXED_DEGREE
    search_degree: int = 15    # SEARCH_DEGREE
    ef_construction: int = 150 # EF_CONSTRUCTION
    pq_size: int = 50          # pq_size
    bf_words: int = 256        # BF_WORDS
    hash_bits: int = 256       # hash_bits

    @property
    def name(self) -> str:
        return (f"bs{self.block_size}_fd{self.fixed_degree}_sd{self.search_degree}"
                f"_efc{self.ef_construction}_pq{self.pq_size}_bf{self.bf_words}"
                f"_hb{self.hash_bits}")

    @property
    def dir(self) -> str:
        return os.path.join(OUT_DIR, self.name)


# Variants the tests, fixtures and benchmarks use.
#  * C1: degree 16 (BLOCK_SIZE 16, FIXED_DEGREE 15), 1,024-bit Bloom filter.
#  * reference defaults with a queue cap large enough for every sweep point.
#  * 512-bit sign-random-projection codes for the Hamming variant.
DEFAULT_VARIANTS = [
    RefVariant(block_size=16, fixed_degree=15, search_degree=15, pq_size=512, bf_words=16),
    RefVariant(pq_size=512),
    RefVariant(pq_size=512, hash_bits=512),
    RefVariant(),
    # the benchmark's operating points (queue cap 1024)
    RefVariant(pq_size=1024, bf_words=256),
    RefVariant(pq_size=1024, bf_words=512),
    RefVariant(pq_size=1024, bf_words=1024),
]


def _rewrite_config(text: str, v: RefVariant) -> str:
    repl = {
        "BLOCK_SIZE": v.block_size, "FIXED_DEGREE": v.fixed_degree,
        "SEARCH_DEGREE": v.search_degree, "EF_CONSTRUCTION": v.ef_construction,
        "pq_size": v.pq_size, "BF_WORDS": v.bf_words, "hash_bits": v.hash_bits,
    }
    for name, val in repl.items():
        text, n = re.subn(rf"(constexpr int {name}\s*=\s*)\d+;", rf"\g<1>{val};", text)
        if n != 1:
            raise RuntimeError(f"config.h: constant {name} not found exactly once")
    return text


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_variant(v: RefVariant, gpu: bool = True, quiet: bool = False) -> str:
    """Copy + configure the reference headers for ``v`` and compile both libraries."""
    if not os.path.isdir(REF_DIR):
        raise FileNotFoundError(f"reference sources not found at {REF_DIR}")
    src = os.path.join(v.dir, "src")
    os.makedirs(src, exist_ok=True)
    for h in HEADERS:
        dst = os.path.join(src, h)
        with open(os.path.join(REF_DIR, h)) as f:
            text = f.read()
        if h == "config.h":
            text = _rewrite_config(text, v)
        old = open(dst).read() if os.path.exists(dst) else None
        if old != text:
            with open(dst, "w") as f:
                f.write(text)
    hdrs = [os.path.join(src, h) for h in HEADERS]
    cpu_so = os.path.join(v.dir, "libref_cpu.so")
    cpu_src = os.path.join(HERE, "ref_cpu.cpp")
    if _stale(cpu_so, hdrs + [cpu_src]):
        cmd = [CXX, "-std=c++17", "-O3", "-shared", "-fPIC", "-pthread", "-I", src,
               cpu_src, "-o", cpu_so]
        if not quiet:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    if gpu:
        gpu_so = os.path.join(v.dir, "libref_gpu.so")
        gpu_src = os.path.join(HERE, "ref_gpu.cu")
        if _stale(gpu_so, hdrs + [gpu_src]):
            cmd = [NVCC, "-std=c++17", "-O3", "-shared", "-Xcompiler", "-fPIC",
                   "-gencode", "arch=compute_100a,code=sm_100a", "-I", src,
                   gpu_src, "-o", gpu_so]
            if not quiet:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    with open(os.path.join(v.dir, "variant.txt"), "w") as f:
        f.write(repr(asdict(v)) + "\n")
    return v.dir


def build_all(gpu: bool = True, quiet: bool = False) -> None:
    for v in DEFAULT_VARIANTS:
        build_variant(v, gpu=gpu, quiet=quiet)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--bs", type=int)
    ap.add_argument("--fd", type=int)
    ap.add_argument("--sd", type=int)
    ap.add_argument("--efc", type=int)
    ap.add_argument("--pq", type=int)
    ap.add_argument("--bfw", type=int)
    ap.add_argument("--hb", type=int)
    ap.add_argument("--no-gpu", action="store_true")
    a = ap.parse_args(argv)
    if all(x is None for x in (a.bs, a.fd, a.sd, a.efc, a.pq, a.bfw, a.hb)):
        build_all(gpu=not a.no_gpu)
        return 0
    base = RefVariant()
    bs = a.bs if a.bs is not None else base.block_size
    v = RefVariant(
        block_size=bs,
        fixed_degree=a.fd if a.fd is not None else bs - 1,
        search_degree=a.sd if a.sd is not None else base.search_degree,
        ef_construction=a.efc if a.efc is not None else base.ef_construction,
        pq_size=a.pq if a.pq is not None else base.pq_size,
        bf_words=a.bfw if a.bfw is not None else base.bf_words,
        hash_bits=a.hb if a.hb is not None else base.hash_bits,
    )
    print(build_variant(v, gpu=not a.no_gpu))
    return 0


if __name__ == "__main__":
    sys.exit(main())
