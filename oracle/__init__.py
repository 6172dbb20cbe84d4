"""Oracle loader: the CPU restatement and the compiled reference, via ctypes.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline / reference legs of ``bench.py`` import this package, and
only to check or to time the reference CPU path; the product
(``2020_song_ex_b200``) never imports it.

* ``libsong_oracle.so`` (``song_oracle.cpp``) restates the reference GPU
  search (kernalGraph.h:184-299, hashKernelGraph.h:238-352) on the CPU.
* ``_ref/<variant>/libref_{cpu,gpu}.so`` (``build_ref.py``) are the
  reference's own sources compiled for one config.h variant.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libsong_oracle.so")
ORACLE_SRC = os.path.join(HERE, "song_oracle.cpp")

TRACE_FIELDS = (
    "seed_count", "visited_nodes", "expanded_nodes", "neighbor_slots_scanned",
    "candidate_nodes", "distance_evals", "frontier_pushes", "result_updates",
    "peak_frontier", "peak_results", "result_count", "early_stopped",
)

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


def build_oracle(force: bool = False) -> str:
    """Compile the CPU restatement (no FP contraction: fmaf is explicit)."""
    if force or not os.path.exists(ORACLE_SO) or \
            os.path.getmtime(ORACLE_SO) < os.path.getmtime(ORACLE_SRC):
        cxx = os.environ.get("CXX", "g++")
        subprocess.check_call([cxx, "-std=c++17", "-O2", "-ffp-contract=off", "-shared", "-fPIC",
                               "-pthread", ORACLE_SRC, "-o", ORACLE_SO])
    return ORACLE_SO


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = C.CDLL(ORACLE_SO)
        L.oracle_clamp_ef.argtypes = [C.c_int, C.c_int, C.c_int]
        L.oracle_clamp_ef.restype = C.c_int
        L.oracle_warp_l2.argtypes = [_f32p, _f32p, C.c_int]
        L.oracle_warp_l2.restype = C.c_float
        L.oracle_search_l2.argtypes = [
            _f32p, C.c_int64, C.c_int, _i32p, C.c_int, _f32p, C.c_int, C.c_int, C.c_int,
            C.c_int, C.c_int, C.c_int, C.c_int, _i32p, C.c_void_p, C.c_int]
        L.oracle_search_l2.restype = C.c_int
        L.oracle_search_hamming.argtypes = [
            _u32p, C.c_int64, C.c_int, _i32p, C.c_int, _u32p, C.c_int, C.c_int, C.c_int,
            C.c_int, C.c_int, C.c_int, C.c_int, _i32p, C.c_void_p, C.c_int]
        L.oracle_search_hamming.restype = C.c_int
        L.oracle_graph_search.argtypes = [_f32p, C.c_int64, C.c_int, _i32p, C.c_int, _f32p,
                                          C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p]
        L.oracle_graph_search.restype = None
        L.oracle_bithash_matrix.argtypes = [C.c_int, C.c_int, C.c_uint, _f32p]
        L.oracle_bithash_matrix.restype = None
        L.oracle_bithash_project.argtypes = [_f32p, C.c_int, C.c_int, _f32p, C.c_int64, _u32p]
        L.oracle_bithash_project.restype = None
        _lib = L
    return _lib


def clamp_ef(ef: int, k: int, pq_size: int) -> int:
    return lib().oracle_clamp_ef(ef, k, pq_size)


def search_l2(data, adj, block_size, queries, k, ef, pq_size=50, bf_words=256, bf_nhash=4,
              n_multiprobe=4, threads=None, with_trace=True):
    """kg_search_kernel semantics for every query; ``ef`` as the kernel receives it."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    queries = np.ascontiguousarray(queries, dtype=np.float32)
    adj = np.ascontiguousarray(adj, dtype=np.int32).reshape(-1)
    n, dim = data.shape
    nq = queries.shape[0]
    ids = np.empty((nq, max(k, 0)), dtype=np.int32)
    trace = np.zeros((nq, 12), dtype=np.int32) if with_trace else None
    rc = lib().oracle_search_l2(
        data, n, dim, adj, block_size, queries, nq, k, ef, pq_size, bf_words, bf_nhash,
        n_multiprobe, ids, trace.ctypes.data if trace is not None else None,
        threads or os.cpu_count() or 1)
    if rc != 0:
        raise ValueError("oracle_search_l2: invalid arguments")
    return ids, trace


def search_hamming(codes, adj, block_size, qcodes, k, ef, pq_size=50, bf_words=256, bf_nhash=4,
                   n_multiprobe=4, threads=None, with_trace=True):
    """hkg_search_kernel semantics for every query."""
    codes = np.ascontiguousarray(codes, dtype=np.uint32)
    qcodes = np.ascontiguousarray(qcodes, dtype=np.uint32)
    adj = np.ascontiguousarray(adj, dtype=np.int32).reshape(-1)
    n, words = codes.shape
    nq = qcodes.shape[0]
    ids = np.empty((nq, max(k, 0)), dtype=np.int32)
    trace = np.zeros((nq, 12), dtype=np.int32) if with_trace else None
    rc = lib().oracle_search_hamming(
        codes, n, words, adj, block_size, qcodes, nq, k, ef, pq_size, bf_words, bf_nhash,
        n_multiprobe, ids, trace.ctypes.data if trace is not None else None,
        threads or os.cpu_count() or 1)
    if rc != 0:
        raise ValueError("oracle_search_hamming: invalid arguments")
    return ids, trace


def graph_search(data, adj, block_size, queries, k, ef, n_multiprobe=4):
    """Graph::search (graph.h:33-115) restated: ids worst-first (-1 padded) and traces."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    queries = np.ascontiguousarray(queries, dtype=np.float32)
    adj = np.ascontiguousarray(adj, dtype=np.int32).reshape(-1)
    n, dim = data.shape
    nq = queries.shape[0]
    ids = np.empty((nq, k), dtype=np.int32)
    trace = np.zeros((nq, 12), dtype=np.int32)
    lib().oracle_graph_search(data, n, dim, adj, block_size, queries, nq, k, ef, n_multiprobe,
                              ids, trace)
    return ids, trace


def bithash_matrix(dim: int, hash_bits: int, seed: int = 42) -> np.ndarray:
    R = np.empty((hash_bits, dim), dtype=np.float32)
    lib().oracle_bithash_matrix(dim, hash_bits, seed, R)
    return R


def bithash_project(R: np.ndarray, x: np.ndarray) -> np.ndarray:
    R = np.ascontiguousarray(R, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    hash_bits, dim = R.shape
    out = np.empty((x.shape[0], hash_bits // 32), dtype=np.uint32)
    lib().oracle_bithash_project(R, dim, hash_bits, x, x.shape[0], out)
    return out


# ------------------------------------------------------------ compiled reference

class RefLib:
    """The reference's own code for one config.h variant (see build_ref.py)."""

    def __init__(self, variant):
        from . import build_ref
        self.variant = variant
        self.dir = variant.dir
        cpu = os.path.join(self.dir, "libref_cpu.so")
        if not os.path.exists(cpu):
            if not os.path.isdir(build_ref.REF_DIR):
                raise FileNotFoundError(f"reference variant {variant.name} not built")
            build_ref.build_variant(variant, gpu=True, quiet=True)
        self.cpu = C.CDLL(cpu)
        self.cpu.ref_config.argtypes = [_i32p]
        self.cpu.ref_cpu_build_graph.argtypes = [_f32p, C.c_int, C.c_int, _i32p]
        self.cpu.ref_cpu_graph_create.argtypes = [_f32p, C.c_int, C.c_int, _i32p]
        self.cpu.ref_cpu_graph_create.restype = C.c_void_p
        self.cpu.ref_cpu_graph_destroy.argtypes = [C.c_void_p]
        self.cpu.ref_cpu_graph_search.argtypes = [C.c_void_p, _f32p, C.c_int, C.c_int, C.c_int,
                                                  C.c_int, _i32p, C.c_void_p]
        gpu = os.path.join(self.dir, "libref_gpu.so")
        self.gpu = None
        if os.path.exists(gpu):
            try:
                self.gpu = C.CDLL(gpu)
            except OSError:
                self.gpu = None
        if self.gpu is not None:
            g = self.gpu
            g.ref_build_kernel_graph.argtypes = [_f32p, C.c_int, C.c_int, _i32p]
            g.ref_build_hashed_graph.argtypes = [_f32p, C.c_int, C.c_int, _i32p, _u32p]
            g.ref_bithash_project.argtypes = [_f32p, C.c_int, C.c_int, C.c_uint, _u32p, C.c_void_p]
            _d = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
            g.ref_gpu_search_l2.argtypes = [_f32p, C.c_int, C.c_int, _i32p, _f32p, C.c_int, C.c_int,
                                            C.c_int, C.c_int, _i32p, _i32p, _d]
            g.ref_gpu_search_hamming.argtypes = [_u32p, C.c_int, _i32p, _u32p, C.c_int, C.c_int,
                                                 C.c_int, C.c_int, _i32p, _i32p, _d]

    def config(self) -> dict:
        v = np.zeros(12, dtype=np.int32)
        self.cpu.ref_config(v)
        keys = ("BLOCK_SIZE", "FIXED_DEGREE", "SEARCH_DEGREE", "EF_CONSTRUCTION", "pq_size", "TOPK",
                "N_MULTIPROBE", "N_MULTIQUERY", "hash_bits", "HASH_WORDS", "BF_WORDS", "BF_NHASH")
        return dict(zip(keys, (int(x) for x in v)))

    @property
    def block_size(self) -> int:
        return self.variant.block_size

    def build_graph(self, data: np.ndarray) -> np.ndarray:
        """build_kernel_graph (kernalGraph.h:140-149) -> adj [n, BLOCK_SIZE]."""
        data = np.ascontiguousarray(data, dtype=np.float32)
        n, dim = data.shape
        adj = np.empty((n, self.block_size), dtype=np.int32)
        fn = self.gpu.ref_build_kernel_graph if self.gpu is not None else self.cpu.ref_cpu_build_graph
        if fn(data, n, dim, adj) != 0:
            raise RuntimeError("reference graph build failed")
        return adj

    def build_hashed_graph(self, data: np.ndarray):
        """build_hashed_graph (hashKernelGraph.h:196-207) -> (adj, codes)."""
        data = np.ascontiguousarray(data, dtype=np.float32)
        n, dim = data.shape
        adj = np.empty((n, self.block_size), dtype=np.int32)
        codes = np.empty((n, self.variant.hash_bits // 32), dtype=np.uint32)
        if self.gpu.ref_build_hashed_graph(data, n, dim, adj, codes) != 0:
            raise RuntimeError("reference hashed graph build failed")
        return adj, codes

    def bithash_project(self, x: np.ndarray, seed: int = 42):
        x = np.ascontiguousarray(x, dtype=np.float32)
        n, dim = x.shape
        codes = np.empty((n, self.variant.hash_bits // 32), dtype=np.uint32)
        R = np.empty((self.variant.hash_bits, dim), dtype=np.float32)
        self.gpu.ref_bithash_project(x, n, dim, seed, codes, R.ctypes.data)
        return codes, R

    def cpu_graph(self, data: np.ndarray, adj: np.ndarray) -> "RefCpuGraph":
        return RefCpuGraph(self, data, adj)

    def gpu_search_l2(self, data, adj, queries, k, ef, n_multiquery=512):
        """gpu_search (kernalGraph.h:307-382): needs a GPU."""
        data = np.ascontiguousarray(data, dtype=np.float32)
        queries = np.ascontiguousarray(queries, dtype=np.float32)
        adj = np.ascontiguousarray(adj, dtype=np.int32).reshape(-1)
        n, dim = data.shape
        nq = queries.shape[0]
        ids = np.empty((nq, k), dtype=np.int32)
        trace = np.zeros((nq, 12), dtype=np.int32)
        timing = np.zeros(6, dtype=np.float64)
        rc = self.gpu.ref_gpu_search_l2(data, n, dim, adj, queries, nq, k, n_multiquery, ef,
                                        ids, trace, timing)
        if rc != 0:
            raise RuntimeError(f"reference gpu_search failed: cuda error {rc}")
        return ids, trace, timing

    def gpu_search_hamming(self, codes, adj, qcodes, k, ef, n_multiquery=512):
        codes = np.ascontiguousarray(codes, dtype=np.uint32)
        qcodes = np.ascontiguousarray(qcodes, dtype=np.uint32)
        adj = np.ascontiguousarray(adj, dtype=np.int32).reshape(-1)
        n = codes.shape[0]
        nq = qcodes.shape[0]
        ids = np.empty((nq, k), dtype=np.int32)
        trace = np.zeros((nq, 12), dtype=np.int32)
        timing = np.zeros(6, dtype=np.float64)
        rc = self.gpu.ref_gpu_search_hamming(codes, n, adj, qcodes, nq, k, n_multiquery, ef,
                                             ids, trace, timing)
        if rc != 0:
            raise RuntimeError(f"reference gpu_search (hash) failed: cuda error {rc}")
        return ids, trace, timing


class RefCpuGraph:
    """A reference ``Graph`` (graph.h:11-20) over a supplied adjacency."""

    def __init__(self, ref: RefLib, data: np.ndarray, adj: np.ndarray):
        self.ref = ref
        data = np.ascontiguousarray(data, dtype=np.float32)
        adj = np.ascontiguousarray(adj, dtype=np.int32).reshape(-1)
        self.n, self.dim = data.shape
        self.h = ref.cpu.ref_cpu_graph_create(data, self.n, self.dim, adj)

    def search(self, queries, k, ef, threads=1, with_trace=False):
        """Graph::search (graph.h:33-115); rows come back worst-first, as the reference returns."""
        queries = np.ascontiguousarray(queries, dtype=np.float32)
        nq = queries.shape[0]
        ids = np.empty((nq, k), dtype=np.int32)
        trace = np.zeros((nq, 12), dtype=np.int32) if with_trace else None
        self.ref.cpu.ref_cpu_graph_search(self.h, queries, nq, k, ef, threads, ids,
                                          trace.ctypes.data if trace is not None else None)
        return ids, trace

    def close(self):
        if self.h:
            self.ref.cpu.ref_cpu_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_refs: dict = {}


def ref(block_size=32, bf_words=256, pq_size=512, hash_bits=256, fixed_degree=None,
        search_degree=15, ef_construction=150) -> RefLib:
    """The compiled reference for one config.h variant (built on first use if possible)."""
    from .build_ref import RefVariant
    v = RefVariant(block_size=block_size,
                   fixed_degree=block_size - 1 if fixed_degree is None else fixed_degree,
                   search_degree=search_degree, ef_construction=ef_construction,
                   pq_size=pq_size, bf_words=bf_words, hash_bits=hash_bits)
    if v not in _refs:
        _refs[v] = RefLib(v)
    return _refs[v]


def ref_available(**kw) -> bool:
    try:
        ref(**kw)
        return True
    except (FileNotFoundError, OSError):
        return False
