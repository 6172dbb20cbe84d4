"""song_b200 -- B200-native SONG graph search behind the reference's interface.

Python mirror of the reference's search entry points (lrlorry/2020_song_ex),
calling the sm_100a kernels through the C ABI of ``include/song_b200.h``
(``libsong_b200.so``, built in-tree by ``build.py``):

* :class:`Params`           -- config.h:9-58 as runtime values.
* :class:`KernelGraph`      -- kernalGraph.h:20-71 (data + adj; ``upload_to_gpu``).
* :class:`HashKernelGraph`  -- hashKernelGraph.h:22-126 (codes + adj).
* :class:`BitHash`          -- bitHash.h:17-56, the projection on the GPU.
* :func:`gpu_search`        -- kernalGraph.h:307-382 and the Hamming overload
  hashKernelGraph.h:360-435: returns the flat ``[nq*k]`` id list, best-first,
  ``-1`` padded, optionally filling a :class:`GpuSearchTrace`.
* :func:`search_device`     -- the same search on device-resident tensors.

There is no CPU fallback: if the library is missing or no GPU is present the
calls raise :class:`SongError`.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field, fields
from typing import List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsong_b200.so")

SONG_OK = 0
SONG_ERR_INVALID_ARG = 1
SONG_ERR_OOM = 2
SONG_ERR_CUDA = 3
SONG_ERR_TIMEOUT = 4
SONG_ERR_BUDGET = 5
SONG_ERR_UNSUPPORTED = 6
KIND_L2 = 0
KIND_HAMMING = 1
PREC_FP32 = 0
PREC_BF16 = 1
PREC_FP8 = 2
ENTRY_MODEL = 0    # learned entry points: the entry model's top hubs
ENTRY_NEAREST = 1  # the entry stage's nearest hubs, no model
ENTRY_SEEDS = 2    # the reference's seeds p*n/N_MULTIPROBE, no entry stage

TRACE_FIELDS = (
    "seed_count", "visited_nodes", "expanded_nodes", "neighbor_slots_scanned",
    "candidate_nodes", "distance_evals", "frontier_pushes", "result_updates",
    "peak_frontier", "peak_results", "result_count", "early_stopped",
)


class SongError(RuntimeError):
    """A song_b200 call failed; ``status`` is the song_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[song status {status}] {message}")
        self.status = status


class _Params(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "block_size", "fixed_degree", "search_degree", "ef_construction", "pq_size", "topk",
        "n_multiprobe", "n_multiquery", "hash_bits", "bf_words", "bf_nhash")]


class _Timing(C.Structure):
    _fields_ = [("alloc_ms", C.c_double), ("h2d_ms", C.c_double), ("memset_ms", C.c_double),
                ("kernel_ms", C.c_double), ("d2h_ms", C.c_double), ("total_ms", C.c_double),
                ("ef_search", C.c_int), ("batch_limit", C.c_int), ("n_batches", C.c_int)]


class _Opts(C.Structure):
    _fields_ = [("precision", C.c_int), ("rerank", C.c_int), ("learned", C.c_int),
                ("stop_threshold", C.c_float), ("beam", C.c_int), ("bloom_hashes", C.c_int),
                ("entry", C.c_int), ("reserved", C.c_int)]


@dataclass
class SearchOpts:
    """Extended search options (song_search_opts): precision form, FP32
    re-rank, learned entry/stop model.  The defaults select the plain search."""
    precision: int = PREC_FP32
    rerank: bool = False
    learned: bool = False
    stop_threshold: float = 0.5
    beam: int = 1  # learned search: 2 expands the two best candidates per step
    bloom_hashes: int = 0  # learned search: Bloom hashes per id (0 = the index's bf_nhash)
    entry: int = 0  # learned search: ENTRY_MODEL, ENTRY_NEAREST (no model) or ENTRY_SEEDS

    def _c(self) -> _Opts:
        return _Opts(int(self.precision), int(bool(self.rerank)), int(bool(self.learned)),
                     float(self.stop_threshold), int(self.beam), int(self.bloom_hashes),
                     int(self.entry))


class _LearnParams(C.Structure):
    _fields_ = [("k", C.c_int), ("ef", C.c_int), ("ckpt_every", C.c_int),
                ("min_expansions", C.c_int), ("max_ckpt", C.c_int), ("entry_steps", C.c_int),
                ("stop_steps", C.c_int), ("batch", C.c_int), ("lr", C.c_float),
                ("seed", C.c_uint), ("entry_hubs", C.c_int)]


class _LearnReport(C.Structure):
    _fields_ = [("n_hubs", C.c_int), ("stop_samples", C.c_longlong),
                ("entry_loss_first", C.c_double), ("entry_loss_last", C.c_double),
                ("stop_loss_first", C.c_double), ("stop_loss_last", C.c_double),
                ("stop_pos_frac", C.c_double)]


class _ServerConfig(C.Structure):
    _fields_ = [("max_k", C.c_int), ("max_ef", C.c_int), ("precision", C.c_int),
                ("stop_threshold", C.c_float), ("ring_slots", C.c_int),
                ("hbm_budget", C.c_longlong), ("max_ctas", C.c_int), ("idle_exit_us", C.c_int)]


class _ServerStats(C.Structure):
    _fields_ = [("launches", C.c_longlong), ("idle_exits", C.c_longlong),
                ("poll_cap_exits", C.c_longlong), ("stop_exits", C.c_longlong),
                ("running", C.c_int)]


_lib: Optional[C.CDLL] = None


def load_library(build_if_missing: bool = True) -> C.CDLL:
    """Load libsong_b200.so (building it first when absent and nvcc is present)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise SongError(SONG_ERR_UNSUPPORTED, f"{LIB_PATH} is missing; run build.py")
        from importlib import import_module
        import_module(__name__ + ".build").build()
    L = C.CDLL(LIB_PATH)
    vp, i64, ci = C.c_void_p, C.c_int64, C.c_int
    L.song_params_default.argtypes = [C.POINTER(_Params)]
    L.song_params_default.restype = None
    L.song_last_error.restype = C.c_char_p
    L.song_version.restype = C.c_char_p
    L.song_index_create_l2.argtypes = [vp, i64, ci, vp, C.POINTER(_Params), C.POINTER(vp)]
    L.song_index_create_hamming.argtypes = [vp, i64, ci, vp, C.POINTER(_Params), C.POINTER(vp)]
    L.song_index_destroy.argtypes = [vp]
    L.song_index_info.argtypes = [vp, C.POINTER(i64), C.POINTER(ci), C.POINTER(ci)]
    L.song_gpu_search.argtypes = [vp, vp, ci, ci, ci, ci, vp, vp, C.POINTER(_Timing)]
    L.song_gpu_search_hamming.argtypes = [vp, vp, ci, ci, ci, ci, vp, vp, C.POINTER(_Timing)]
    L.song_search_device.argtypes = [vp, vp, ci, ci, ci, vp, vp, vp]
    L.song_kernel_launch_count.restype = C.c_int64
    L.song_build_graph.argtypes = [ci, vp, i64, ci, C.POINTER(_Params), ci, ci, vp]
    L.song_build_graph.restype = C.c_int
    L.song_index_set_precision.argtypes = [vp, ci]
    L.song_index_set_precision.restype = C.c_int
    L.song_search_device_ex.argtypes = [vp, C.POINTER(_Opts), vp, ci, ci, ci, vp, vp, vp, vp]
    L.song_search_device_ex.restype = C.c_int
    L.song_gpu_search_ex.argtypes = [vp, C.POINTER(_Opts), vp, ci, ci, ci, ci, vp, vp, vp,
                                     C.POINTER(_Timing)]
    L.song_gpu_search_ex.restype = C.c_int
    L.song_learn_params_default.argtypes = [C.POINTER(_LearnParams)]
    L.song_learn_params_default.restype = None
    L.song_index_learn.argtypes = [vp, C.POINTER(_LearnParams), vp, ci, vp, C.POINTER(_LearnReport)]
    L.song_index_learn.restype = C.c_int
    L.song_index_get_model.argtypes = [vp, vp, ci, C.POINTER(ci)]
    L.song_index_get_model.restype = C.c_int
    L.song_index_set_model.argtypes = [vp, vp, ci]
    L.song_index_set_model.restype = C.c_int
    L.song_mlp_grad.argtypes = [ci, ci, vp, vp, vp, vp, ci, vp, C.POINTER(C.c_double)]
    L.song_mlp_grad.restype = C.c_int
    L.song_server_config_default.argtypes = [C.POINTER(_ServerConfig)]
    L.song_server_config_default.restype = None
    L.song_server_create.argtypes = [vp, C.POINTER(_ServerConfig), C.POINTER(vp)]
    L.song_server_submit.argtypes = [vp, vp, ci, vp, vp, vp, C.POINTER(C.c_longlong)]
    L.song_server_poll.argtypes = [vp, C.c_longlong, vp, vp, vp, C.POINTER(ci)]
    L.song_server_run_poisson.argtypes = [vp, vp, ci, vp, vp, vp, C.c_double, C.c_uint, vp, vp,
                                          C.POINTER(C.c_double)]
    L.song_server_destroy.argtypes = [vp]
    L.song_server_wait.argtypes = [vp, C.c_longlong, C.c_longlong, vp, vp, vp]
    L.song_server_get_stats.argtypes = [vp, C.POINTER(_ServerStats)]
    L.song_search_device_seeded.argtypes = [vp, C.POINTER(_Opts), vp, ci, ci, ci, vp, ci, vp, vp,
                                            vp, vp]
    L.song_search_device_seeded.restype = C.c_int
    L.song_index_set_entry_hubs.argtypes = [vp, vp, ci]
    L.song_index_set_entry_hubs.restype = C.c_int
    L.song_index_entry_candidates.argtypes = [vp, vp, ci, vp, vp, vp]
    L.song_index_entry_candidates.restype = C.c_int
    L.song_graph_search.argtypes = [vp, vp, ci, ci, ci, vp, vp]
    L.song_graph_search.restype = C.c_int
    L.song_graph_search_device.argtypes = [vp, vp, ci, ci, ci, vp, vp, vp]
    L.song_graph_search_device.restype = C.c_int
    L.song_index_u8_rows.argtypes = [vp, C.POINTER(ci), C.POINTER(ci)]
    L.song_index_u8_rows.restype = C.c_int
    L.song_bithash_matrix.argtypes = [ci, ci, C.c_uint, vp]
    L.song_bithash_project.argtypes = [vp, ci, ci, vp, i64, vp]
    L.song_bithash_project_device.argtypes = [vp, ci, ci, vp, i64, i64, vp, i64, vp]
    for name in ("song_bithash_matrix", "song_bithash_project", "song_bithash_project_device"):
        getattr(L, name).restype = C.c_int
    L.song_exact_knn_device.argtypes = [vp, i64, i64, ci, vp, ci, i64, ci, vp, vp, vp]
    L.song_exact_knn_device.restype = C.c_int
    L.song_exact_knn.argtypes = [vp, i64, ci, vp, ci, ci, vp, vp]
    L.song_exact_knn.restype = C.c_int
    for name in ("song_server_create", "song_server_submit", "song_server_poll",
                 "song_server_run_poisson", "song_server_destroy", "song_server_wait",
                 "song_server_get_stats"):
        getattr(L, name).restype = C.c_int
    for name in ("song_index_create_l2", "song_index_create_hamming", "song_index_destroy",
                 "song_index_info", "song_gpu_search", "song_gpu_search_hamming",
                 "song_search_device"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def _check(status: int) -> None:
    if status != SONG_OK:
        msg = load_library().song_last_error().decode(errors="replace")
        raise SongError(status, msg)


def launch_count() -> int:
    """Search-kernel launches issued by the library in this process."""
    return int(load_library().song_kernel_launch_count())


@dataclass
class Params:
    """config.h:9-58 as runtime values; defaults are the reference's."""
    block_size: int = 32       # BLOCK_SIZE
    fixed_degree: int = 31     # FIXED_DEGREE
    search_degree: int = 15    # SEARCH_DEGREE
    ef_construction: int = 150 # EF_CONSTRUCTION
    pq_size: int = 50          # pq_size
    topk: int = 10             # TOPK
    n_multiprobe: int = 4      # N_MULTIPROBE
    n_multiquery: int = 512    # N_MULTIQUERY
    hash_bits: int = 256       # hash_bits
    bf_words: int = 256        # BF_WORDS
    bf_nhash: int = 4          # BF_NHASH

    @property
    def hash_words(self) -> int:  # HASH_WORDS, config.h:44
        return self.hash_bits // 32

    def _c(self) -> _Params:
        return _Params(**{f.name: int(getattr(self, f.name)) for f in fields(self)})


@dataclass
class QueryTrace:
    """telemetry.h:5-18."""
    seed_count: int = 0
    visited_nodes: int = 0
    expanded_nodes: int = 0
    neighbor_slots_scanned: int = 0
    candidate_nodes: int = 0
    distance_evals: int = 0
    frontier_pushes: int = 0
    result_updates: int = 0
    peak_frontier: int = 0
    peak_results: int = 0
    result_count: int = 0
    early_stopped: int = 0


@dataclass
class GpuSearchTrace:
    """telemetry.h:30-41; ``queries`` is an int32 array [nq, 12] in QueryTrace order."""
    ef_search: int = 0
    batch_limit: int = 0
    alloc_ms: float = 0.0
    h2d_ms: float = 0.0
    memset_ms: float = 0.0
    kernel_ms: float = 0.0
    d2h_ms: float = 0.0
    total_ms: float = 0.0
    n_batches: int = 0
    queries: np.ndarray = field(default_factory=lambda: np.zeros((0, 12), np.int32))

    def query(self, i: int) -> QueryTrace:
        return QueryTrace(*(int(v) for v in self.queries[i]))


class _Index:
    kind = KIND_L2

    def __init__(self, params: Optional[Params]):
        self.params = params or Params()
        self._h = C.c_void_p()

    @property
    def uploaded(self) -> bool:
        return bool(self._h)

    def close(self) -> None:
        if self._h:
            load_library().song_index_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class KernelGraph(_Index):
    """kernalGraph.h:20-71: FP32 ``data [n, dim]`` + ``adj [n, block_size]``."""
    kind = KIND_L2

    def __init__(self, num_nodes: int, dim: int, data, params: Optional[Params] = None,
                 adj=None):
        super().__init__(params)
        self.num_nodes = int(num_nodes)
        self.dim = int(dim)
        self.data = np.ascontiguousarray(np.asarray(data, dtype=np.float32).reshape(num_nodes, dim))
        bs = self.params.block_size
        self.adj = (np.full((num_nodes, bs), -1, np.int32) if adj is None
                    else np.ascontiguousarray(np.asarray(adj, dtype=np.int32).reshape(num_nodes, bs)))

    def add_vertex(self, u: int, neighbors) -> None:
        """kernalGraph.h:32-35."""
        m = min(len(neighbors), self.params.fixed_degree)
        self.adj[u, :m] = np.asarray(neighbors[:m], dtype=np.int32)

    def upload_to_gpu(self) -> None:
        """kernalGraph.h:38-43 (replaces any earlier upload)."""
        self.close()
        L = load_library()
        _check(L.song_index_create_l2(self.data.ctypes.data, self.num_nodes, self.dim,
                                      self.adj.ctypes.data, C.byref(self.params._c()),
                                      C.byref(self._h)))

    def u8_rows(self) -> int:
        """Bytes per row of the exact byte copy of the rows (0 when the base is
        not integer-valued in [0, 255]): the row size the plain and learned
        searches gather for integer queries in [0, 255]."""
        has, rb = C.c_int(), C.c_int()
        _check(load_library().song_index_u8_rows(self._h, C.byref(has), C.byref(rb)))
        return rb.value if has.value else 0


class HashKernelGraph(_Index):
    """hashKernelGraph.h:22-126: packed ``hashed [n, hash_words]`` codes + ``adj``."""
    kind = KIND_HAMMING

    def __init__(self, num_nodes: int, hashed, params: Optional[Params] = None, adj=None):
        super().__init__(params)
        self.num_nodes = int(num_nodes)
        self.hashed = np.ascontiguousarray(np.asarray(hashed, dtype=np.uint32).reshape(num_nodes, -1))
        self.hash_words = self.hashed.shape[1]
        bs = self.params.block_size
        self.adj = (np.full((num_nodes, bs), -1, np.int32) if adj is None
                    else np.ascontiguousarray(np.asarray(adj, dtype=np.int32).reshape(num_nodes, bs)))

    def upload_to_gpu(self) -> None:
        self.close()
        L = load_library()
        _check(L.song_index_create_hamming(self.hashed.ctypes.data, self.num_nodes,
                                           self.hash_words, self.adj.ctypes.data,
                                           C.byref(self.params._c()), C.byref(self._h)))


class BitHash:
    """BitHash (bitHash.h:17-56): 1-bit Gaussian random projection to
    ``hash_bits`` sign bits packed in u32 words.  The matrix ``R`` is drawn
    exactly as the reference's constructor draws it (bitHash.h:23-27); the
    projection runs on the GPU and is bit-identical to ``BitHash::project``
    (sequential FP32 dot, separate multiply and add, ``dot > 0``)."""

    def __init__(self, dim: int, seed: int = 42, hash_bits: int = 256):
        self.dim = int(dim)
        self.hash_bits = int(hash_bits)
        self.R = np.empty((self.hash_bits, self.dim), np.float32)
        _check(load_library().song_bithash_matrix(self.dim, self.hash_bits, int(seed),
                                                  self.R.ctypes.data))

    @property
    def hash_words(self) -> int:  # HASH_WORDS, config.h:44
        return self.hash_bits // 32

    def project_all(self, data, n: Optional[int] = None) -> np.ndarray:
        """bitHash.h:51-56: codes [n, hash_words] (u32) of data [n, dim]."""
        x = np.ascontiguousarray(np.asarray(data, np.float32).reshape(-1, self.dim))
        if n is not None:
            x = x[:n]
        out = np.empty((x.shape[0], self.hash_words), np.uint32)
        _check(load_library().song_bithash_project(self.R.ctypes.data, self.dim, self.hash_bits,
                                                   x.ctypes.data, x.shape[0], out.ctypes.data))
        return out

    def project(self, vec) -> np.ndarray:
        """bitHash.h:32-44: the code words of one vector."""
        return self.project_all(np.asarray(vec, np.float32).reshape(1, self.dim))[0]

    def project_device(self, d_R, d_x, n: int, d_codes, ldx: Optional[int] = None,
                       ldc: Optional[int] = None, stream=None) -> None:
        """project_all on device tensors (R as uploaded by the caller), async."""
        def ptr(t):
            return C.c_void_p(t.data_ptr() if hasattr(t, "data_ptr") else int(t))
        st = C.c_void_p(stream.cuda_stream if stream is not None else 0)
        _check(load_library().song_bithash_project_device(
            ptr(d_R), self.dim, self.hash_bits, ptr(d_x), int(n),
            int(ldx if ldx is not None else self.dim), ptr(d_codes),
            int(ldc if ldc is not None else self.hash_words), st))


def build_graph(rows, params: Optional[Params] = None, kind: int = KIND_L2,
                batch_ratio: int = 32, build_bf_words: int = 1024) -> np.ndarray:
    """NSW adjacency [n, block_size] built on the GPU (song_build_graph).

    The reference's insertion algorithm (kernalGraph.h:140-149) run in
    batches of max(1, inserted/batch_ratio) nodes; ``rows`` is FP32
    ``[n, dim]`` for KIND_L2 or uint32 codes ``[n, words]`` for KIND_HAMMING.
    """
    params = params or Params()
    dt = np.float32 if kind == KIND_L2 else np.uint32
    rows = np.ascontiguousarray(np.asarray(rows, dtype=dt))
    n, dim = rows.shape
    adj = np.empty((n, params.block_size), dtype=np.int32)
    _check(load_library().song_build_graph(kind, rows.ctypes.data, n, dim,
                                           C.byref(params._c()), batch_ratio, build_bf_words,
                                           adj.ctypes.data))
    return adj


def build_kernel_graph(data, n: int, dim: int, params: Optional[Params] = None,
                       batch_ratio: int = 32) -> KernelGraph:
    """build_kernel_graph (kernalGraph.h:140-149), built on the GPU."""
    params = params or Params()
    data = np.ascontiguousarray(np.asarray(data, dtype=np.float32).reshape(n, dim))
    adj = build_graph(data, params, KIND_L2, batch_ratio)
    return KernelGraph(n, dim, data, params, adj=adj)


def gpu_search(g, queries, nq: int, k: int, N_MULTIQUERY: int = 512, ef_search: Optional[int] = None,
               trace: Optional[GpuSearchTrace] = None) -> np.ndarray:
    """gpu_search (kernalGraph.h:307-382 / hashKernelGraph.h:360-435).

    ``queries`` is ``[nq, dim]`` FP32 for a :class:`KernelGraph` or
    ``[nq, hash_words]`` uint32 codes for a :class:`HashKernelGraph`.
    ``ef_search`` defaults to ``pq_size`` and is clamped like the reference.
    Returns the flat ``[nq*k]`` int32 ids, best-first, -1 padded.
    """
    if not g.uploaded:
        raise SongError(SONG_ERR_INVALID_ARG, "graph not uploaded (call upload_to_gpu first)")
    L = load_library()
    ef = g.params.pq_size if ef_search is None else int(ef_search)
    if g.kind == KIND_L2:
        q = np.ascontiguousarray(np.asarray(queries, dtype=np.float32).reshape(nq, g.dim))
        fn = L.song_gpu_search
    else:
        q = np.ascontiguousarray(np.asarray(queries, dtype=np.uint32).reshape(nq, g.hash_words))
        fn = L.song_gpu_search_hamming
    ids = np.empty(max(nq * k, 1), dtype=np.int32)
    tq = np.zeros((nq, 12), dtype=np.int32) if trace is not None else None
    t = _Timing()
    _check(fn(g._h, q.ctypes.data, nq, k, N_MULTIQUERY, ef, ids.ctypes.data,
              tq.ctypes.data if tq is not None else None, C.byref(t)))
    if trace is not None:
        trace.ef_search, trace.batch_limit = t.ef_search, t.batch_limit
        trace.alloc_ms, trace.h2d_ms, trace.memset_ms = t.alloc_ms, t.h2d_ms, t.memset_ms
        trace.kernel_ms, trace.d2h_ms, trace.total_ms = t.kernel_ms, t.d2h_ms, t.total_ms
        trace.n_batches = t.n_batches
        trace.queries = tq
    return ids[: nq * k]


def search_device(g, d_queries, nq: int, k: int, ef_search: int, d_ids, d_traces=None,
                  stream=None) -> None:
    """Asynchronous search on device pointers (ints) or torch CUDA tensors."""
    def ptr(x):
        if x is None:
            return None
        return int(x.data_ptr()) if hasattr(x, "data_ptr") else int(x)
    st = None
    if stream is not None:
        st = int(getattr(stream, "cuda_stream", stream))
    _check(load_library().song_search_device(g._h, ptr(d_queries), nq, k, ef_search, ptr(d_ids),
                                             ptr(d_traces), st))


def set_precision(g: KernelGraph, precision: int) -> None:
    """Attach a BF16 or FP8 (per-vector scale) copy of the rows for the precision form."""
    _check(load_library().song_index_set_precision(g._h, int(precision)))


def search_device_ex(g, opts: Optional[SearchOpts], d_queries, nq: int, k: int, ef_search: int,
                     d_ids, d_dists=None, d_traces=None, stream=None) -> None:
    """song_search_device_ex on device pointers / torch CUDA tensors (asynchronous)."""
    def ptr(x):
        if x is None:
            return None
        return int(x.data_ptr()) if hasattr(x, "data_ptr") else int(x)
    st = None
    if stream is not None:
        st = int(getattr(stream, "cuda_stream", stream))
    o = (opts or SearchOpts())._c()
    _check(load_library().song_search_device_ex(g._h, C.byref(o), ptr(d_queries), nq, k,
                                                ef_search, ptr(d_ids), ptr(d_dists),
                                                ptr(d_traces), st))


def graph_search(g: KernelGraph, queries, nq: int, k: int, ef_search: int = 0):
    """Graph::search (graph.h:33-115) on the GPU: returns (ids [nq, k] worst-first
    as the reference returns them, -1 padded; traces int32 [nq, 12])."""
    q = np.ascontiguousarray(np.asarray(queries, np.float32).reshape(nq, -1))
    ids = np.empty((nq, k), np.int32)
    tr = np.zeros((nq, 12), np.int32)
    _check(load_library().song_graph_search(g._h, q.ctypes.data, nq, k, ef_search,
                                            ids.ctypes.data, tr.ctypes.data))
    return ids, tr


def exact_knn_device(d_base, n: int, dim: int, d_queries, nq: int, k: int, d_ids, d_dists,
                     ldb: Optional[int] = None, ldq: Optional[int] = None, stream=None) -> None:
    """Exact kNN (squared L2) of device rows on the tensor cores: ids [nq, k]
    int32 ascending by (distance, id) and their FP32 distances.  Replaces the
    reference's brute force (bench_cpu.cpp:158-175, run_compare.py:199-213)."""
    def ptr(t):
        return C.c_void_p(t.data_ptr() if hasattr(t, "data_ptr") else int(t))
    st = C.c_void_p(stream.cuda_stream if stream is not None else 0)
    _check(load_library().song_exact_knn_device(
        ptr(d_base), int(n), int(ldb if ldb is not None else dim), int(dim), ptr(d_queries),
        int(nq), int(ldq if ldq is not None else dim), int(k), ptr(d_ids), ptr(d_dists), st))


def exact_knn(base, queries, k: int):
    """exact_knn_device on host arrays: returns (ids [nq, k] int32, dists [nq, k] f32)."""
    b = np.ascontiguousarray(np.asarray(base, np.float32))
    q = np.ascontiguousarray(np.asarray(queries, np.float32).reshape(-1, b.shape[1]))
    ids = np.empty((q.shape[0], k), np.int32)
    d = np.empty((q.shape[0], k), np.float32)
    _check(load_library().song_exact_knn(b.ctypes.data, b.shape[0], b.shape[1], q.ctypes.data,
                                         q.shape[0], int(k), ids.ctypes.data, d.ctypes.data))
    return ids, d


ENTRY_K = 24  # entry candidates per query (the entry model's inputs)


def set_entry_hubs(g: KernelGraph, hub_ids) -> None:
    """Attach the hub set of the learned entry stage (node ids)."""
    h = np.ascontiguousarray(np.asarray(hub_ids, np.int32).reshape(-1))
    _check(load_library().song_index_set_entry_hubs(g._h, h.ctypes.data, int(h.size)))


def entry_candidates(g: KernelGraph, d_queries, nq: int, d_ids, d_dists, stream=None) -> None:
    """The entry stage alone: each query's 24 nearest hubs (device int32 /
    float32 [nq, 24]), from the tensor-core kernel."""
    st = None
    if stream is not None:
        st = int(getattr(stream, "cuda_stream", stream))
    _check(load_library().song_index_entry_candidates(
        g._h, int(d_queries.data_ptr()), nq, int(d_ids.data_ptr()), int(d_dists.data_ptr()), st))


def search_device_seeded(g, opts: Optional[SearchOpts], d_queries, nq: int, k: int,
                         ef_search: int, d_seeds, n_seeds: int, d_ids, d_dists=None,
                         d_traces=None, stream=None) -> None:
    """song_search_device_seeded: the extended search from per-query entry
    points d_seeds [nq, n_seeds] (device int32) instead of p*n/N_MULTIPROBE."""
    def ptr(x):
        if x is None:
            return None
        return int(x.data_ptr()) if hasattr(x, "data_ptr") else int(x)
    st = None
    if stream is not None:
        st = int(getattr(stream, "cuda_stream", stream))
    o = (opts or SearchOpts())._c()
    _check(load_library().song_search_device_seeded(g._h, C.byref(o), ptr(d_queries), nq, k,
                                                    ef_search, ptr(d_seeds), n_seeds, ptr(d_ids),
                                                    ptr(d_dists), ptr(d_traces), st))


def gpu_search_ex(g, opts: Optional[SearchOpts], queries, nq: int, k: int,
                  ef_search: Optional[int] = None, N_MULTIQUERY: int = 512,
                  trace: Optional[GpuSearchTrace] = None):
    """Host-buffer extended search; returns (ids [nq, k], dists [nq, k])."""
    L = load_library()
    ef = g.params.pq_size if ef_search is None else int(ef_search)
    q = np.ascontiguousarray(np.asarray(queries, dtype=np.float32).reshape(nq, -1))
    ids = np.empty((nq, max(k, 1)), dtype=np.int32)
    dists = np.empty((nq, max(k, 1)), dtype=np.float32)
    tq = np.zeros((nq, 12), dtype=np.int32) if trace is not None else None
    t = _Timing()
    o = (opts or SearchOpts())._c()
    _check(L.song_gpu_search_ex(g._h, C.byref(o), q.ctypes.data, nq, k, N_MULTIQUERY, ef,
                                ids.ctypes.data, dists.ctypes.data,
                                tq.ctypes.data if tq is not None else None, C.byref(t)))
    if trace is not None:
        trace.ef_search, trace.kernel_ms, trace.total_ms = t.ef_search, t.kernel_ms, t.total_ms
        trace.queries = tq
    return ids[:, :k], dists[:, :k]


@dataclass
class LearnParams:
    """song_learn_params: traces come from the plain search at (k, ef)."""
    k: int = 10
    ef: int = 128
    ckpt_every: int = 8
    min_expansions: int = 8
    max_ckpt: int = 256
    entry_steps: int = 1500
    stop_steps: int = 3000
    batch: int = 4096
    lr: float = 2e-3
    seed: int = 2020
    entry_hubs: int = 8192  # hub set of the tensor-core entry stage; 0 = 24 in-kernel hubs

    def _c(self) -> _LearnParams:
        return _LearnParams(self.k, self.ef, self.ckpt_every, self.min_expansions, self.max_ckpt,
                            self.entry_steps, self.stop_steps, self.batch, float(self.lr),
                            int(self.seed), int(self.entry_hubs))


def learn(g: KernelGraph, d_train_queries, nq: int, d_train_nn1,
          params: Optional[LearnParams] = None) -> dict:
    """Train the entry and stop models on the GPU (song_index_learn).

    ``d_train_queries`` [nq, dim] FP32 and ``d_train_nn1`` [nq] int32 (the
    exact nearest neighbour of each training query) are device tensors.
    """
    p = (params or LearnParams())._c()
    rep = _LearnReport()
    _check(load_library().song_index_learn(g._h, C.byref(p), int(d_train_queries.data_ptr()), nq,
                                           int(d_train_nn1.data_ptr()), C.byref(rep)))
    return {f: getattr(rep, f) for f, _ in _LearnReport._fields_}


def get_model(g: KernelGraph) -> np.ndarray:
    """The attached learned models as a flat float32 array (save with np.save)."""
    L = load_library()
    n = C.c_int()
    _check(L.song_index_get_model(g._h, None, 0, C.byref(n)))
    blob = np.empty(n.value, dtype=np.float32)
    _check(L.song_index_get_model(g._h, blob.ctypes.data, n.value, C.byref(n)))
    return blob


def set_model(g: KernelGraph, blob: np.ndarray) -> None:
    blob = np.ascontiguousarray(blob, dtype=np.float32)
    _check(load_library().song_index_set_model(g._h, blob.ctypes.data, blob.size))


def mlp_grad(params: np.ndarray, out: int, loss_kind: int, x, y, w=None):
    """Mean loss and parameter gradient of the learned-model MLP from the GPU
    training kernels (song_mlp_grad)."""
    params = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    wp = None if w is None else np.ascontiguousarray(w, dtype=np.float32)
    g = np.empty_like(params)
    loss = C.c_double()
    _check(load_library().song_mlp_grad(out, loss_kind, params.ctypes.data, x.ctypes.data,
                                        y.ctypes.data, wp.ctypes.data if wp is not None else None,
                                        x.shape[0], g.ctypes.data, C.byref(loss)))
    return g, loss.value


REQ_LEARNED = 1


@dataclass
class ServerConfig:
    """song_server_config (see include/song_b200.h)."""
    max_k: int = 100
    max_ef: int = 256
    precision: int = PREC_FP32
    stop_threshold: float = 0.85
    ring_slots: int = 4096
    hbm_budget: int = 0
    max_ctas: int = 0
    idle_exit_us: int = 200000

    def _c(self) -> _ServerConfig:
        return _ServerConfig(self.max_k, self.max_ef, self.precision, float(self.stop_threshold),
                             self.ring_slots, int(self.hbm_budget), self.max_ctas,
                             self.idle_exit_us)


class Server:
    """Serving loop with continuous batching over an uploaded L2 index."""

    def __init__(self, g: KernelGraph, config: Optional[ServerConfig] = None):
        self.config = config or ServerConfig()
        self.g = g
        self._h = C.c_void_p()
        _check(load_library().song_server_create(g._h, C.byref(self.config._c()),
                                                 C.byref(self._h)))

    def submit(self, queries, ks, efs, flags=None) -> int:
        q = np.ascontiguousarray(np.asarray(queries, dtype=np.float32).reshape(len(ks), -1))
        ks = np.ascontiguousarray(ks, dtype=np.int32)
        efs = np.ascontiguousarray(efs, dtype=np.int32)
        fl = None if flags is None else np.ascontiguousarray(flags, dtype=np.int32)
        t = C.c_longlong()
        _check(load_library().song_server_submit(self._h, q.ctypes.data, len(ks), ks.ctypes.data,
                                                 efs.ctypes.data,
                                                 fl.ctypes.data if fl is not None else None,
                                                 C.byref(t)))
        return t.value

    def poll(self, ticket: int, k: int):
        """(done, ids[:k], dists[:k], QueryTrace row) of a ticket."""
        ids = np.empty(self.config.max_k, dtype=np.int32)
        d = np.empty(self.config.max_k, dtype=np.float32)
        tr = np.zeros(12, dtype=np.int32)
        done = C.c_int()
        _check(load_library().song_server_poll(self._h, ticket, ids.ctypes.data, d.ctypes.data,
                                               tr.ctypes.data, C.byref(done)))
        return bool(done.value), ids[:k], d[:k], tr

    def wait(self, ticket: int, k: int, timeout_us: int):
        """(ids[:k], dists[:k], QueryTrace row) once the ticket finished; raises
        SongError(SONG_ERR_TIMEOUT) if it has not within timeout_us."""
        ids = np.empty(self.config.max_k, dtype=np.int32)
        d = np.empty(self.config.max_k, dtype=np.float32)
        tr = np.zeros(12, dtype=np.int32)
        _check(load_library().song_server_wait(self._h, ticket, int(timeout_us), ids.ctypes.data,
                                               d.ctypes.data, tr.ctypes.data))
        return ids[:k], d[:k], tr

    def stats(self) -> dict:
        """Launch count, running flag and why the kernel's warps left (song_server_get_stats)."""
        st = _ServerStats()
        _check(load_library().song_server_get_stats(self._h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in _ServerStats._fields_}

    def run_poisson(self, queries, ks, efs, flags, rate_qps: float, seed: int = 0):
        """Native Poisson-arrival driver: (latency_ms [nq], ids [nq, max_k], wall_s)."""
        q = np.ascontiguousarray(np.asarray(queries, dtype=np.float32))
        nq = q.shape[0]
        ks = np.ascontiguousarray(ks, dtype=np.int32)
        efs = np.ascontiguousarray(efs, dtype=np.int32)
        fl = None if flags is None else np.ascontiguousarray(flags, dtype=np.int32)
        lat = np.empty(nq, dtype=np.float64)
        ids = np.empty((nq, self.config.max_k), dtype=np.int32)
        wall = C.c_double()
        _check(load_library().song_server_run_poisson(
            self._h, q.ctypes.data, nq, ks.ctypes.data, efs.ctypes.data,
            fl.ctypes.data if fl is not None else None, float(rate_qps), int(seed),
            lat.ctypes.data, ids.ctypes.data, C.byref(wall)))
        return lat, ids, wall.value

    def close(self) -> None:
        if self._h:
            load_library().song_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
