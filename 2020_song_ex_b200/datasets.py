"""Seeded synthetic base/query sets with the shapes of the reference's benchmarks.

The reference benchmarks on SIFT1M, GIST1M, GloVe-200 and NYTimes-256
(run_compare.py:23-60).  Those datasets are not available here, so every
workload is a seeded synthetic mixture with the same shape, size and value
distribution class:

* ``int_mixture``   -- SIFT-shaped: isotropic Gaussian mixture, centres
  uniform in [0, 255], sigma 20, clipped and rounded to integers 0..255
  (stored as FP32, like fvecs).  With dim 128 every squared L2 distance is an
  integer below 2**24, so FP32 sums are exact in any order.
* ``l1_mixture``    -- GIST-shaped: non-negative mixture, L1-normalised.
* ``angular_mixture`` -- GloVe-shaped: anisotropic mixture, L2-normalised
  (the reference L2-normalises cosine sets, run_compare.py:183-186).

Also the reference's file formats: fvecs/ivecs (parser.h:10-38) and the
int32 ``.npy`` ground truth (bench_cpu.cpp:177-233).
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Mixture:
    """Base and query draws from one mixture (independent component picks)."""
    base: np.ndarray     # float32 [n, dim], C-contiguous
    queries: np.ndarray  # float32 [nq, dim]
    seed: int


def _pick(rng: np.random.Generator, n: int, n_comp: int) -> np.ndarray:
    return rng.integers(0, n_comp, size=n)


def int_mixture(n: int, nq: int, dim: int = 128, n_comp: int = 64, sigma: float = 20.0,
                seed: int = 0, chunk: int = 1 << 18, query_seed=None,
                with_base: bool = True) -> Mixture:
    """Integer-valued FP32 points: centre ~ U[0,255]^dim + N(0, sigma^2), clip, round.

    ``query_seed`` draws the queries from the same mixture with a separate
    generator (independent query sets over one base, e.g. one per GPU); with
    it, ``with_base=False`` skips drawing the base (``base`` is then empty)
    and the queries are the same as with it.
    """
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, 255.0, size=(n_comp, dim))

    def draw(m: int) -> np.ndarray:
        out = np.empty((m, dim), dtype=np.float32)
        for s in range(0, m, chunk):
            e = min(m, s + chunk)
            c = centres[_pick(rng, e - s, n_comp)]
            x = c + rng.normal(0.0, sigma, size=(e - s, dim))
            np.clip(np.rint(x), 0.0, 255.0, out=x)
            out[s:e] = x
        return out

    if query_seed is not None and not with_base:
        base = np.zeros((0, dim), dtype=np.float32)
    else:
        base = draw(n)
    if query_seed is not None:
        rng = np.random.default_rng(query_seed)
    queries = draw(nq)
    return Mixture(base, queries, seed)


def l1_mixture(n: int, nq: int, dim: int = 960, n_comp: int = 256, seed: int = 0,
               chunk: int = 1 << 16, rank: int = 16) -> Mixture:
    """Non-negative mixture, each vector L1-normalised (GIST-shaped).

    Centres are Gamma(2, 1) per dimension.  Each component spreads mostly
    along `rank` random directions of its own (per-dimension scale about
    0.7) plus a small isotropic part (0.1 per dimension): a Gaussian mixture
    whose neighbourhoods have the low intrinsic dimension of real image
    descriptors.  A purely isotropic spread in 960 dimensions would make all
    points of a component nearly equidistant, which no graph search (nor the
    reference's) can rank.  Values are clipped at 0, then each vector is
    divided by its sum.
    """
    rng = np.random.default_rng(seed)
    centres = rng.gamma(2.0, 1.0, size=(n_comp, dim))
    basis = rng.normal(0.0, 0.7 / np.sqrt(rank), size=(n_comp, rank, dim))

    def draw(m: int) -> np.ndarray:
        out = np.empty((m, dim), dtype=np.float32)
        for s in range(0, m, chunk):
            e = min(m, s + chunk)
            c = _pick(rng, e - s, n_comp)
            z = rng.normal(0.0, 1.0, size=(e - s, rank))
            x = centres[c] + rng.normal(0.0, 0.1, size=(e - s, dim))
            for k in np.unique(c):
                sel = np.nonzero(c == k)[0]
                x[sel] += z[sel] @ basis[k]
            np.maximum(x, 0.0, out=x)
            x /= np.maximum(x.sum(axis=1, keepdims=True), 1e-12)
            out[s:e] = x
        return out

    return Mixture(draw(n), draw(nq), seed)


def angular_mixture(n: int, nq: int, dim: int = 200, n_comp: int = 512, seed: int = 0,
                    chunk: int = 1 << 16) -> Mixture:
    """Anisotropic Gaussian mixture, each vector L2-normalised (GloVe-shaped)."""
    rng = np.random.default_rng(seed)
    centres = rng.normal(0.0, 1.0, size=(n_comp, dim))
    scales = np.exp(rng.normal(-0.5, 0.5, size=(n_comp, dim)))

    def draw(m: int) -> np.ndarray:
        out = np.empty((m, dim), dtype=np.float32)
        for s in range(0, m, chunk):
            e = min(m, s + chunk)
            c = _pick(rng, e - s, n_comp)
            x = centres[c] + scales[c] * rng.normal(0.0, 1.0, size=(e - s, dim))
            x /= np.maximum(np.linalg.norm(x, axis=1, keepdims=True), 1e-12)
            out[s:e] = x
        return out

    return Mixture(draw(n), draw(nq), seed)


# ---------------------------------------------------------------- file formats

def write_fvecs(path: str, x: np.ndarray) -> None:
    """fvecs: per vector int32 dim then dim float32 values (parser.h:10-21)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    n, d = x.shape
    rec = np.empty((n, d + 1), dtype=np.float32)
    rec[:, 0] = np.frombuffer(struct.pack("<i", d), dtype=np.float32)[0]
    rec[:, 1:] = x
    rec.tofile(path)


def read_fvecs(path: str) -> np.ndarray:
    """Read an fvecs file (parser.h:10-21); raises on a malformed size."""
    raw = np.fromfile(path, dtype=np.int32)
    if raw.size == 0:
        return np.zeros((0, 0), dtype=np.float32)
    d = int(raw[0])
    if d <= 0 or raw.size % (d + 1) != 0:
        raise ValueError(f"{path}: not an fvecs file (dim {d}, {raw.size} words)")
    rec = raw.reshape(-1, d + 1)
    if np.any(rec[:, 0] != d):
        raise ValueError(f"{path}: ragged fvecs records")
    return rec[:, 1:].view(np.float32).copy()


def write_ivecs(path: str, x: np.ndarray) -> None:
    x = np.ascontiguousarray(x, dtype=np.int32)
    n, d = x.shape
    rec = np.empty((n, d + 1), dtype=np.int32)
    rec[:, 0] = d
    rec[:, 1:] = x
    rec.tofile(path)


def read_ivecs(path: str) -> np.ndarray:
    """Read an ivecs file (parser.h:27-38)."""
    raw = np.fromfile(path, dtype=np.int32)
    if raw.size == 0:
        return np.zeros((0, 0), dtype=np.int32)
    d = int(raw[0])
    if d <= 0 or raw.size % (d + 1) != 0:
        raise ValueError(f"{path}: not an ivecs file")
    rec = raw.reshape(-1, d + 1)
    if np.any(rec[:, 0] != d):
        raise ValueError(f"{path}: ragged ivecs records")
    return rec[:, 1:].copy()


def write_gt_npy(path: str, gt: np.ndarray) -> None:
    """Ground truth as an int32 ``.npy`` (the format bench_cpu --gt-npy reads)."""
    np.save(path, np.ascontiguousarray(gt, dtype=np.int32))


def load_gt_npy(path: str, nq: int, k: int) -> np.ndarray:
    """Mirror of load_gt_npy (bench_cpu.cpp:177-233): int32 [rows, cols], rows>=nq, cols>=k."""
    gt = np.load(path)
    if gt.ndim != 2 or gt.shape[0] < nq or gt.shape[1] < k:
        raise ValueError(f"gt npy smaller than requested nq/k: {path}")
    return np.ascontiguousarray(gt[:nq, :k], dtype=np.int32)


def recall_at_k(ids: np.ndarray, gt: np.ndarray, k: int) -> np.ndarray:
    """Per-query recall@k = |ids[:k] ∩ gt[:k]| / k (bench_cpu.cpp:235-247)."""
    ids = np.asarray(ids)[:, :k]
    gt = np.asarray(gt)[:, :k]
    hits = (ids[:, :, None] == gt[:, None, :]).any(axis=2).sum(axis=1)
    return hits / float(k)


GRAPH_MAGIC = 0x3148505247474E53  # the bytes "SNGGRPH1" read as a little-endian u64


def save_graph(path: str, adj: np.ndarray) -> None:
    """Write an adjacency in the ``song_graph`` v1 format: u64 magic, u32
    version (1), u32 block_size, u64 n, then int32 [n x block_size] exactly as
    the reference's in-memory ``adj`` (graph.h:14-15; -1 = empty slot).  The
    reference itself never serialises its graph (it rebuilds it every run)."""
    adj = np.ascontiguousarray(adj, dtype=np.int32)
    n, bs = adj.shape
    with open(path, "wb") as f:
        np.array([GRAPH_MAGIC], dtype=np.uint64).tofile(f)
        np.array([1, bs], dtype=np.uint32).tofile(f)
        np.array([n], dtype=np.uint64).tofile(f)
        adj.tofile(f)


def load_graph(path: str) -> np.ndarray:
    """Read a ``song_graph`` v1 file; raises ValueError on a malformed file."""
    with open(path, "rb") as f:
        head = f.read(24)
        if len(head) != 24:
            raise ValueError(f"{path}: truncated graph header")
        magic = int(np.frombuffer(head[:8], dtype=np.uint64)[0])
        ver, bs = (int(x) for x in np.frombuffer(head[8:16], dtype=np.uint32))
        n = int(np.frombuffer(head[16:24], dtype=np.uint64)[0])
        if magic != GRAPH_MAGIC or ver != 1 or bs < 1:
            raise ValueError(f"{path}: not a song_graph v1 file")
        adj = np.fromfile(f, dtype=np.int32)
    if adj.size != n * bs:
        raise ValueError(f"{path}: expected {n * bs} entries, found {adj.size}")
    adj = adj.reshape(n, bs)
    if adj.size and (adj.min() < -1 or adj.max() >= n):
        raise ValueError(f"{path}: neighbour id out of range")
    return adj


def cache_dir() -> str:
    d = os.environ.get("SONG_CACHE_DIR") or os.path.join(
        os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "_cache")
    os.makedirs(d, exist_ok=True)
    return d
