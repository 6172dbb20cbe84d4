"""Exact k-nearest-neighbour ground truth on the GPU, for recall.

The reference computes ground truth by sequential brute force on the CPU
(bench_cpu.cpp:158-175) or in numpy (run_compare.py:199-213).  ``knn`` runs
the library's tensor-core kernel (``song_exact_knn_device``):
``||q - b||^2 = ||q||^2 - 2 q.b + ||b||^2`` with the cross term from 3xBF16
split operands, x = hi + lo with hi = bf16(x) and lo = bf16(x - hi), and
q.b ~= hi_q.hi_b + hi_q.lo_b + lo_q.hi_b accumulated in FP32 (the lo.lo term
is below FP32 resolution), the k smallest kept per query in the kernel's
epilogue, ties broken by the lower id.  For integer data in [0, 255] (the
SIFT-shaped workloads) lo is exactly zero and every sum is an integer below
2^24, so the distances are exact.  ``knn_torch`` computes the same split
products with library GEMMs (a cross-check for tests).  ``spot_check``
recomputes a sample of queries in FP64 and reports how many true top-k ids
the GPU ground truth misses.
"""
from __future__ import annotations

import numpy as np


def _split(x):
    import torch
    hi = x.to(torch.bfloat16)
    lo = (x - hi.float()).to(torch.bfloat16)
    return hi, lo


def _mm(a, b):
    """BF16 x BF16 tensor-core GEMM with an FP32 result (not rounded to BF16)."""
    import torch
    return torch.mm(a, b, out_dtype=torch.float32)


def knn(base, queries, k: int, device: str = "cuda"):
    """Exact top-k ids [nq, k] int32 (ascending (distance, id)) and their FP32
    distances, from the tensor-core kernel."""
    import torch
    from . import exact_knn_device
    b = torch.as_tensor(np.ascontiguousarray(base, dtype=np.float32), device=device)
    q = torch.as_tensor(np.ascontiguousarray(queries, dtype=np.float32), device=device)
    q = q.reshape(-1, b.shape[1])
    ids = torch.empty((q.shape[0], k), dtype=torch.int32, device=device)
    dists = torch.empty((q.shape[0], k), dtype=torch.float32, device=device)
    exact_knn_device(b, b.shape[0], b.shape[1], q, q.shape[0], k, ids, dists,
                     stream=torch.cuda.current_stream())
    return ids.cpu().numpy(), dists.cpu().numpy()


def knn_torch(base, queries, k: int, chunk: int = 2048, device: str = "cuda"):
    """The same split products with library GEMMs and torch.topk (ties in
    arbitrary order): top-k ids [nq, k] and FP32 distances."""
    import torch
    b = torch.as_tensor(np.ascontiguousarray(base, dtype=np.float32), device=device)
    q_all = torch.as_tensor(np.ascontiguousarray(queries, dtype=np.float32), device=device)
    bh, bl = _split(b)
    bn = (b.double() ** 2).sum(1).float()
    need_lo = bool((bl != 0).any())
    ids = torch.empty((q_all.shape[0], k), dtype=torch.int64, device=device)
    dists = torch.empty((q_all.shape[0], k), dtype=torch.float32, device=device)
    for s in range(0, q_all.shape[0], chunk):
        q = q_all[s:s + chunk]
        qh, ql = _split(q)
        cross = _mm(qh, bh.T)
        if need_lo or bool((ql != 0).any()):
            cross += _mm(qh, bl.T)
            cross += _mm(ql, bh.T)
        qn = (q.double() ** 2).sum(1).float()
        d = qn[:, None] - 2.0 * cross + bn[None, :]
        v, i = torch.topk(d, k, dim=1, largest=False, sorted=True)
        ids[s:s + chunk] = i
        dists[s:s + chunk] = v
    return ids.to(torch.int32).cpu().numpy(), dists.cpu().numpy()


def spot_check(base, queries, gt_ids, sample: int = 32, seed: int = 0, device: str = "cuda"):
    """FP64 brute force on `sample` queries; returns (queries checked, ids missed,
    max |d_fp32 - d_fp64| relative at the k-th neighbour)."""
    import torch
    rng = np.random.default_rng(seed)
    nq, k = gt_ids.shape
    pick = rng.choice(nq, size=min(sample, nq), replace=False)
    b = torch.as_tensor(np.ascontiguousarray(base), device=device).double()
    missed = 0
    for qi in pick:
        q = torch.as_tensor(np.ascontiguousarray(queries[qi]), device=device).double()
        d = ((b - q[None, :]) ** 2).sum(1)
        kth = torch.topk(d, k, largest=False).values[-1]
        true_set = set(torch.nonzero(d <= kth).flatten().tolist())  # ties at the k-th count as true
        missed += sum(1 for x in gt_ids[qi] if int(x) not in true_set)
    return len(pick), missed
