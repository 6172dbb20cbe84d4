"""The precision form (BF16 / FP8 storage, FP32 accumulation, FP32 re-rank).

* On integer vectors in [0, 255] every value is exact in BF16, so the BF16
  traversal must reproduce the plain (reference-exact) search bit for bit.
* Distances reported for the output ids are checked against float64: the
  re-ranked ones are exact FP32 L2 (relative tolerance 1e-5), the
  un-re-ranked ones match the quantised rows (BF16 round-to-nearest-even,
  FP8 e4m3 with scale amax/448) within 1e-4 relative.
* Recall@10 against exact ground truth stays within 0.02 (BF16) and 0.05
  (FP8) of the plain search at the same queue size.
"""
import numpy as np
import pytest

from conftest import knn_graph

pytestmark = pytest.mark.gpu


def _graph(song, base, adj, pq=512):
    g = song.KernelGraph(base.shape[0], base.shape[1], base, song.Params(pq_size=pq), adj=adj)
    g.upload_to_gpu()
    return g


def _exact(base, q, ids):
    b = base.astype(np.float64)[np.clip(ids, 0, None)]
    return ((b - q.astype(np.float64)[:, None, :]) ** 2).sum(-1)


def test_bf16_on_integer_data_equals_plain(cuda, song, ds):
    m = ds.int_mixture(3000, 200, dim=128, n_comp=8, seed=41)
    adj = knn_graph(m.base, 32, 31, seed=4)
    g = _graph(song, m.base, adj)
    song.set_precision(g, song.PREC_BF16)
    tr0, tr1 = song.GpuSearchTrace(), song.GpuSearchTrace()
    ids0, d0 = song.gpu_search_ex(g, song.SearchOpts(), m.queries, 200, 10, 128, trace=tr0)
    ids1, d1 = song.gpu_search_ex(g, song.SearchOpts(precision=song.PREC_BF16), m.queries, 200,
                                  10, 128, trace=tr1)
    np.testing.assert_array_equal(ids1, ids0)
    np.testing.assert_array_equal(d1, d0)
    np.testing.assert_array_equal(tr1.queries, tr0.queries)
    plain = song.gpu_search(g, m.queries, 200, 10, 512, 128).reshape(200, 10)
    np.testing.assert_array_equal(ids0, plain)
    g.close()


@pytest.mark.parametrize("prec", ["bf16", "fp8"])
def test_precision_form_distances_and_recall(cuda, song, ds, prec):
    import torch
    gtm = __import__("importlib").import_module("2020_song_ex_b200.groundtruth")
    m = ds.angular_mixture(4000, 200, dim=96, n_comp=16, seed=43)
    adj = knn_graph(m.base, 32, 31, seed=5)
    g = _graph(song, m.base, adj)
    P = song.PREC_BF16 if prec == "bf16" else song.PREC_FP8
    song.set_precision(g, P)
    gt, _ = gtm.knn(m.base, m.queries, 10)
    ids_p, d_p = song.gpu_search_ex(g, song.SearchOpts(), m.queries, 200, 10, 96)
    ids_r, d_r = song.gpu_search_ex(g, song.SearchOpts(precision=P, rerank=True), m.queries,
                                    200, 10, 96)
    ids_a, d_a = song.gpu_search_ex(g, song.SearchOpts(precision=P), m.queries, 200, 10, 96)
    # re-ranked distances are exact FP32 L2 of the returned ids, ascending
    ex = _exact(m.base, m.queries, ids_r)
    np.testing.assert_allclose(d_r, ex, rtol=1e-5, atol=1e-7)
    assert (np.diff(d_r, axis=1) >= 0).all()
    # un-re-ranked distances are those of the quantised rows
    xb = torch.from_numpy(m.base)
    if P == song.PREC_BF16:
        deq = xb.to(torch.bfloat16).float().numpy()
    else:
        scale = xb.abs().amax(1, keepdim=True) / 448.0
        deq = ((xb * (1.0 / scale)).to(torch.float8_e4m3fn).float() * scale).numpy()
    qa = _exact(deq, m.queries, ids_a)
    np.testing.assert_allclose(d_a, qa, rtol=1e-4, atol=1e-6)
    rec_p = ds.recall_at_k(ids_p, gt, 10).mean()
    rec_r = ds.recall_at_k(ids_r, gt, 10).mean()
    tol = 0.02 if P == song.PREC_BF16 else 0.05
    assert rec_r >= rec_p - tol, (rec_p, rec_r)
    g.close()


def test_precision_requires_attached_rows(cuda, song, ds):
    m = ds.int_mixture(500, 4, dim=32, n_comp=4, seed=44)
    adj = knn_graph(m.base, 16, 12, seed=6)
    g = song.KernelGraph(500, 32, m.base, song.Params(block_size=16, fixed_degree=15), adj=adj)
    g.upload_to_gpu()
    with pytest.raises(song.SongError):
        song.gpu_search_ex(g, song.SearchOpts(precision=song.PREC_FP8), m.queries, 4, 5, 16)
    g.close()
