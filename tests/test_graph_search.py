"""The reference's CPU search, Graph::search (graph.h:33-115): exact visited
set, unbounded (distance, id)-ordered frontier and top-ef, dimension-order
FP32 distances, worst-first results.

* CPU: the oracle's restatement equals the compiled reference's own
  Graph::search (ids and all twelve QueryTrace counters).
* GPU: song_graph_search equals both, bit for bit, on integer and
  non-integer vectors, distance ties, BLOCK_SIZE 16 and 32, k above ef,
  tiny graphs with repeated entry points, and queues large enough that the
  frontier must drop never-expandable entries.
"""
import numpy as np
import pytest

from conftest import knn_graph


def _ref(oracle, bs):
    kw = dict(block_size=16, fixed_degree=15, search_degree=15, pq_size=512, bf_words=16) \
        if bs == 16 else dict(pq_size=512)
    if not oracle.ref_available(**kw):
        pytest.skip("compiled reference not available")
    return oracle.ref(**kw)


CASES = [
    # kind, n, nq, dim, bs, degree, k, ef
    ("int", 3000, 120, 128, 32, 31, 10, 64),
    ("int", 3000, 80, 128, 16, 15, 10, 128),
    ("angular", 2500, 80, 100, 32, 28, 10, 50),
    ("int", 2000, 60, 37, 32, 20, 25, 10),       # k > ef: raised to k
    ("angular", 4000, 40, 64, 32, 31, 10, 400),  # large queue
]


def _case(ds, kind, n, nq, dim, seed):
    m = (ds.int_mixture if kind == "int" else ds.angular_mixture)(n, nq, dim=dim, n_comp=8, seed=seed)
    return m.base, m.queries


@pytest.mark.parametrize("case", CASES[:3], ids=[f"cpu_{i}" for i in range(3)])
def test_oracle_restatement_matches_reference(oracle, ds, case):
    kind, n, nq, dim, bs, deg, k, ef = case
    r = _ref(oracle, bs)
    base, q = _case(ds, kind, n, nq, dim, seed=n + dim)
    adj = knn_graph(base, bs, deg, seed=dim)
    ids, tr = oracle.graph_search(base, adj, bs, q, k, ef)
    g = r.cpu_graph(base, adj)
    rids, rtr = g.search(q, k, ef, threads=4, with_trace=True)
    g.close()
    np.testing.assert_array_equal(ids, rids)
    np.testing.assert_array_equal(tr, rtr)


def _gpu(song, base, adj, bs, q, k, ef):
    p = song.Params(block_size=bs, pq_size=1024)
    g = song.KernelGraph(base.shape[0], base.shape[1], base, p, adj=adj)
    g.upload_to_gpu()
    out = song.graph_search(g, q, q.shape[0], k, ef)
    g.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[f"gpu_{i}" for i in range(len(CASES))])
def test_gpu_matches_reference(cuda, song, oracle, ds, case):
    kind, n, nq, dim, bs, deg, k, ef = case
    base, q = _case(ds, kind, n, nq, dim, seed=n + dim)
    adj = knn_graph(base, bs, deg, seed=dim)
    ids, tr = _gpu(song, base, adj, bs, q, k, ef)
    oids, otr = oracle.graph_search(base, adj, bs, q, k, ef)
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_array_equal(tr, otr)
    if oracle.ref_available(**(dict(block_size=16, fixed_degree=15, search_degree=15, pq_size=512,
                                    bf_words=16) if bs == 16 else dict(pq_size=512))):
        r = _ref(oracle, bs)
        g = r.cpu_graph(base, adj)
        rids, rtr = g.search(q, k, ef, threads=4, with_trace=True)
        g.close()
        np.testing.assert_array_equal(ids, rids)
        np.testing.assert_array_equal(tr, rtr)


@pytest.mark.gpu
def test_gpu_ties_and_small_graphs(cuda, song, oracle):
    rng = np.random.default_rng(3)
    rows = np.rint(rng.uniform(0, 255, (40, 16))).astype(np.float32)
    base = rows[rng.integers(0, 40, 1500)]
    q = rows[rng.integers(0, 40, 50)]
    adj = knn_graph(base + rng.normal(0, 1e-3, base.shape), 32, 28, seed=1)
    ids, tr = _gpu(song, base, adj, 32, q, 10, 32)
    oids, otr = oracle.graph_search(base, adj, 32, q, 10, 32)
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_array_equal(tr, otr)
    for n in (1, 2, 3, 5):  # fewer nodes than entry points
        b = np.arange(n * 4, dtype=np.float32).reshape(n, 4)
        a = np.full((n, 32), -1, np.int32)
        if n > 2:
            a[0, 5] = n - 1
        qq = np.array([[0, 1, 2, 3], [100, 0, 0, 0]], np.float32)
        ids, tr = _gpu(song, b, a, 32, qq, 3, 4)
        oids, otr = oracle.graph_search(b, a, 32, qq, 3, 4)
        np.testing.assert_array_equal(ids, oids)
        np.testing.assert_array_equal(tr, otr)
