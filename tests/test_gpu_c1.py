"""C1 at full size against the reference itself, and the GPU builder's graph
against the reference builder's (GPU).

Workload C1: 100,000 x 128 integer vectors (64-component Gaussian mixture,
centres U[0,255], sigma 20, clipped and rounded), 1,000 queries from the same
mixture, NSW graph made by the reference's own builder (build_kernel_graph,
kernalGraph.h:140-149) with BLOCK_SIZE 16, FIXED_DEGREE 15 and
SEARCH_DEGREE 15; k = 10, queue 64, a 1,024-bit Bloom filter (BF_WORDS 16).

* Every one of the 1,000 queries returns the same ids and the same twelve
  QueryTrace counters as the reference's own GPU kernel (kg_search_kernel
  through gpu_search, kernalGraph.h:184-382, compiled for sm_100a from the
  reference sources with this config.h).
* Graph quality of the library's GPU builder (batched insertion) against
  the reference builder on the same data.  C1's own graph (FIXED_DEGREE =
  SEARCH_DEGREE = 15) loses its long links to reverse-edge eviction on this
  well-separated 64-cluster mixture, so every search -- the reference's
  included -- stays near its seeds (recall@10 about 0.01 for both builders)
  and says nothing about quality.  The comparison therefore uses the C2
  graph shape (BLOCK_SIZE 32, FIXED_DEGREE 31) on the same data: recall@10
  at queues 64, 128 and 256 with a 16,384-bit Bloom filter, both graphs
  searched by the same bit-exact kernel; the GPU builder may trail the
  reference builder by at most GRAPH_RECALL_BOUND.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, NQ, DIM = 100_000, 1_000, 128
GRAPH_RECALL_BOUND = 0.01


@pytest.fixture(scope="module")
def c1(ds, oracle):
    m = ds.int_mixture(N, NQ, dim=DIM, n_comp=64, seed=1100)
    r = oracle.ref(block_size=16, fixed_degree=15, search_degree=15, pq_size=512, bf_words=16)
    assert r.config()["BF_WORDS"] == 16 and r.config()["BLOCK_SIZE"] == 16
    adj = r.build_graph(m.base)  # the reference builder: sequential insertion on the host
    return m, r, adj


def _index(song, m, adj):
    p = song.Params(block_size=16, fixed_degree=15, search_degree=15, pq_size=512, bf_words=16)
    g = song.KernelGraph(N, DIM, m.base, p, adj=adj)
    g.upload_to_gpu()
    return g


def test_all_queries_match_the_reference_gpu_kernel(cuda, song, c1):
    m, r, adj = c1
    ref_ids, ref_tr, _ = r.gpu_search_l2(m.base, adj, m.queries, 10, 64)
    with _index(song, m, adj) as g:
        tr = song.GpuSearchTrace()
        ids = song.gpu_search(g, m.queries, NQ, 10, 512, 64, tr).reshape(NQ, 10)
    assert tr.ef_search == 64
    np.testing.assert_array_equal(ids, ref_ids)
    np.testing.assert_array_equal(tr.queries, ref_tr)


def test_gpu_builder_graph_recall_against_the_reference_builder(cuda, song, oracle, c1):
    m = c1[0]
    r32 = oracle.ref(block_size=32, fixed_degree=31, search_degree=15, pq_size=512, bf_words=256)
    adj_ref = r32.build_graph(m.base)
    gtm = importlib.import_module("2020_song_ex_b200.groundtruth")
    gt, _ = gtm.knn(m.base, m.queries, 10)
    ds = importlib.import_module("2020_song_ex_b200.datasets")
    adj_gpu = song.build_graph(m.base, song.Params(block_size=32, fixed_degree=31, search_degree=15),
                               batch_ratio=32)
    p = song.Params(block_size=32, fixed_degree=31, search_degree=15, pq_size=512, bf_words=256)
    rows = []
    for ef in (64, 128, 256):
        rec = {}
        for name, adj in (("reference_builder", adj_ref), ("gpu_builder", adj_gpu)):
            with song.KernelGraph(N, DIM, m.base, p, adj=adj) as g:
                g.upload_to_gpu()
                ids = song.gpu_search(g, m.queries, NQ, 10, 512, ef).reshape(NQ, 10)
            rec[name] = float(ds.recall_at_k(ids, gt, 10).mean())
        rows.append((ef, rec["reference_builder"], rec["gpu_builder"]))
    print("recall@10 on C1 data, degree-31 graphs (ef, reference builder, GPU builder):", rows)
    for ef, rr, rg in rows:
        assert rg >= rr - GRAPH_RECALL_BOUND, (ef, rr, rg)
