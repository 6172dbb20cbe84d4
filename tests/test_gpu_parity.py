"""Parity of the sm_100a search with the reference, through the C ABI (GPU).

Bit-exact: top-k ids (best-first, -1 padded, ties included) and all twelve
QueryTrace counters, against
  * the golden fixtures made by the reference's own GPU kernel, and
  * the oracle (CPU restatement) on seeded inputs across the parameter space:
    block sizes around the 32-lane width, Bloom filters from saturated to
    sparse (power-of-two and not), 1-4 hashes, queue caps, k above ef and
    above pq_size, dims that are not multiples of 4 or 32, non-integer FP32
    data, exact distance ties, Hamming codes of 1-32 words, fewer nodes than
    entry points, empty and ragged adjacency rows.
"""
import numpy as np
import pytest

from conftest import knn_graph
from test_oracle import golden_names, load_golden, oracle_run

pytestmark = pytest.mark.gpu


def song_search(song, meta, a, n_multiquery=512):
    p = song.Params(block_size=meta["block_size"], pq_size=meta["pq_size"],
                    bf_words=meta["bf_words"], bf_nhash=meta["bf_nhash"],
                    n_multiprobe=meta["n_multiprobe"])
    tr = song.GpuSearchTrace()
    if meta["kind"] == "l2":
        base, q = a["base"], a["queries"]
        g = song.KernelGraph(base.shape[0], base.shape[1], base, p, adj=a["adj"])
    else:
        base, q = a["codes"], a["qcodes"]
        g = song.HashKernelGraph(base.shape[0], base, p, adj=a["adj"])
    with g:
        g.upload_to_gpu()
        ids = song.gpu_search(g, q, q.shape[0], meta["k"], n_multiquery, meta["ef"], tr)
    return ids.reshape(q.shape[0], meta["k"]), tr


@pytest.mark.parametrize("name", golden_names())
def test_matches_reference_gpu_kernel(cuda, song, name):
    meta, a = load_golden(name)
    ids, tr = song_search(song, meta, a)
    assert tr.ef_search == meta["ef_effective"]
    np.testing.assert_array_equal(ids, a["ids"])
    np.testing.assert_array_equal(tr.queries, a["trace"])


def _case(ds, kind, n, nq, dim, seed):
    if kind == "int":
        m = ds.int_mixture(n, nq, dim=dim, n_comp=8, seed=seed)
    elif kind == "angular":
        m = ds.angular_mixture(n, nq, dim=dim, n_comp=8, seed=seed)
    else:
        m = ds.l1_mixture(n, nq, dim=dim, n_comp=8, seed=seed)
    return m.base, m.queries


L2_CASES = [
    # kind, n, nq, dim, bs, degree, bf_words, nhash, pq, ef, k, nmp
    ("int", 3000, 200, 128, 16, 15, 16, 4, 512, 64, 10, 4),      # C1 shape
    ("int", 3000, 200, 128, 32, 31, 256, 4, 512, 256, 10, 4),    # C2 shape, big queue
    ("int", 3000, 100, 128, 32, 31, 256, 4, 512, 256, 100, 4),   # k = 100
    ("int", 2000, 100, 128, 32, 24, 24, 3, 300, 300, 10, 4),     # non-power-of-two filter
    ("int", 2000, 100, 64, 40, 36, 64, 2, 128, 100, 7, 4),       # block_size > 32
    ("int", 2000, 100, 64, 64, 50, 1024, 1, 700, 600, 12, 40),   # 2 chunks, 40 entry points
    ("int", 1500, 100, 37, 32, 20, 256, 4, 64, 5, 1, 4),         # odd dim, k = 1
    ("int", 1500, 100, 3, 8, 6, 4, 4, 32, 16, 4, 4),             # tiny dim, tiny filter
    ("angular", 2000, 100, 200, 32, 31, 256, 4, 512, 128, 10, 4),  # non-integer FP32
    ("l1", 1200, 60, 300, 32, 31, 256, 4, 512, 96, 10, 4),       # generic (dim > 256) path
    ("angular", 2000, 100, 64, 32, 31, 256, 4, 512, 1, 10, 4),   # ef < k: raised to k
    ("int", 1000, 50, 64, 32, 31, 256, 4, 50, 10, 60, 4),        # k > pq_size: -1 padding
]


@pytest.mark.parametrize("case", L2_CASES, ids=[f"l2_{i}" for i in range(len(L2_CASES))])
def test_l2_matches_oracle(cuda, song, ds, oracle, case):
    kind, n, nq, dim, bs, deg, bfw, nh, pq, ef, k, nmp = case
    base, q = _case(ds, kind, n, nq, dim, seed=n + dim)
    adj = knn_graph(base, bs, deg, seed=dim)
    meta = dict(kind="l2", block_size=bs, pq_size=pq, bf_words=bfw, bf_nhash=nh,
                n_multiprobe=nmp, k=k, ef=ef)
    a = dict(base=base, queries=q, adj=adj)
    ids, tr = song_search(song, meta, a)
    oids, otr = oracle_run(oracle, meta, a)
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_array_equal(tr.queries, otr)


@pytest.mark.parametrize("ef,bfw", [(256, 256), (576, 512), (1024, 1024)])
def test_untraced_search_matches_oracle(cuda, song, ds, oracle, ef, bfw):
    """Searches without a trace run the trace-free instances (fewer
    registers, more resident queries), and at large queues and filters the
    launcher keeps the result distances in TMEM as well: the ids equal the
    oracle's, as the traced search's do."""
    base, q = _case(ds, "int", 4000, 100, 128, seed=ef + bfw)
    adj = knn_graph(base, 32, 31, seed=ef)
    meta = dict(kind="l2", block_size=32, pq_size=ef, bf_words=bfw, bf_nhash=4,
                n_multiprobe=4, k=10, ef=ef)
    a = dict(base=base, queries=q, adj=adj)
    ids_tr, tr = song_search(song, meta, a)
    p = song.Params(block_size=32, pq_size=ef, bf_words=bfw, bf_nhash=4, n_multiprobe=4)
    with song.KernelGraph(base.shape[0], base.shape[1], base, p, adj=adj) as g:
        g.upload_to_gpu()
        ids = song.gpu_search(g, q, q.shape[0], 10, 512, ef).reshape(q.shape[0], 10)
    oids, otr = oracle_run(oracle, meta, a)
    np.testing.assert_array_equal(ids_tr, oids)
    np.testing.assert_array_equal(tr.queries, otr)
    np.testing.assert_array_equal(ids, oids)


@pytest.mark.parametrize("words", [1, 3, 8, 16, 32])
def test_hamming_matches_oracle(cuda, song, oracle, words):
    rng = np.random.default_rng(words)
    n, nq = 2000, 100
    bits = rng.random((n, words * 32)) < 0.5
    codes = np.packbits(bits, axis=1, bitorder="little").view(np.uint32).reshape(n, words)
    qcodes = codes[rng.integers(0, n, nq)] ^ (rng.random((nq, words)) < 0.02).astype(np.uint32)
    x = bits.astype(np.float32)
    adj = knn_graph(x, 32, 24, seed=words)
    meta = dict(kind="hamming", block_size=32, pq_size=512, bf_words=256, bf_nhash=4,
                n_multiprobe=4, k=10, ef=64)
    a = dict(codes=codes, qcodes=qcodes, adj=adj)
    ids, tr = song_search(song, meta, a)
    oids, otr = oracle_run(oracle, meta, a)
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_array_equal(tr.queries, otr)


def test_ties_and_duplicates(cuda, song, oracle):
    """Duplicate vectors give equal distances everywhere: slot order decides."""
    rng = np.random.default_rng(3)
    rows = np.rint(rng.uniform(0, 255, (50, 32))).astype(np.float32)
    base = rows[rng.integers(0, 50, 2000)]
    q = rows[rng.integers(0, 50, 100)]
    adj = knn_graph(base + rng.normal(0, 1e-3, base.shape), 32, 28, seed=1)
    meta = dict(kind="l2", block_size=32, pq_size=512, bf_words=256, bf_nhash=4,
                n_multiprobe=4, k=10, ef=64)
    a = dict(base=base, queries=q, adj=adj)
    ids, tr = song_search(song, meta, a)
    oids, otr = oracle_run(oracle, meta, a)
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_array_equal(tr.queries, otr)


def test_small_graphs(cuda, song, oracle):
    """n below N_MULTIPROBE (repeated entry points), isolated nodes, empty rows."""
    for n in (1, 2, 3, 5):
        base = np.arange(n * 4, dtype=np.float32).reshape(n, 4)
        adj = np.full((n, 32), -1, np.int32)
        if n > 2:
            adj[0, 5] = n - 1
        q = np.array([[0, 1, 2, 3], [100, 0, 0, 0]], np.float32)
        meta = dict(kind="l2", block_size=32, pq_size=512, bf_words=256, bf_nhash=4,
                    n_multiprobe=4, k=3, ef=4)
        a = dict(base=base, queries=q, adj=adj)
        ids, tr = song_search(song, meta, a)
        oids, otr = oracle_run(oracle, meta, a)
        np.testing.assert_array_equal(ids, oids)
        np.testing.assert_array_equal(tr.queries, otr)


def test_batching_and_device_path_agree(cuda, song, ds):
    """Results do not depend on n_multiquery staging, and the device-pointer
    entry point returns the same as the host one."""
    torch = cuda
    base, q = _case(ds, "int", 3000, 700, 128, seed=21)
    adj = knn_graph(base, 32, 31, seed=2)
    p = song.Params(pq_size=256)
    g = song.KernelGraph(3000, 128, base, p, adj=adj)
    g.upload_to_gpu()
    tr = song.GpuSearchTrace()
    a = song.gpu_search(g, q, 700, 10, 512, 128, tr)
    b = song.gpu_search(g, q, 700, 10, 7, 128)
    np.testing.assert_array_equal(a, b)
    dq = torch.from_numpy(q).cuda()
    dids = torch.empty((700, 10), dtype=torch.int32, device="cuda")
    dtr = torch.empty((700, 12), dtype=torch.int32, device="cuda")
    s = torch.cuda.Stream()
    song.search_device(g, dq, 700, 10, 128, dids, dtr, stream=s)
    s.synchronize()
    np.testing.assert_array_equal(dids.cpu().numpy().reshape(-1), a)
    np.testing.assert_array_equal(dtr.cpu().numpy(), tr.queries)
    g.close()


def test_empty_and_zero_k(cuda, song):
    base = np.ones((10, 8), np.float32)
    adj = np.full((10, 32), -1, np.int32)
    g = song.KernelGraph(10, 8, base, song.Params(), adj=adj)
    g.upload_to_gpu()
    assert song.gpu_search(g, np.zeros((0, 8), np.float32), 0, 10).size == 0
    assert song.gpu_search(g, np.zeros((3, 8), np.float32), 3, 0).size == 0
    g.close()


@pytest.mark.parametrize("dim", [128, 200, 37])
def test_byte_rows_and_their_fallbacks(cuda, song, ds, oracle, dim):
    """Integer rows in [0, 255] get an exact byte copy; queries in [0, 255]
    use it, queries outside that range (but integral) and non-integral
    queries fall back to the FP32 rows -- all bit-exact with the oracle,
    including the QueryTrace counters, in one batch."""
    base, q = _case(ds, "int", 2500, 90, dim, seed=dim + 7)
    q = q.copy()
    q[30:45, 0] = 300.0                   # integral, outside the byte range
    q[45:60, 1] = -3.0
    q[60:75, 2] += 0.5                    # not integral
    adj = knn_graph(base, 32, 31, seed=dim)
    meta = dict(kind="l2", block_size=32, pq_size=512, bf_words=512, bf_nhash=4,
                n_multiprobe=4, k=10, ef=128)
    a = dict(base=base, queries=q, adj=adj)
    g = song.KernelGraph(base.shape[0], dim, base, song.Params(pq_size=512), adj=adj)
    g.upload_to_gpu()
    assert g.u8_rows() == (dim + 15) // 16 * 16
    g.close()
    ids, tr = song_search(song, meta, a)
    oids, otr = oracle_run(oracle, meta, a)
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_array_equal(tr.queries, otr)


def test_no_byte_rows_outside_range(cuda, song):
    base = np.full((50, 16), 256.0, np.float32)
    g = song.KernelGraph(50, 16, base, song.Params(), adj=np.full((50, 32), -1, np.int32))
    g.upload_to_gpu()
    assert g.u8_rows() == 0
    g.close()
