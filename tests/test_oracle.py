"""The oracle (CPU restatement of the reference GPU search), pinned (CPU only).

* against the golden fixtures made by the reference's own GPU kernel
  (tests/golden/make_golden.py): ids AND QueryTrace counters bit-exact;
* against the reference's BitHash compiled here: codes bit-exact;
* against the reference's CPU Graph::search compiled here: the documented
  relation (same algorithm up to the Bloom filter and the bounded frontier).
"""
import glob
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    meta = json.loads(str(z["meta"]))
    arrays = {k: z[k] for k in z.files if k != "meta"}
    if "base_u8" in arrays:
        arrays["base"] = arrays.pop("base_u8").astype(np.float32)
    return meta, arrays


def golden_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def oracle_run(oracle, meta, a):
    ef = oracle.clamp_ef(meta["ef"], meta["k"], meta["pq_size"])
    kw = dict(pq_size=meta["pq_size"], bf_words=meta["bf_words"], bf_nhash=meta["bf_nhash"],
              n_multiprobe=meta["n_multiprobe"])
    if meta["kind"] == "l2":
        return oracle.search_l2(a["base"], a["adj"], meta["block_size"], a["queries"], meta["k"],
                                ef, **kw)
    return oracle.search_hamming(a["codes"], a["adj"], meta["block_size"], a["qcodes"],
                                 meta["k"], ef, **kw)


def test_goldens_present():
    names = golden_names()
    assert {"c1_small", "ref_defaults", "float_angular", "hamming512", "ties"} <= set(names), names


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference_gpu_kernel(oracle, name):
    meta, a = load_golden(name)
    ids, trace = oracle_run(oracle, meta, a)
    assert meta["ef_effective"] == oracle.clamp_ef(meta["ef"], meta["k"], meta["pq_size"])
    np.testing.assert_array_equal(ids, a["ids"])
    np.testing.assert_array_equal(trace, a["trace"])


def test_clamp_ef(oracle):
    assert oracle.clamp_ef(5, 10, 50) == 10      # raised to k
    assert oracle.clamp_ef(100, 10, 50) == 50    # capped at pq_size
    assert oracle.clamp_ef(10, 60, 50) == 50     # k > pq_size: cap wins (clamped after)


def _tree_l2(q, b):
    """numpy statement of warp_l2: per-lane FMA chains, then the 16,8,4,2,1 tree."""
    q = q.astype(np.float32)
    b = b.astype(np.float32)
    part = np.zeros(32, np.float32)
    for lane in range(32):
        s = np.float32(0)
        for i in range(lane, q.size, 32):
            t = np.float32(q[i] - b[i])
            s = np.float32(np.float64(t) * np.float64(t) + np.float64(s))  # one rounding = FMA
        part[lane] = s
    off = 16
    while off:
        part[:off] = part[:off] + part[off:2 * off]
        off //= 2
    return part[0]


def test_warp_l2_order(oracle):
    rng = np.random.default_rng(5)
    for dim in (1, 7, 32, 40, 100, 128, 200):
        q = rng.normal(size=dim).astype(np.float32)
        b = rng.normal(size=dim).astype(np.float32)
        assert oracle.lib().oracle_warp_l2(q, b, dim) == _tree_l2(q, b)
    # integer data: exact integer value
    q = np.rint(rng.uniform(0, 255, 128)).astype(np.float32)
    b = np.rint(rng.uniform(0, 255, 128)).astype(np.float32)
    assert oracle.lib().oracle_warp_l2(q, b, 128) == float(((q.astype(np.int64) - b) ** 2).sum())


def test_bithash_matches_reference(oracle, ds):
    if not oracle.ref_available(hash_bits=512, pq_size=512):
        pytest.skip("compiled reference not available")
    r = oracle.ref(hash_bits=512, pq_size=512)
    if r.gpu is None:
        pytest.skip("reference BitHash library not built")
    x = ds.angular_mixture(300, 1, dim=64, n_comp=4, seed=2).base
    codes, R = r.bithash_project(x)
    R2 = oracle.bithash_matrix(64, 512, 42)
    np.testing.assert_array_equal(R, R2)
    np.testing.assert_array_equal(oracle.bithash_project(R2, x), codes)


@pytest.mark.parametrize("bs,bfw", [(16, 16), (32, 256)])
def test_relation_to_reference_cpu_search(oracle, ds, bs, bfw):
    """Graph::search (graph.h:33-115) differs by design (exact visited set,
    unbounded frontier, lexicographic ties, worst-first output), so only most
    queries agree exactly; the rest must still overlap heavily."""
    if not oracle.ref_available(block_size=bs, bf_words=bfw, pq_size=512):
        pytest.skip("compiled reference not available")
    r = oracle.ref(block_size=bs, bf_words=bfw, pq_size=512)
    m = ds.int_mixture(3000, 100, dim=64, n_comp=16, seed=9)
    adj = r.build_graph(m.base)
    ids, _ = oracle.search_l2(m.base, adj, bs, m.queries, 10, 64, pq_size=512, bf_words=bfw)
    cpu, _ = r.cpu_graph(m.base, adj).search(m.queries, 10, 64, threads=4)
    cpu = cpu[:, ::-1]  # best-first
    exact = (ids == cpu).all(axis=1).mean()
    overlap = np.mean([len(set(a) & set(b)) / 10 for a, b in zip(ids, cpu)])
    assert exact >= 0.6 and overlap >= 0.9, (exact, overlap)


def test_reference_builders_agree(oracle, ds):
    """build_graph (graph.h) and build_kernel_graph (kernalGraph.h) are the
    same algorithm; the fixtures use the latter."""
    if not oracle.ref_available(block_size=16, bf_words=16, pq_size=512):
        pytest.skip("compiled reference not available")
    r = oracle.ref(block_size=16, bf_words=16, pq_size=512)
    if r.gpu is None:
        pytest.skip("reference kernel-graph library not built")
    m = ds.int_mixture(800, 1, dim=32, n_comp=4, seed=4)
    a1 = r.build_graph(m.base)
    a2 = np.empty_like(a1)
    r.cpu.ref_cpu_build_graph(np.ascontiguousarray(m.base), 800, 32, a2)
    np.testing.assert_array_equal(a1, a2)
