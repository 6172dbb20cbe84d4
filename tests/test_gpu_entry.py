"""The learned search's entry stage: every query's 24 nearest hubs from the
tcgen05 tensor-core kernel (BF16 operands, FP32 accumulation in TMEM).

* Integer vectors in [0, 255] with dim <= 128: BF16 is exact and every FP32
  sum stays below 2^24, so ids and squared distances must equal an exact
  int64 computation, ties ordered by hub index.
* Non-integer vectors: the distances of the returned hubs match a float64
  computation on the same BF16-rounded operands within 1e-4 relative, and
  no hub is missed by more than that tolerance.
* Ragged shapes: dims that are not multiples of 16, hub counts that are not
  whole tiles or below 24, query counts that are not whole 128-query tiles.
  Batches of up to 128 queries spread the hub tiles over several CTAs and
  merge their lists; the result must not change.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _bf16(x):
    return torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(torch.bfloat16).float().numpy()


def _run(song, base, hubs, q):
    n, dim = base.shape
    g = song.KernelGraph(n, dim, base, song.Params(), adj=np.full((n, 32), -1, np.int32))
    g.upload_to_gpu()
    song.set_entry_hubs(g, hubs)
    dq = torch.from_numpy(np.ascontiguousarray(q, np.float32)).cuda()
    ids = torch.empty((q.shape[0], 24), dtype=torch.int32, device="cuda")
    dd = torch.empty((q.shape[0], 24), dtype=torch.float32, device="cuda")
    st = torch.cuda.Stream()
    song.entry_candidates(g, dq, q.shape[0], ids, dd, stream=st)
    st.synchronize()
    g.close()
    return ids.cpu().numpy(), dd.cpu().numpy()


@pytest.mark.parametrize("n,dim,nh,nq", [(20000, 128, 1000, 300), (3000, 37, 700, 129),
                                         (2000, 64, 10, 5), (5000, 96, 256, 128),
                                         (30000, 128, 4096, 100), (9000, 80, 2100, 1)])
def test_integer_vectors_exact(cuda, song, ds, n, dim, nh, nq):
    m = ds.int_mixture(n, nq, dim=dim, n_comp=16, seed=n + dim)
    rng = np.random.default_rng(dim)
    hubs = rng.choice(n, nh, replace=False).astype(np.int32)
    ids, dd = _run(song, m.base, hubs, m.queries)
    h = m.base[hubs].astype(np.int64)
    qq = m.queries.astype(np.int64)
    d = (qq * qq).sum(1)[:, None] + (h * h).sum(1)[None] - 2 * qq @ h.T
    order = np.argsort(d, axis=1, kind="stable")[:, :24]   # ties: lower hub index first
    want_ids = np.full((nq, 24), -1, np.int64)
    want_d = np.full((nq, 24), np.inf)
    k = min(24, nh)
    want_ids[:, :k] = hubs[order[:, :k]]
    want_d[:, :k] = np.take_along_axis(d, order, 1)[:, :k]
    np.testing.assert_array_equal(ids, want_ids)
    np.testing.assert_array_equal(dd, want_d.astype(np.float32))


def test_float_vectors_bf16(cuda, song, ds):
    m = ds.angular_mixture(6000, 200, dim=200, n_comp=16, seed=3)
    hubs = np.random.default_rng(1).choice(6000, 1500, replace=False).astype(np.int32)
    ids, dd = _run(song, m.base, hubs, m.queries)
    qb = _bf16(m.queries).astype(np.float64)
    hb = _bf16(m.base[hubs]).astype(np.float64)
    qn = (m.queries.astype(np.float64) ** 2).sum(1)
    ref = qn[:, None] + (hb * hb).sum(1)[None] - 2 * qb @ hb.T
    pos = {int(h): i for i, h in enumerate(hubs)}
    got_ref = np.array([[ref[r, pos[int(i)]] for i in row] for r, row in enumerate(ids)])
    scale = np.abs(ref).max()
    np.testing.assert_allclose(dd, got_ref, atol=1e-4 * scale, rtol=0)
    kth = np.sort(ref, axis=1)[:, 23]
    assert (got_ref[:, 23] <= kth + 1e-4 * scale).all()
    assert (np.diff(dd, axis=1) >= 0).all()


def test_bad_hub_sets(cuda, song):
    base = np.zeros((10, 8), np.float32)
    g = song.KernelGraph(10, 8, base, song.Params(), adj=np.full((10, 32), -1, np.int32))
    g.upload_to_gpu()
    with pytest.raises(song.SongError):
        song.set_entry_hubs(g, [3, 10])
    with pytest.raises(song.SongError):
        song.set_entry_hubs(g, [])
    g.close()
    wide = np.zeros((10, 300), np.float32)
    g = song.KernelGraph(10, 300, wide, song.Params(), adj=np.full((10, 32), -1, np.int32))
    g.upload_to_gpu()
    with pytest.raises(song.SongError):
        song.set_entry_hubs(g, [1, 2])
    g.close()
