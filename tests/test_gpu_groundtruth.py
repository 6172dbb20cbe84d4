"""Exact kNN ground truth on the tensor cores (song_exact_knn_device).

The reference's ground truth is a brute force over every base vector
(bench_cpu.cpp:158-175; numpy in run_compare.py:199-213).  Checks:

* integer vectors in [0, 255], dim <= 128: ids and distances equal an
  int64 brute force exactly, ties ordered by the lower id;
* ragged sizes (n, nq not multiples of 128), k > n (-1 / +inf padding),
  k = 1, k = 128, dimensions that are not multiples of 32 and a 960-dim case;
* float vectors (every split product used, and the one-sided cases where
  only the queries or only the bases have a nonzero lo part): each returned
  id is a true top-k neighbour in float64 up to distance ties within
  1e-5 relative (3e-5 at 960 dimensions), and distances agree with float64
  within the same tolerance, relative to the k-th distance;
* the result equals the library-GEMM path (``knn_torch``) wherever no two
  distances tie.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gt():
    return importlib.import_module("2020_song_ex_b200.groundtruth")


def _exact_int(base, q, k):
    """int64 brute force: ids ascending by (distance, id), -1 padded."""
    b = base.astype(np.int64)
    qq = q.astype(np.int64)
    d = (qq * qq).sum(1)[:, None] - 2 * qq @ b.T + (b * b).sum(1)[None, :]
    n = b.shape[0]
    ids = np.full((q.shape[0], k), -1, np.int64)
    dd = np.full((q.shape[0], k), np.inf)
    idx = np.arange(n)
    for i in range(q.shape[0]):
        o = np.lexsort((idx, d[i]))[:k]
        ids[i, :len(o)] = o
        dd[i, :len(o)] = d[i, o]
    return ids, dd


def _int_data(n, nq, dim, seed):
    rng = np.random.default_rng(seed)
    base = rng.integers(0, 256, size=(n, dim)).astype(np.float32)
    q = rng.integers(0, 256, size=(nq, dim)).astype(np.float32)
    return base, q


@pytest.mark.parametrize("n,nq,dim,k", [
    (5000, 300, 128, 100),   # SIFT-shaped, several splits
    (1037, 129, 96, 10),     # ragged n and nq
    (777, 5, 40, 128),       # dim not a multiple of 32, k at its maximum
    (50, 17, 128, 100),      # k > n: padding
    (20000, 64, 128, 1),     # nearest neighbour only
])
def test_integer_data_exact(cuda, n, nq, dim, k):
    base, q = _int_data(n, nq, dim, seed=n + dim)
    ids, d = _gt().knn(base, q, k)
    ref_ids, ref_d = _exact_int(base, q, k)
    np.testing.assert_array_equal(ids, ref_ids)
    np.testing.assert_array_equal(d, ref_d.astype(np.float32))


def test_integer_ties_lower_id_first(cuda):
    # many duplicate rows: equal distances must come out by increasing id
    rng = np.random.default_rng(3)
    proto = rng.integers(0, 256, size=(40, 64)).astype(np.float32)
    base = proto[rng.integers(0, 40, size=3000)]
    q = proto[:20] + 1.0
    ids, d = _gt().knn(base, q, 50)
    ref_ids, ref_d = _exact_int(base, q, 50)
    np.testing.assert_array_equal(ids, ref_ids)
    np.testing.assert_array_equal(d, ref_d.astype(np.float32))


def _check_float(base, q, ids, d, k, rel=1e-5):
    b = base.astype(np.float64)
    qq = q.astype(np.float64)
    for i in range(q.shape[0]):
        full = ((b - qq[i]) ** 2).sum(1)
        kth = np.sort(full)[k - 1]
        tol = rel * max(kth, 1e-30)
        # every returned id is within the true top-k up to near-ties
        assert np.all(full[ids[i]] <= kth + tol), i
        assert len(set(ids[i].tolist())) == k
        np.testing.assert_allclose(d[i], full[ids[i]], rtol=0, atol=tol)
        assert np.all(np.diff(d[i]) >= 0)


@pytest.mark.parametrize("qkind,bkind", [("f", "f"), ("f", "i"), ("i", "f")])
def test_float_data_within_tolerance(cuda, qkind, bkind):
    rng = np.random.default_rng(11)
    n, nq, dim, k = 4000, 130, 200, 20
    fb = rng.normal(size=(n, dim)).astype(np.float32)
    fq = rng.normal(size=(nq, dim)).astype(np.float32)
    ib = rng.integers(0, 4, size=(n, dim)).astype(np.float32)
    iq = rng.integers(0, 4, size=(nq, dim)).astype(np.float32)
    base = fb if bkind == "f" else ib
    q = fq if qkind == "f" else iq
    ids, d = _gt().knn(base, q, k)
    _check_float(base, q, ids, d, k)


def test_wide_vectors(cuda):
    rng = np.random.default_rng(5)
    base = rng.random(size=(2000, 960), dtype=np.float32)
    q = rng.random(size=(40, 960), dtype=np.float32)
    ids, d = _gt().knn(base, q, 10)
    _check_float(base, q, ids, d, 10, rel=3e-5)


def test_matches_library_gemm_path(cuda, ds):
    m = ds.int_mixture(30000, 256, dim=128, n_comp=16, seed=9)
    ids, d = _gt().knn(m.base, m.queries, 10)
    ids_t, d_t = _gt().knn_torch(m.base, m.queries, 10)
    np.testing.assert_array_equal(d, d_t)
    # ids agree wherever the distance is not tied inside the row
    for i in range(ids.shape[0]):
        untied = np.array([np.sum(d[i] == x) == 1 for x in d[i]])
        np.testing.assert_array_equal(ids[i][untied], ids_t[i][untied])


def test_device_strides(cuda, song):
    import torch
    base, q = _int_data(3000, 70, 100, seed=2)
    wide_b = np.zeros((3000, 128), np.float32)
    wide_b[:, :100] = base
    wide_q = np.zeros((70, 112), np.float32)
    wide_q[:, :100] = q
    db = torch.as_tensor(wide_b, device="cuda")
    dq = torch.as_tensor(wide_q, device="cuda")
    ids = torch.empty((70, 16), dtype=torch.int32, device="cuda")
    dd = torch.empty((70, 16), dtype=torch.float32, device="cuda")
    song.exact_knn_device(db, 3000, 100, dq, 70, 16, ids, dd, ldb=128, ldq=112)
    ref_ids, ref_d = _exact_int(base, q, 16)
    np.testing.assert_array_equal(ids.cpu().numpy(), ref_ids)
    np.testing.assert_array_equal(dd.cpu().numpy(), ref_d.astype(np.float32))


def test_rejects_bad_arguments(cuda, song):
    base, q = _int_data(100, 4, 16, seed=1)
    with pytest.raises(song.SongError):
        song.exact_knn(base, q, 129)
    with pytest.raises(song.SongError):
        song.exact_knn(base, q, 0)
