"""File formats and recall definition (CPU)."""
import numpy as np
import pytest


def test_fvecs_roundtrip(ds, tmp_path):
    x = np.random.default_rng(0).normal(size=(17, 5)).astype(np.float32)
    p = str(tmp_path / "a.fvecs")
    ds.write_fvecs(p, x)
    assert np.array_equal(ds.read_fvecs(p), x)
    # layout: int32 dim then the floats (parser.h:10-21)
    raw = np.fromfile(p, dtype=np.int32).reshape(17, 6)
    assert (raw[:, 0] == 5).all()


def test_ivecs_roundtrip(ds, tmp_path):
    x = np.arange(12, dtype=np.int32).reshape(3, 4)
    p = str(tmp_path / "a.ivecs")
    ds.write_ivecs(p, x)
    assert np.array_equal(ds.read_ivecs(p), x)


def test_fvecs_malformed(ds, tmp_path):
    p = tmp_path / "bad.fvecs"
    np.array([3, 0, 0], dtype=np.int32).tofile(p)  # dim 3 but only 2 values
    with pytest.raises(ValueError):
        ds.read_fvecs(str(p))


def test_gt_npy(ds, tmp_path):
    gt = np.arange(40, dtype=np.int32).reshape(4, 10)
    p = str(tmp_path / "gt.npy")
    ds.write_gt_npy(p, gt)
    assert np.array_equal(ds.load_gt_npy(p, 3, 5), gt[:3, :5])
    with pytest.raises(ValueError):
        ds.load_gt_npy(p, 5, 10)


def test_recall(ds):
    ids = np.array([[1, 2, 3], [4, 5, 6]])
    gt = np.array([[3, 2, 9], [7, 8, 9]])
    assert np.allclose(ds.recall_at_k(ids, gt, 3), [2 / 3, 0.0])


def test_int_mixture_properties(ds):
    m = ds.int_mixture(2000, 50, dim=128, n_comp=8, seed=3)
    assert m.base.dtype == np.float32 and m.base.shape == (2000, 128)
    assert (m.base == np.rint(m.base)).all() and m.base.min() >= 0 and m.base.max() <= 255
    # every squared L2 distance is an integer < 2^24: FP32 sums are exact in any order
    assert 128 * 255 ** 2 < 2 ** 24
    m2 = ds.int_mixture(2000, 50, dim=128, n_comp=8, seed=3)
    assert np.array_equal(m.base, m2.base)


def test_other_mixtures(ds):
    g = ds.l1_mixture(300, 10, dim=96, n_comp=4, seed=1)
    assert (g.base >= 0).all() and np.allclose(g.base.sum(1), 1.0, atol=1e-4)
    a = ds.angular_mixture(300, 10, dim=40, n_comp=4, seed=1)
    assert np.allclose(np.linalg.norm(a.base, axis=1), 1.0, atol=1e-4)


def test_graph_file_roundtrip(ds, tmp_path):
    adj = np.random.default_rng(1).integers(-1, 50, size=(50, 16)).astype(np.int32)
    p = str(tmp_path / "g.song")
    ds.save_graph(p, adj)
    np.testing.assert_array_equal(ds.load_graph(p), adj)
    raw = bytearray(open(p, "rb").read())
    raw[-4:] = np.array([99], np.int32).tobytes()  # out-of-range neighbour
    open(p, "wb").write(bytes(raw))
    with pytest.raises(ValueError):
        ds.load_graph(p)
    open(p, "wb").write(b"not a graph file at all.")
    with pytest.raises(ValueError):
        ds.load_graph(p)
