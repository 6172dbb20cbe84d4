"""The reference-shaped C++ interface (include/song_b200.hpp) compiles
against the C ABI, fails loudly without a GPU, and on a GPU returns exactly
what the oracle returns."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, knn_graph

SRC = os.path.join(ROOT, "tests", "cpp", "shim_search.cpp")


@pytest.fixture(scope="module")
def shim_bin(song, tmp_path_factory):
    song.load_library()  # builds libsong_b200.so when missing
    libdir = os.path.dirname(song.LIB_PATH)
    out = str(tmp_path_factory.mktemp("shim") / "shim_search")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SRC,
                           "-o", out, "-L", libdir, "-l:libsong_b200.so",
                           f"-Wl,-rpath,{libdir}"])
    return out


def _write_case(path, data, adj, q, k, ef):
    n, dim = data.shape
    with open(path, "wb") as f:
        np.array([n, dim, q.shape[0], k, ef, adj.shape[1]], np.int32).tofile(f)
        data.astype(np.float32).tofile(f)
        adj.astype(np.int32).tofile(f)
        q.astype(np.float32).tofile(f)


def test_shim_fails_loudly_without_gpu(shim_bin, ds, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    m = ds.int_mixture(200, 4, dim=16, n_comp=2, seed=1)
    adj = knn_graph(m.base, 8, 6)
    inp = str(tmp_path / "in.bin")
    _write_case(inp, m.base, adj, m.queries, 5, 16)
    r = subprocess.run([shim_bin, inp, str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 2 and "song_b200" in r.stderr


@pytest.mark.gpu
def test_shim_matches_oracle(cuda, shim_bin, ds, oracle, tmp_path):
    m = ds.int_mixture(3000, 100, dim=128, n_comp=8, seed=8)
    adj = knn_graph(m.base, 32, 31, seed=3)
    inp, outp = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    _write_case(inp, m.base, adj, m.queries, 10, 64)
    subprocess.check_call([shim_bin, inp, outp])
    raw = np.fromfile(outp, dtype=np.int32)
    ids = raw[:1000].reshape(100, 10)
    tr = raw[1000:].reshape(100, 12)
    oids, otr = oracle.search_l2(m.base, adj, 32, m.queries, 10, 64, pq_size=512, bf_words=256)
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_array_equal(tr, otr)


@pytest.mark.gpu
def test_shim_graph_search_and_bithash(cuda, shim_bin, ds, oracle, tmp_path):
    """graph_search (Graph::search's results) and BitHash through the C++ shim."""
    m = ds.angular_mixture(2500, 60, dim=64, n_comp=8, seed=9)
    adj = knn_graph(m.base, 32, 28, seed=4)
    inp, outp = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    _write_case(inp, m.base, adj, m.queries, 10, 40)
    subprocess.check_call([shim_bin, inp, outp, "extras"])
    raw = np.fromfile(outp, dtype=np.int32)
    o = 60 * 10 + 60 * 12
    gids = raw[o:o + 600].reshape(60, 10)
    gtr = raw[o + 600:o + 600 + 720].reshape(60, 12)
    codes = raw[o + 1320:].view(np.uint32).reshape(60, 8)
    oids, otr = oracle.graph_search(m.base, adj, 32, m.queries, 10, 40)
    np.testing.assert_array_equal(gids, oids)
    np.testing.assert_array_equal(gtr, otr)
    np.testing.assert_array_equal(codes, oracle.bithash_project(oracle.bithash_matrix(64, 256, 42),
                                                                 m.queries))
