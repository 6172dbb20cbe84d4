"""The C ABI library: loads, exports what include/*.h declares, and rejects
bad arguments before touching the GPU (CPU only; no compute calls)."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(song_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("song_index_create_l2", "song_gpu_search", "song_gpu_search_hamming",
              "song_search_device", "song_index_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol(song):
    L = song.load_library()
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing


def test_params_default_matches_config_h(song):
    L = song.load_library()
    p = song._Params()
    L.song_params_default(C.byref(p))
    assert (p.block_size, p.fixed_degree, p.search_degree, p.ef_construction, p.pq_size,
            p.topk, p.n_multiprobe, p.n_multiquery, p.hash_bits, p.bf_words, p.bf_nhash) == \
        (32, 31, 15, 150, 50, 10, 4, 512, 256, 256, 4)
    assert song.Params() == song.Params(**{f: getattr(p, f) for f, _ in p._fields_})


def _create(song, data, adj, params):
    h = C.c_void_p()
    L = song.load_library()
    st = L.song_index_create_l2(data.ctypes.data if data is not None else None,
                                data.shape[0] if data is not None else 0,
                                data.shape[1] if data is not None else 0,
                                adj.ctypes.data if adj is not None else None,
                                C.byref(params._c()), C.byref(h))
    return st, h, L.song_last_error().decode()


def test_rejects_out_of_range_adjacency(song):
    data = np.zeros((4, 8), np.float32)
    adj = np.full((4, 32), -1, np.int32)
    adj[2, 3] = 4  # == n
    st, h, msg = _create(song, data, adj, song.Params())
    assert st == song.SONG_ERR_INVALID_ARG and "adj[67]" in msg and not h


def test_rejects_bad_params(song):
    data = np.zeros((4, 8), np.float32)
    adj = np.full((4, 32), -1, np.int32)
    st, _, msg = _create(song, data, adj, song.Params(bf_nhash=5))
    assert st == song.SONG_ERR_UNSUPPORTED
    st, _, msg = _create(song, data, adj, song.Params(pq_size=0))
    assert st == song.SONG_ERR_INVALID_ARG
    st, _, msg = _create(song, None, None, song.Params())
    assert st == song.SONG_ERR_INVALID_ARG


def test_search_requires_upload(song):
    g = song.KernelGraph(4, 8, np.zeros((4, 8), np.float32))
    with pytest.raises(song.SongError):
        song.gpu_search(g, np.zeros((1, 8), np.float32), 1, 1)


def test_no_cpu_fallback_without_gpu(song):
    """Without a CUDA device the library fails loudly (no silent CPU path)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    g = song.KernelGraph(4, 8, np.zeros((4, 8), np.float32))
    with pytest.raises(song.SongError) as ei:
        g.upload_to_gpu()
    assert ei.value.status in (song.SONG_ERR_CUDA, song.SONG_ERR_OOM)
