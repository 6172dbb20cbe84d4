"""The allocation-free graph build (song_build_graph_noalloc), through the C ABI.

Callers that cannot call cudaMalloc while they build (a serving process whose
device memory belongs to its own pool, or one that must not let an
allocation synchronise the device under live traffic) pass device buffers
for the rows and the adjacency; every temporary lives in the library's fixed
16 MiB device array.  This test checks that two calls in a row each produce
exactly the graph of the allocating entry point song_build_graph (the build
is deterministic, so the comparison is exact), also for rows wider than dim
whose padding holds garbage and for a single node, and that a build whose
temporaries do not fit is refused with a clear message.  The file name makes
pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(song):
    L = song.load_library()
    fn = L.song_build_graph_noalloc
    fn.argtypes = [C.c_int, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.POINTER(song._Params),
                   C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    return L, fn


def _case(song, ds, kind, n, dim, ld):
    """(rows [n, dim] for song_build_graph, padded rows [n, ld] with non-zero
    padding for the no-alloc call, kind constant)."""
    rng = np.random.default_rng(32 + dim + ld)
    if kind == "l2":
        rows = ds.int_mixture(n, 1, dim=dim, n_comp=16, seed=31).base
        padded = np.full((n, ld), 77.0, np.float32)
        padded[:, :dim] = rows
        return rows, padded.view(np.int32), song.KIND_L2
    rows = rng.integers(0, 2 ** 32, size=(n, dim), dtype=np.uint64).astype(np.uint32)
    padded = np.full((n, ld), 0xA5A5A5A5, np.uint32)
    padded[:, :dim] = rows
    return rows, padded.view(np.int32), song.KIND_HAMMING


@pytest.mark.parametrize("kind,n,dim,ld", [
    ("l2", 12000, 64, 64),
    ("hamming", 12000, 8, 8),
    ("l2", 6000, 60, 64),       # padding floats past dim hold 77.0
    ("hamming", 6000, 5, 8),    # padding words past dim hold 0xA5A5A5A5
    ("l2", 1, 16, 16),          # a single node: nothing to insert
])
def test_noalloc_build_matches_song_build_graph(cuda, song, ds, kind, n, dim, ld):
    torch = cuda
    L, fn = _noalloc(song)
    rows, padded, k = _case(song, ds, kind, n, dim, ld)
    p = song.Params(block_size=32, fixed_degree=31)
    expect = song.build_graph(rows, p, kind=k)          # the allocating entry point
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):                     # inputs written on the build's stream
        t = torch.from_numpy(padded).cuda()
    for call in range(2):                               # two calls in a row share the array
        with torch.cuda.stream(stream):
            d_adj = torch.full((n, 32), 12345, dtype=torch.int32, device="cuda")
        st = fn(k, t.data_ptr(), n, dim, ld, C.byref(p._c()), 32, 1024,
                d_adj.data_ptr(), stream.cuda_stream)
        assert st == song.SONG_OK, L.song_last_error().decode()
        stream.synchronize()
        np.testing.assert_array_equal(d_adj.cpu().numpy(), expect, err_msg=f"call {call}")


def test_noalloc_rejects_builds_beyond_the_scratch(cuda, song):
    torch = cuda
    L, fn = _noalloc(song)
    t = torch.zeros((4, 4), dtype=torch.float32, device="cuda")
    d_adj = torch.zeros((4, 32), dtype=torch.int32, device="cuda")
    p = song.Params(block_size=32, fixed_degree=31)
    # 50M nodes inserted one at a time: far more temporaries than the array holds;
    # refused before any work is queued (the small buffers are never touched).
    st = fn(song.KIND_L2, t.data_ptr(), 50_000_000, 4, 4, C.byref(p._c()), 1, 1024,
            d_adj.data_ptr(), None)
    assert st == song.SONG_ERR_BUDGET
    msg = L.song_last_error().decode()
    assert ("scratch" in msg and "16777216" in msg) or "too large" in msg, msg
