"""BitHash (bitHash.h:17-56): sign-random-projection codes.

* The projection matrix comes from the same generator calls as the
  reference's constructor (bitHash.h:23-27): identical to the oracle's and to
  the compiled reference's matrix, bit for bit (CPU, no GPU needed).
* The GPU projection (song_bithash_project) is bit-identical to the oracle's
  sequential FP32 dot (bitHash.h:32-44, multiply then add per step), on
  ragged shapes, on vectors whose dot products land on or near zero, and on
  subnormal inputs; and to the compiled reference's own project_all.
* Argument errors are refused before any device work.
"""
import ctypes as C

import numpy as np
import pytest


def _x(rng, n, dim):
    x = rng.normal(size=(n, dim)).astype(np.float32)
    if n >= 8:
        x[0] = 0.0                                   # every dot is exactly 0: no bit set
        x[1, : dim // 2] = 0.0                       # half the terms vanish
        x[2] = np.float32(1e-39) * np.sign(x[2])     # subnormal inputs
        x[3] = np.rint(x[3] * 2.0) / 2.0             # coarse values: cancellations happen
        x[4] = x[3]                                  # duplicates give duplicate codes
        x[5] = -x[3]                                 # negated vector: complement where dot != 0
    return x


@pytest.mark.parametrize("dim,bits", [(128, 256), (200, 512), (7, 32)])
def test_matrix_matches_oracle(song, oracle, dim, bits):
    bh = song.BitHash(dim, seed=42, hash_bits=bits)
    np.testing.assert_array_equal(bh.R.view(np.uint32),
                                  oracle.bithash_matrix(dim, bits, 42).view(np.uint32))
    assert bh.hash_words == bits // 32


def test_matrix_matches_reference(song, oracle):
    if not oracle.ref_available(hash_bits=512, pq_size=512):
        pytest.skip("compiled reference not available")
    r = oracle.ref(hash_bits=512, pq_size=512)
    if r.gpu is None:
        pytest.skip("reference BitHash library not built")
    x = np.zeros((1, 64), np.float32)
    _, R = r.bithash_project(x)
    np.testing.assert_array_equal(song.BitHash(64, 42, 512).R, R)


def test_argument_errors(song):
    L = song.load_library()
    R = np.zeros((33, 8), np.float32)
    x = np.zeros((4, 8), np.float32)
    out = np.zeros((4, 2), np.uint32)
    assert L.song_bithash_project(R.ctypes.data, 8, 33, x.ctypes.data, 4, out.ctypes.data) == \
        song.SONG_ERR_INVALID_ARG
    assert L.song_bithash_project(R.ctypes.data, 0, 32, x.ctypes.data, 4, out.ctypes.data) == \
        song.SONG_ERR_INVALID_ARG
    assert L.song_bithash_project(None, 8, 32, x.ctypes.data, 4, out.ctypes.data) == \
        song.SONG_ERR_INVALID_ARG
    assert L.song_bithash_matrix(8, 0, 1, R.ctypes.data) == song.SONG_ERR_INVALID_ARG
    # n == 0 is a no-op
    assert L.song_bithash_project(R.ctypes.data, 8, 32, x.ctypes.data, 0, out.ctypes.data) == 0
    with pytest.raises(song.SongError):
        song.BitHash(8, hash_bits=48)


@pytest.mark.gpu
@pytest.mark.parametrize("n,dim,bits", [
    (1000, 128, 256), (777, 200, 512), (65, 33, 64), (130, 960, 256), (3, 7, 32), (64, 32, 160)])
def test_gpu_projection_bit_exact(cuda, song, oracle, n, dim, bits):
    rng = np.random.default_rng(n * 7 + dim)
    x = _x(rng, n, dim)
    bh = song.BitHash(dim, seed=42, hash_bits=bits)
    codes = bh.project_all(x)
    want = oracle.bithash_project(bh.R, x)
    np.testing.assert_array_equal(codes, want)
    if n >= 8:
        assert not codes[0].any()
        np.testing.assert_array_equal(codes[3], codes[4])
    np.testing.assert_array_equal(bh.project(x[n // 2]), want[n // 2])


@pytest.mark.gpu
def test_gpu_projection_matches_reference(cuda, song, oracle, ds):
    if not oracle.ref_available(hash_bits=512, pq_size=512):
        pytest.skip("compiled reference not available")
    r = oracle.ref(hash_bits=512, pq_size=512)
    if r.gpu is None:
        pytest.skip("reference BitHash library not built")
    x = ds.angular_mixture(2000, 1, dim=256, n_comp=16, seed=5).base
    codes, R = r.bithash_project(x)
    np.testing.assert_array_equal(song.BitHash(256, 42, 512).project_all(x), codes)


@pytest.mark.gpu
def test_gpu_projection_device_strides(cuda, song, oracle):
    torch = cuda
    n, dim, bits, ldx, ldc = 300, 100, 256, 104, 12
    rng = np.random.default_rng(3)
    x = _x(rng, n, dim)
    xp = np.zeros((n, ldx), np.float32)
    xp[:, :dim] = x
    bh = song.BitHash(dim, seed=7, hash_bits=bits)
    dev = torch.device("cuda", 0)
    d_R = torch.from_numpy(bh.R).to(dev)
    d_x = torch.from_numpy(xp).to(dev)
    d_c = torch.full((n, ldc), 0x5A5A5A5A, dtype=torch.int32, device=dev)
    st = torch.cuda.Stream()
    bh.project_device(d_R, d_x, n, d_c, ldx=ldx, ldc=ldc, stream=st)
    st.synchronize()
    got = d_c.cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(got[:, :bits // 32], oracle.bithash_project(bh.R, x))
    assert (got[:, bits // 32:] == 0x5A5A5A5A).all()  # padding words untouched
