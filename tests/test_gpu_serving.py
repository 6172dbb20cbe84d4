"""Serving loop with continuous batching (song_server_*).

Requests of mixed k and queue size are submitted in bursts while earlier
ones are still running; each result must be the same as the same query
searched alone (gpu_search / gpu_search_ex with that k and queue size):
ids and QueryTrace bit for bit, for plain and learned requests.  The
Poisson driver completes every request with positive latency, and requests
beyond the ring or max_k are refused.
"""
import importlib

import numpy as np
import pytest

from conftest import knn_graph

pytestmark = pytest.mark.gpu

KS = (1, 10, 100)
EFS = (32, 64, 128, 256)


@pytest.fixture(scope="module")
def setup(song, ds):
    torch = importlib.import_module("torch")
    gtm = importlib.import_module("2020_song_ex_b200.groundtruth")
    m = ds.int_mixture(20000, 600, dim=128, n_comp=32, seed=71)
    train = ds.int_mixture(20000, 2000, dim=128, n_comp=32, seed=71, query_seed=72).queries
    adj = song.build_graph(m.base, song.Params(), batch_ratio=32)
    g = song.KernelGraph(20000, 128, m.base, song.Params(pq_size=256), adj=adj)
    g.upload_to_gpu()
    nn1, _ = gtm.knn(m.base, train, 1)
    song.learn(g, torch.from_numpy(train).cuda(), 2000, torch.from_numpy(nn1[:, 0].copy()).cuda(),
               song.LearnParams(k=10, ef=128, entry_steps=200, stop_steps=300))
    rng = np.random.default_rng(5)
    ks = rng.choice(KS, 600).astype(np.int32)
    efs = rng.choice(EFS, 600).astype(np.int32)
    flags = (rng.random(600) < 0.5).astype(np.int32)
    yield m, g, ks, efs, flags
    g.close()


def alone(song, g, q, k, ef, learned, thr):
    opts = song.SearchOpts(learned=bool(learned), stop_threshold=thr)
    tr = song.GpuSearchTrace()
    ids, d = song.gpu_search_ex(g, opts, q[None, :], 1, int(k), int(ef), trace=tr)
    return ids[0], tr.queries[0]


def test_each_result_same_alone_and_in_mix(cuda, song, setup):
    m, g, ks, efs, flags = setup
    cfg = song.ServerConfig(max_k=100, max_ef=256, stop_threshold=0.85)
    with song.Server(g, cfg) as srv:
        tickets = []
        for s in range(0, 600, 50):  # bursts, no waiting in between
            t0 = srv.submit(m.queries[s:s + 50], ks[s:s + 50], efs[s:s + 50], flags[s:s + 50])
            tickets += list(range(t0, t0 + 50))
        got = {}
        import time
        deadline = time.time() + 60
        while len(got) < 600 and time.time() < deadline:
            for i, t in enumerate(tickets):
                if i in got:
                    continue
                done, ids, _, tr = srv.poll(t, int(ks[i]))
                if done:
                    got[i] = (ids.copy(), tr.copy())
        assert len(got) == 600
    for i in range(600):
        ids_a, tr_a = alone(song, g, m.queries[i], ks[i], efs[i], flags[i], 0.85)
        np.testing.assert_array_equal(got[i][0], ids_a, err_msg=f"request {i}")
        np.testing.assert_array_equal(got[i][1], tr_a, err_msg=f"trace {i}")


def test_poisson_driver(cuda, song, setup):
    m, g, ks, efs, flags = setup
    cfg = song.ServerConfig(max_k=100, max_ef=256, ring_slots=64)
    with song.Server(g, cfg) as srv:
        lat, ids, wall = srv.run_poisson(m.queries, ks, efs, flags, rate_qps=20000.0, seed=3)
    assert (lat > 0).all() and wall > 0
    for i in range(0, 600, 37):
        ids_a, _ = alone(song, g, m.queries[i], ks[i], efs[i], flags[i], cfg.stop_threshold)
        np.testing.assert_array_equal(ids[i, :ks[i]], ids_a)


def test_admission_limits(cuda, song, setup):
    m, g, ks, efs, flags = setup
    with song.Server(g, song.ServerConfig(max_k=10, max_ef=64, ring_slots=16)) as srv:
        with pytest.raises(song.SongError) as e:
            srv.submit(m.queries[:17], np.full(17, 10), np.full(17, 32))
        assert e.value.status == song.SONG_ERR_BUDGET
        with pytest.raises(song.SongError) as e:
            srv.submit(m.queries[:1], np.array([11]), np.array([32]))
        assert e.value.status == song.SONG_ERR_INVALID_ARG
    with pytest.raises(song.SongError) as e:  # a budget that holds no slot
        song.Server(g, song.ServerConfig(hbm_budget=64))
    assert e.value.status == song.SONG_ERR_BUDGET


def test_idle_wait_runs_out_then_relaunch(cuda, song, setup):
    """The persistent kernel's idle wait is bounded: with nothing to claim its
    warps leave after idle_exit_us and the kernel ends cleanly; a later submit
    relaunches it and the results are the same as searched alone.  A wait on
    the host with a deadline that passes first reports SONG_ERR_TIMEOUT."""
    import time
    m, g, ks, efs, flags = setup
    cfg = song.ServerConfig(max_k=100, max_ef=256, idle_exit_us=2000)
    with song.Server(g, cfg) as srv:
        for rnd in range(2):
            t0 = srv.submit(m.queries[:32], ks[:32], efs[:32], flags[:32])
            for i in range(32):
                ids, _, tr = srv.wait(t0 + i, int(ks[i]), timeout_us=30_000_000)
                ids_a, tr_a = alone(song, g, m.queries[i], ks[i], efs[i], flags[i], 0.85)
                np.testing.assert_array_equal(ids, ids_a, err_msg=f"round {rnd} request {i}")
                np.testing.assert_array_equal(tr, tr_a, err_msg=f"round {rnd} trace {i}")
            deadline = time.time() + 10
            st = srv.stats()
            while st["running"] and time.time() < deadline:  # the idle wait runs out
                time.sleep(0.01)
                st = srv.stats()
            assert st["running"] == 0
            assert st["launches"] == rnd + 1
            assert st["idle_exits"] + st["poll_cap_exits"] > 0
            assert st["stop_exits"] == 0
        # a deadline of zero: the request was only just published
        t1 = srv.submit(m.queries[40:41], ks[40:41], efs[40:41], flags[40:41])
        with pytest.raises(song.SongError) as e:
            srv.wait(t1, int(ks[40]), timeout_us=0)
        assert e.value.status == song.SONG_ERR_TIMEOUT
        ids, _, _ = srv.wait(t1, int(ks[40]), timeout_us=30_000_000)
        ids_a, _ = alone(song, g, m.queries[40], ks[40], efs[40], flags[40], 0.85)
        np.testing.assert_array_equal(ids, ids_a)


def test_bf16_serving_same_alone_and_in_mix(cuda, song, setup):
    """The serving loop on BF16 rows (the precision form's storage) with the
    learned entry/stop: each result equals the same request searched alone
    with the same options."""
    m, g, ks, efs, flags = setup
    song.set_precision(g, song.PREC_BF16)
    cfg = song.ServerConfig(max_k=100, max_ef=256, stop_threshold=0.85, precision=song.PREC_BF16)
    n = 200
    with song.Server(g, cfg) as srv:
        t0 = srv.submit(m.queries[:n], ks[:n], efs[:n], flags[:n])
        got = [srv.wait(t0 + i, int(ks[i]), timeout_us=30_000_000) for i in range(n)]
    for i in range(n):
        opts = song.SearchOpts(precision=song.PREC_BF16, learned=bool(flags[i]), stop_threshold=0.85)
        tr = song.GpuSearchTrace()
        ids, _ = song.gpu_search_ex(g, opts, m.queries[i][None, :], 1, int(ks[i]), int(efs[i]), trace=tr)
        np.testing.assert_array_equal(got[i][0], ids[0], err_msg=f"request {i}")
        np.testing.assert_array_equal(got[i][2], tr.queries[0], err_msg=f"trace {i}")
