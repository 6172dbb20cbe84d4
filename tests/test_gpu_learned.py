"""The learned entry/stop models: GPU training kernels against the float64
oracle, and what the trained models gain over the plain search."""
import importlib

import numpy as np
import pytest

from conftest import knn_graph
from oracle import mlp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("out,loss_kind", [(1, 0), (24, 1)])
def test_training_gradients_match_oracle(cuda, song, out, loss_kind):
    rng = np.random.default_rng(7 + out)
    p = rng.normal(0, 0.2, mlp.n_params(out)).astype(np.float32)
    x = rng.normal(0, 1, (300, mlp.FEAT)).astype(np.float32)
    y = (rng.random(300) if loss_kind == 0 else rng.integers(0, out, 300)).astype(np.float32)
    w = (rng.random(300) + 0.5).astype(np.float32)
    g, loss = song.mlp_grad(p, out, loss_kind, x, y, w)
    lo, go = mlp.loss_and_grad(p.astype(np.float64), out, loss_kind, x, y, w)
    assert abs(loss - lo) <= 1e-5 * max(1.0, abs(lo))
    np.testing.assert_allclose(g, go, rtol=2e-4, atol=2e-6)


def _setup(song, ds, n=30000, nq=400, ntrain=4000, entry_hubs=4096):
    torch = importlib.import_module("torch")
    gtm = importlib.import_module("2020_song_ex_b200.groundtruth")
    m = ds.int_mixture(n, nq, dim=128, n_comp=64, seed=61)
    train = ds.int_mixture(n, ntrain, dim=128, n_comp=64, seed=61, query_seed=62).queries
    adj = song.build_graph(m.base, song.Params(), batch_ratio=32)
    g = song.KernelGraph(n, 128, m.base, song.Params(pq_size=512), adj=adj)
    g.upload_to_gpu()
    nn1, _ = gtm.knn(m.base, train, 1)
    gt, _ = gtm.knn(m.base, m.queries, 10)
    rep = song.learn(g, torch.from_numpy(train).cuda(), ntrain,
                     torch.from_numpy(nn1[:, 0].copy()).cuda(),
                     song.LearnParams(k=10, ef=128, entry_steps=600, stop_steps=1200,
                                      entry_hubs=entry_hubs))
    return m, g, gt, rep


@pytest.mark.parametrize("entry_hubs", [4096, 0])
def test_learned_models_gain_over_plain(cuda, song, ds, entry_hubs):
    """entry_hubs 4096: the tensor-core entry stage proposes 24 candidates per
    query and the entry model scores them; 0: the entry model scores 24
    farthest-point hubs inside the search kernel."""
    m, g, gt, rep = _setup(song, ds, entry_hubs=entry_hubs)
    assert rep["n_hubs"] == (entry_hubs if entry_hubs else 24)
    assert rep["stop_loss_last"] < rep["stop_loss_first"]
    assert rep["entry_loss_last"] < rep["entry_loss_first"]
    assert 0.0 < rep["stop_pos_frac"] < 1.0 and rep["stop_samples"] > 0
    nq = m.queries.shape[0]
    tp, tl = song.GpuSearchTrace(), song.GpuSearchTrace()
    ids_p, _ = song.gpu_search_ex(g, song.SearchOpts(), m.queries, nq, 10, 128, trace=tp)
    ids_l, _ = song.gpu_search_ex(g, song.SearchOpts(learned=True, stop_threshold=0.8),
                                  m.queries, nq, 10, 128, trace=tl)
    rec_p = ds.recall_at_k(ids_p, gt, 10).mean()
    rec_l = ds.recall_at_k(ids_l, gt, 10).mean()
    exp_p = tp.queries[:, 2].mean()
    exp_l = tl.queries[:, 2].mean()
    # the gain: far fewer expansions for nearly the same recall
    assert exp_l < 0.8 * exp_p, (exp_p, exp_l)
    assert rec_l >= rec_p - 0.03, (rec_p, rec_l)
    assert (tl.queries[:, 11] == 2).mean() > 0.3  # most queries stopped by the model
    # threshold 1.0 never stops early: the full-budget search with the learned entry
    ids_f, _ = song.gpu_search_ex(g, song.SearchOpts(learned=True, stop_threshold=1.0),
                                  m.queries, nq, 10, 128)
    assert ds.recall_at_k(ids_f, gt, 10).mean() >= rec_p - 0.02
    # saved models reproduce the same search
    blob = song.get_model(g)
    g2 = song.KernelGraph(g.num_nodes, 128, m.base, song.Params(pq_size=512), adj=g.adj)
    g2.upload_to_gpu()
    song.set_model(g2, blob)
    ids_2, _ = song.gpu_search_ex(g2, song.SearchOpts(learned=True, stop_threshold=0.8),
                                  m.queries, nq, 10, 128)
    np.testing.assert_array_equal(ids_2, ids_l)
    g.close()
    g2.close()


def test_entry_stage_cuts_work_at_equal_recall(cuda, song, ds):
    """The entry stage's nearest hubs as entry points: at a quarter of the
    queue size the search reaches the plain search's recall with far fewer
    distance evaluations."""
    m, g, gt, rep = _setup(song, ds, n=30000, nq=400, ntrain=2000)
    nq = m.queries.shape[0]
    tp, tl = song.GpuSearchTrace(), song.GpuSearchTrace()
    ids_p, _ = song.gpu_search_ex(g, song.SearchOpts(), m.queries, nq, 10, 256, trace=tp)
    ids_l, _ = song.gpu_search_ex(g, song.SearchOpts(learned=True, stop_threshold=1.0),
                                  m.queries, nq, 10, 64, trace=tl)
    rec_p = ds.recall_at_k(ids_p, gt, 10).mean()
    rec_l = ds.recall_at_k(ids_l, gt, 10).mean()
    assert rec_l >= rec_p - 0.01, (rec_p, rec_l)
    assert tl.queries[:, 5].mean() < 0.6 * tp.queries[:, 5].mean()
    g.close()


def test_beam_two_expands_pairs(cuda, song, ds):
    """Beam 2 expands the two best candidates per step: same recall within
    0.01, and the search ends in fewer steps (expansions counted singly)."""
    m, g, gt, rep = _setup(song, ds, n=30000, nq=400, ntrain=2000)
    nq = m.queries.shape[0]
    t1, t2 = song.GpuSearchTrace(), song.GpuSearchTrace()
    ids1, _ = song.gpu_search_ex(g, song.SearchOpts(learned=True, stop_threshold=1.0),
                                 m.queries, nq, 10, 64, trace=t1)
    ids2, d2 = song.gpu_search_ex(g, song.SearchOpts(learned=True, stop_threshold=1.0, beam=2),
                                  m.queries, nq, 10, 64, trace=t2)
    r1 = ds.recall_at_k(ids1, gt, 10).mean()
    r2 = ds.recall_at_k(ids2, gt, 10).mean()
    assert r2 >= r1 - 0.01, (r1, r2)
    assert ((ids2 >= 0) & (ids2 < g.num_nodes)).all()
    assert (np.diff(d2, axis=1) >= 0).all()          # best-first
    assert t2.queries[:, 2].mean() > 0.8 * t1.queries[:, 2].mean()
    # beams 3 and 4: valid best-first output, recall not below beam 1's
    for beam in (3, 4):
        ids_b, d_b = song.gpu_search_ex(g, song.SearchOpts(learned=True, stop_threshold=1.0,
                                                           beam=beam), m.queries, nq, 10, 64)
        assert ((ids_b >= 0) & (ids_b < g.num_nodes)).all()
        assert (np.diff(d_b, axis=1) >= 0).all()
        assert ds.recall_at_k(ids_b, gt, 10).mean() >= r1 - 0.01
    # with a stop model too: checkpoints are still reached in steps of two
    ids3, _ = song.gpu_search_ex(g, song.SearchOpts(learned=True, stop_threshold=0.8, beam=2),
                                 m.queries, nq, 10, 128)
    assert ds.recall_at_k(ids3, gt, 10).mean() >= r1 - 0.05
    g.close()


def test_bloom_hashes_option(cuda, song, ds):
    """A learned search may test visited ids with fewer Bloom hashes than the
    index's BF_NHASH (a cheaper test, a few more false 'visited'): recall stays
    within 0.01 (0.02 with one hash) and the output stays valid; the default (0) is the index's
    value, bit for bit; a plain search refuses the option, so it keeps the
    reference's visited set."""
    m, g, gt, rep = _setup(song, ds, n=30000, nq=400, ntrain=2000)
    nq = m.queries.shape[0]
    o4 = song.SearchOpts(learned=True, stop_threshold=1.0)
    ids4, _ = song.gpu_search_ex(g, o4, m.queries, nq, 10, 64)
    ids4b, _ = song.gpu_search_ex(g, song.SearchOpts(learned=True, stop_threshold=1.0,
                                                     bloom_hashes=4), m.queries, nq, 10, 64)
    np.testing.assert_array_equal(ids4, ids4b)
    for nh in (1, 2, 3):
        ids, d = song.gpu_search_ex(g, song.SearchOpts(learned=True, stop_threshold=1.0,
                                                       bloom_hashes=nh), m.queries, nq, 10, 64)
        assert ((ids >= 0) & (ids < g.num_nodes)).all()
        assert (np.diff(d, axis=1) >= 0).all()
        tol = 0.02 if nh == 1 else 0.01
        assert ds.recall_at_k(ids, gt, 10).mean() >= ds.recall_at_k(ids4, gt, 10).mean() - tol
    with pytest.raises(song.SongError):
        song.gpu_search_ex(g, song.SearchOpts(learned=True, bloom_hashes=5), m.queries, nq, 10, 64)
    with pytest.raises(song.SongError):
        song.gpu_search_ex(g, song.SearchOpts(bloom_hashes=2), m.queries, nq, 10, 64)
    g.close()


def test_concurrent_streams_share_no_buffers(cuda, song, ds):
    """Searches of one index issued on two streams at once -- learned ones,
    each with its own entry-stage launch, and plain ones -- return exactly
    what the same queries return one call at a time: every launch takes its
    own work counter and its own entry-stage scratch."""
    torch = importlib.import_module("torch")
    m, g, gt, rep = _setup(song, ds, n=30000, nq=400, ntrain=2000)
    nq = m.queries.shape[0]
    h = nq // 2
    dq = torch.from_numpy(m.queries).cuda()
    for opts, ef in ((song.SearchOpts(learned=True, stop_threshold=1.0, beam=2), 64),
                     (song.SearchOpts(), 128)):
        ref = torch.empty((nq, 10), dtype=torch.int32, device="cuda")
        song.search_device_ex(g, opts, dq, nq, 10, ef, ref, None, None)
        torch.cuda.synchronize()
        s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
        for _ in range(3):
            o1 = torch.full((h, 10), -7, dtype=torch.int32, device="cuda")
            o2 = torch.full((nq - h, 10), -7, dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            song.search_device_ex(g, opts, dq[:h], h, 10, ef, o1, None, None, stream=s1)
            song.search_device_ex(g, opts, dq[h:], nq - h, 10, ef, o2, None, None, stream=s2)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(torch.cat([o1, o2]).cpu().numpy(), ref.cpu().numpy())
    g.close()


def test_entry_choices_are_exact_ablations(cuda, song, ds):
    """The ablation options change only the entry points: with the
    reference's seeds (SONG_ENTRY_SEEDS) a learned search without a stop is
    the plain search, ids and traces bit for bit; with the entry stage's
    nearest hubs (SONG_ENTRY_NEAREST) it is the seeded search from those
    hubs."""
    torch = importlib.import_module("torch")
    m, g, gt, rep = _setup(song, ds, n=30000, nq=400, ntrain=2000)
    nq = m.queries.shape[0]
    tp, ts = song.GpuSearchTrace(), song.GpuSearchTrace()
    ids_p, _ = song.gpu_search_ex(g, song.SearchOpts(), m.queries, nq, 10, 96, trace=tp)
    ids_s, _ = song.gpu_search_ex(g, song.SearchOpts(learned=True, stop_threshold=1.0,
                                                     entry=song.ENTRY_SEEDS),
                                  m.queries, nq, 10, 96, trace=ts)
    np.testing.assert_array_equal(ids_s, ids_p)
    np.testing.assert_array_equal(ts.queries, tp.queries)
    dq = torch.from_numpy(m.queries).cuda()
    cid = torch.empty((nq, song.ENTRY_K), dtype=torch.int32, device="cuda")
    cd = torch.empty((nq, song.ENTRY_K), dtype=torch.float32, device="cuda")
    song.entry_candidates(g, dq, nq, cid, cd)
    seeds = cid[:, :4].contiguous()
    out_n = torch.empty((nq, 10), dtype=torch.int32, device="cuda")
    out_s = torch.empty((nq, 10), dtype=torch.int32, device="cuda")
    tr_n = torch.empty((nq, 12), dtype=torch.int32, device="cuda")
    tr_s = torch.empty((nq, 12), dtype=torch.int32, device="cuda")
    song.search_device_ex(g, song.SearchOpts(learned=True, stop_threshold=1.0, entry=song.ENTRY_NEAREST),
                          dq, nq, 10, 64, out_n, None, tr_n)
    song.search_device_seeded(g, song.SearchOpts(), dq, nq, 10, 64, seeds, 4, out_s, None, tr_s)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out_n.cpu().numpy(), out_s.cpu().numpy())
    np.testing.assert_array_equal(tr_n.cpu().numpy(), tr_s.cpu().numpy())
    with pytest.raises(song.SongError):  # entry choices beyond the three are refused
        song.gpu_search_ex(g, song.SearchOpts(learned=True, entry=3), m.queries, nq, 10, 64)
    g.close()


def test_nearest_entry_keeps_the_nearest_hubs(cuda, song, ds):
    """Without the entry model the entry stage keeps only the n_multiprobe
    nearest hubs per query (less insertion work); they are the head of the
    full 24-hub list, at every split of the hub tiles over CTAs (16 splits
    at 400 queries, 3 at 10,000, 1 at 40,000), so the search from them is
    the seeded search from that head."""
    torch = importlib.import_module("torch")
    m, g, gt, rep = _setup(song, ds, n=30000, nq=400, ntrain=2000)
    for reps in (1, 25, 100):
        q = np.ascontiguousarray(np.tile(m.queries, (reps, 1)))
        nq = q.shape[0]
        dq = torch.from_numpy(q).cuda()
        cid = torch.empty((nq, song.ENTRY_K), dtype=torch.int32, device="cuda")
        cd = torch.empty((nq, song.ENTRY_K), dtype=torch.float32, device="cuda")
        song.entry_candidates(g, dq, nq, cid, cd)
        seeds = cid[:, :4].contiguous()
        out_n = torch.empty((nq, 10), dtype=torch.int32, device="cuda")
        out_s = torch.empty((nq, 10), dtype=torch.int32, device="cuda")
        song.search_device_ex(g, song.SearchOpts(learned=True, stop_threshold=1.0,
                                                 entry=song.ENTRY_NEAREST),
                              dq, nq, 10, 64, out_n, None, None)
        song.search_device_seeded(g, song.SearchOpts(), dq, nq, 10, 64, seeds, 4, out_s, None, None)
        torch.cuda.synchronize()
        a_n, a_s = out_n.cpu().numpy(), out_s.cpu().numpy()
        np.testing.assert_array_equal(a_n, a_s)
        # every copy of a query found the same neighbours
        np.testing.assert_array_equal(a_n.reshape(reps, 400, 10),
                                      np.broadcast_to(a_n[:400], (reps, 400, 10)))
    g.close()
