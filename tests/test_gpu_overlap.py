"""Consecutive plain searches on one stream may overlap (GPU).

A plain search launch signals, once all of its queries are claimed, that
the next search launch on the stream may start on the SMs its tail leaves
idle; the later launch writes nothing until the earlier one has finished,
and every launch leaves its work-counter slot at zero for the launch that
takes the slot next (a ring of 1024).  These tests launch back to back
without synchronising and compare with launches made one at a time:
different output buffers, one shared output buffer (the last launch's
results must be what remains), traces, more launches than the counter ring
holds, and Graph::search launches (which use the same ring) in between.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def index(song, ds):
    m = ds.int_mixture(20000, 4000, dim=128, n_comp=32, seed=91)
    adj = song.build_graph(m.base, song.Params(), batch_ratio=32)
    g = song.KernelGraph(20000, 128, m.base, song.Params(pq_size=256, bf_words=256), adj=adj)
    g.upload_to_gpu()
    yield m, g
    g.close()


def _alone(cuda, song, g, dq, nq, ef, k=10):
    torch = cuda
    ids = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    tr = torch.empty((nq, 12), dtype=torch.int32, device="cuda")
    song.search_device(g, dq, nq, k, ef, ids, tr)
    torch.cuda.synchronize()
    return ids.cpu().numpy(), tr.cpu().numpy()


def test_back_to_back_launches_match_single_launches(cuda, song, index):
    torch = cuda
    m, g = index
    qa = torch.from_numpy(m.queries[:2000]).cuda()
    qb = torch.from_numpy(m.queries[2000:]).cuda()
    ra, ta = _alone(torch, song, g, qa, 2000, 128)
    rb, tb = _alone(torch, song, g, qb, 2000, 64)
    st = torch.cuda.Stream()
    outs = [torch.empty((2000, 10), dtype=torch.int32, device="cuda") for _ in range(4)]
    trs = [torch.empty((2000, 12), dtype=torch.int32, device="cuda") for _ in range(4)]
    torch.cuda.synchronize()
    for i in range(4):
        song.search_device(g, qa if i % 2 == 0 else qb, 2000, 10, 128 if i % 2 == 0 else 64, outs[i], trs[i],
                           stream=st)
    st.synchronize()
    for i in range(4):
        np.testing.assert_array_equal(outs[i].cpu().numpy(), ra if i % 2 == 0 else rb, err_msg=f"launch {i}")
        np.testing.assert_array_equal(trs[i].cpu().numpy(), ta if i % 2 == 0 else tb, err_msg=f"trace {i}")


def test_shared_output_buffer_holds_the_last_launch(cuda, song, index):
    torch = cuda
    m, g = index
    qa = torch.from_numpy(m.queries[:2000]).cuda()
    qb = torch.from_numpy(m.queries[2000:]).cuda()
    rb, _ = _alone(torch, song, g, qb, 2000, 64)
    out = torch.empty((2000, 10), dtype=torch.int32, device="cuda")
    st = torch.cuda.Stream()
    torch.cuda.synchronize()
    for _ in range(5):  # a long search, then a short one into the same rows
        song.search_device(g, qa, 2000, 10, 256, out, None, stream=st)
        song.search_device(g, qb, 2000, 10, 64, out, None, stream=st)
    st.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), rb)


def test_more_launches_than_the_counter_ring(cuda, song, index):
    torch = cuda
    m, g = index
    n_launch, nq = 2100, 64
    dq = torch.from_numpy(m.queries[:nq]).cuda()
    ref, _ = _alone(torch, song, g, dq, nq, 32)
    out = torch.empty((n_launch, nq, 10), dtype=torch.int32, device="cuda")
    gs_ids = torch.empty((nq, 10), dtype=torch.int32, device="cuda")
    st = torch.cuda.Stream()
    torch.cuda.synchronize()
    L = song.load_library()
    for i in range(n_launch):
        song.search_device(g, dq, nq, 10, 32, out[i], None, stream=st)
        if i % 700 == 350:  # Graph::search launches take slots of the same ring
            assert L.song_graph_search_device(g._h, dq.data_ptr(), nq, 10, 32, gs_ids.data_ptr(), None,
                                              st.cuda_stream) == 0
    st.synchronize()
    got = out.cpu().numpy()
    for i in range(n_launch):
        np.testing.assert_array_equal(got[i], ref, err_msg=f"launch {i}")


def test_learned_back_to_back_through_the_entry_ring(cuda, song, ds, index):
    """Learned searches take their entry-stage buffers from a ring of 16
    slots, and each entry stage may start while the previous search finishes:
    40 calls back to back (the ring wraps twice), alternating two batch
    sizes, give exactly what each call gives alone; so does a stop model."""
    torch = cuda
    gtm = __import__("importlib").import_module("2020_song_ex_b200.groundtruth")
    m, g = index
    train = ds.int_mixture(20000, 2000, dim=128, n_comp=32, seed=91, query_seed=92).queries
    nn1, _ = gtm.knn(m.base, train, 1)
    song.learn(g, torch.from_numpy(train).cuda(), 2000, torch.from_numpy(nn1[:, 0].copy()).cuda(),
               song.LearnParams(k=10, ef=64, entry_steps=200, stop_steps=300, entry_hubs=2048))
    qs = [torch.from_numpy(m.queries[:1500]).cuda(), torch.from_numpy(m.queries[1500:3500]).cuda()]
    for opts in (song.SearchOpts(learned=True, stop_threshold=1.0, beam=4, bloom_hashes=2,
                                 entry=song.ENTRY_NEAREST),
                 song.SearchOpts(learned=True, stop_threshold=0.9, beam=2)):
        refs = []
        for q in qs:
            r = torch.empty((q.shape[0], 10), dtype=torch.int32, device="cuda")
            song.search_device_ex(g, opts, q, q.shape[0], 10, 64, r, None, None)
            torch.cuda.synchronize()
            refs.append(r.cpu().numpy())
        st = torch.cuda.Stream()
        outs = [torch.full((qs[i % 2].shape[0], 10), -7, dtype=torch.int32, device="cuda") for i in range(40)]
        torch.cuda.synchronize()
        for i in range(40):
            q = qs[i % 2]
            song.search_device_ex(g, opts, q, q.shape[0], 10, 64, outs[i], None, None, stream=st)
        st.synchronize()
        for i in range(40):
            np.testing.assert_array_equal(outs[i].cpu().numpy(), refs[i % 2], err_msg=f"call {i}")
