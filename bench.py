"""Benchmark: QPS at recall@10 >= 0.95 of the SONG graph search on B200.

Workload (one "step" = one pass of the search over the whole query batch):
1,000,000 x 128 integer-valued FP32 base vectors from a 1,024-component
Gaussian mixture (centres U[0,255], sigma 20, clipped and rounded), 10,000
queries from the same mixture, NSW graph with BLOCK_SIZE 32 (degree 31) built
on the GPU, k = 10.  Synthetic, seeded stand-in for SIFT1M-shaped data (the
public set is not available).  The queue size ef (and the Bloom filter size)
is the smallest point of a sweep whose recall@10 against exact GPU
brute-force ground truth reaches 0.95.

Two forms are measured.  The plain form is bit-exact with the reference
search.  The learned form keeps BF16 rows (exact for these integer vectors)
and uses the learned entry and stop models, trained on the GPU from traces of
50,000 held-out queries searched by the plain form; its stop threshold is the
fastest one whose recall@10 reaches 0.95.

Outputs one JSON line (rank 0).  ``value`` is device-resident QPS (queries
and graph already in HBM) of the fastest form meeting the recall target,
with both forms under ``forms``; ``e2e`` is the same through the host C-ABI
call (pinned host queries, H2D + kernel + D2H in the timed region).

``--impl reference`` times the reference's own CPU search (Graph::search,
graph.h:33-115, compiled from the reference sources into oracle/_ref) on the
host cores, at the ef where IT reaches recall@10 0.95 on the same graph.

Multi-GPU (torchrun): replicas only -- each rank searches its own 10,000
queries on its own copy of the graph; no collective on the data path.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_BASE = 1_000_000
DIM = 128
N_COMP = 1024
NQ = 10_000
K = 10
SEED = 2020
BLOCK_SIZE = 32
TARGET_RECALL = 0.95
EF_SWEEP = (64, 96, 128, 192, 256, 320, 384, 448, 480, 512, 640, 768, 1024)
BF_SWEEP = (256, 512, 1024)
LEARN_THRESHOLDS = (0.8, 0.9, 0.95, 0.98, 1.0)   # 1.0: entry stage alone, no learned stop
LEARN_EFS = (96, 160)                              # queue sizes the models are trained at
LEARN_SWEEP_EFS = {96: (64, 72, 80, 88, 96, 128), 160: (160, 192, 256)}
LEARN_BEAMS = (1, 2, 3, 4)                         # candidates expanded per step
LEARN_BLOOM_HASHES = (4, 2)                        # BF_NHASH, and the learned search's cheaper test
WORKLOAD = "plain-L2 1M x 128 int-mixture(1024 comps), 10k queries, NSW deg 31 (BLOCK_SIZE 32), k=10"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.p = None
        self.path = os.path.join(tempfile.gettempdir(), f"song_clocks_{os.getpid()}.csv")

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p is not None:
            time.sleep(0.25)
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
            self.f.close()

    def summary(self) -> dict:
        if self.p is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_workload(rank: int):
    """Same base on every rank (replicas); rank r > 0 draws its own queries
    from the same mixture."""
    ds = importlib.import_module("2020_song_ex_b200.datasets")
    rep = importlib.import_module("2020_song_ex_b200.replicas")
    m = ds.int_mixture(N_BASE, NQ, dim=DIM, n_comp=N_COMP, seed=SEED,
                       query_seed=rep.query_seed(SEED, rank))
    return m.base, m.queries


def build_graph(song, base):
    return song.build_graph(base, song.Params(block_size=BLOCK_SIZE, fixed_degree=BLOCK_SIZE - 1),
                            batch_ratio=32)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(ef: int, bf_words: int, form: str = "plain"):
    """Per-launch DRAM bytes of the search kernel from the committed ncu
    summary, when it was captured at this workload, form and operating point."""
    p = os.path.join(ROOT, "profiles", "search_kernel_traffic.json")
    if os.path.exists(p):
        try:
            d = json.load(open(p))
            entries = d if isinstance(d, list) else [d]
            for e in entries:
                c = e.get("config", {})
                if (c.get("n"), c.get("nq"), c.get("ef"), c.get("bf_words"), c.get("form", "plain")) == \
                        (N_BASE, NQ, ef, bf_words, form):
                    return e.get("bytes_per_launch_scaled"), e.get("source")
        except (OSError, ValueError):
            pass
    return None, None


def bytes_per_query(trace: np.ndarray, k: int, row_bytes: int = DIM * 4) -> np.ndarray:
    """Algorithmic bytes: E*row + X*BLOCK_SIZE*4 + dim*4 + k*4 per query, where
    row is the bytes of one gathered vector: dim*4 for FP32 rows, or the byte
    row (dim rounded up to 16) that integer vectors in [0, 255] are read from."""
    E = trace[:, 5].astype(np.float64)
    X = trace[:, 2].astype(np.float64)
    return E * row_bytes + X * BLOCK_SIZE * 4 + DIM * 4 + k * 4


def _gpu_index(local: int) -> int:
    cvd = os.environ.get("CUDA_VISIBLE_DEVICES")
    if cvd:
        try:
            return int(cvd.split(",")[local])
        except (ValueError, IndexError):
            pass
    return local


def timed_device(torch, dist, ws, dev, stream, steps, warmup, launch, clocks_gpu=None, count=None):
    """Warm up, then time `steps` launches on `stream` with CUDA events
    (barrier + synchronize on both sides, max over ranks).  Returns
    (total_ms, per-step kernel ms list, clock summary or None).  With
    `count` (the library's launch counter), timed_device.last_launches is the
    number of kernels launched inside the timed loop."""
    for _ in range(warmup):
        launch()
    stream.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed")
    clk = Clocks(clocks_gpu) if clocks_gpu is not None else None
    if clk:
        clk.__enter__()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    n_before = count() if count is not None else 0
    t_start.record(stream)
    for i in range(steps):
        evs[i][0].record(stream)
        launch()
        evs[i][1].record(stream)
    t_end.record(stream)
    timed_device.last_launches = (count() - n_before) if count is not None else None
    stream.synchronize()
    torch.cuda.synchronize()
    if clk:
        clk.__exit__(None, None, None)
    torch.cuda.nvtx.range_pop()
    if ws > 1:
        dist.barrier()
    rep = importlib.import_module("2020_song_ex_b200.replicas")
    total = rep.max_over_ranks(t_start.elapsed_time(t_end), device=dev)
    return total, [a.elapsed_time(b) for a, b in evs], (clk.summary() if clk else None)


def timed_host(torch, dist, ws, dev, steps, warmup, call):
    """Time `steps` synchronous host-API calls (wall clock, max over ranks)."""
    for _ in range(warmup):
        call()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    h0 = time.perf_counter()
    for _ in range(steps):
        call()
    dt = time.perf_counter() - h0
    rep = importlib.import_module("2020_song_ex_b200.replicas")
    return rep.max_over_ranks(dt, device=dev)


def run_ours(args, ws, rank, local):
    import ctypes as C

    import torch
    import torch.distributed as dist
    song = importlib.import_module("2020_song_ex_b200")
    ds = importlib.import_module("2020_song_ex_b200.datasets")
    gtm = importlib.import_module("2020_song_ex_b200.groundtruth")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L = song.load_library()

    t0 = time.time()
    base, queries = make_workload(rank)
    adj = build_graph(song, base)
    torch.cuda.synchronize()
    build_s = time.time() - t0
    gt, _ = gtm.knn(base, queries, K)
    spot = gtm.spot_check(base, queries, gt, sample=16)
    torch.cuda.empty_cache()
    log(f"[rank {rank}] workload+graph {build_s:.1f}s, gt spot-check {spot}")

    dq = torch.from_numpy(queries).to(dev)
    d_ids = torch.empty((NQ, K), dtype=torch.int32, device=dev)
    d_tr = torch.empty((NQ, 12), dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)

    # ---------------- plain form: fastest (ef, bf_words) with recall@10 >= 0.95
    curve, best = [], None
    graphs = {}
    sweep = BF_SWEEP if not args.ef else (args.bf_words,)
    for bfw in sweep:
        g = song.KernelGraph(N_BASE, DIM, base, song.Params(pq_size=1024, bf_words=bfw), adj=adj)
        g.upload_to_gpu()
        graphs[bfw] = g
        for ef in (EF_SWEEP if not args.ef else (args.ef,)):
            song.search_device(g, dq, NQ, K, ef, d_ids, d_tr, stream=stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            song.search_device(g, dq, NQ, K, ef, d_ids, None, stream=stream)
            e1.record(stream)
            stream.synchronize()
            ms = e0.elapsed_time(e1)
            rec = float(ds.recall_at_k(d_ids.cpu().numpy(), gt, K).mean())
            pt = {"ef": ef, "bf_words": bfw, "recall": round(rec, 4), "qps": round(NQ / ms * 1e3)}
            curve.append(pt)
            if (rec >= TARGET_RECALL or args.ef) and (best is None or pt["qps"] > best["qps"]):
                best = pt
            if rec >= TARGET_RECALL:
                break
    if best is None:  # not reached: report the highest-recall point
        best = max(curve, key=lambda p: (p["recall"], p["qps"]))
    for bfw, g in graphs.items():
        if bfw != best["bf_words"]:
            g.close()
    g = graphs[best["bf_words"]]
    ef = best["ef"]
    log(f"[rank {rank}] plain operating point {best}")

    song.search_device(g, dq, NQ, K, ef, d_ids, d_tr, stream=stream)
    stream.synchronize()
    trace = d_tr.cpu().numpy()
    ids_op = d_ids.cpu().numpy()
    recall = float(ds.recall_at_k(ids_op, gt, K).mean())
    row_bytes = g.u8_rows() or DIM * 4  # the bench vectors and queries are integers in [0, 255]
    launch_bytes = float(bytes_per_query(trace, K, row_bytes).sum())

    parity = None
    if rank == 0 and not args.no_parity:  # bit-exactness at full size (oracle = checker)
        import oracle
        sample = 64
        oids, otr = oracle.search_l2(base, adj, BLOCK_SIZE, queries[:sample], K, ef, pq_size=1024,
                                     bf_words=best["bf_words"])
        parity = bool((oids == ids_op[:sample]).all() and (otr == trace[:sample]).all())

    plain_ms, plain_kern, clocks = timed_device(
        torch, dist, ws, dev, stream, args.steps, args.warmup,
        lambda: song.search_device(g, dq, NQ, K, ef, d_ids, None, stream=stream),
        clocks_gpu=_gpu_index(local), count=song.launch_count)
    plain_launches = timed_device.last_launches
    plain_qps = ws * NQ * args.steps / (plain_ms / 1e3)
    if args.no_e2e:
        g.close()
        return {"value": round(plain_qps, 1), "note": "profiling case"} if rank == 0 else None

    hq = torch.from_numpy(queries).pin_memory()
    hids = torch.empty((NQ, K), dtype=torch.int32).pin_memory()
    hdist = torch.empty((NQ, K), dtype=torch.float32).pin_memory()
    timing = song._Timing()

    def host_plain():
        st = L.song_gpu_search(g._h, C.c_void_p(hq.data_ptr()), NQ, K, NQ, ef,
                               C.c_void_p(hids.data_ptr()), None, C.byref(timing))
        if st != 0:
            raise song.SongError(st, L.song_last_error().decode())

    plain_e2e_s = timed_host(torch, dist, ws, dev, args.steps, args.warmup, host_plain)
    assert np.array_equal(hids.numpy(), ids_op), "host-API ids differ from the device path"
    plain_e2e = ws * NQ * args.steps / plain_e2e_s

    # ---------------- learned form: BF16 rows + learned entry/stop
    learned = None
    if not args.no_learned:
        ntrain = args.train_queries
        train = importlib.import_module("2020_song_ex_b200.datasets").int_mixture(
            N_BASE, ntrain, dim=DIM, n_comp=N_COMP, seed=SEED,
            query_seed=SEED + 104729 + rank).queries
        nn1, _ = gtm.knn(base, train, 1)
        torch.cuda.empty_cache()
        lcurve, lbest, learn_s, reps, blobs = [], None, 0.0, {}, {}
        prec = song.PREC_FP32  # the byte rows (exact for these vectors) are read either way
        for tef in LEARN_EFS:
            tl0 = time.time()
            reps[tef] = song.learn(g, torch.from_numpy(train).to(dev), ntrain,
                                   torch.from_numpy(np.ascontiguousarray(nn1[:, 0])).to(dev),
                                   song.LearnParams(k=K, ef=tef))
            torch.cuda.synchronize()
            learn_s += time.time() - tl0
            blobs[tef] = song.get_model(g)
            # threshold 1.0 (entry model only): every beam and Bloom hash count;
            # learned stop: beam 1 and 2 with 2 hashes
            for lef, thr, beam, nh in [(e, t, b, h) for e in LEARN_SWEEP_EFS[tef]
                                       for t in LEARN_THRESHOLDS
                                       for b in (LEARN_BEAMS if t >= 1.0 else (1, 2))
                                       for h in (LEARN_BLOOM_HASHES if t >= 1.0 else (2,))]:
                    opts = song.SearchOpts(precision=prec, learned=True, stop_threshold=thr, beam=beam,
                                           bloom_hashes=nh)
                    song.search_device_ex(g, opts, dq, NQ, K, lef, d_ids, None, d_tr, stream=stream)
                    stream.synchronize()  # the ids and traces of this point, not the previous one
                    rec = float(ds.recall_at_k(d_ids.cpu().numpy(), gt, K).mean())
                    trl = d_tr.cpu().numpy()
                    mss = []
                    for _ in range(3):  # median of three launches
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record(stream)
                        song.search_device_ex(g, opts, dq, NQ, K, lef, d_ids, None, None, stream=stream)
                        e1.record(stream)
                        stream.synchronize()
                        mss.append(e0.elapsed_time(e1))
                    ms = statistics.median(mss)
                    pt = {"ef": lef, "trained_ef": tef, "threshold": thr, "beam": beam,
                          "bloom_hashes": nh, "recall": round(rec, 4),
                          "qps": round(NQ / ms * 1e3),
                          "mean_expanded": round(float(trl[:, 2].mean()), 1),
                          "mean_distance_evals": round(float(trl[:, 5].mean()), 1),
                          "learned_stop_rate": round(float((trl[:, 11] == 2).mean()), 3)}
                    lcurve.append(pt)
                    if rec >= TARGET_RECALL and (lbest is None or pt["qps"] > lbest["qps"]):
                        lbest = pt
        if lbest is not None:
            lef = lbest["ef"]
            song.set_model(g, blobs[lbest["trained_ef"]])
            rep = reps[lbest["trained_ef"]]
            lprec = prec
            lopts = song.SearchOpts(precision=lprec, learned=True, stop_threshold=lbest["threshold"],
                                    beam=lbest["beam"], bloom_hashes=lbest["bloom_hashes"])
            lms, lkern, _ = timed_device(
                torch, dist, ws, dev, stream, args.steps, args.warmup,
                lambda: song.search_device_ex(g, lopts, dq, NQ, K, lef, d_ids, None, None,
                                              stream=stream), count=song.launch_count)
            l_launches = timed_device.last_launches
            ids_l = d_ids.cpu().numpy()
            song.search_device_ex(g, lopts, dq, NQ, K, lef, d_ids, None, d_tr, stream=stream)
            stream.synchronize()
            # gathered rows + the entry stage's hub tiles (hubs x dim BF16 per 128 queries)
            l_bytes = float(bytes_per_query(d_tr.cpu().numpy(), K, row_bytes).sum()) + \
                (NQ + 127) // 128 * int(rep.get("n_hubs", 0) or 0) * DIM * 2
            copts = lopts._c()

            def host_learned():
                st = L.song_gpu_search_ex(g._h, C.byref(copts), C.c_void_p(hq.data_ptr()), NQ, K,
                                          NQ, lef, C.c_void_p(hids.data_ptr()),
                                          C.c_void_p(hdist.data_ptr()), None, C.byref(timing))
                if st != 0:
                    raise song.SongError(st, L.song_last_error().decode())

            l_e2e_s = timed_host(torch, dist, ws, dev, args.steps, args.warmup, host_learned)
            learned = {
                "form": f"tensor-core entry stage ({int(rep.get('n_hubs', 0) or 0)} hubs) + learned entry/stop model, byte rows",
                "precision": "u8 rows (exact for these integer vectors)" if row_bytes < DIM * 4 else "fp32",
                "threshold": lbest["threshold"], "beam": lbest["beam"],
                "bloom_hashes": lbest["bloom_hashes"], "ef": lef,
                "trained_ef": lbest["trained_ef"],
                "qps": round(ws * NQ * args.steps / (lms / 1e3), 1),
                "e2e_qps": round(ws * NQ * args.steps / l_e2e_s, 1),
                "recall_at_10": round(float(ds.recall_at_k(ids_l, gt, K).mean()), 4),
                "ms_per_step": round(lms / args.steps, 4), "gpu_launches": int(l_launches),
                "algorithmic_bytes_per_launch": round(l_bytes),
                "kernel_ms_avg": round(statistics.mean(lkern), 4),
                "kernel_ms": [round(x, 3) for x in lkern],
                "curve": lcurve, "learn_s": round(learn_s, 2), "train_queries": ntrain,
                "learn_report": {k2: (round(v, 5) if isinstance(v, float) else v)
                                 for k2, v in rep.items()},
            }
        else:
            learned = {"curve": lcurve, "note": "no threshold reached recall 0.95",
                       "learn_report": reps}
        log(f"[rank {rank}] learned form {lbest}")

    # ---------------- serving: Poisson arrivals, mixed k / queue size, p50/p99 latency
    serving = None
    if not args.no_serving:
        serving = run_serving(song, ds, gtm, torch, g, base, queries, dev, args, rank)

    out = None
    if rank == 0:
        peak, peak_kind = peaks()
        avg_kern_s = statistics.mean(plain_kern) / 1e3
        achieved = launch_bytes / avg_kern_s / 1e9
        traffic, traffic_src = ncu_traffic(ef, best["bf_words"])
        roof_plain = {
            "kernel": "plain search_kernel<0,4,1,0,0,0> (bit-exact form)",
            "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
            "traffic": traffic, "traffic_source": traffic_src,
            "algorithmic_bytes_per_launch": round(launch_bytes),
            "kernel_ms_avg": round(avg_kern_s * 1e3, 4),
        }
        cpu = None if args.no_cpu_baseline else cpu_baseline(base, adj, queries, gt, ef)
        refgpu = None if args.no_ref_gpu else reference_gpu(base, adj, queries, gt, ef,
                                                            best["bf_words"], ids_op)
        use_learned = learned is not None and "qps" in learned and learned["qps"] > plain_qps
        roof_learned = None
        if learned is not None and "qps" in learned:
            la = learned["algorithmic_bytes_per_launch"] / (learned["kernel_ms_avg"] / 1e3) / 1e9
            lt, lsrc = ncu_traffic(learned["ef"], best["bf_words"], form="learned")
            roof_learned = {
                "kernel": ("entry_kernel + search_kernel<0,4,1,0,3,0> (entry model; the stop cannot fire)"
                           if learned["threshold"] >= 1.0 else
                           "entry_kernel + search_kernel<0,4,1,0,2,0> (entry + stop models)"),
                "bound": "hbm", "achieved": round(la, 1), "peak": peak, "unit": "GB/s",
                "frac": round(la / peak, 4), "peak_kind": peak_kind,
                "traffic": lt, "traffic_source": lsrc,
                "algorithmic_bytes_per_launch": learned["algorithmic_bytes_per_launch"],
                "kernel_ms_avg": learned["kernel_ms_avg"],
            }
        value = learned["qps"] if use_learned else plain_qps
        e2e_v = learned["e2e_qps"] if use_learned else plain_e2e
        out = {
            "metric": "QPS at recall@10>=0.95 (fastest form: plain bit-exact, or tensor-core entry + learned stop)",
            "value": round(value, 1),
            "unit": "queries/s",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round((learned["ms_per_step"] if use_learned else plain_ms / args.steps), 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "u8" if row_bytes < DIM * 4 else "f32",
            "data": "synthetic (seeded 1,024-component integer Gaussian mixture; SIFT1M-shaped stand-in)",
            "config": {
                "workload": WORKLOAD, "n": N_BASE, "dim": DIM, "nq_per_gpu": NQ, "k": K,
                "form": "learned" if use_learned else "plain",
                "ef": learned["ef"] if use_learned else ef, "bf_words": best["bf_words"],
                "bloom_hashes": learned["bloom_hashes"] if use_learned else 4,
                "beam": learned["beam"] if use_learned else 1, "pq_size": 1024,
                "graph": "GPU batched-insertion NSW (ratio 32)",
                "l2": "inputs larger than L2 (data 512 MB + adj 128 MB per GPU)",
                "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
            },
            "recall_at_10": learned["recall_at_10"] if use_learned else round(recall, 4),
            "forms": {
                "plain": {"qps": round(plain_qps, 1), "e2e_qps": round(plain_e2e, 1),
                          "recall_at_10": round(recall, 4), "operating_point": best,
                          "ms_per_step": round(plain_ms / args.steps, 4),
                          "gpu_launches": int(plain_launches),
                          "parity_sample_bit_exact": parity},
                "learned": learned,
                "learned_over_plain": (round(learned["qps"] / plain_qps, 3)
                                       if learned and "qps" in learned else None),
            },
            "recall_curve": curve,
            "gt_fp64_spot_check": {"queries": spot[0], "ids_missed": spot[1]},
            "e2e": {"value": round(e2e_v, 1), "unit": "queries/s",
                    "h2d_bytes_per_step": int(queries.nbytes),
                    "d2h_bytes_per_step": int(NQ * K * (8 if use_learned else 4))},
            "gpu_launches": int(learned["gpu_launches"] if use_learned else plain_launches),
            "roofline": roof_learned if use_learned else roof_plain,
            "roofline_plain": roof_plain,
            "serving": serving,
            "cpu_baseline": cpu,
            "reference_gpu_kernel": refgpu,
            "clocks": clocks,
            "trace_means": {k2: round(float(v), 2) for k2, v in
                            zip(song.TRACE_FIELDS, trace.mean(axis=0))},
            "build_s": round(build_s, 2),
        }
    g.close()
    return out


SERVE_KS = (1, 10, 100)
SERVE_EFS = (32, 64, 128, 256)
SERVE_RATES = (5_000, 20_000, 50_000, 100_000, 200_000)


def run_serving(song, ds, gtm, torch, g, base, queries, dev, args, rank):
    """Continuous-batching server over the same index: Poisson arrivals at
    several rates, k ~ U{1,10,100}, queue ~ U{32,...,256}; every request uses
    the learned entry/stop (trained here at queue 256, k 10) and falls back to
    the full search when not confident.  Per rate: achieved QPS, p50/p99
    latency (arrival to completion seen by the host), recall@k per k."""
    ntrain = min(args.train_queries, 20_000)
    train = ds.int_mixture(N_BASE, ntrain, dim=DIM, n_comp=N_COMP, seed=SEED,
                           query_seed=SEED + 7 * 104729 + rank).queries
    nn1, _ = gtm.knn(base, train, 1)
    gt100, _ = gtm.knn(base, queries, 100)
    torch.cuda.empty_cache()
    song.learn(g, torch.from_numpy(train).to(dev), ntrain,
               torch.from_numpy(np.ascontiguousarray(nn1[:, 0])).to(dev),
               song.LearnParams(k=10, ef=max(SERVE_EFS)))
    rng = np.random.default_rng(SEED + rank)
    out = []
    cfg = song.ServerConfig(max_k=max(SERVE_KS), max_ef=max(SERVE_EFS), stop_threshold=0.85)
    with song.Server(g, cfg) as srv:
        for rate in SERVE_RATES:
            nreq = int(min(len(queries), max(2000, rate * args.serve_seconds)))
            idx = rng.integers(0, len(queries), nreq)
            ks = rng.choice(SERVE_KS, nreq).astype(np.int32)
            efs = rng.choice(SERVE_EFS, nreq).astype(np.int32)
            flags = np.full(nreq, song.REQ_LEARNED, np.int32)
            lat, ids, wall = srv.run_poisson(queries[idx], ks, efs, flags, float(rate),
                                             seed=int(rate))
            rec = {}
            for k in SERVE_KS:
                sel = ks == k
                if sel.any():
                    rec[f"recall@{k}"] = round(float(ds.recall_at_k(ids[sel, :k], gt100[idx[sel], :k], k).mean()), 4)
            out.append({"offered_qps": rate, "requests": nreq,
                        "achieved_qps": round(nreq / wall, 1) if wall > 0 else None,
                        "p50_ms": round(float(np.percentile(lat, 50)), 3),
                        "p99_ms": round(float(np.percentile(lat, 99)), 3),
                        "mean_ms": round(float(lat.mean()), 3), **rec})
            log(f"[rank {rank}] serving {out[-1]}")
    return {"form": "FP32 + learned entry/stop (full search when not confident)",
            "k_choices": list(SERVE_KS), "queue_choices": list(SERVE_EFS), "points": out}


def cpu_baseline(base, adj, queries, gt, ef, sample=3000):
    """Reference CPU search (Graph::search) on a bounded sample, all host threads."""
    try:
        import oracle
        r = oracle.ref(block_size=BLOCK_SIZE, bf_words=256, pq_size=512)
    except Exception as e:  # reference not built
        return {"value": None, "unit": "queries/s", "cores": 0, "kind": "reference",
                "sample": f"unavailable: {e}"}
    ds = importlib.import_module("2020_song_ex_b200.datasets")
    threads = os.cpu_count() or 1
    cg = r.cpu_graph(base, adj)
    cg.search(queries[:64], K, ef, threads=threads)  # warm
    t0 = time.perf_counter()
    ids, _ = cg.search(queries[:sample], K, ef, threads=threads)
    dt = time.perf_counter() - t0
    rec = float(ds.recall_at_k(ids, gt[:sample], K).mean())
    cg.close()
    return {"value": round(sample / dt, 1), "unit": "queries/s", "cores": threads,
            "kind": "reference",
            "sample": f"{sample} of the {NQ} queries at ef={ef}, Graph::search (graph.h:33) "
                      f"from oracle/_ref on {threads} threads; its recall@10 {rec:.4f}"}


def reference_gpu(base, adj, queries, gt, ef, bf_words, ours):
    """The reference's own GPU kernel (kg_search_kernel via gpu_search, compiled
    for sm_100a), same graph and parameters: QPS and id agreement."""
    try:
        import oracle
        r = oracle.ref(block_size=BLOCK_SIZE, bf_words=bf_words, pq_size=1024)
        if r.gpu is None:
            raise FileNotFoundError("libref_gpu.so not built")
    except Exception as e:
        return {"unavailable": str(e)}
    ids, _tr, timing = r.gpu_search_l2(base, adj, queries, K, ef)  # warm (JIT-free: sm_100a SASS)
    ids, _tr, timing = r.gpu_search_l2(base, adj, queries, K, ef)
    return {"qps_total": round(NQ / (timing[4] / 1e3), 1), "kernel_ms": round(timing[2], 3),
            "total_ms": round(timing[4], 3), "ids_identical_to_ours": bool((ids == ours).all()),
            "note": "gpu_search (kernalGraph.h:307) on the same graph: 512-query batches, H2D+kernel+D2H"}


def run_reference(args, ws, rank, local):
    """--impl reference: the reference CPU search on the host cores."""
    if rank != 0:
        return None
    ds = importlib.import_module("2020_song_ex_b200.datasets")
    try:
        import oracle
        r = oracle.ref(block_size=BLOCK_SIZE, bf_words=256, pq_size=512)
    except Exception as e:
        return {"impl": "reference", "unavailable": f"compiled reference not available: {e}"}
    song = importlib.import_module("2020_song_ex_b200")
    gtm = importlib.import_module("2020_song_ex_b200.groundtruth")
    base, queries = make_workload(0)
    adj = build_graph(song, base)  # setup only (same graph as our arm); untimed
    gt, _ = gtm.knn(base, queries, K)
    threads = os.cpu_count() or 1
    cg = r.cpu_graph(base, adj)
    rng = np.random.default_rng(1)
    sweep_q = rng.choice(NQ, 400, replace=False)
    ef_op, curve = None, []
    for ef in EF_SWEEP:
        ids, _ = cg.search(queries[sweep_q], K, ef, threads=threads)
        rec = float(ds.recall_at_k(ids, gt[sweep_q], K).mean())
        curve.append({"ef": ef, "recall": round(rec, 4)})
        if rec >= TARGET_RECALL:
            ef_op = ef
            break
    if ef_op is None:
        ef_op = EF_SWEEP[-1]
    per_step = args.ref_step_queries
    times = []
    for i in range(args.warmup + args.steps):
        sel = np.arange(i * per_step, (i + 1) * per_step) % NQ
        t0 = time.perf_counter()
        cg.search(queries[sel], K, ef_op, threads=threads)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    total = sum(times)
    qps = per_step * args.steps / total
    ids, _ = cg.search(queries[:per_step], K, ef_op, threads=threads)
    rec = float(ds.recall_at_k(ids, gt[:per_step], K).mean())
    cg.close()
    return {
        "metric": "QPS at recall@10>=0.95 (plain bit-exact form)",
        "value": round(qps, 1), "unit": "queries/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded 1,024-component integer Gaussian mixture; SIFT1M-shaped stand-in)",
        "config": {"workload": WORKLOAD, "n": N_BASE, "dim": DIM, "k": K, "ef": ef_op,
                   "step": f"{per_step} queries"},
        "impl": "reference",
        "recall_at_10": round(rec, 4),
        "ef_curve": curve,
        "cpu_baseline": {"value": round(qps, 1), "unit": "queries/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"{per_step} queries per step, Graph::search (graph.h:33) from "
                                   f"oracle/_ref on {threads} threads, ef={ef_op}"},
        "e2e": {"value": round(qps, 1), "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main(argv=None):
    global N_BASE, NQ
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--ref-step-queries", type=int, default=1000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned form")
    ap.add_argument("--train-queries", type=int, default=50_000)
    ap.add_argument("--no-serving", action="store_true", help="skip the serving measurement")
    ap.add_argument("--serve-seconds", type=float, default=1.0)
    ap.add_argument("--n", type=int, default=N_BASE, help="base size (profiling cases)")
    ap.add_argument("--nq", type=int, default=NQ, help="queries per GPU (profiling cases)")
    ap.add_argument("--ef", type=int, default=0, help="fixed queue size: skip the sweep")
    ap.add_argument("--bf-words", type=int, default=1024, help="Bloom words with --ef")
    args = ap.parse_args(argv)
    N_BASE, NQ = args.n, args.nq
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        backend = "gloo" if args.impl == "reference" else "nccl"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            out = run_reference(args, ws, rank, local)
        else:
            out = run_ours(args, ws, rank, local)
        if rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
