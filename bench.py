"""Benchmark: QPS at recall@10 >= 0.95 of the SONG graph search on one B200.

Workload (one "step" = one pass of the search over the whole query batch):
1,000,000 x 128 integer-valued FP32 base vectors from a 1,024-component
Gaussian mixture (centres U[0,255], sigma 20, clipped and rounded), 10,000
evaluation queries from the same mixture, NSW graph with BLOCK_SIZE 32
(degree 31), k = 10.  Synthetic, seeded stand-in for SIFT1M-shaped data (the
public set is not available).

Operating points (queue size ef, Bloom size, and the learned form's knobs)
are chosen on 10,000 separate calibration queries (another seed) as the
fastest point whose calibration recall@10 reaches 0.95 plus a small margin;
the numbers reported are those of the 10,000 evaluation queries at that
point.  Recall is against exact GPU brute-force ground truth.

Two forms are measured.  The plain form is bit-exact with the reference
search (kernalGraph.h:184-299).  The learned form adds the tensor-core entry
stage, the learned entry model and (when it pays) the learned stop, trained
on the GPU from traces of 50,000 held-out queries searched by the plain form.
Ablations measure the entry model and the stop model against the same
search without them.

The graph: when the reference arm ran first on the same machine it leaves
the graph the reference's own builder made (build_graph, graph.h:190-199) in
the cache directory, and this arm searches that graph; otherwise the graph
comes from the library's GPU builder.  ``config.graph`` says which.

Output: ONE compact JSON line on stdout (rank 0; a few KB at most).  Curves,
sweeps, per-step times and the serving points go to a side file
(``--details``, default ``gpurun_out/bench_details.json``) and to stderr.
``value`` is device-resident QPS of the fastest form meeting the recall
target (queries and graph already in HBM); ``e2e`` is the same through the
host C-ABI call (pinned host queries, H2D + kernels + D2H timed).

``--impl reference`` runs the reference's own CPU code only (oracle/_ref,
compiled from the reference sources; none of this library): its graph
builder, then Graph::search (graph.h:33-115) timed on all host cores and on
one core (bench_cpu semantics, bench_cpu.cpp:444-451), at the ef where it
reaches recall@10 0.95 on the same data.

Extra workloads (``--configs``, all by default; one summary each in the
line's ``configs``): C3, the precision form on 1M x 960 L1-normalised vectors
(BF16 and per-vector FP8 rows, FP32 re-rank, distance error against FP64);
C4, 1,183,514 x 200 angular vectors at k 10 and 100 (plain and entry-stage
forms, models trained on 50,000 held-out queries); C4's Hamming variant,
512-bit BitHash codes of 290,000 x 256 vectors.  Their graphs come from the
GPU builder.

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
NCAL = 10_000
K = 10
SEED = 2020
CAL_SEED = SEED + 31337         # calibration queries: same mixture, separate generator
TRAIN_SEED = SEED + 104729      # training queries of the learned models
BLOCK_SIZE = 32
TARGET_RECALL = 0.95
SELECT_MARGIN = 0.002           # points are chosen at calibration recall >= target + margin
EF_SWEEP = (64, 96, 128, 192, 256, 320, 384, 448, 480, 512, 576, 640, 768, 1024)
BF_SWEEP = (256, 512, 1024)
QUEUE_SWEEP = (32, 64, 128, 256)
EF_SWEEP_K100 = (128, 192, 256, 320, 384, 448, 512, 640, 768, 1024)
LEARN_THRESHOLDS = (0.8, 0.9, 0.95, 0.98, 1.0)   # 1.0: entry stage alone, no learned stop
LEARN_EFS = (96, 160)                              # queue sizes the models are trained at
LEARN_SWEEP_EFS = {96: (64, 72, 80, 88, 96, 128), 160: (160, 192, 256)}
LEARN_BEAMS = (1, 2, 3, 4)                         # candidates expanded per step
LEARN_BLOOM_HASHES = (4, 2)                        # BF_NHASH, and the learned search's cheaper test
# The learned form's own Bloom filter: its searches insert about 69 x 31 ids, 1.5 % false
# positives with 2 hashes in 32,768 bits; a larger filter (the plain form's choice may be
# 1,024 words) would only cost resident warps (8 KB of shared memory per query instead of 4).
LEARN_BF_WORDS = 512
ABLATION_EFS = (64, 72, 80, 88, 96, 112, 128, 160, 192, 256, 320, 384, 512)
WORKLOAD = "plain-L2 1M x 128 int-mixture(1024 comps), 10k queries, NSW deg 31 (BLOCK_SIZE 32), k=10"
METRIC = "QPS at recall@10>=0.95 (fastest form: plain bit-exact, or the entry-stage/learned form)"
DATA = "synthetic, seeded (1,024-component integer Gaussian mixture, SIFT1M-shaped)"
LINE_LIMIT = 4000                                  # bytes of the stdout JSON line


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


# ------------------------------------------------------------------ workload

def datasets():
    return importlib.import_module("2020_song_ex_b200.datasets")


def make_workload(rank: int):
    """Same base on every rank (replicas); rank r > 0 draws its own queries
    from the same mixture."""
    ds = datasets()
    rep = importlib.import_module("2020_song_ex_b200.replicas")
    m = ds.int_mixture(N_BASE, NQ, dim=DIM, n_comp=N_COMP, seed=SEED,
                       query_seed=rep.query_seed(SEED, rank))
    return m.base, m.queries


def draw_queries(n: int, query_seed: int) -> np.ndarray:
    """Extra queries from the workload's mixture with their own generator."""
    return datasets().int_mixture(N_BASE, n, dim=DIM, n_comp=N_COMP, seed=SEED,
                                  query_seed=query_seed, with_base=False).queries


def ref_graph_path() -> str:
    """Where the reference arm leaves the graph its own builder made."""
    return os.path.join(datasets().cache_dir(),
                        f"c2_ref_build_graph_n{N_BASE}_d{DIM}_c{N_COMP}_s{SEED}_bs{BLOCK_SIZE}.song")


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
                    return e.get("bytes_per_launch_scaled"), "profiles/search_kernel_traffic.json"
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


def choose(points, key="recall_cal"):
    """Fastest point whose calibration recall reaches the target plus the
    margin; else the highest-recall point (flagged)."""
    ok = [p for p in points if p[key] >= TARGET_RECALL + SELECT_MARGIN]
    if ok:
        return max(ok, key=lambda p: p["qps"]), True
    return max(points, key=lambda p: (p[key], p["qps"])), False


def timed_device(torch, dist, ws, dev, stream, steps, warmup, launch, clocks_gpu=None, count=None):
    """Warm up, then time `steps` launches on `stream` with CUDA events
    (barrier + synchronize on both sides, max over ranks).  Only the start
    and the end of the region are recorded: an event between two steps would
    keep a step's launch from overlapping the previous step's tail.  Returns
    (total_ms, per-step average ms repeated per step, clock summary or None).
    With `count` (the library's launch counter), timed_device.last_launches
    is the number of kernels launched inside the timed loop."""
    for _ in range(warmup):
        launch()
    stream.synchronize()
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
    for _ in range(steps):
        launch()
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
    return total, [total / steps] * steps, (clk.summary() if clk else None)


def timed_host(torch, dist, ws, dev, steps, warmup, call):
    """Time `steps` synchronous host-API calls (wall clock, max over ranks)."""
    for _ in range(warmup):
        call()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    calls = []
    h0 = time.perf_counter()
    for _ in range(steps):
        c0 = time.perf_counter()
        call()
        calls.append(time.perf_counter() - c0)
    dt = time.perf_counter() - h0
    timed_host.last_calls_ms = [round(x * 1e3, 4) for x in calls]
    rep = importlib.import_module("2020_song_ex_b200.replicas")
    return rep.max_over_ranks(dt, device=dev)


def launch_ms(torch, stream, fn, reps=3):
    """CUDA-event time per launch of `reps` launches of fn issued back to back
    (one untimed first): the same overlap of consecutive launches as the timed
    region, so the calibration ranks points by what is then reported."""
    fn()
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    stream.synchronize()
    return e0.elapsed_time(e1) / reps


# ------------------------------------------------------------------ our arm

class Ctx:
    """Per-run state shared by the measurement sections."""
    pass


def run_ours(args, ws, rank, local):
    import torch
    import torch.distributed as dist
    song = importlib.import_module("2020_song_ex_b200")
    ds = datasets()
    gtm = importlib.import_module("2020_song_ex_b200.groundtruth")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    song.load_library()

    c = Ctx()
    c.torch, c.dist, c.song, c.ds, c.gtm, c.dev, c.ws, c.rank, c.local, c.args = \
        torch, dist, song, ds, gtm, dev, ws, rank, local, args
    details = {}

    t0 = time.time()
    base, queries = make_workload(rank)
    cal = draw_queries(NCAL, CAL_SEED + rank)
    rp = ref_graph_path()
    if args.graph in ("auto", "ref") and os.path.exists(rp):
        adj = ds.load_graph(rp)
        graph_src = "reference build_graph (graph.h:190-199), made by the reference arm"
    elif args.graph == "ref":
        raise SystemExit(f"--graph ref: {rp} not found (run --impl reference first)")
    else:
        adj = song.build_graph(base, song.Params(block_size=BLOCK_SIZE, fixed_degree=BLOCK_SIZE - 1),
                               batch_ratio=32)
        graph_src = "library GPU builder (batched insertion, ratio 32)"
    torch.cuda.synchronize()
    setup_s = time.time() - t0
    gt100, _ = gtm.knn(base, queries, 100)
    gt = np.ascontiguousarray(gt100[:, :K])
    gt_cal, _ = gtm.knn(base, cal, K)
    spot = gtm.spot_check(base, queries, gt100, sample=16)
    torch.cuda.empty_cache()
    log(f"[rank {rank}] workload+graph {setup_s:.1f}s ({graph_src}), gt spot-check {spot}")
    c.base, c.queries, c.cal, c.adj, c.gt, c.gt100, c.gt_cal = base, queries, cal, adj, gt, gt100, gt_cal
    c.dq = torch.from_numpy(queries).to(dev)
    c.dcal = torch.from_numpy(cal).to(dev)
    c.d_ids = torch.empty((max(NQ, NCAL), K), dtype=torch.int32, device=dev)     # row slices stay contiguous
    c.d_ids100 = torch.empty((max(NQ, NCAL), 100), dtype=torch.int32, device=dev)
    c.d_tr = torch.empty((max(NQ, NCAL), 12), dtype=torch.int32, device=dev)
    c.stream = torch.cuda.Stream(device=dev)

    plain = measure_plain(c, details)
    c.g = plain.pop("_graph")
    queue = measure_queue_sweep(c, details, plain["bf_words"]) if not args.no_queue_sweep else None
    c.gl = None
    if not args.no_learned:  # the learned form's index: the same rows and graph, its own filter size
        c.gl = song.KernelGraph(N_BASE, DIM, c.base, song.Params(pq_size=1024, bf_words=LEARN_BF_WORDS),
                                adj=c.adj)
        c.gl.upload_to_gpu()
    learned = None if args.no_learned else measure_learned(c, details, plain)
    serving = None if args.no_serving else measure_serving(c, details)
    c.g.close()
    if c.gl is not None:
        c.gl.close()

    out = None
    if rank == 0:
        peak, peak_kind = peaks()
        roof_plain = roofline(plain, peak, peak_kind, "plain search_kernel (bit-exact form)",
                              ncu_traffic(plain["ef"], plain["bf_words"]))
        cpu = None if args.no_cpu_baseline else cpu_baseline(base, adj, queries, gt, plain["ef"])
        refgpu = None if args.no_ref_gpu else reference_gpu(base, adj, queries, plain["ef"],
                                                            plain["bf_words"], plain["_ids"])
        use_learned = learned is not None and "qps" in learned and learned["qps"] > plain["qps"]
        roof_learned = None
        if learned is not None and "qps" in learned:
            roof_learned = roofline(learned, peak, peak_kind, learned["kernels"],
                                    ncu_traffic(learned["ef"], LEARN_BF_WORDS, form="learned"))
        best = learned if use_learned else plain
        details.update({"plain": strip(plain), "learned": strip(learned), "queue_sweep": queue,
                        "serving": serving, "cpu_baseline": cpu, "reference_gpu_kernel": refgpu,
                        "roofline_plain": roof_plain, "roofline_learned": roof_learned,
                        "gt_fp64_spot_check": {"queries": spot[0], "ids_missed": spot[1]},
                        "graph": graph_src, "setup_s": round(setup_s, 2)})
        out = {
            "metric": METRIC,
            "value": round(best["qps"], 1),
            "unit": "queries/s",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": best["ms_per_step"],
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": DATA,
            "config": {
                "workload": WORKLOAD, "n": N_BASE, "dim": DIM, "nq_per_gpu": NQ, "k": K,
                "form": "learned" if use_learned else "plain",
                "ef": best["ef"], "bf_words": LEARN_BF_WORDS if use_learned else plain["bf_words"],
                "bloom_hashes": best.get("bloom_hashes", 4), "beam": best.get("beam", 1),
                "graph": graph_src,
                "storage": "u8 byte rows (integer base 0-255)" if plain["row_bytes"] < DIM * 4
                           else "fp32 rows",
                "arithmetic": "exact integer distances (= reference FP32)",
                "selection": f"knobs chosen on {NCAL} calibration queries (recall >= "
                             f"{TARGET_RECALL}+{SELECT_MARGIN}), reported on evaluation queries",
                "l2": "inputs larger than L2 (data 512 MB + adj 128 MB per GPU)",
                "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
            },
            "recall_at_10": best["recall_at_10"],
            "e2e": {"value": round(best["e2e_qps"], 1), "unit": "queries/s",
                    "h2d_bytes_per_step": int(queries.nbytes),
                    "d2h_bytes_per_step": int(NQ * K * (8 if use_learned else 4))},
            "gpu_launches": int(best["gpu_launches"]),
            "roofline": roof_learned if use_learned else roof_plain,
            "roofline_plain": roof_plain,
            "cpu_baseline": cpu,
            "clocks": plain["clocks"],
            "forms": {"plain": summary_plain(plain),
                      "learned": summary_learned(learned),
                      "learned_over_plain": (round(learned["qps"] / plain["qps"], 3)
                                             if learned and "qps" in learned else None)},
            "configs": {"c2_queue_sweep": summary_queue(queue), "c5_serving": summary_serving(serving)},
            "reference_gpu_kernel": ({"qps": refgpu.get("qps_total"),
                                      "ids_identical": refgpu.get("ids_identical_to_ours")}
                                     if refgpu and "qps_total" in refgpu else refgpu),
        }
        if args.configs:
            ex = measure_extra_configs(c, details, args.configs.split(","))
            out["configs"].update(ex)
    return out, details


def strip(d):
    if d is None:
        return None
    return {k: v for k, v in d.items() if not k.startswith("_")}


def roofline(form, peak, peak_kind, kernel, traffic_src):
    achieved = form["algorithmic_bytes_per_launch"] / (form["kernel_ms_avg"] / 1e3) / 1e9
    traffic, src = traffic_src
    return {"kernel": kernel, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
            "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
            "traffic": traffic, "traffic_source": src,
            "algorithmic_bytes_per_launch": form["algorithmic_bytes_per_launch"],
            "kernel_ms_avg": form["kernel_ms_avg"]}


def measure_plain(c, details):
    """The plain bit-exact form: (ef, bf_words) chosen on calibration queries,
    then timed and checked on the evaluation queries."""
    torch, song, ds, args = c.torch, c.song, c.ds, c.args
    import ctypes as C
    L = song.load_library()
    stream, d_ids, d_tr = c.stream, c.d_ids, c.d_tr
    curve, graphs = [], {}
    bfs = BF_SWEEP if not args.ef else (args.bf_words,)
    efs = EF_SWEEP if not args.ef else (args.ef,)
    for bfw in bfs:
        g = song.KernelGraph(N_BASE, DIM, c.base, song.Params(pq_size=1024, bf_words=bfw), adj=c.adj)
        g.upload_to_gpu()
        graphs[bfw] = g
        for ef in efs:
            ids_v = d_ids[:NCAL]
            ms = launch_ms(torch, stream, lambda: song.search_device(g, c.dcal, NCAL, K, ef, ids_v, None,
                                                                     stream=stream), reps=3)
            rec = float(ds.recall_at_k(ids_v.cpu().numpy(), c.gt_cal, K).mean())
            curve.append({"ef": ef, "bf_words": bfw, "recall_cal": round(rec, 4),
                          "qps": round(NCAL / ms * 1e3)})
            if rec >= TARGET_RECALL + SELECT_MARGIN:
                break
    op, reached = choose(curve) if not args.ef else (curve[0], True)
    for bfw, g in graphs.items():
        if bfw != op["bf_words"]:
            g.close()
    g = graphs[op["bf_words"]]
    ef = op["ef"]
    log(f"[rank {c.rank}] plain operating point {op}")
    ids_v = d_ids[:NQ]
    song.search_device(g, c.dq, NQ, K, ef, ids_v, d_tr[:NQ], stream=stream)
    stream.synchronize()
    trace = d_tr[:NQ].cpu().numpy()
    ids_op = ids_v.cpu().numpy()
    recall = float(ds.recall_at_k(ids_op, c.gt, K).mean())
    row_bytes = g.u8_rows() or DIM * 4  # the bench vectors and queries are integers in [0, 255]
    launch_bytes = float(bytes_per_query(trace, K, row_bytes).sum())
    parity = None
    if c.rank == 0 and not args.no_parity:  # bit-exactness at full size (oracle = checker)
        import oracle
        sample = 64
        oids, otr = oracle.search_l2(c.base, c.adj, BLOCK_SIZE, c.queries[:sample], K, ef,
                                     pq_size=1024, bf_words=op["bf_words"])
        parity = bool((oids == ids_op[:sample]).all() and (otr == trace[:sample]).all())
    total_ms, kern, clocks = timed_device(
        torch, c.dist, c.ws, c.dev, stream, args.steps, args.warmup,
        lambda: song.search_device(g, c.dq, NQ, K, ef, ids_v, None, stream=stream),
        clocks_gpu=_gpu_index(c.local), count=song.launch_count)
    launches = timed_device.last_launches
    qps = c.ws * NQ * args.steps / (total_ms / 1e3)
    e2e = None
    if not args.no_e2e:
        hq = torch.from_numpy(c.queries).pin_memory()
        hids = torch.empty((NQ, K), dtype=torch.int32).pin_memory()
        timing = song._Timing()

        def host_plain():
            st = L.song_gpu_search(g._h, C.c_void_p(hq.data_ptr()), NQ, K, NQ, ef,
                                   C.c_void_p(hids.data_ptr()), None, C.byref(timing))
            if st != 0:
                raise song.SongError(st, L.song_last_error().decode())

        e2e_s = timed_host(torch, c.dist, c.ws, c.dev, args.steps, args.warmup, host_plain)
        details["plain_e2e_call_ms"] = timed_host.last_calls_ms
        details["plain_e2e_last_timing"] = {f: round(getattr(timing, f), 4) for f in
                                            ("h2d_ms", "kernel_ms", "d2h_ms", "total_ms")}
        assert np.array_equal(hids.numpy(), ids_op), "host-API ids differ from the device path"
        e2e = c.ws * NQ * args.steps / e2e_s
    details["plain_curve"] = curve
    details["plain_kernel_ms"] = [round(x, 3) for x in kern]
    details["plain_trace_means"] = {k2: round(float(v), 2) for k2, v in
                                    zip(song.TRACE_FIELDS, trace.mean(axis=0))}
    return {"_graph": g, "_ids": ids_op, "ef": ef, "bf_words": op["bf_words"],
            "reached_on_calibration": reached, "recall_cal": op["recall_cal"],
            "qps": qps, "e2e_qps": e2e if e2e is not None else qps,
            "recall_at_10": round(recall, 4), "ms_per_step": round(total_ms / args.steps, 4),
            "gpu_launches": int(launches), "algorithmic_bytes_per_launch": round(launch_bytes),
            "kernel_ms_avg": round(statistics.mean(kern), 4), "row_bytes": row_bytes,
            "parity_sample_bit_exact": parity, "clocks": clocks,
            "mean_expanded": round(float(trace[:, 2].mean()), 1),
            "mean_distance_evals": round(float(trace[:, 5].mean()), 1)}


def measure_queue_sweep(c, details, bf_words):
    """Plain form at queue sizes 32..256 for k = 10 and k = 100 (recall@k on
    the evaluation queries), and the k = 100 operating point for recall@100
    >= 0.95 (chosen on calibration queries)."""
    torch, song, ds = c.torch, c.song, c.ds
    g = c.g
    stream = c.stream
    pts = []
    for k in (10, 100):
        gtk = c.gt100[:, :k]
        for ef in QUEUE_SWEEP:
            ids_v = (c.d_ids if k == K else c.d_ids100)[:NQ]
            ms = launch_ms(torch, stream, lambda: song.search_device(g, c.dq, NQ, k, ef, ids_v, None,
                                                                     stream=stream))
            rec = float(ds.recall_at_k(ids_v.cpu().numpy(), gtk, k).mean())
            pts.append({"k": k, "ef": ef, "ef_effective": min(max(ef, k), 1024),
                        f"recall@{k}": round(rec, 4), "qps": round(NQ / ms * 1e3)})
    # k = 100: calibration sweep for recall@100 >= target
    gt_cal100, _ = c.gtm.knn(c.base, c.cal, 100)
    cal_pts = []
    for ef in EF_SWEEP_K100:
        ids_v = c.d_ids100[:NCAL]
        ms = launch_ms(torch, stream, lambda: song.search_device(g, c.dcal, NCAL, 100, ef, ids_v, None,
                                                                 stream=stream), reps=3)
        rec = float(ds.recall_at_k(ids_v.cpu().numpy(), gt_cal100, 100).mean())
        cal_pts.append({"ef": ef, "recall_cal": round(rec, 4), "qps": round(NCAL / ms * 1e3)})
        if rec >= TARGET_RECALL + SELECT_MARGIN:
            break
    op, reached = choose(cal_pts)
    ids_v = c.d_ids100[:NQ]
    ms = launch_ms(torch, stream, lambda: song.search_device(g, c.dq, NQ, 100, op["ef"], ids_v, None,
                                                             stream=stream), reps=5)
    rec = float(ds.recall_at_k(ids_v.cpu().numpy(), c.gt100, 100).mean())
    k100 = {"ef": op["ef"], "qps": round(NQ / ms * 1e3), "recall@100": round(rec, 4),
            "reached_on_calibration": reached}
    details["queue_sweep"] = pts
    details["k100_calibration_curve"] = cal_pts
    log(f"[rank {c.rank}] k=100 operating point {k100}")
    return {"points": pts, "k100": k100, "bf_words": bf_words}


def summary_queue(q):
    if q is None:
        return None
    s = {"cols": "ef,qps,recall@k"}
    for k in (10, 100):
        s[f"k{k}"] = [[p["ef"], p["qps"], p[f"recall@{k}"]] for p in q["points"] if p["k"] == k]
    s["k100_at_target"] = [q["k100"]["ef"], q["k100"]["qps"], q["k100"]["recall@100"]]
    return s


def measure_learned(c, details, plain):
    """Learned form: models trained on 50,000 held-out queries; the knobs are
    chosen on calibration queries; then timed, and ablated, on the
    evaluation queries."""
    torch, song, ds, gtm, args = c.torch, c.song, c.ds, c.gtm, c.args
    import ctypes as C
    L = song.load_library()
    g, stream, dev = c.gl, c.stream, c.dev
    ntrain = args.train_queries
    train = draw_queries(ntrain, TRAIN_SEED + c.rank)
    nn1, _ = gtm.knn(c.base, train, 1)
    torch.cuda.empty_cache()
    ids_cal = c.d_ids[:NCAL]
    ids_ev = c.d_ids[:NQ]
    tr_cal = c.d_tr[:NCAL]
    lcurve, reps, blobs, learn_s = [], {}, {}, 0.0
    prec = song.PREC_FP32  # the byte rows (exact for these vectors) are read either way
    fixed = None
    if args.learned_fixed:  # profiling cases: one point, no sweep, no ablation
        f = args.learned_fixed.split(",")
        fixed = (int(f[0]), float(f[3]), int(f[1]), int(f[2]), int(f[4]))
    for tef in (LEARN_EFS[:1] if fixed else LEARN_EFS):
        tl0 = time.time()
        reps[tef] = song.learn(g, torch.from_numpy(train).to(dev), ntrain,
                               torch.from_numpy(np.ascontiguousarray(nn1[:, 0])).to(dev),
                               song.LearnParams(k=K, ef=tef))
        torch.cuda.synchronize()
        learn_s += time.time() - tl0
        blobs[tef] = song.get_model(g)
        # threshold 1.0 (no stop): every beam and Bloom hash count, entry points from
        # the entry model or the entry stage's nearest hubs; learned stop: beams 1, 2
        # and 4 with 2 hashes and the entry model
        points = [fixed] if fixed else [
            (e, t, b, h, en) for e in LEARN_SWEEP_EFS[tef]
            for t in LEARN_THRESHOLDS
            for b in (LEARN_BEAMS if t >= 1.0 else (1, 2, 4))
            for h in (LEARN_BLOOM_HASHES if t >= 1.0 else (2,))
            for en in ((song.ENTRY_MODEL, song.ENTRY_NEAREST) if t >= 1.0 else (song.ENTRY_MODEL,))]
        for lef, thr, beam, nh, ent in points:
            opts = song.SearchOpts(precision=prec, learned=True, stop_threshold=thr, beam=beam,
                                   bloom_hashes=nh, entry=ent)
            song.search_device_ex(g, opts, c.dcal, NCAL, K, lef, ids_cal, None, tr_cal, stream=stream)
            stream.synchronize()
            rec = float(ds.recall_at_k(ids_cal.cpu().numpy(), c.gt_cal, K).mean())
            trl = tr_cal.cpu().numpy()
            ms = launch_ms(torch, stream, lambda: song.search_device_ex(
                g, opts, c.dcal, NCAL, K, lef, ids_cal, None, None, stream=stream))
            lcurve.append({"ef": lef, "trained_ef": tef, "threshold": thr, "beam": beam,
                           "bloom_hashes": nh, "entry": ent, "recall_cal": round(rec, 4),
                           "qps": round(NCAL / ms * 1e3),
                           "mean_expanded": round(float(trl[:, 2].mean()), 1),
                           "learned_stop_rate": round(float((trl[:, 11] == 2).mean()), 3)})
    details["learned_curve"] = lcurve
    details["learn_reports"] = {str(t): {k2: (round(v, 5) if isinstance(v, float) else v)
                                         for k2, v in r.items()} for t, r in reps.items()}
    op, reached = (lcurve[0], True) if fixed else choose(lcurve)
    stop_pts = [p for p in lcurve if p["threshold"] < 1.0]
    nostop_pts = [p for p in lcurve if p["threshold"] >= 1.0 and p["entry"] == song.ENTRY_MODEL]
    log(f"[rank {c.rank}] learned operating point {op}")

    def opts_of(p, entry=None, precision=None):
        return song.SearchOpts(precision=prec if precision is None else precision, learned=True,
                               stop_threshold=p["threshold"], beam=p["beam"],
                               bloom_hashes=p["bloom_hashes"],
                               entry=p["entry"] if entry is None else entry)

    def evaluate(p, entry=None, reps_=5, precision=None):
        """Recall, QPS and trace means of point p on the evaluation queries."""
        song.set_model(g, blobs[p["trained_ef"]])
        o = opts_of(p, entry, precision)
        song.search_device_ex(g, o, c.dq, NQ, K, p["ef"], ids_ev, None, c.d_tr[:NQ], stream=stream)
        stream.synchronize()
        rec = float(ds.recall_at_k(ids_ev.cpu().numpy(), c.gt, K).mean())
        tr = c.d_tr[:NQ].cpu().numpy()
        ms = launch_ms(torch, stream, lambda: song.search_device_ex(
            g, o, c.dq, NQ, K, p["ef"], ids_ev, None, None, stream=stream), reps=reps_)
        return {"ef": p["ef"], "trained_ef": p["trained_ef"], "threshold": p["threshold"],
                "beam": p["beam"], "bloom_hashes": p["bloom_hashes"],
                "entry": p["entry"] if entry is None else entry, "recall_at_10": round(rec, 4),
                "qps": round(NQ / ms * 1e3), "mean_expanded": round(float(tr[:, 2].mean()), 1),
                "learned_stop_rate": round(float((tr[:, 11] == 2).mean()), 3)}, tr

    def ablate(entry):
        """The op point's knobs with another entry choice, ef re-chosen on the
        calibration queries for the same recall target, evaluated."""
        song.set_model(g, blobs[op["trained_ef"]])
        pts = []
        for ef in ABLATION_EFS:
            p = dict(op, ef=ef)
            o = opts_of(p, entry)
            song.search_device_ex(g, o, c.dcal, NCAL, K, ef, ids_cal, None, None, stream=stream)
            stream.synchronize()
            rec = float(ds.recall_at_k(ids_cal.cpu().numpy(), c.gt_cal, K).mean())
            ms = launch_ms(torch, stream, lambda: song.search_device_ex(
                g, o, c.dcal, NCAL, K, ef, ids_cal, None, None, stream=stream), reps=3)
            pts.append(dict(p, recall_cal=round(rec, 4), qps=round(NCAL / ms * 1e3)))
            if rec >= TARGET_RECALL + SELECT_MARGIN:
                break
        best, ok = choose(pts)
        ev, _ = evaluate(best, entry)
        ev["reached_on_calibration"] = ok
        same_ef, _ = evaluate(op, entry, reps_=3)
        return {"at_target": ev, "at_op_ef": {"ef": op["ef"], "recall_at_10": same_ef["recall_at_10"],
                                              "qps": same_ef["qps"]}}

    # the same knobs with each entry choice, each at the queue size that reaches the target
    ablation = {} if fixed else {"entry_model": ablate(song.ENTRY_MODEL),
                                 "nearest_hubs": ablate(song.ENTRY_NEAREST),
                                 "reference_seeds": ablate(song.ENTRY_SEEDS)}
    if stop_pts and nostop_pts and not fixed:
        bs, oks = choose(stop_pts)
        bn, okn = choose(nostop_pts)
        es, _ = evaluate(bs)
        en, _ = evaluate(bn)
        es["reached_on_calibration"], en["reached_on_calibration"] = oks, okn
        ablation["stop_model_on"] = es
        ablation["stop_model_off"] = en
        # the precision form's storage with the learned stop: BF16 rows (exact for
        # these integer vectors) at the stop model's operating point
        song.set_precision(g, song.PREC_BF16)
        eb, _ = evaluate(bs, precision=song.PREC_BF16)
        eb["reached_on_calibration"] = oks
        eb["precision"] = "bf16"
        ablation["bf16_stop_model_on"] = eb
    details["learned_ablation"] = ablation

    # the operating point, timed on the evaluation queries
    song.set_model(g, blobs[op["trained_ef"]])
    lopts = opts_of(op)
    lef = op["ef"]
    total_ms, kern, _ = timed_device(
        torch, c.dist, c.ws, dev, stream, args.steps, args.warmup,
        lambda: song.search_device_ex(g, lopts, c.dq, NQ, K, lef, ids_ev, None, None, stream=stream),
        count=song.launch_count)
    launches = timed_device.last_launches
    ids_l = ids_ev.cpu().numpy()
    song.search_device_ex(g, lopts, c.dq, NQ, K, lef, ids_ev, None, c.d_tr[:NQ], stream=stream)
    stream.synchronize()
    tr = c.d_tr[:NQ].cpu().numpy()
    rep = reps[op["trained_ef"]]
    n_hubs = int(rep.get("n_hubs", 0) or 0)
    # gathered rows + the entry stage's hub tiles (hubs x dim BF16 per 128 queries)
    l_bytes = float(bytes_per_query(tr, K, plain["row_bytes"]).sum()) + \
        (NQ + 127) // 128 * n_hubs * DIM * 2
    e2e = None
    if not args.no_e2e:
        hq = torch.from_numpy(c.queries).pin_memory()
        hids = torch.empty((NQ, K), dtype=torch.int32).pin_memory()
        hdist = torch.empty((NQ, K), dtype=torch.float32).pin_memory()
        timing = song._Timing()
        copts = lopts._c()

        def host_learned():
            st = L.song_gpu_search_ex(g._h, C.byref(copts), C.c_void_p(hq.data_ptr()), NQ, K,
                                      NQ, lef, C.c_void_p(hids.data_ptr()),
                                      C.c_void_p(hdist.data_ptr()), None, C.byref(timing))
            if st != 0:
                raise song.SongError(st, L.song_last_error().decode())

        e2e = c.ws * NQ * args.steps / timed_host(torch, c.dist, c.ws, dev, args.steps, args.warmup,
                                                  host_learned)
        details["learned_e2e_call_ms"] = timed_host.last_calls_ms
        details["learned_e2e_last_timing"] = {f: round(getattr(timing, f), 4) for f in
                                              ("h2d_ms", "kernel_ms", "d2h_ms", "total_ms")}
    details["learned_kernel_ms"] = [round(x, 3) for x in kern]
    entry_name = "learned entry model" if op["entry"] == song.ENTRY_MODEL else "nearest hubs (no model)"
    return {
        "form": f"tensor-core entry stage ({n_hubs} hubs), {entry_name}"
                + (" + learned stop" if op["threshold"] < 1.0 else "") + ", byte rows",
        "kernels": ("entry_kernel + search_kernel<0,-1,1,0,3,0> (no stop model)"
                    if op["threshold"] >= 1.0 else
                    "entry_kernel + search_kernel<0,-1,1,0,2,0> (stop model)"),
        "entry": entry_name,
        "threshold": op["threshold"], "beam": op["beam"], "bloom_hashes": op["bloom_hashes"],
        "bf_words": LEARN_BF_WORDS,
        "ef": lef, "trained_ef": op["trained_ef"], "recall_cal": op["recall_cal"],
        "reached_on_calibration": reached,
        "qps": c.ws * NQ * args.steps / (total_ms / 1e3),
        "e2e_qps": e2e if e2e is not None else c.ws * NQ * args.steps / (total_ms / 1e3),
        "recall_at_10": round(float(ds.recall_at_k(ids_l, c.gt, K).mean()), 4),
        "ms_per_step": round(total_ms / args.steps, 4), "gpu_launches": int(launches),
        "algorithmic_bytes_per_launch": round(l_bytes),
        "kernel_ms_avg": round(statistics.mean(kern), 4),
        "mean_expanded": round(float(tr[:, 2].mean()), 1),
        "learned_stop_rate": round(float((tr[:, 11] == 2).mean()), 3),
        "learn_s": round(learn_s, 2), "train_queries": ntrain, "ablation": ablation,
    }


def summary_plain(p):
    return {"qps": round(p["qps"], 1), "e2e_qps": round(p["e2e_qps"], 1),
            "recall_at_10": p["recall_at_10"], "ef": p["ef"], "bf_words": p["bf_words"],
            "bit_exact_sample": p["parity_sample_bit_exact"],
            "mean_expanded": p["mean_expanded"]}


def summary_learned(l):
    if l is None or "qps" not in l:
        return l
    ab = l.get("ablation", {})

    def short(e, stop=False):
        if e is None:
            return None
        e = e.get("at_target", e)
        out = [e["qps"], e["recall_at_10"], e["ef"]]
        if stop:  # the stop threshold and the share of queries the model stopped
            out += [e["threshold"], e["learned_stop_rate"]]
        return out

    return {"qps": round(l["qps"], 1), "e2e_qps": round(l["e2e_qps"], 1),
            "recall_at_10": l["recall_at_10"], "ef": l["ef"], "beam": l["beam"],
            "bloom_hashes": l["bloom_hashes"], "bf_words": l.get("bf_words"), "stop_threshold": l["threshold"],
            "entry": l["entry"], "learned_stop_rate": l["learned_stop_rate"],
            "mean_expanded": l["mean_expanded"],
            "ablation_cols": "qps,recall,ef[,stop thr,share stopped]",
            "ablation_qps_recall_ef": {
                "entry_model": short(ab.get("entry_model")),
                "nearest_hubs_no_model": short(ab.get("nearest_hubs")),
                "reference_seeds_no_entry_stage": short(ab.get("reference_seeds")),
                "stop_model_on": short(ab.get("stop_model_on"), True),
                "bf16_rows_stop_model_on": short(ab.get("bf16_stop_model_on"), True),
                "stop_model_off": short(ab.get("stop_model_off"))}}


SERVE_KS = (1, 10, 100)
SERVE_EFS = (32, 64, 128, 256)
SERVE_RATES = (5_000, 20_000, 50_000, 100_000, 200_000)


def measure_serving(c, details):
    """Continuous-batching server over the same index: Poisson arrivals at
    several rates, k ~ U{1,10,100}, queue ~ U{32,...,256}; every request uses
    the learned entry/stop (trained here at queue 256, k 10) and falls back to
    the full search when not confident.  Per rate: achieved QPS, p50/p99
    latency (arrival to completion seen by the host), recall@k per k and per
    queue size."""
    torch, song, ds, gtm, args = c.torch, c.song, c.ds, c.gtm, c.args
    g = c.g
    ntrain = min(args.train_queries, 20_000)
    train = draw_queries(ntrain, SEED + 7 * 104729 + c.rank)
    nn1, _ = gtm.knn(c.base, train, 1)
    torch.cuda.empty_cache()
    song.learn(g, torch.from_numpy(train).to(c.dev), ntrain,
               torch.from_numpy(np.ascontiguousarray(nn1[:, 0])).to(c.dev),
               song.LearnParams(k=10, ef=max(SERVE_EFS)))
    rng = np.random.default_rng(SEED + c.rank)
    out = []
    # BF16 rows, the precision form's storage (exact for these integer vectors)
    song.set_precision(g, song.PREC_BF16)
    cfg = song.ServerConfig(max_k=max(SERVE_KS), max_ef=max(SERVE_EFS), stop_threshold=0.85,
                            precision=song.PREC_BF16)
    with song.Server(g, cfg) as srv:
        for rate in SERVE_RATES:
            nreq = int(min(NQ, max(2000, rate * args.serve_seconds)))
            idx = rng.integers(0, NQ, nreq)
            ks = rng.choice(SERVE_KS, nreq).astype(np.int32)
            efs = rng.choice(SERVE_EFS, nreq).astype(np.int32)
            flags = np.full(nreq, song.REQ_LEARNED, np.int32)
            lat, ids, wall = srv.run_poisson(c.queries[idx], ks, efs, flags, float(rate), seed=int(rate))
            rec = {}
            for k in SERVE_KS:
                sel = ks == k
                if sel.any():
                    rec[f"recall@{k}"] = round(float(ds.recall_at_k(ids[sel, :k], c.gt100[idx[sel], :k],
                                                                     k).mean()), 4)
            by_ef = {}
            for ef in SERVE_EFS:  # recall@min(k,10) per queue size: the latency-recall trade
                sel = efs == ef
                if sel.any():
                    kk = np.minimum(ks[sel], 10)
                    r = [float(ds.recall_at_k(ids[sel][kk == k, :k], c.gt100[idx[sel]][kk == k, :k],
                                              k).sum()) for k in np.unique(kk)]
                    by_ef[str(ef)] = {"recall": round(sum(r) / int(sel.sum()), 4),
                                      "p50_ms": round(float(np.percentile(lat[sel], 50)), 3),
                                      "p99_ms": round(float(np.percentile(lat[sel], 99)), 3)}
            out.append({"offered_qps": rate, "requests": nreq,
                        "achieved_qps": round(nreq / wall, 1) if wall > 0 else None,
                        "p50_ms": round(float(np.percentile(lat, 50)), 3),
                        "p99_ms": round(float(np.percentile(lat, 99)), 3),
                        "mean_ms": round(float(lat.mean()), 3), **rec, "by_queue": by_ef})
            log(f"[rank {c.rank}] serving {out[-1]}")
    details["serving"] = out
    return {"form": "BF16 rows, learned entry/stop at threshold 0.85, full search when not confident",
            "k_choices": list(SERVE_KS), "queue_choices": list(SERVE_EFS), "points": out}


def summary_serving(s):
    if s is None:
        return None
    return {"cols": "offered,achieved,p50 ms,p99 ms,recall@10",
            "points": [[p["offered_qps"], round(p["achieved_qps"] or 0), round(p["p50_ms"], 2),
                        round(p["p99_ms"], 2), p.get("recall@10")] for p in s["points"]]}


C3 = {"n": 1_000_000, "dim": 960, "n_comp": 256, "nq": 1000, "seed": 960}
C4 = {"n": 1_183_514, "dim": 200, "n_comp": 512, "nq": 10_000, "ntrain": 50_000, "seed": 200}
C4H = {"n": 290_000, "dim": 256, "n_comp": 256, "nq": 10_000, "bits": 512, "seed": 256}
C3_EFS = (32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024, 1536, 2048, 3072, 4096)
C4_EFS = (32, 48, 64, 96, 128, 192, 256, 320, 384, 512, 768, 1024)
HAM_EFS = (32, 50, 64, 128, 256, 512, 1024)


def measure_extra_configs(c, details, names):
    """The other workloads, each summarised in one entry of the line's
    `configs` (the curves go to the side file)."""
    out = {}
    for name in names:
        name = name.strip().lower()
        t0 = time.time()
        key = {"c3": "c3_precision", "c4": "c4_angular", "c4h": "c4_hamming"}.get(name, name)
        try:
            if name == "c3":
                out[key] = measure_c3(c, details)
            elif name == "c4":
                out[key] = measure_c4(c, details)
            elif name == "c4h":
                out[key] = measure_c4h(c, details)
            elif name:
                out[key] = {"unavailable": "unknown config"}
        except Exception as e:  # one workload failing must not lose the line
            out[key] = {"error": f"{type(e).__name__}: {e}"[:200]}
        log(f"[configs] {name} {time.time() - t0:.1f} s: {out.get(key)}")
        c.torch.cuda.empty_cache()
    return out


def _sweep(c, efs, run, gt, k, nq):
    """Points (ef, recall, qps) of `run(ef)` (which searches the calibration
    queries and returns (ids, ms)) until recall@k reaches the target plus the
    margin."""
    pts = []
    for ef in efs:
        ids, ms = run(ef)
        rec = float(c.ds.recall_at_k(ids, gt, k).mean())
        pts.append({"ef": ef, "recall": round(rec, 4), "qps": round(nq / ms * 1e3)})
        if rec >= TARGET_RECALL + SELECT_MARGIN:
            break
    return pts


def _op(pts):
    ok = [p for p in pts if p["recall"] >= TARGET_RECALL + SELECT_MARGIN]
    return (max(ok, key=lambda p: p["qps"]), True) if ok else (max(pts, key=lambda p: p["recall"]), False)


def measure_c3(c, details):
    """C3, precision form: 1M x 960 non-negative mixture, L1-normalised; BF16
    and per-vector-scaled FP8 rows with FP32 accumulation and an exact FP32
    re-rank of the final results queue, against the plain FP32 form on the
    same graph.  Operating points on 1,000 calibration queries, reported on
    1,000 others; distance error of the returned results against FP64."""
    torch, song, ds = c.torch, c.song, c.ds
    n, dim, nq = c.args.c3_n or C3["n"], C3["dim"], C3["nq"]
    t0 = time.time()
    m = ds.l1_mixture(n, 2 * nq, dim=dim, n_comp=C3["n_comp"], seed=C3["seed"])
    gen_s = time.time() - t0
    t0 = time.time()
    adj = song.build_graph(m.base, song.Params(block_size=32, fixed_degree=31), batch_ratio=32)
    build_s = time.time() - t0
    cal, ev = m.queries[:nq], m.queries[nq:]
    gt_ev, _ = c.gtm.knn(m.base, ev, K)
    gt_cal, _ = c.gtm.knn(m.base, cal, K)
    g = song.KernelGraph(n, dim, m.base, song.Params(pq_size=4096, bf_words=512), adj=adj)
    g.upload_to_gpu()
    dcal, dev_q = torch.from_numpy(cal).to(c.dev), torch.from_numpy(ev).to(c.dev)
    ids_d = torch.empty((nq, K), dtype=torch.int32, device=c.dev)
    dist_d = torch.empty((nq, K), dtype=torch.float32, device=c.dev)
    tr_d = torch.empty((nq, 12), dtype=torch.int32, device=c.dev)
    st = c.stream
    base_t = torch.from_numpy(m.base).to(c.dev)
    res, curves = {}, {}
    for form, prec, rerank in (("fp32_plain", song.PREC_FP32, False), ("bf16_rerank", song.PREC_BF16, True),
                               ("fp8_rerank", song.PREC_FP8, True), ("fp8_no_rerank", song.PREC_FP8, False)):
        if prec != song.PREC_FP32:
            song.set_precision(g, prec)
        opts = song.SearchOpts(precision=prec, rerank=rerank)

        def run(ef, q=dcal):
            ms = launch_ms(torch, st, lambda: song.search_device_ex(g, opts, q, nq, K, ef, ids_d, dist_d,
                                                                     None, stream=st))
            return ids_d.cpu().numpy(), ms

        pts = _sweep(c, C3_EFS, run, gt_cal, K, nq)
        op, ok = _op(pts)
        song.search_device_ex(g, opts, dev_q, nq, K, op["ef"], ids_d, dist_d, tr_d, stream=st)
        st.synchronize()
        ids = ids_d.cpu().numpy()
        tr = tr_d.cpu().numpy()
        d32 = dist_d.clone()
        ms = launch_ms(torch, st, lambda: song.search_device_ex(g, opts, dev_q, nq, K, op["ef"], ids_d,
                                                                 dist_d, None, stream=st), reps=5)
        rec = float(ds.recall_at_k(ids, gt_ev, K).mean())
        # distance error of every returned result against FP64
        valid = torch.from_numpy(ids >= 0).to(c.dev)
        sel = torch.from_numpy(np.maximum(ids, 0).astype(np.int64)).to(c.dev)
        d64 = ((base_t[sel].double() - dev_q[:, None, :].double()) ** 2).sum(-1)
        rel = ((d32.double() - d64).abs() / d64.clamp_min(1e-300))[valid]
        E, X = tr[:, 5].astype(np.float64), tr[:, 2].astype(np.float64)
        s_bytes = {song.PREC_FP32: dim * 4, song.PREC_BF16: dim * 2, song.PREC_FP8: dim + 4}[prec]
        b = E * s_bytes + X * BLOCK_SIZE * 4 + dim * 4 + K * 4
        if rerank:
            b = b + np.minimum(op["ef"], 4096) * dim * 4
        res[form] = {"ef": op["ef"], "reached_on_calibration": ok, "recall_at_10": round(rec, 4),
                     "qps": round(nq / ms * 1e3), "kernel_ms": round(ms, 4),
                     "dist_rel_err_max": float(f"{rel.max().item():.3e}"),
                     "dist_rel_err_mean": float(f"{rel.mean().item():.3e}"),
                     "gather_gbs": round(float(b.sum()) / (ms / 1e3) / 1e9, 1),
                     "mean_expanded": round(float(X.mean()), 1)}
        curves[form] = pts
    g.close()
    del base_t
    details["c3"] = {"forms": res, "curves": curves,
                     "timing_s": {"generate": round(gen_s, 1), "gpu_build": round(build_s, 1)}}
    best = max((v for k2, v in res.items() if k2 in ("bf16_rerank", "fp8_rerank")), key=lambda v: v["qps"])
    return {"n": n, "cols": "ef,recall,qps,max rel err vs fp64",
            **{k2: [v["ef"], v["recall_at_10"], v["qps"], v["dist_rel_err_max"]] for k2, v in res.items()},
            "lowp_rerank_over_fp32": round(best["qps"] / max(res["fp32_plain"]["qps"], 1), 2)}


def measure_c4(c, details):
    """C4, learned form on angular data: 1,183,514 x 200 L2-normalised
    anisotropic mixture; models trained on 50,000 held-out queries; plain and
    learned forms at recall@k >= 0.95 (chosen on calibration queries) for
    k = 10 and 100 (k = 100: the learned entry without the stop model)."""
    torch, song, ds, gtm = c.torch, c.song, c.ds, c.gtm
    n, dim, nq, ntr = c.args.c4_n or C4["n"], C4["dim"], C4["nq"], C4["ntrain"]
    t0 = time.time()
    m = ds.angular_mixture(n, 2 * nq + ntr, dim=dim, n_comp=C4["n_comp"], seed=C4["seed"])
    ev, cal, train = m.queries[:nq], m.queries[nq:2 * nq], m.queries[2 * nq:]
    gen_s = time.time() - t0
    t0 = time.time()
    adj = song.build_graph(m.base, song.Params(block_size=32, fixed_degree=31), batch_ratio=32)
    build_s = time.time() - t0
    gt100, _ = gtm.knn(m.base, ev, 100)
    gt_cal, _ = gtm.knn(m.base, cal, 100)
    nn1, _ = gtm.knn(m.base, train, 1)
    g = song.KernelGraph(n, dim, m.base, song.Params(pq_size=1024, bf_words=512), adj=adj)
    g.upload_to_gpu()
    dev_q, dcal = torch.from_numpy(ev).to(c.dev), torch.from_numpy(cal).to(c.dev)
    st = c.stream
    out, curves = {}, {}
    for k in (10, 100):
        ids_d = torch.empty((nq, k), dtype=torch.int32, device=c.dev)

        def plain(ef, q=dcal):
            ms = launch_ms(torch, st, lambda: song.search_device(g, q, nq, k, ef, ids_d, None, stream=st))
            return ids_d.cpu().numpy(), ms

        pts = _sweep(c, [e for e in C4_EFS if e >= k], plain, gt_cal[:, :k], k, nq)
        op, ok = _op(pts)
        ids, ms = plain(op["ef"], dev_q)
        out[f"plain_k{k}"] = {"ef": op["ef"], "qps": round(nq / ms * 1e3), "reached": ok,
                              "recall": round(float(ds.recall_at_k(ids, gt100[:, :k], k).mean()), 4)}
        curves[f"plain_k{k}"] = pts
    t1 = time.time()
    song.learn(g, torch.from_numpy(train).to(c.dev), ntr,
               torch.from_numpy(np.ascontiguousarray(nn1[:, 0])).to(c.dev),
               song.LearnParams(k=K, ef=128))
    learn_s = time.time() - t1
    for k, thr in ((10, 0.9), (10, 1.0), (100, 1.0)):
        ids_d = torch.empty((nq, k), dtype=torch.int32, device=c.dev)
        best = None
        for beam in (1, 2, 4):
            opts = song.SearchOpts(learned=True, stop_threshold=thr, beam=beam, bloom_hashes=2)

            def learned(ef, q=dcal):
                ms = launch_ms(torch, st, lambda: song.search_device_ex(g, opts, q, nq, k, ef, ids_d, None,
                                                                         None, stream=st))
                return ids_d.cpu().numpy(), ms

            pts = _sweep(c, [e for e in C4_EFS if e >= k], learned, gt_cal[:, :k], k, nq)
            op, ok = _op(pts)
            curves[f"learned_k{k}_thr{thr}_beam{beam}"] = pts
            if ok and (best is None or op["qps"] > best[0]["qps"]):
                best = (op, beam, opts)
        if best is None:
            out[f"learned_k{k}_thr{thr}"] = {"reached": False}
            continue
        op, beam, opts = best
        ms = launch_ms(torch, st, lambda: song.search_device_ex(g, opts, dev_q, nq, k, op["ef"], ids_d, None,
                                                                 None, stream=st), reps=5)
        ids = ids_d.cpu().numpy()
        out[f"learned_k{k}_thr{thr}"] = {"ef": op["ef"], "beam": beam, "qps": round(nq / ms * 1e3),
                                         "recall": round(float(ds.recall_at_k(ids, gt100[:, :k], k).mean()), 4)}
    g.close()
    details["c4"] = {"points": out, "curves": curves,
                     "timing_s": {"generate": round(gen_s, 1), "gpu_build": round(build_s, 1),
                                  "learn": round(learn_s, 1)}}
    return {"n": n, "cols": "ef,qps,recall@k",
            **{k2: [v.get("ef"), v.get("qps"), v.get("recall")] for k2, v in out.items()
               if v.get("qps") is not None}}


def measure_c4h(c, details):
    """C4, Hamming variant: 512-bit sign-random-projection codes (BitHash,
    bitHash.h:17-56, seed 42) of a 290,000 x 256 L2-normalised base; NSW graph
    on the codes (hashKernelGraph.h:196-207); recall@10 against the exact L2
    neighbours of the vectors, as the reference measures it."""
    torch, song, ds, gtm = c.torch, c.song, c.ds, c.gtm
    n, dim, nq, bits = C4H["n"], C4H["dim"], C4H["nq"], C4H["bits"]
    m = ds.angular_mixture(n, nq, dim=dim, n_comp=C4H["n_comp"], seed=C4H["seed"])
    bh = song.BitHash(dim, seed=42, hash_bits=bits)
    codes, qcodes = bh.project_all(m.base), bh.project_all(m.queries)
    t0 = time.time()
    adj = song.build_graph(codes, song.Params(block_size=32, fixed_degree=31), kind=song.KIND_HAMMING,
                           batch_ratio=32)
    build_s = time.time() - t0
    gt, _ = gtm.knn(m.base, m.queries, K)
    g = song.HashKernelGraph(n, codes, song.Params(pq_size=1024, bf_words=512), adj=adj)
    g.upload_to_gpu()
    dq = torch.from_numpy(np.ascontiguousarray(qcodes).view(np.int32)).to(c.dev)
    ids_d = torch.empty((nq, K), dtype=torch.int32, device=c.dev)
    pts = []
    for ef in HAM_EFS:
        ms = launch_ms(torch, c.stream, lambda: song.search_device(g, dq, nq, K, ef, ids_d, None,
                                                                   stream=c.stream), reps=3)
        rec = float(ds.recall_at_k(ids_d.cpu().numpy(), gt, K).mean())
        pts.append({"ef": ef, "recall": round(rec, 4), "qps": round(nq / ms * 1e3)})
    g.close()
    details["c4_hamming"] = {"curve": pts, "gpu_build_s": round(build_s, 1)}
    return {"n": n, "cols": "ef,qps,recall vs exact L2",
            "points": [[p["ef"], p["qps"], p["recall"]] for p in pts]}


def cpu_baseline(base, adj, queries, gt, ef, sample=3000):
    """Reference CPU search (Graph::search) on a bounded sample, all host threads."""
    try:
        import oracle
        r = oracle.ref(block_size=BLOCK_SIZE, bf_words=256, pq_size=512)
    except Exception as e:  # reference not built
        return {"value": None, "unit": "queries/s", "cores": 0, "kind": "reference",
                "sample": f"unavailable: {e}"}
    ds = datasets()
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
            "sample": f"{sample} eval queries, ef={ef}, Graph::search (graph.h:33), "
                      f"oracle/_ref, {threads} threads; recall@10 {rec:.4f}"}


def reference_gpu(base, adj, queries, ef, bf_words, ours):
    """The reference's own GPU kernel (kg_search_kernel via gpu_search, compiled
    for sm_100a), same graph and parameters: QPS and id agreement."""
    try:
        import oracle
        r = oracle.ref(block_size=BLOCK_SIZE, bf_words=bf_words, pq_size=1024)
        if r.gpu is None:
            raise FileNotFoundError("libref_gpu.so not built")
    except Exception as e:
        return {"unavailable": str(e)}
    ids, _tr, timing = r.gpu_search_l2(base, adj, queries, K, ef)  # warm
    ids, _tr, timing = r.gpu_search_l2(base, adj, queries, K, ef)
    return {"qps_total": round(NQ / (timing[4] / 1e3), 1), "kernel_ms": round(timing[2], 3),
            "total_ms": round(timing[4], 3), "ids_identical_to_ours": bool((ids == ours).all()),
            "note": "gpu_search (kernalGraph.h:307) on the same graph: 512-query batches, H2D+kernel+D2H"}


# ------------------------------------------------------------------ reference arm

def cpu_info() -> dict:
    model = None
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in out.splitlines():
            if line.lower().startswith("model name"):
                model = line.split(":", 1)[1].strip()
    except (OSError, subprocess.SubprocessError):
        pass
    return {"model": model, "cores_visible": os.cpu_count(),
            "cores_usable": len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else None}


def exact_knn_cpu(base, queries, k, chunk=512):
    """Exact top-k on the host with FP32 GEMMs (torch on CPU, all threads).
    For integer vectors in [0, 255] of dim 128 every term of
    |q|^2 + |b|^2 - 2 q.b is an integer below 2^24, so the FP32 values are
    exact; ties go to the lower id."""
    import torch
    b = torch.from_numpy(np.ascontiguousarray(base, dtype=np.float32))
    bn = (b * b).sum(1)
    out = np.empty((queries.shape[0], k), np.int32)
    for s in range(0, queries.shape[0], chunk):
        q = torch.from_numpy(np.ascontiguousarray(queries[s:s + chunk], dtype=np.float32))
        d = (q * q).sum(1)[:, None] + bn[None, :] - 2.0 * (q @ b.T)
        v, i = torch.topk(d, k + 8, dim=1, largest=False, sorted=True)
        v, i = v.numpy(), i.numpy()
        for r in range(v.shape[0]):  # (distance, id) order among the candidates
            o = np.lexsort((i[r], v[r]))[:k]
            out[s + r] = i[r][o]
    return out


def run_reference(args, ws, rank, local):
    """--impl reference: the reference's own CPU code on the host cores --
    its graph builder and Graph::search -- and nothing of this library."""
    if rank != 0:
        return None, None
    ds = datasets()
    try:
        import oracle
        r = oracle.ref(block_size=BLOCK_SIZE, bf_words=256, pq_size=512)
    except Exception as e:
        return {"impl": "reference", "unavailable": f"compiled reference not available: {e}"}, None
    base, queries = make_workload(0)
    cal = draw_queries(NCAL, CAL_SEED)
    rp = ref_graph_path()
    t0 = time.time()
    if os.path.exists(rp):
        adj = ds.load_graph(rp)
        build_s = None
    else:
        adj = np.empty((N_BASE, BLOCK_SIZE), np.int32)
        if r.cpu.ref_cpu_build_graph(np.ascontiguousarray(base), N_BASE, DIM, adj) != 0:
            raise RuntimeError("reference build_graph failed")
        build_s = round(time.time() - t0, 1)
        tmp = rp + f".tmp{os.getpid()}"
        ds.save_graph(tmp, adj)
        os.replace(tmp, rp)
    log(f"[reference] graph: build_graph {build_s} s")
    t1 = time.time()
    gt = exact_knn_cpu(base, queries, K)
    rng = np.random.default_rng(1)
    sweep_q = rng.choice(NCAL, 500, replace=False)
    gt_cal = exact_knn_cpu(base, cal[sweep_q], K)
    log(f"[reference] exact kNN on the host {time.time() - t1:.1f} s")
    threads = os.cpu_count() or 1
    if hasattr(os, "sched_getaffinity"):
        threads = len(os.sched_getaffinity(0))
    cg = r.cpu_graph(base, adj)
    ef_op, curve = None, []
    for ef in EF_SWEEP:
        ids, _ = cg.search(cal[sweep_q], K, ef, threads=threads)
        rec = float(ds.recall_at_k(ids, gt_cal, K).mean())
        curve.append({"ef": ef, "recall_cal": round(rec, 4)})
        if rec >= TARGET_RECALL + SELECT_MARGIN:
            ef_op = ef
            break
    if ef_op is None:
        ef_op = EF_SWEEP[-1]
    per_step = args.ref_step_queries
    times = []
    for i in range(args.warmup + args.steps):
        sel = np.arange(i * per_step, (i + 1) * per_step) % NQ
        ts = time.perf_counter()
        cg.search(queries[sel], K, ef_op, threads=threads)
        if i >= args.warmup:
            times.append(time.perf_counter() - ts)
    total = sum(times)
    qps = per_step * args.steps / total
    ids, _ = cg.search(queries[:per_step], K, ef_op, threads=threads)
    rec = float(ds.recall_at_k(ids, gt[:per_step], K).mean())
    # bench_cpu semantics: one thread, per-query latency (bench_cpu.cpp:444-451)
    n1 = args.ref_single_queries
    lat = []
    for i in range(n1):
        ts = time.perf_counter()
        cg.search(queries[i:i + 1], K, ef_op, threads=1)
        lat.append(time.perf_counter() - ts)
    lat = np.array(lat)
    single = {"qps": round(n1 / lat.sum(), 1), "p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 3),
              "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 3), "queries": n1, "ef": ef_op}
    cg.close()
    info = cpu_info()
    out = {
        "metric": "QPS at recall@10>=0.95 (reference CPU search, Graph::search)",
        "value": round(qps, 1), "unit": "queries/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": DATA,
        "config": {"workload": WORKLOAD, "n": N_BASE, "dim": DIM, "k": K, "ef": ef_op,
                   "step": f"{per_step} queries", "graph": "reference build_graph (graph.h:190-199)",
                   "graph_build_s": build_s,
                   "selection": f"smallest ef with recall@10 >= {TARGET_RECALL}+{SELECT_MARGIN} on 500 "
                                f"calibration queries"},
        "impl": "reference",
        "recall_at_10": round(rec, 4),
        "cpu": info,
        "single_thread": single,
        "cpu_baseline": {"value": round(qps, 1), "unit": "queries/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"{per_step} queries per step, Graph::search (graph.h:33) from "
                                   f"oracle/_ref on {threads} threads, ef={ef_op}"},
        "e2e": {"value": round(qps, 1), "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    return out, {"ef_curve": curve, "step_s": [round(t, 4) for t in times]}


# ------------------------------------------------------------------ output

def compact_line(out: dict, limit: int = LINE_LIMIT) -> str:
    """The stdout JSON line: `out` as is when it fits `limit` bytes; else the
    optional per-config summaries are dropped, largest first."""
    line = json.dumps(out, separators=(",", ":"))
    if len(line) <= limit:
        return line
    out = json.loads(line)
    for key in ("configs", "reference_gpu_kernel", "roofline_plain", "forms"):
        sub = out.get(key)
        if isinstance(sub, dict):
            for k2 in sorted(sub, key=lambda s: -len(json.dumps(sub[s]))):
                sub[k2] = "in the details file"
                line = json.dumps(out, separators=(",", ":"))
                if len(line) <= limit:
                    return line
        out.pop(key, None)
        line = json.dumps(out, separators=(",", ":"))
        if len(line) <= limit:
            return line
    return line


def write_details(path: str, details) -> None:
    if not path or details is None:
        return
    try:
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        with open(path, "w") as f:
            json.dump(details, f, indent=1, default=str)
    except OSError as e:
        log(f"details file not written: {e}")


def main(argv=None):
    global N_BASE, NQ, NCAL
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--details", default=os.path.join(ROOT, "gpurun_out", "bench_details.json"),
                    help="side file for curves, sweeps and per-step times ('' = none)")
    ap.add_argument("--graph", choices=("auto", "gpu", "ref"), default="auto",
                    help="auto: the reference arm's graph when present, else the GPU builder")
    ap.add_argument("--ref-step-queries", type=int, default=1000)
    ap.add_argument("--ref-single-queries", type=int, default=200)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned form")
    ap.add_argument("--learned-fixed", default="",
                    help="profiling cases: one learned point EF,BEAM,HASHES,THRESHOLD,ENTRY (no sweep)")
    ap.add_argument("--no-queue-sweep", action="store_true")
    ap.add_argument("--train-queries", type=int, default=50_000)
    ap.add_argument("--no-serving", action="store_true", help="skip the serving measurement")
    ap.add_argument("--serve-seconds", type=float, default=1.0)
    ap.add_argument("--configs", default="c3,c4,c4h",
                    help="extra workloads, comma separated (c3, c4, c4h; '' = none)")
    ap.add_argument("--c3-n", type=int, default=0, help="C3 base size (0 = 1,000,000)")
    ap.add_argument("--c4-n", type=int, default=0, help="C4 base size (0 = 1,183,514)")
    ap.add_argument("--n", type=int, default=N_BASE, help="base size (profiling cases)")
    ap.add_argument("--nq", type=int, default=NQ, help="queries per GPU (profiling cases)")
    ap.add_argument("--ef", type=int, default=0, help="fixed queue size: skip the sweep")
    ap.add_argument("--bf-words", type=int, default=1024, help="Bloom words with --ef")
    args = ap.parse_args(argv)
    N_BASE, NQ = args.n, args.nq
    NCAL = min(NCAL, max(NQ, 1000))
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "gloo" if args.impl == "reference" else "nccl"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            out, details = run_reference(args, ws, rank, local)
        else:
            out, details = run_ours(args, ws, rank, local)
        if rank == 0 and out is not None:
            write_details(args.details, {"line": out, **(details or {})})
            print(compact_line(out), flush=True)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
