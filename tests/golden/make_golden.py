"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the UNMODIFIED reference -- its NSW builders (kernalGraph.h:140-149,
hashKernelGraph.h:196-207), its BitHash (bitHash.h:17-56) and its GPU search
``gpu_search`` with ``kg_search_kernel`` / ``hkg_search_kernel``
(kernalGraph.h:307-382, hashKernelGraph.h:360-435) -- compiled from the
reference sources by ``oracle/build_ref.py`` for each config.h variant, on
seeded synthetic inputs.  Needs a CUDA GPU (the reference search is a GPU
kernel) and the built ``oracle/_ref`` libraries.

Each fixture ``<case>.npz`` holds the inputs (base vectors or codes, graph,
queries), the parameters, and the reference outputs: ``ids`` [nq, k]
best-first and ``trace`` [nq, 12] (QueryTrace).  The reference CPU search
``Graph::search`` (graph.h:33-115) ids are stored too (``cpu_ids``, as
returned: worst-first) for the relation tests.

Usage (on a GPU host):  python tests/golden/make_golden.py --out DIR
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

ds = importlib.import_module("2020_song_ex_b200.datasets")


def _ties_data(n, nq, dim, distinct, seed):
    """Integer data built from few distinct rows, so many distances tie."""
    rng = np.random.default_rng(seed)
    rows = np.rint(rng.uniform(0, 255, size=(distinct, dim))).astype(np.float32)
    base = rows[rng.integers(0, distinct, size=n)]
    queries = np.rint(rng.uniform(0, 255, size=(nq, dim))).astype(np.float32)
    return base, queries


CASES = {
    # C1 shape scaled down: degree 16, 1,024-bit Bloom filter, queue 64.
    "c1_small": dict(kind="l2", data=("int", 2000, 100, 128, 16, 11), bs=16, bfw=16, pq=512,
                     k=10, ef=64),
    # reference defaults (pq_size 50, 16,384-bit filter), ef defaults to pq_size.
    "ref_defaults": dict(kind="l2", data=("int", 2000, 100, 128, 16, 12), bs=32, bfw=256, pq=50,
                         k=10, ef=50),
    # non-integer FP32 data: checks the warp_l2 FMA/tree order bit for bit.
    "float_angular": dict(kind="l2", data=("angular", 1500, 100, 40, 12, 13), bs=32, bfw=256,
                          pq=512, k=10, ef=64),
    "float_l1_d100": dict(kind="l2", data=("l1", 1200, 80, 100, 12, 14), bs=32, bfw=256,
                          pq=512, k=10, ef=96),
    # Hamming on 512-bit sign-random-projection codes.
    "hamming512": dict(kind="hamming", data=("angular", 2000, 100, 64, 12, 15), bs=32, bfw=256,
                       pq=512, hb=512, k=10, ef=64),
    # ef clamp: k above ef, and k above pq_size (ef = pq_size, -1 padding).
    "clamp_k20": dict(kind="l2", data=("int", 1000, 60, 64, 8, 16), bs=32, bfw=256, pq=50,
                      k=20, ef=10),
    "clamp_k60": dict(kind="l2", data=("int", 1000, 60, 64, 8, 16), bs=32, bfw=256, pq=50,
                      k=60, ef=10),
    # many exact distance ties: tie order is decided by the slot arrays.
    "ties": dict(kind="l2", data=("ties", 1500, 80, 32, 60, 17), bs=32, bfw=256, pq=512,
                 k=10, ef=48),
    # fewer nodes than entry points: duplicated seeds p*n/4.
    "tiny_n3": dict(kind="l2", data=("int", 3, 5, 8, 2, 18), bs=32, bfw=256, pq=512, k=5,
                    ef=8),
}


def make_inputs(spec):
    kind, n, nq, dim, comp, seed = spec
    if kind == "int":
        m = ds.int_mixture(n, nq, dim=dim, n_comp=comp, seed=seed)
        return m.base, m.queries
    if kind == "angular":
        m = ds.angular_mixture(n, nq, dim=dim, n_comp=comp, seed=seed)
        return m.base, m.queries
    if kind == "l1":
        m = ds.l1_mixture(n, nq, dim=dim, n_comp=comp, seed=seed)
        return m.base, m.queries
    if kind == "ties":
        return _ties_data(n, nq, dim, comp, seed)
    raise ValueError(kind)


def make_case(name, c):
    base, queries = make_inputs(c["data"])
    r = oracle.ref(block_size=c["bs"], bf_words=c["bfw"], pq_size=c["pq"],
                   hash_bits=c.get("hb", 256))
    out = dict(name=name, kind=c["kind"], block_size=c["bs"], bf_words=c["bfw"],
               pq_size=c["pq"], k=c["k"], ef=c["ef"], bf_nhash=4, n_multiprobe=4)
    if c["kind"] == "l2":
        adj = r.build_graph(base)
        ids, trace, timing = r.gpu_search_l2(base, adj, queries, c["k"], c["ef"])
        cpu_ids, _ = r.cpu_graph(base, adj).search(queries, c["k"], c["ef"])
        arrays = dict(adj=adj, ids=ids, trace=trace, cpu_ids=cpu_ids, queries=queries)
        if c["data"][0] in ("int", "ties"):
            arrays["base_u8"] = base.astype(np.uint8)
        else:
            arrays["base"] = base
    else:
        adj, codes = r.build_hashed_graph(base)
        qcodes, _R = r.bithash_project(queries)
        ids, trace, timing = r.gpu_search_hamming(codes, adj, qcodes, c["k"], c["ef"])
        arrays = dict(adj=adj, ids=ids, trace=trace, codes=codes, qcodes=qcodes,
                      raw_base=base, raw_queries=queries)
    out["ef_effective"] = int(timing[5])
    return out, arrays


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--only", nargs="*")
    a = ap.parse_args(argv)
    os.makedirs(a.out, exist_ok=True)
    for name, c in CASES.items():
        if a.only and name not in a.only:
            continue
        meta, arrays = make_case(name, c)
        np.savez_compressed(os.path.join(a.out, f"{name}.npz"), meta=json.dumps(meta), **arrays)
        print(name, {k: v.shape for k, v in arrays.items()}, "ef_effective", meta["ef_effective"])
    return 0


if __name__ == "__main__":
    sys.exit(main())
