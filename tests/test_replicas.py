"""Replica logic of the multi-GPU bench on CPU: two gloo ranks (world size 2).

Each rank draws its own queries over the same base, the maximum-over-ranks
reduction picks the slowest rank, and the aggregate counts every rank's
queries over that time."""
import importlib
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, port, outdir):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE="2", LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=2)
    rep = importlib.import_module("2020_song_ex_b200.replicas")
    ds = importlib.import_module("2020_song_ex_b200.datasets")
    ws, r, _ = rep.env()
    m = ds.int_mixture(500, 20, dim=16, n_comp=4, seed=9, query_seed=rep.query_seed(9, r))
    mx = rep.max_over_ranks(1.0 + r)  # rank 1 is the slower one
    np.savez(os.path.join(outdir, f"r{r}.npz"), base=m.base, q=m.queries, mx=mx, ws=ws,
             agg=rep.aggregate_qps(ws, 20, 3, mx))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(port, str(tmp_path)), nprocs=2, start_method="spawn",
                       join=True)
    a, b = (np.load(tmp_path / f"r{i}.npz") for i in (0, 1))
    np.testing.assert_array_equal(a["base"], b["base"])           # same replica
    assert not np.array_equal(a["q"], b["q"])                      # own queries per rank
    assert float(a["mx"]) == float(b["mx"]) == 2.0                 # max over ranks
    assert int(a["ws"]) == 2 and float(a["agg"]) == pytest.approx(2 * 20 * 3 / 2.0)
