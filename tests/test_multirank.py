"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (one process
each, as torchrun starts them) shard the batched-acceleration workload into
independent batches (weak scaling, no data-path collective) and agree on the
max-over-ranks time and the summed work through the process group."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    w, r, local, pg = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank) and pg is not None
    # each rank's shard: the bench derives its cells from seed + 1000 * rank
    mesh, offs, gids, data, B, dt = bench.workload(8, 2026 + 1000 * rank)
    t = 1.0 + rank  # a per-rank "time"
    out[rank] = (float(gids.astype(np.float64).sum()), bench.allreduce_max(pg, t),
                 bench.allreduce_sum(pg, float(offs[-1])), float(offs[-1]))
    pg.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:  # no fork of a process that holds CUDA
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] != res[1][0]                      # different cells on each rank
    assert res[0][1] == res[1][1] == pytest.approx(2.0)  # max over ranks
    assert res[0][2] == res[1][2] == pytest.approx(res[0][3] + res[1][3])  # whole-job work
