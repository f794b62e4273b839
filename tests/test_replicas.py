"""Multi-rank path (replicas only), on CPU with the gloo backend: every rank
builds its own operator plan, the ranks agree on the slowest time, and the
job throughput counts every replica's points."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from defmm_b200 import IBFMM_Mat, replicas, workloads as W


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = W.cube_surface(4000, seed=3)
        A = IBFMM_Mat()
        A.addSourceParticles(w.points)
        A.addTargetParticles(w.points)
        A.prcmpt(4, 32, 2 * np.pi * 4)
        q = W.charges(w.n, replicas.replica_seed(rank))
        fake_seconds = 0.5 + rank  # per-rank time of the timed region
        dist.barrier()
        tmax = replicas.max_over_ranks(fake_seconds, dist)
        cells = A.info("cells_T")
        out[rank] = (tmax, cells, float(np.abs(q).sum()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_run_independent_replicas():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    # both ranks see the slowest rank's time; same plan; different charges
    assert res[0][0] == res[1][0] == 1.5
    assert res[0][1] == res[1][1]
    assert res[0][2] != res[1][2]
    assert replicas.job_throughput(4000, world, res[0][0]) == pytest.approx(2 * 4000 / 1.5)


def test_single_process_max_is_identity():
    assert replicas.max_over_ranks(3.25) == 3.25
