"""The multi-GPU bench path's host logic on CPU ranks (gloo, world size 2).

Each rank is an independent replica (weak scaling): it samples the same
workload from its own Philox key (bench.replica_seed) into its own buffer,
and the whole-job figures are the per-dimension ESS summed over all ranks'
chains and the maximum device time over ranks (bench.reduce_over_ranks).
Here the CPU oracle stands in for the GPU sampler on each rank.
"""
import datetime
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import oracle.oracle as O
        from naja_b200 import synth

        A, b, x0 = synth.simplex(5)
        S = O.chr_run(A, b, x0, 120, 3, 2, seed=bench.replica_seed(7, rank), precision="fp64")
        ess = O.ess(S.astype(np.float32), 2, layout=1)
        per_dim, ms = bench.reduce_over_ranks(ess.sum(axis=1), 10.0 + rank, world, torch.device("cpu"))
        q.put((rank, ess.sum(axis=1), per_dim, ms, S))
    finally:
        dist.destroy_process_group()


def test_replicas_and_reductions_two_ranks():
    import torch.multiprocessing as mp

    import bench
    import oracle.oracle as O
    from naja_b200 import synth

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        r, own, per_dim, ms, S = q.get(timeout=120)
        got[r] = (own, per_dim, ms, S)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # sums over ranks, max time over ranks, identical on both ranks
    total = got[0][0] + got[1][0]
    for r in range(2):
        assert np.allclose(got[r][1], total)
        assert got[r][2] == 11.0
    # independent streams per replica, each reproducible alone
    assert not np.array_equal(got[0][3], got[1][3])
    A, b, x0 = synth.simplex(5)
    alone = O.chr_run(A, b, x0, 120, 3, 2, seed=bench.replica_seed(7, 1), precision="fp64")
    assert np.array_equal(alone, got[1][3])
    assert bench.replica_seed(7, 0) == 7


def test_single_rank_reduction_is_identity():
    import bench

    per_dim, ms = bench.reduce_over_ranks(np.array([3.0, 4.0]), 5.0, 1, None)
    assert per_dim.tolist() == [3.0, 4.0] and ms == 5.0
