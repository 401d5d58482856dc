"""Multi-rank harness of bench.py on CPU: two gloo ranks, as torchrun would
start them.  The solve does not shard (one mesh needs one sparse
factorization), so N GPUs run N replicas; what crosses ranks is only the
timing and unit count: the slowest rank's time and the element-iterations
of all replicas."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench
    from wrapd_b200 import bars

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bar = bars.bar_8x8x32(seed=rank)   # each replica its own seeded bar, as bench.py builds them
        bench.barrier(dist)
        ms = bench.max_over_ranks(dist, 10.0 + rank)          # rank r "took" 10 + r ms
        units = bench.sum_over_ranks(dist, float(bar.n_tets * (3 + rank)))
        out[rank] = (ms, units, bar.n_tets, float(np.abs(bar.init).sum()))
        bench.barrier(dist)
    finally:
        dist.destroy_process_group()


def test_two_replicas_reduce_time_and_units():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    (ms0, u0, ne0, g0), (ms1, u1, ne1, g1) = res[0], res[1]
    # every rank sees the slowest rank's time and the units of all replicas
    assert ms0 == ms1 == 11.0
    assert ne0 == ne1 == 12288
    assert u0 == u1 == 12288 * 3 + 12288 * 4
    # the replicas are different meshes of the same size (seed = rank)
    assert g0 != g1


def test_single_process_needs_no_group():
    import bench
    assert bench.max_over_ranks(None, 3.5) == 3.5
    assert bench.sum_over_ranks(None, 7.0) == 7.0
    bench.barrier(None)
