"""Multi-process replica plumbing of bench.py on CPU (gloo, world size 2).

On N GPUs every rank solves its own seeded batch (weak scaling, no
collective on the data path); only the timing is reduced: the job time is
the max over ranks and the work the sum.  This runs those pieces in two
gloo processes.
"""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys

    import numpy as np
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from shearwave_b200 import workloads as W

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        probs = W.batch_c3(seed=rank, n=3, shrink=0.25)  # this rank's replica batch
        cells = sum(W.cell_steps(p) for p in probs)
        t = 1.0 + rank  # a per-rank "elapsed time"
        tmax = bench.reduce_scalar(t, "max", "cpu", world)
        total = bench.reduce_scalar(cells, "sum", "cpu", world)
        fp = float(np.sum(probs[0]["mu"][:4, :4, :4]))
        out[rank] = (tmax, total, cells, fp)
    finally:
        dist.destroy_process_group()


def test_replica_reductions_two_ranks():
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    r0, r1 = out[0], out[1]
    assert r0[0] == r1[0] == 2.0                # max of the per-rank times
    assert r0[1] == r1[1] == r0[2] + r1[2]      # total work = sum of replica work
    assert r0[3] != r1[3]                       # ranks solve different seeded problems


def test_single_rank_reduction_is_identity():
    import bench

    assert bench.reduce_scalar(3.5, "max", "cpu", 1) == 3.5
    with pytest.raises(Exception):
        bench.reduce_scalar(1.0, "max", "cpu", 2)  # no process group
