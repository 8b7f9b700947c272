"""Multi-process host logic of bench.py on CPU: two gloo ranks go through
the same process-group set-up, barrier and max-over-ranks timing that the
NCCL run uses, get their own weak-scaling share of nets, and the reference
arm does its work on rank 0 only."""
import os
import socket
import sys
import types

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    args = types.SimpleNamespace(impl="reference", gpus=world, steps=1, warmup=0)
    w, r, _ = bench.dist_setup(args)
    try:
        bench.barrier(w)
        mx = bench.max_over_ranks(w, 0.5 + r)
        ns = bench.rank_nets(r, 1000, 2, 4096)
        if r != 0:
            bench.run_reference(args, w, r)  # returns at once: rank 0 alone works
        q.put((r, w, mx, int(ns[-1]), len(ns), dist.get_backend()))
        bench.barrier(w)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [x[0] for x in res] == [0, 1]
    assert all(x[1] == world and x[5] == "gloo" for x in res)
    assert all(x[2] == 1.5 for x in res)                  # max over ranks
    assert res[0][4] == res[1][4] == 1001                 # same net count per rank
    assert res[0][3] != res[1][3]                         # but its own nets
    assert np.isfinite([x[2] for x in res]).all()
