"""Multi-process host logic on CPU (gloo, world size 2).

Each rank traces its own Philox stream of the small field with the FP64
oracle (no GPU here), the maps are all-reduced, and rank 0 checks the result
against one process tracing both streams.  This is the sharding/reduction
logic bench.py runs over NCCL on N GPUs.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from onemirror_b200 import dist as D
from onemirror_b200 import workloads as W
from oracle import oracle as O

RAYS = 1 << 14


def trace_item(item):
    w = W.small()
    sc = O.Scene(w.pos, w.size, w.sigma, w.receiver, 10.0, 1.0, list(w.sun.dir))
    xz, helio = O.points_poisson(w.size, int(w.params.rays // 256), 0.3, w.params.seed)
    weight = np.asarray(w.size[:, 0] * w.size[:, 2], np.float64) / np.bincount(helio, minlength=w.n)
    cfg = sc.cfg(w.sun.csr, w.params.seed, int(w.params.rays), 256, xz, helio, weight, threads=1, ray_end=RAYS,
                 item=item)
    r = sc.trace_philox(cfg, records=False)
    return r["counts"].astype(np.int64), r["energy"]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        item = D.shard_item(rank, 0)
        c, e = trace_item(item)
        ct, et = D.reduce_maps(torch.from_numpy(c), torch.from_numpy(e))
        slow = D.max_over_ranks(1.0 + rank)
        if rank == 0:
            out.put((ct.numpy(), et.numpy(), slow))
    finally:
        dist.destroy_process_group()


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_items_are_disjoint_across_ranks_and_steps():
    seen = {D.shard_item(r, s) for r in range(8) for s in range(100)}
    assert len(seen) == 800
    with pytest.raises(ValueError):
        D.shard_item(0, D.ITEMS_PER_RANK)


def test_two_rank_reduction_equals_one_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    counts, energy, slow = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    c0, e0 = trace_item(D.shard_item(0, 0))
    c1, e1 = trace_item(D.shard_item(1, 0))
    assert np.array_equal(counts, c0 + c1)
    assert np.allclose(energy, e0 + e1, rtol=1e-12, atol=1e-12)
    assert slow == 2.0
    assert not np.array_equal(c0, c1)  # the two ranks traced different rays
