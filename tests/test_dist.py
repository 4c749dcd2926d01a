"""Multi-process host logic on CPU (gloo, world size 2).

Each rank traces its own Philox stream of the small field with the FP64
oracle (no GPU here), the maps are all-reduced, and rank 0 checks the result
against one process tracing both streams.  This is the sharding/reduction
logic bench.py runs over NCCL on N GPUs, and its step composition: the
exchange first, then the trimmed-mean smoothing of the summed count map
(dist.step_maps, with the oracle's smoother standing in for the GPU's).
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


def oracle_smooth(counts):
    """The bench's smoothing (5x5 window, 20 % trimmed at each end, exact order
    statistics) by the oracle, on an int32 tensor of uint32 counts."""
    m = counts.numpy().astype(np.int32).view(np.uint32).reshape(W.small().res)
    return torch.from_numpy(O.smooth_u32(np.ascontiguousarray(m), 2, 0.2, 0))


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        item = D.shard_item(rank, 0)
        c, e = trace_item(item)
        tc, te = torch.from_numpy(c), torch.from_numpy(e)
        ct, et = D.reduce_maps(tc, te)
        untouched = np.array_equal(tc.numpy(), c) and np.array_equal(te.numpy(), e)
        # the bench step: exchange, then smooth the summed map
        sc, se, sm = D.step_maps(torch.from_numpy(c.astype(np.int32)), te, oracle_smooth)
        slow = D.max_over_ranks(1.0 + rank)
        out.put((rank, ct.numpy(), et.numpy(), slow, untouched, sc.numpy(), se.numpy(), sm.numpy()))
    except BaseException as ex:  # report instead of leaving the parent waiting
        out.put((rank, "error: %r" % (ex,)))
        raise
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
    res = sorted([q.get(timeout=300) for _ in procs], key=lambda r: r[0])
    assert all(len(r) > 2 for r in res), res
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    c0, e0 = trace_item(D.shard_item(0, 0))
    c1, e1 = trace_item(D.shard_item(1, 0))
    assert not np.array_equal(c0, c1)  # the two ranks traced different rays
    one = oracle_smooth(torch.from_numpy((c0 + c1).astype(np.int32))).numpy()
    for rank, counts, energy, slow, untouched, sc, se, sm in res:
        assert np.array_equal(counts, c0 + c1)
        assert np.allclose(energy, e0 + e1, rtol=1e-12, atol=1e-12)
        assert slow == 2.0
        assert untouched  # reduce_maps returns new tensors
        # step order: the smoothed map is the one process's smoothing of the sum
        assert np.array_equal(sc, c0 + c1) and np.allclose(se, e0 + e1, rtol=1e-12, atol=1e-12)
        assert sm.tobytes() == one.tobytes()
    # smoothing each rank's map and summing would give another map
    per_rank = oracle_smooth(torch.from_numpy(c0.astype(np.int32))).numpy() + \
        oracle_smooth(torch.from_numpy(c1.astype(np.int32))).numpy()
    assert not np.array_equal(per_rank, one)


def test_single_process_step_smooths_its_own_map():
    c, e = trace_item(D.shard_item(0, 0))
    tc = torch.from_numpy(c.astype(np.int32))
    sc, se, sm = D.step_maps(tc, torch.from_numpy(e), oracle_smooth)
    assert sc is tc and sm.numpy().tobytes() == oracle_smooth(tc).numpy().tobytes()
