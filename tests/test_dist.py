"""Multi-process host logic on CPU (gloo, world size 2).

Each rank traces its own Philox stream of the small field with the FP64
oracle (no GPU here), the maps are all-reduced, and rank 0 checks the result
against one process tracing both streams.  This is the sharding/reduction
logic bench.py runs over NCCL on N GPUs, and its step composition: the
exchange first, then the trimmed-mean smoothing of the summed count map
(dist.step_maps, with the oracle's smoother standing in for the GPU's).
The sharded adjoint (dist.adjoint_step) runs on two and three ranks with a
CPU stand-in for the scene's adjoint calls, against one process.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from onemirror_b200 import capi
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


class ToyAdjoint:
    """CPU stand-in for SolarScene's adjoint calls, with the same signatures:
    ray i of a trace of R rays deposits c_i + d_i . theta[h_i] into pixel p_i
    (theta: 4 parameters per heliostat), flux = s x energy, and the loss
    L = sum (flux - T)^2 with its exact gradient.  A tape is a dict."""

    def __init__(self, n=40, res=64, rays=(1 << 12) + 77, seed=3):
        rng = np.random.default_rng(seed)
        self.n, self.res, self.s = n, res, 0.5
        self.h = rng.integers(0, n, rays)
        self.p = rng.integers(0, res, rays)
        self.c = rng.random(rays)
        self.d = rng.normal(size=(rays, 4))
        self.theta = rng.normal(size=(n, 4))

    def adjoint_forward(self, sun, params, target, want_loss=True, flux=True, tape=None):
        b, e = (params.ray_begin, params.ray_end) if params.ray_end else (0, params.rays)
        energy = np.zeros(self.res)
        np.add.at(energy, self.p[b:e], self.c[b:e] + (self.d[b:e] * self.theta[self.h[b:e]]).sum(1))
        return {"range": (b, e), "energy": torch.from_numpy(energy)}, None, None

    def tape_energy(self, tape):
        return tape["energy"].clone()

    def adjoint_loss(self, tape, target, energy=None, want_loss=True, flux=False):
        if energy is not None:
            tape["energy"] = energy.clone()
        f = self.s * tape["energy"]
        tape["G"] = 2 * (f - target) * self.s
        return float(((f - target) ** 2).sum()), f

    def adjoint_backward(self, tape):
        b, e = tape["range"]
        g = np.zeros((self.n, 4))
        np.add.at(g, self.h[b:e], tape["G"].numpy()[self.p[b:e], None] * self.d[b:e])
        g = torch.from_numpy(g)
        return g[:, :2].contiguous(), g[:, 2:].contiguous()


def toy_params(rays):
    p = capi.TraceParams()
    p.rays = rays
    p.rays_per_point = 256
    return p


def _adjoint_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        toy = ToyAdjoint()
        target = torch.full((toy.res,), 1.5, dtype=torch.float64)
        params = toy_params(len(toy.h))
        tape, loss, flux, ga, gt = D.adjoint_step(toy, None, params, target)
        # what a rank would get without the energy exchange: the loss of its own partial map
        own, _ = toy.adjoint_loss(toy.adjoint_forward(None, _ranged(params, rank, world), target)[0], target)
        out.put((rank, tape["range"], loss, flux.numpy(), ga.numpy(), gt.numpy(), own, params.ray_end))
    except BaseException as ex:  # report instead of leaving the parent waiting
        out.put((rank, "error: %r" % (ex,)))
        raise
    finally:
        dist.destroy_process_group()


def _ranged(params, rank, world):
    p = type(params).from_buffer_copy(params)
    p.ray_begin, p.ray_end = D.shard_range(rank, world, int(params.rays))
    return p


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_adjoint_equals_one_process(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_adjoint_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in procs], key=lambda r: r[0])
    assert all(len(r) > 2 for r in res), res
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    toy = ToyAdjoint()
    target = torch.full((toy.res,), 1.5, dtype=torch.float64)
    params = toy_params(len(toy.h))
    _, loss, flux, ga, gt = D.adjoint_step(toy, None, params, target)  # one process, every ray
    ranges = [r[1] for r in res]
    assert ranges[0][0] == 0 and ranges[-1][1] == len(toy.h)
    assert all(ranges[k][1] == ranges[k + 1][0] for k in range(world - 1))
    assert all(b % 256 == 0 for b, _ in ranges)
    for rank, rng, l, f, a, t, own, caller_end in res:
        assert caller_end == 0  # the caller's parameters are left as they were
        assert abs(l - loss) <= 1e-12 * loss
        assert np.allclose(f, flux.numpy(), rtol=1e-12, atol=0)
        assert np.allclose(a, ga.numpy(), rtol=1e-10, atol=1e-12 * np.abs(ga.numpy()).max())
        assert np.allclose(t, gt.numpy(), rtol=1e-10, atol=1e-12 * np.abs(gt.numpy()).max())
        assert abs(own - loss) > 1e-3 * loss  # a rank's own partial map gives another loss


def test_shard_ranges_cover_every_ray_once():
    for rays in (256, 1000, (1 << 20) + 77):
        for world in (1, 2, 3, 8):
            if rays < 256 * world:
                continue
            rs = [D.shard_range(r, world, rays) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == rays
            assert all(rs[k][1] == rs[k + 1][0] and rs[k][0] < rs[k][1] for k in range(world - 1))
