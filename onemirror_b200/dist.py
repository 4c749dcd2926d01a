"""Multi-GPU plumbing: one process per GPU, ray streams sharded by rank.

Rays are independent, so N GPUs trace N disjoint Philox streams of the same
field (the stream id is the trace's `item`), and the per-rank flux maps are
summed with one all-reduce -- the only exchange the path has.  Counts are
integers (exact in any order); energies are summed in float64 on the wire so
the result does not depend on the reduction order beyond float64 rounding.
The smoothing of a step (ImageSmoother::image_smooth, image_smooth.cu:60-115)
runs on the summed count map, after the exchange: a trimmed mean of per-rank
maps is not the trimmed mean of their sum.

The adjoint shards one trace by ray ranges instead (adjoint_step): its loss
is a function of the whole flux map, so the ranks sum their energy maps
before the loss and the adjoint map are formed, then sum the gradients of
their backward passes -- two exchanges, and the result of one GPU tracing
every ray.
"""
import torch
import torch.distributed as dist

ITEMS_PER_RANK = 1 << 16


def shard_item(rank, step):
    """Philox stream of `rank` at `step`: disjoint across ranks and steps."""
    if not 0 <= step < ITEMS_PER_RANK - 1:
        raise ValueError("step out of range for the per-rank item space")
    return rank * ITEMS_PER_RANK + 1 + step


def reduce_maps(counts, energy, group=None):
    """Sum count and energy maps over the process group.

    counts: integer tensor; energy: float32/float64 tensor.  Returns NEW
    tensors holding the sums, counts as int64 and energy as float64; the
    inputs are left as they were.  With one rank (or no process group) the
    returned tensors are converted copies of the inputs."""
    c = counts.to(torch.int64, copy=True)
    e = energy.to(torch.float64, copy=True)
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(c, group=group)
        dist.all_reduce(e, group=group)
    return c, e


def step_maps(counts, energy, smooth, group=None):
    """The exchange and smoothing of one step: sum the ranks' maps, then smooth
    the summed count map with `smooth` (a function of an int32 count map).
    Returns (summed counts int64, summed energy float64, smoothed map).  Every
    rank runs the same collectives in the same order and gets the same maps.
    The int64 sums go to the smoother as 32-bit words, which hold the uint32
    count of any pixel below 2^32 rays (the conversion keeps the low 32 bits).
    With one rank nothing is exchanged or converted: the inputs are returned
    with the smoothing of `counts` itself."""
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return counts, energy, smooth(counts)
    c, e = reduce_maps(counts, energy, group)
    return c, e, smooth(c.to(torch.int32))


def shard_range(rank, world, rays, align=256):
    """Rays [begin, end) of `rank` when `world` ranks split one trace of
    `rays` rays: contiguous ranges covering every ray once, cut at multiples
    of `align` rays (one sample point's rays stay on one rank)."""
    blocks = (rays + align - 1) // align
    return min(rays, blocks * rank // world * align), min(rays, blocks * (rank + 1) // world * align)


def adjoint_step(scene, sun, params, target, tape=None, group=None):
    """One gradient evaluation of the flux-map loss, sharded over the process
    group: this rank's forward pass over its ray range, the energy maps
    summed over the ranks, the loss and adjoint map formed from the sum, this
    rank's backward pass and the gradients summed over the ranks.  `scene`
    provides adjoint_forward, tape_energy, adjoint_loss and adjoint_backward
    (onemirror_b200.scene.SolarScene).  Returns (tape, loss, flux, grad_aim,
    grad_tilt), the same on every rank; every rank runs the same three
    all-reduces in the same order.  With one rank (or no process group) it is
    the single-GPU adjoint and nothing is exchanged."""
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    if world > 1 and int(params.rays) < 256 * world:  # the same on every rank: all raise before any exchange
        raise ValueError("a sharded adjoint needs at least 256 rays per rank")
    p = type(params).from_buffer_copy(params)
    if world > 1:
        p.ray_begin, p.ray_end = shard_range(dist.get_rank(group), world, int(params.rays))
    tape, _, _ = scene.adjoint_forward(sun, p, target, want_loss=False, flux=False, tape=tape)
    energy = None
    if world > 1:
        energy = scene.tape_energy(tape)
        dist.all_reduce(energy, group=group)
    loss, flux = scene.adjoint_loss(tape, target, energy=energy, flux=True)
    ga, gt = scene.adjoint_backward(tape)
    if world > 1:
        dist.all_reduce(ga, group=group)
        dist.all_reduce(gt, group=group)
    return tape, loss, flux, ga, gt


def max_over_ranks(value, device=None):
    """Max of a per-rank float (timings are reported as the slowest rank)."""
    if not dist.is_initialized():
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
