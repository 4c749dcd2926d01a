"""Multi-GPU plumbing: one process per GPU, ray streams sharded by rank.

Rays are independent, so N GPUs trace N disjoint Philox streams of the same
field (the stream id is the trace's `item`), and the per-rank flux maps are
summed with one all-reduce -- the only exchange the path has.  Counts are
integers (exact in any order); energies are summed in float64 on the wire so
the result does not depend on the reduction order beyond float64 rounding.
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
    """Sum count and energy maps over the process group, in place.

    counts: int32/int64 tensor; energy: float32/float64 tensor.  Returns the
    reduced tensors (energy as float64)."""
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return counts, energy.double()
    c = counts.to(torch.int64)
    e = energy.to(torch.float64)
    dist.all_reduce(c, group=group)
    dist.all_reduce(e, group=group)
    return c, e


def max_over_ranks(value, device=None):
    """Max of a per-rank float (timings are reported as the slowest rank)."""
    if not dist.is_initialized():
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
