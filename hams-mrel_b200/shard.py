"""Frequency sharding across ranks (one process per GPU).

Frequencies are independent, so a deck's frequency list is cut into
contiguous blocks, one per rank; each rank solves its block with its own
context, and the per-frequency results (added mass, damping, excitation --
a few tens of KB per frequency) are gathered on rank 0 in frequency order.
There is no collective on the data path; the only exchanges are this final
gather and the max-over-ranks of timings.
"""
import numpy as np


def block(n, rank, world):
    """Indices [lo, hi) of rank's contiguous share of n items (the first n % world ranks get one more)."""
    q, r = divmod(n, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def gather_results(local, lo, dist=None, n=None):
    """Rank 0 receives every rank's (lo, results) and returns the full list in frequency order; the
    other ranks return None.  `local` is a list of per-frequency tuples of arrays."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return list(local)
    world = dist.get_world_size()
    parts = [None] * world if dist.get_rank() == 0 else None
    dist.gather_object((lo, [tuple(np.asarray(a) for a in r) for r in local]), parts, dst=0)
    if dist.get_rank() != 0:
        return None
    out = []
    for lo_k, res in sorted(parts, key=lambda t: t[0]):
        out.extend(res)
    if n is not None and len(out) != n:
        raise RuntimeError(f"gathered {len(out)} frequencies, expected {n}")
    return out


def max_over_ranks(x, dist=None, device=None):
    """The largest value of x over all ranks (timings are reported as the slowest rank)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
