"""Host-side logic of multi-GPU runs: replicas, one process per GPU.

The path has no exchange step: every rank holds the whole compressed index
(it fits one B200 many times over) and answers its own queries, so there is no
data-path collective. The process group is used only to line the ranks up
around the timed region and to combine results for checking:

- `shard_queries` gives a rank its contiguous block of a query stream;
- `max_over_ranks` is the job time (the slowest rank), `sum_over_ranks`
  the job's total work;
- `combine_checksums` merges per-rank checksum triples into the triple of
  the whole stream (counts add, the docID fingerprint XORs), so a sharded
  run can be checked against a single-GPU run of the same queries.
"""
from __future__ import annotations

import numpy as np


def shard_queries(terms, term_offsets, rank: int, world: int):
    """Queries [q0, q1) of rank `rank` out of `world`, as (terms, offsets, q0, q1)
    with offsets rebased to 0."""
    toff = np.asarray(term_offsets)
    nq = len(toff) - 1
    q0 = nq * rank // world
    q1 = nq * (rank + 1) // world
    t = np.asarray(terms)[int(toff[q0]):int(toff[q1])]
    o = (toff[q0:q1 + 1] - toff[q0]).astype(toff.dtype)
    return t, o, q0, q1


def max_over_ranks(value: float, group=None, device=None) -> float:
    """The largest `value` over the ranks of the default (or given) group."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t[0])


def sum_over_ranks(value: float, group=None, device=None) -> float:
    """The sum of `value` over the ranks of the default (or given) group."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t[0])


def combine_checksums(triples) -> tuple[int, int, int]:
    """Merge excl_checksum triples of disjoint query shards."""
    c0 = c1 = c2 = 0
    for a, b, c in triples:
        c0 += int(a)
        c1 += int(b)
        c2 ^= int(c)
    return c0, c1, c2


def gather_checksums(triple, group=None) -> tuple[int, int, int]:
    """All ranks' checksum triples combined (every rank gets the result)."""
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return tuple(int(x) for x in triple)
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, tuple(int(x) for x in triple), group=group)
    return combine_checksums(out)
