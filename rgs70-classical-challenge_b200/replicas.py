"""Replica parallelism over GPUs (one process per GPU): the scan state does not shard
(every position gathers through an arbitrary GF(2) map), but bitstrings, samples and
instances are independent, so N GPUs run N replicas on disjoint work with no data-path
collective.  The only collectives are a timing reduction (max over ranks) and an
optional gather of results.

Work split: contiguous shards of a global index range (bitstrings, instances) or
independent seed streams per rank (samples), spawned from one base seed the way the
reference's production manifests spawn per-group PCG64 streams
(``W/production_seed_manifest.json``, ``W/born_production.py:20-23``).
Works with the ``nccl`` backend on GPUs and with ``gloo`` on CPU (the tests).
"""
import numpy as np
import torch
import torch.distributed as dist

__all__ = ["world", "shard", "rank_seeds", "max_over_ranks", "gather"]


def world():
    """(rank, world size) of the default process group, or (0, 1) without one."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard(count, rank, size):
    """[first, last) of rank's contiguous share of ``count`` items (sizes differ by <= 1)."""
    if not (0 <= rank < size):
        raise ValueError("rank out of range")
    base, extra = divmod(int(count), int(size))
    first = rank * base + min(rank, extra)
    return first, first + base + (1 if rank < extra else 0)


def rank_seeds(base_seed, size):
    """One independent 64-bit seed per rank, spawned from ``base_seed`` (SeedSequence)."""
    children = np.random.SeedSequence(int(base_seed)).spawn(int(size))
    return [int(c.generate_state(1, dtype=np.uint64)[0]) for c in children]


def max_over_ranks(x, device=None):
    """Maximum of a per-rank float over all ranks (the job's time is its slowest rank)."""
    r, n = world()
    if n == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather(obj):
    """List of every rank's ``obj`` (picklable), in rank order."""
    r, n = world()
    if n == 1:
        return [obj]
    out = [None] * n
    dist.all_gather_object(out, obj)
    return out
