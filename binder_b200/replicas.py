"""Replica parallelism for independent registrations and Gibbs chains.

One volume's registration has no exchange step worth a collective: sharding it would need a
halo exchange for the E-step, a K x L histogram all-reduce and a transpose per DCT axis every
iteration.  The units that do parallelise are whole image pairs and whole chains, so several
GPUs run independent replicas.  Each rank takes a static block of the work list, runs it alone
on its own GPU, and the only collectives are host-side bookkeeping after the work: the max of
the ranks' elapsed times and a gather of small per-unit results.

Works with any torch.distributed backend (nccl on the GPU nodes, gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def partition(n_units: int, rank: int, world: int) -> range:
    """Contiguous block of unit indices owned by `rank`; blocks differ in size by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of size {world}")
    if n_units < 0:
        raise ValueError("negative unit count")
    base, extra = divmod(n_units, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def unit_seed(base_seed: int, unit: int) -> int:
    """Seed of work unit `unit` (pair or chain): independent of how units map to ranks."""
    return int(base_seed) + int(unit)


def _device_for(dist):
    import torch
    return "cuda" if dist.get_backend() == "nccl" and torch.cuda.is_available() else "cpu"


def max_over_ranks(x: float, dist=None) -> float:
    """max of a per-rank scalar (elapsed time) over all ranks; `x` itself without a group."""
    if dist is None or not dist.is_initialized():
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(local: dict, n_units: int, dist=None) -> dict | None:
    """Collect {unit index: small numpy result} from every rank on rank 0 (None elsewhere).

    Every rank must call it (it is a collective).  Rank 0 checks that each unit arrived exactly
    once.
    """
    if dist is None or not dist.is_initialized():
        merged = dict(local)
    else:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, {int(k): np.asarray(v) for k, v in local.items()})
        if dist.get_rank() != 0:
            return None
        merged = {}
        for p in parts:
            for k, v in p.items():
                if k in merged:
                    raise RuntimeError(f"unit {k} reported by two ranks")
                merged[k] = v
    missing = sorted(set(range(n_units)) - set(merged))
    if missing:
        raise RuntimeError(f"units {missing[:8]} were not reported by any rank")
    return merged
