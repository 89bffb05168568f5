"""Several GPUs: each rank integrates its own contiguous block of Sobol indices and the
ranks combine their sums with one all_reduce.

keldy's integrator keeps point i on rank i % size (integrator.hpp:84-88) and sums with
mpi::all_reduce in reduce_result (integrator.hpp:123-131). Contiguous blocks cover the
same points (each once) without every rank generating every point; the sum over ranks is
the same set of evaluations, added in a different order.
"""
from __future__ import annotations


def shard(n_points, rank, world, k_first=1):
    """(k_first, count) of rank's contiguous block of n_points Sobol indices starting at
    k_first: the first n_points % world ranks take one extra point."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(int(n_points), world)
    start = rank * base + min(rank, extra)
    count = base + (1 if rank < extra else 0)
    return k_first + start, count


def allreduce_sums(sums, group=None, device=None):
    """Element-wise sum over ranks of a list of (complex sum, n_points, n_in_domain) tuples
    (torch.distributed, any backend). Returns the reduced list in the same layout."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return list(sums)
    flat = []
    for s, n, d in sums:
        flat += [complex(s).real, complex(s).imag, float(n), float(d)]
    t = torch.tensor(flat, dtype=torch.float64, device=device)
    dist.all_reduce(t, group=group)
    v = t.tolist()
    return [(complex(v[4 * i], v[4 * i + 1]), int(round(v[4 * i + 2])), int(round(v[4 * i + 3])))
            for i in range(len(sums))]


def integrate_sharded(ctx, items, rank, world, group=None, device=None, algo=0):
    """capi.integrate over this rank's share of every item, then the all_reduce: each item
    dict's n_points/k_first describe the whole job."""
    from . import capi
    mine = []
    for it in items:
        k0, cnt = shard(it["n_points"], rank, world, it.get("k_first", 1))
        mine.append(dict(it, k_first=k0, n_points=cnt))
    res = capi.integrate(ctx, mine, algo)
    return allreduce_sums([(s, n, d) for s, n, d, _ in res], group, device)
