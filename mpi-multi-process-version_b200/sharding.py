"""Spreading independent cavities over ranks (one process per GPU).

The reference decomposes ONE cavity over MPI ranks (1D slabs or 2D/3D
blocks with a ghost-layer exchange every step, natural-convection_2dim_block
.f90:602-658).  On B200 one cavity of the reference's sizes fits one GPU many
times over, so a multi-GPU job here runs whole cavities per rank: the batch is
split by longest-processing-time-first over the node counts (a cavity's cost
per iteration is proportional to its nodes), each rank advances its share with
the persistent batch kernel and no data crosses between ranks while stepping;
the only collective is the final gather of the per-cavity results.
"""
from __future__ import annotations

import numpy as np


def lpt_shards(weights, world):
    """Indices per rank: cavities in decreasing weight order, each to the rank
    with the smallest load so far (ties to the lower rank / lower index).
    Every index appears exactly once; each rank's list is sorted."""
    if world < 1:
        raise ValueError("world must be >= 1")
    w = [float(x) for x in weights]
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    loads = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        out[r].append(i)
        loads[r] += w[i]
    return [sorted(o) for o in out]


def case_nodes(case):
    return int(case["nx"]) * int(case["ny"]) * int(case.get("nz", 1))


def my_share(cases, world, rank):
    """(indices, cases) of this rank's share of `cases` (LPT over node counts)."""
    idx = lpt_shards([case_nodes(c) for c in cases], world)[rank]
    return idx, [cases[i] for i in idx]


def gather_by_index(idx_local, values_local, n_total):
    """Reassemble per-cavity results computed on every rank.

    values_local: {name: sequence aligned with idx_local}.  Returns
    {name: ndarray of n_total} on every rank (all_gather of Python objects over
    the default process group; without one, the local values are placed)."""
    import torch.distributed as dist
    parts = [(list(idx_local), {k: list(np.asarray(v).tolist()) for k, v in values_local.items()})]
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, (list(idx_local), {k: list(np.asarray(v).tolist())
                                                         for k, v in values_local.items()}))
    out = {}
    seen = np.zeros(n_total, dtype=bool)
    for idx, vals in parts:
        for k, v in vals.items():
            arr = out.setdefault(k, np.full(n_total, np.nan))
            arr[np.asarray(idx, dtype=np.int64)] = v
        seen[np.asarray(idx, dtype=np.int64)] = True
    if not seen.all():
        raise RuntimeError(f"gather_by_index: {int((~seen).sum())} cavities have no result")
    return out
