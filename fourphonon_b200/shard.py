"""Multi-GPU host logic: how a solve's irreducible modes are split across
ranks and joined again.

The reference splits the modes mm in [1, Nbands*Nlist] into contiguous
chunks per MPI rank (Src/ShengBTE.f90:176-177, loops such as
Src/processes.f90:1722-1725) and joins the per-mode rates with
MPI_ALLREDUCE(SUM) (e.g. processes.f90:5296-5308).  Here a rank owns a
contiguous range of irreducible q-points (all branches of each, so a work
item never spans ranks), balanced by the number of candidate q'' per point,
and the rates are joined with one all-gather of the per-mode vectors.  The
same functions run over NCCL (one process per GPU) and over gloo (CPU tests).
"""
from __future__ import annotations

import numpy as np


def partition_qpoints(nlist: int, world: int, weights=None):
    """Contiguous [begin, end) ranges of irreducible q-points, one per rank,
    with nearly equal total weight (default weight 1 per point)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    w = np.ones(nlist) if weights is None else np.asarray(weights, dtype=np.float64)
    if w.shape != (nlist,):
        raise ValueError("weights must have one entry per irreducible q-point")
    c = np.concatenate([[0.0], np.cumsum(w)])
    total = c[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.searchsorted(c, target, side="left"))
        if b > 0 and abs(c[b - 1] - target) <= abs(c[min(b, nlist)] - target):
            b -= 1
        b = min(max(b, bounds[-1]), nlist)
        bounds.append(b)
    bounds.append(nlist)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def mode_range(qrange, nbands: int):
    """Irreducible modes (0-based, mm = ll*nbands + i) of a q-point range."""
    return qrange[0] * nbands, qrange[1] * nbands


def gather_modes(local: np.ndarray, qrange, nbands: int, nlist: int, group=None):
    """All-gather per-mode values owned by each rank into the full (nlist*nbands)
    vector (rank r contributes its own mode range; other entries are zero
    before the reduction)."""
    import torch
    import torch.distributed as dist

    full = np.zeros(nlist * nbands, dtype=np.float64)
    m0, m1 = mode_range(qrange, nbands)
    full[m0:m1] = local[m0:m1]
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return full
    backend = dist.get_backend(group)
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.from_numpy(full).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def reduce_max(x: float, group=None) -> float:
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(x)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def rank_temperatures(base, rank: int, step: float = 10.0):
    """Temperatures of rank r's independent solve in the weak-scaling benchmark."""
    return [float(t) + step * rank for t in base]
