"""Point sharding across GPUs: one process per GPU, torch.distributed plumbing.

Grid points are independent, so every local descriptor and the electrostatic
potential shard with no collective: each rank evaluates its own contiguous
slice of the points (``shard_bounds``) and keeps its results.  The adjoint's
outputs are sums over points, so a sharded adjoint ends with one all-reduce
(sum) of dL/dD (M x M) and dL/dR (natom x 3) -- over NCCL on GPUs.  Timings
of a multi-GPU run are reduced with ``max_over_ranks``.

The reference is single-GPU; this module has no counterpart there.
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple


def rank_world(group=None) -> Tuple[int, int]:
    """(rank, world size) of the default or given process group; (0, 1) without one."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def shard_bounds(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous slice [lo, hi) of n points owned by rank: sizes differ by at most one."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError(f"rank {rank} outside a world of {world}")
    if n < 0:
        raise ValueError("negative point count")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _collective_device(group=None):
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)
    if backend == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x: float, group=None) -> float:
    """Maximum of a host scalar (e.g. a per-rank device time) over the ranks."""
    import torch
    import torch.distributed as dist
    _, world = rank_world(group)
    if world == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_collective_device(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sum_over_ranks_(t, group=None):
    """In-place sum of a tensor over the ranks (no-op on one rank); returns t."""
    import torch.distributed as dist
    _, world = rank_world(group)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def device_adjoint(mol) -> Callable:
    """Adjoint of one shard on the GPU through the C ABI (``ctc_adjoint``):
    f(points, v_rho, v_grad) -> (dL/dD, dL/dR) as CUDA float64 tensors."""
    import torch

    def f(points, v_rho, v_grad):
        dev = points.device
        M = mol.nbasis
        dD = torch.zeros(M, M, dtype=torch.float64, device=dev)
        dR = torch.zeros(mol.natom, 3, dtype=torch.float64, device=dev)
        n = points.shape[0]
        if n:
            stream = torch.cuda.current_stream(dev).cuda_stream
            mol.adjoint_device(points.data_ptr(), n, v_rho.data_ptr(),
                               0 if v_grad is None else v_grad.data_ptr(),
                               dD.data_ptr(), dR.data_ptr(), stream=stream)
        return dD, dR

    return f


def sharded_adjoint(points, v_rho, v_grad=None, *, mol=None,
                    adjoint: Optional[Callable] = None, group=None):
    """dL/dD and dL/dR of a grid functional whose points are split over the ranks.

    Every rank passes the full point set (or any set of the same length and
    order) and its matching v_rho = dL/drho and v_grad = dL/d(grad rho); it
    evaluates the adjoint of its own slice only and the partial sums are
    all-reduced, so every rank returns the totals.  ``adjoint`` computes one
    slice (default: the GPU kernels of ``mol``).
    """
    if adjoint is None:
        if mol is None:
            raise ValueError("sharded_adjoint needs mol or adjoint")
        adjoint = device_adjoint(mol)
    rank, world = rank_world(group)
    n = points.shape[0]
    if v_rho.shape[0] != n or (v_grad is not None and v_grad.shape[0] != n):
        raise ValueError("points, v_rho and v_grad must have the same length")
    lo, hi = shard_bounds(n, rank, world)
    vg = None if v_grad is None else v_grad[lo:hi].contiguous()
    dD, dR = adjoint(points[lo:hi].contiguous(), v_rho[lo:hi].contiguous(), vg)
    sum_over_ranks_(dD, group)
    sum_over_ranks_(dR, group)
    return dD, dR
