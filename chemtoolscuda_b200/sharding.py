"""Point sharding across GPUs: one process per GPU, torch.distributed plumbing.

Grid points are independent, so every local descriptor and the electrostatic
potential shard with no collective: each rank evaluates its own contiguous
slice of the points (``shard_bounds``, ``sharded_points``) or its own slab of
x-planes of a cubic grid (``slab_bounds``, ``sharded_cubic``; x is the
slowest grid index, the axis the reference's cubic driver chunks along,
src/evaluate_density.cu:496-501) and keeps its results; the optional gather
collects the slices on every rank.  The adjoint's outputs are sums over
points, so a sharded adjoint ends with one all-reduce (sum) of dL/dD (M x M)
and dL/dR (natom x 3) -- over NCCL on GPUs.  Timings of a multi-GPU run are
reduced with ``max_over_ranks``.

Basis, density matrix and atoms are replicated: every rank builds the same
molecule.  No cross-GPU data reaches a kernel: the collectives are NCCL's.

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


def slab_bounds(nx: int, rank: int, world: int) -> Tuple[int, int]:
    """x-planes [lo, hi) of a cubic grid owned by rank (sizes differ by at most one).
    The outputs of planes lo..hi-1 are one contiguous range of the grid's C-order
    output: flat indices [lo * ny * nz, hi * ny * nz)."""
    return shard_bounds(nx, rank, world)


def _slab_grid(origin, axes, shape, lo, hi):
    import numpy as np
    o = np.asarray(origin, dtype=np.float64) + lo * np.asarray(axes, dtype=np.float64).reshape(3, 3)[0]
    return o, np.asarray(axes, dtype=np.float64).reshape(3, 3), (hi - lo, int(shape[1]), int(shape[2]))


def device_cubic(mol, keys=("rho",), precision: str = "tc", params=None) -> Callable:
    """Descriptors of one slab on the GPU through the library (``ctc_eval_cubic``):
    f(origin, axes, shape) -> {key: CUDA float64 tensor of shape (n,) + per-point shape}."""
    import numpy as np
    import torch
    width = dict(rho=1, grad=3, hess=9, lap=1, tau_pd=1, tau_alpha=1, rdg=1, shannon=1,
                 weizsacker=1, thomas_fermi=1, gge=1, general_ked=1)

    def f(origin, axes, shape):
        n = int(np.prod(shape))
        dev = torch.device("cuda", torch.cuda.current_device())
        outs = {k: torch.empty(n * width[k], dtype=torch.float64, device=dev) for k in keys}
        if n:
            stream = torch.cuda.current_stream(dev).cuda_stream
            mol.eval_cubic_device(np.ascontiguousarray(origin), np.ascontiguousarray(axes),
                                  np.ascontiguousarray(shape, dtype=np.int32), precision,
                                  {k: t.data_ptr() for k, t in outs.items()}, **_prm(params),
                                  stream=stream)
        return {k: _shape(t, k) for k, t in outs.items()}

    return f


def device_points(mol, keys=("rho",), precision: str = "tc", params=None) -> Callable:
    """Descriptors of a slice of points on the GPU (``ctc_eval_local``):
    f(points (n, 3) CUDA float64) -> {key: CUDA float64 tensor}."""
    import torch
    width = dict(rho=1, grad=3, hess=9, lap=1, tau_pd=1, tau_alpha=1, rdg=1, shannon=1,
                 weizsacker=1, thomas_fermi=1, gge=1, general_ked=1)

    def f(points):
        n = points.shape[0]
        outs = {k: torch.empty(n * width[k], dtype=torch.float64, device=points.device) for k in keys}
        if n:
            stream = torch.cuda.current_stream(points.device).cuda_stream
            mol.eval_local_device(points.data_ptr(), n, precision,
                                  {k: t.data_ptr() for k, t in outs.items()}, **_prm(params),
                                  stream=stream)
        return {k: _shape(t, k) for k, t in outs.items()}

    return f


def _prm(params):
    """(alpha, gge_a, gge_b, ked_a) -> keyword arguments of the device methods."""
    if params is None:
        return {}
    return dict(zip(("alpha", "gge_a", "gge_b", "ked_a"), params))


def _shape(t, key):
    return t.view(-1, 3) if key == "grad" else (t.view(-1, 3, 3) if key == "hess" else t)


def _gather_rows(local: dict, counts, group=None) -> dict:
    """Concatenation over ranks (in rank order) of each rank's rows; counts[r] = rows of rank r."""
    import torch
    import torch.distributed as dist
    _, world = rank_world(group)
    if world == 1:
        return local
    out = {}
    cmax = max(counts)
    for k, t in local.items():
        pad = torch.zeros((cmax,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
        pad[: t.shape[0]] = t
        parts = [torch.empty_like(pad) for _ in range(world)]
        dist.all_gather(parts, pad, group=group)
        out[k] = torch.cat([p[:c] for p, c in zip(parts, counts)])
    return out


def sharded_cubic(origin, axes, shape, *, mol=None, evaluate: Optional[Callable] = None,
                  keys=("rho",), precision: str = "tc", params=None, gather: bool = False,
                  group=None):
    """Descriptors on one cubic grid split into x-slabs over the ranks.

    Every rank passes the same grid (point (i, j, k) = origin + i a0 + j a1 + k a2,
    k fastest) and evaluates only its slab of x-planes (``slab_bounds``); no data
    crosses GPUs.  Returns (lo, hi, outputs): the rank's planes and its outputs in
    the grid's C order, i.e. flat indices [lo ny nz, hi ny nz) of the whole grid.
    With ``gather=True`` every rank receives the whole grid's outputs instead
    (one all-gather per output; NCCL on GPUs).  ``evaluate(origin, axes, shape)``
    computes one slab (default: the GPU kernels of ``mol``).
    """
    if evaluate is None:
        if mol is None:
            raise ValueError("sharded_cubic needs mol or evaluate")
        evaluate = device_cubic(mol, keys, precision, params)
    rank, world = rank_world(group)
    nx = int(shape[0])
    lo, hi = slab_bounds(nx, rank, world)
    o, a, sh = _slab_grid(origin, axes, shape, lo, hi)
    res = evaluate(o, a, sh)
    if gather:
        plane = int(shape[1]) * int(shape[2])
        counts = [(slab_bounds(nx, r, world)[1] - slab_bounds(nx, r, world)[0]) * plane
                  for r in range(world)]
        return 0, nx, _gather_rows(res, counts, group)
    return lo, hi, res


def sharded_points(points, *, mol=None, evaluate: Optional[Callable] = None, keys=("rho",),
                   precision: str = "tc", params=None, gather: bool = False, group=None):
    """Descriptors at arbitrary points split into contiguous slices over the ranks.

    Every rank passes the same points; each evaluates rows [lo, hi) of them
    (``shard_bounds``).  Returns (lo, hi, outputs of those rows), or with
    ``gather=True`` (0, n, outputs of every row) on every rank."""
    if evaluate is None:
        if mol is None:
            raise ValueError("sharded_points needs mol or evaluate")
        evaluate = device_points(mol, keys, precision, params)
    rank, world = rank_world(group)
    n = points.shape[0]
    lo, hi = shard_bounds(n, rank, world)
    res = evaluate(points[lo:hi].contiguous())
    if gather:
        counts = [shard_bounds(n, r, world)[1] - shard_bounds(n, r, world)[0] for r in range(world)]
        return 0, n, _gather_rows(res, counts, group)
    return lo, hi, res
