"""torch.autograd binding of the density evaluation (no counterpart in the reference).

``density_and_gradient(mol, points, D, coords)`` returns (rho, grad rho) at
``points`` for density matrix ``D`` and atom positions ``coords``; its
backward pass calls the hand-written adjoint kernels (``ctc_adjoint`` in the C
ABI) and returns dL/dD (entries treated as independent) and dL/dR (grid
points and weights held fixed).  Any grid functional written in torch on top
of (rho, grad rho) -- e.g. L = sum_g w_g (c1 rho^(4/3) + c2 |grad rho|^2 / rho^(4/3))
-- then differentiates through it.

PyTorch is plumbing here: device memory, streams and the autograd graph.  The
arithmetic runs in the sm_100a library.
"""
from __future__ import annotations

import numpy as np
import torch


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class _Density(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mol, points, D, coords):
        if points.dtype != torch.float64 or not points.is_cuda:
            raise TypeError("points must be a CUDA float64 tensor")
        points = points.contiguous()
        Dc = D.detach().to(device=points.device, dtype=torch.float64).contiguous()
        mol.set_density_matrix_device(Dc.data_ptr(), _stream())
        mol.set_coordinates(np.ascontiguousarray(coords.detach().cpu().numpy(), dtype=np.float64))
        n = points.shape[0]
        rho = torch.empty(n, dtype=torch.float64, device=points.device)
        grad = torch.empty(n, 3, dtype=torch.float64, device=points.device)
        if n:
            mol.eval_local_device(points.data_ptr(), n, "fp64",
                                  {"rho": rho.data_ptr(), "grad": grad.data_ptr()}, stream=_stream())
        ctx.mol = mol
        ctx.coords_device = coords.device
        ctx.save_for_backward(points, Dc)
        return rho, grad

    @staticmethod
    def backward(ctx, g_rho, g_grad):
        points, Dc = ctx.saved_tensors
        mol = ctx.mol
        n = points.shape[0]
        M = Dc.shape[0]
        need_D = ctx.needs_input_grad[2]
        need_R = ctx.needs_input_grad[3]
        dev = points.device
        if g_rho is None:
            g_rho = torch.zeros(n, dtype=torch.float64, device=dev)
        g_rho = g_rho.contiguous().to(torch.float64)
        g_grad = None if g_grad is None else g_grad.contiguous().to(torch.float64)
        dD = torch.zeros(M, M, dtype=torch.float64, device=dev) if need_D else None
        dR = torch.zeros(mol.natom, 3, dtype=torch.float64, device=dev) if need_R else None
        # the molecule may have been changed by other calls since forward
        mol.set_density_matrix_device(Dc.data_ptr(), _stream())
        if n and (need_D or need_R):
            mol.adjoint_device(points.data_ptr(), n, g_rho.data_ptr(),
                               0 if g_grad is None else g_grad.data_ptr(),
                               0 if dD is None else dD.data_ptr(),
                               0 if dR is None else dR.data_ptr(), stream=_stream())
        if dR is not None:
            dR = dR.to(ctx.coords_device)
        return None, None, dD, dR


def density_and_gradient(mol, points: torch.Tensor, D: torch.Tensor, coords: torch.Tensor):
    """(rho, grad rho) with autograd support for D and coords."""
    return _Density.apply(mol, points, D, coords)


def gga_functional(rho, grad, weights, c1=-0.7386, c2=0.0042, rho_min=1e-10):
    """L = sum_g w_g (c1 rho^(4/3) + c2 |grad rho|^2 / rho^(4/3)) over points with rho > rho_min."""
    mask = rho > rho_min
    r = torch.where(mask, rho, torch.ones_like(rho))
    r43 = r ** (4.0 / 3.0)
    f = c1 * r43 + c2 * (grad * grad).sum(-1) / r43
    return (weights * torch.where(mask, f, torch.zeros_like(f))).sum()
