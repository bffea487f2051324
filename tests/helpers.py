"""Shared checking helpers: per-point error scales for the descriptor comparisons.

Relative error is measured against the sum of the absolute values of the
terms that make up each descriptor (e.g. for rho = sum_{mu nu} phi_mu D_{mu nu}
phi_nu the scale is sum |phi_mu| |D_{mu nu}| |phi_nu|).  This is the quantity
floating-point rounding is proportional to, it is well defined where a
descriptor crosses zero (gradient components, Laplacian), and it equals
|rho| wherever no cancellation happens.  Derived descriptors (RDG, Shannon,
Weizsacker, Thomas-Fermi, GGE, general KED) use first-order propagation of
those scales.
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as O


def term_scales(flat, D, pts, alpha=0.5, gge=(1 / 9, 1 / 6), ked_a=1.0, ref=None):
    ao = O.eval_ao(flat, pts, 2)
    A = np.abs(ao)
    aD = np.abs(np.asarray(D))
    phi, d1, d2 = A[0], A[1:4], A[4:10]
    G0 = phi @ aD
    Gk = [d1[k] @ aD for k in range(3)]
    s = {}
    s["rho"] = (G0 * phi).sum(1)
    s["grad"] = np.stack([2 * (G0 * d1[k]).sum(1) for k in range(3)], 1)
    idx = {(0, 0): 0, (0, 1): 1, (0, 2): 2, (1, 1): 3, (1, 2): 4, (2, 2): 5}
    H = np.zeros((len(pts), 3, 3))
    for i in range(3):
        for j in range(3):
            k = idx[(min(i, j), max(i, j))]
            H[:, i, j] = 2 * ((Gk[i] * d1[j]).sum(1) + (G0 * d2[k]).sum(1))
    s["hess"] = H
    s["lap"] = H[:, 0, 0] + H[:, 1, 1] + H[:, 2, 2]
    s["tau_pd"] = 0.5 * sum((Gk[k] * d1[k]).sum(1) for k in range(3))
    s["tau_alpha"] = s["tau_pd"] + abs(alpha) * s["lap"]
    s["general_ked"] = s["tau_pd"] + abs(ked_a - 1) / 4 * s["lap"]
    if ref is not None:
        rho = np.abs(ref["rho"]) + 1e-300
        g = np.linalg.norm(ref["grad"], axis=1) + 1e-300
        sg = np.linalg.norm(s["grad"], axis=1)
        if "rdg" in ref:
            s["rdg"] = np.abs(ref["rdg"]) * (sg / g + 4 / 3 * s["rho"] / rho)
        s["shannon"] = np.abs(np.log(rho) + 1) * s["rho"]
        w = g ** 2 / (8 * rho)
        s["weizsacker"] = w * (2 * sg / g + s["rho"] / rho)
        tf = 0.3 * (3 * np.pi ** 2) ** (2 / 3) * rho ** (5 / 3)
        s["thomas_fermi"] = 5 / 3 * tf * s["rho"] / rho
        s["gge"] = s["thomas_fermi"] + abs(gge[0]) * s["weizsacker"] + abs(gge[1]) * s["lap"]
    return s


def rel_err(x, ref, scale, floor=0.0):
    x = np.asarray(x)
    ref = np.asarray(ref)
    scale = np.asarray(scale)
    return np.abs(x - ref) / np.maximum(scale, floor)


def assert_close(name, x, ref, scale, rtol, atol=0.0, mask=None):
    x = np.asarray(x, float)
    ref = np.asarray(ref, float)
    scale = np.broadcast_to(np.asarray(scale, float), ref.shape)
    bad = np.abs(x - ref) > rtol * scale + atol
    if mask is not None:
        m = np.asarray(mask)
        while m.ndim < bad.ndim:
            m = m[..., None]
        bad &= np.broadcast_to(m, bad.shape)
    if bad.any():
        i = np.argwhere(bad)[0]
        i = tuple(i)
        raise AssertionError(f"{name}: {bad.sum()} of {bad.size} entries out of tolerance "
                             f"(rtol={rtol:g}, atol={atol:g}); first at {i}: got {x[i]!r}, "
                             f"want {ref[i]!r}, scale {scale[i]!r}")
