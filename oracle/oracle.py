"""TEST INFRASTRUCTURE ONLY: ctypes front-end of the CPU FP64 oracle.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only as the checker.  The oracle restates the
reference's algorithms (citations in ``oracle/ctc_oracle.cpp``); its parity
pin is the set of golden vectors in ``tests/golden/`` that the reference's own
CUDA drivers produced.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "libctc_oracle.so")
_lib = None


class CtcoBasis(C.Structure):
    _fields_ = [("nshell", C.c_int32), ("centers", C.c_void_p), ("shell_atom", C.c_void_p),
                ("nprim", C.c_void_p), ("nseg", C.c_void_p), ("angmoms", C.c_void_p),
                ("exps", C.c_void_p), ("coeffs", C.c_void_p)]


def build() -> str:
    """Compile the oracle library (idempotent)."""
    src = os.path.join(_HERE, "ctc_oracle.cpp")
    if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_LIB)
        vp, i64, i32, dbl = C.c_void_p, C.c_int64, C.c_int, C.c_double
        _lib.ctco_nbasis.argtypes = [vp]
        _lib.ctco_eval_ao.argtypes = [vp, vp, i64, i32, vp, i32]
        _lib.ctco_eval_local.argtypes = [vp, vp, i32, vp, i64, dbl] + [vp] * 8 + [i32]
        _lib.ctco_eval_esp.argtypes = [vp, vp, i32, i32, vp, vp, vp, i64, vp, i32]
        _lib.ctco_adjoint.argtypes = [vp, vp, i32, i32, vp, i64, vp, vp, vp, vp, i32]
    return _lib


class _Basis:
    """Keeps the numpy arrays alive while the C struct points at them."""

    def __init__(self, flat: dict):
        self.arrs = dict(
            centers=np.ascontiguousarray(flat["centers"], np.float64),
            shell_atom=np.ascontiguousarray(flat["shell_atom"], np.int32),
            nprim=np.ascontiguousarray(flat["nprim"], np.int32),
            nseg=np.ascontiguousarray(flat["nseg"], np.int32),
            angmoms=np.ascontiguousarray(flat["angmoms"], np.int32),
            exps=np.ascontiguousarray(flat["exps"], np.float64),
            coeffs=np.ascontiguousarray(flat["coeffs"], np.float64))
        a = self.arrs
        self.s = CtcoBasis(len(a["nprim"]), *[a[k].ctypes.data for k in
                                                ("centers", "shell_atom", "nprim", "nseg",
                                                 "angmoms", "exps", "coeffs")])

    @property
    def ptr(self):
        return C.addressof(self.s)


def _p(x):
    return None if x is None else x.ctypes.data


def nbasis(flat: dict) -> int:
    b = _Basis(flat)
    return lib().ctco_nbasis(b.ptr)


def eval_ao(flat: dict, points: np.ndarray, deriv: int = 0, nthreads: int = 0) -> np.ndarray:
    """AO values (+ derivatives): array (nq, N, M), nq = 1, 4 or 10."""
    b = _Basis(flat)
    pts = np.ascontiguousarray(points, np.float64)
    M = lib().ctco_nbasis(b.ptr)
    nq = {0: 1, 1: 4, 2: 10}[deriv]
    out = np.zeros((nq, len(pts), M))
    rc = lib().ctco_eval_ao(b.ptr, _p(pts), len(pts), deriv, _p(out), nthreads)
    if rc < 0:
        raise ValueError("oracle: bad basis")
    return out


LOCAL_KEYS = ("rho", "grad", "hess", "lap", "tau_pd", "tau_alpha", "rdg", "shannon")
# Pointwise kinetic-energy densities formed from the C oracle's rho, grad rho,
# lap rho and tau_PD (src/evaluate_densbased.cu:91-208):
#   weizsacker   |grad rho|^2 / (8 rho), set to 1e-20 where 8 rho <= 1e-20
#                (divide_inplace with mask 1e-20, :129-131, src/cuda_utils.cu:71-84)
#   thomas_fermi 0.3 (3 pi^2)^(2/3) rho^(5/3)                           (:159-163)
#   gge          thomas_fermi + a weizsacker + b lap                   (:173-191)
#   general_ked  tau_PD + (a - 1)/4 lap                                (:195-208)
DERIVED_KEYS = ("weizsacker", "thomas_fermi", "gge", "general_ked")
ALL_KEYS = LOCAL_KEYS + DERIVED_KEYS


def eval_local(flat: dict, D: np.ndarray, points: np.ndarray, alpha: float = 0.5,
               keys=LOCAL_KEYS, nthreads: int = 0, gge_ab=(1 / 9, 1 / 6),
               ked_a: float = 1.0) -> dict:
    """Local descriptors at points; keys may name any of ALL_KEYS."""
    b = _Basis(flat)
    pts = np.ascontiguousarray(points, np.float64)
    Dm = np.ascontiguousarray(D, np.float64)
    n = len(pts)
    keys = tuple(keys)
    derived = [k for k in keys if k in DERIVED_KEYS]
    need = set(k for k in keys if k in LOCAL_KEYS)
    if derived:
        need |= {"rho", "grad", "lap", "tau_pd"}
    shapes = dict(rho=(n,), grad=(n, 3), hess=(n, 3, 3), lap=(n,), tau_pd=(n,), tau_alpha=(n,),
                  rdg=(n,), shannon=(n,))
    out = {k: np.zeros(shapes[k]) for k in LOCAL_KEYS if k in need}
    rc = lib().ctco_eval_local(b.ptr, _p(Dm), Dm.shape[0], _p(pts), n, float(alpha),
                               *[_p(out.get(k)) for k in LOCAL_KEYS], nthreads)
    if rc != 0:
        raise ValueError("oracle: basis size does not match D")
    if derived:
        rho, lap, tau = out["rho"], out["lap"], out["tau_pd"]
        g2 = (out["grad"] ** 2).sum(1)
        den = 8.0 * rho
        w = np.where(den > 1e-20, g2 / np.where(den > 1e-20, den, 1.0), 1e-20)
        with np.errstate(invalid="ignore"):  # pow of a negative rho is NaN, as in the reference
            tf = 0.3 * (3.0 * np.pi ** 2) ** (2.0 / 3.0) * np.power(rho, 5.0 / 3.0)
        extra = dict(weizsacker=w, thomas_fermi=tf, gge=tf + gge_ab[0] * w + gge_ab[1] * lap,
                     general_ked=tau + 0.25 * (ked_a - 1.0) * lap)
        out.update({k: extra[k] for k in derived})
    return {k: out[k] for k in keys}


def eval_esp(flat: dict, D: np.ndarray, coords: np.ndarray, charges: np.ndarray,
             points: np.ndarray, nthreads: int = 0) -> np.ndarray:
    b = _Basis(flat)
    pts = np.ascontiguousarray(points, np.float64)
    Dm = np.ascontiguousarray(D, np.float64)
    xyz = np.ascontiguousarray(coords, np.float64)
    q = np.ascontiguousarray(charges, np.float64)
    out = np.zeros(len(pts))
    rc = lib().ctco_eval_esp(b.ptr, _p(Dm), Dm.shape[0], len(xyz), _p(xyz), _p(q), _p(pts),
                             len(pts), _p(out), nthreads)
    if rc != 0:
        raise ValueError("oracle: basis size does not match D")
    return out


def adjoint(flat: dict, D: np.ndarray, natom: int, points: np.ndarray, v_rho: np.ndarray,
            v_grad: np.ndarray | None = None, want_D: bool = True, want_R: bool = True,
            nthreads: int = 0):
    b = _Basis(flat)
    pts = np.ascontiguousarray(points, np.float64)
    Dm = np.ascontiguousarray(D, np.float64)
    M = Dm.shape[0]
    vr = np.ascontiguousarray(v_rho, np.float64)
    vg = None if v_grad is None else np.ascontiguousarray(v_grad, np.float64)
    dD = np.zeros((M, M)) if want_D else None
    dR = np.zeros((natom, 3)) if want_R else None
    rc = lib().ctco_adjoint(b.ptr, _p(Dm), M, natom, _p(pts), len(pts), _p(vr), _p(vg),
                            _p(dD), _p(dR), nthreads)
    if rc != 0:
        raise ValueError("oracle: basis size does not match D")
    return dD, dR
