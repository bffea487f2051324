"""ctypes view of include/chemtools_cuda.h for the tests.

The GPU parity tests call the library through this C ABI (not through the
pybind11 module) with torch CUDA tensors as device memory.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "chemtools_cuda.h")
LIB = os.path.join(ROOT, "chemtoolscuda_b200", "libchemtools_cuda.so")

OUT_KEYS = ("rho", "grad", "hess", "lap", "tau_pd", "tau_alpha", "rdg", "shannon", "weizsacker",
            "thomas_fermi", "gge", "general_ked")
OUT_WIDTH = dict(rho=1, grad=3, hess=9, lap=1, tau_pd=1, tau_alpha=1, rdg=1, shannon=1,
                 weizsacker=1, thomas_fermi=1, gge=1, general_ked=1)
PREC_FP64, PREC_TC = 0, 1


class Basis(C.Structure):
    _fields_ = [("nshell", C.c_int32), ("centers", C.c_void_p), ("shell_atom", C.c_void_p),
                ("nprim", C.c_void_p), ("nseg", C.c_void_p), ("angmoms", C.c_void_p),
                ("exps", C.c_void_p), ("coeffs", C.c_void_p)]


class FchkView(C.Structure):
    _fields_ = [("basis", Basis), ("natom", C.c_int32), ("atom_xyz", C.c_void_p),
                ("atom_charges", C.c_void_p), ("atomic_numbers", C.c_void_p), ("nbasis", C.c_int32),
                ("nalpha", C.c_int32), ("nbeta", C.c_int32), ("density", C.c_void_p)]


class Outputs(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in OUT_KEYS]


class Params(C.Structure):
    _fields_ = [("alpha", C.c_double), ("gge_a", C.c_double), ("gge_b", C.c_double),
                ("ked_a", C.c_double)]


def header_symbols() -> list[str]:
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(ctc_[a-z0-9_]+)\s*\(", txt)))


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(LIB)
        vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
        L = _lib
        L.ctc_last_error.restype = C.c_char_p
        L.ctc_version.restype = C.c_char_p
        L.ctc_molecule_create.argtypes = [vp, i32, vp, vp, vp, i32, vp]
        L.ctc_molecule_destroy.argtypes = [vp]
        L.ctc_molecule_nbasis.argtypes = [vp]
        L.ctc_molecule_natom.argtypes = [vp]
        L.ctc_molecule_set_density_matrix.argtypes = [vp, vp, vp]
        L.ctc_molecule_set_coordinates.argtypes = [vp, vp]
        L.ctc_molecule_prepare.argtypes = [vp, i32]
        L.ctc_eval_local.argtypes = [vp, vp, i64, i32, vp, vp, vp]
        L.ctc_eval_local_host.argtypes = [vp, vp, i64, i32, vp, vp]
        L.ctc_eval_cubic.argtypes = [vp, vp, vp, vp, i32, vp, vp, vp]
        L.ctc_eval_ao.argtypes = [vp, vp, i64, i32, vp, vp]
        L.ctc_eval_esp.argtypes = [vp, vp, i64, vp, vp]
        L.ctc_eval_esp_host.argtypes = [vp, vp, i64, vp]
        L.ctc_adjoint.argtypes = [vp, vp, i64, vp, vp, vp, vp, vp]
        L.ctc_fchk_load.argtypes = [C.c_char_p, vp]
        L.ctc_fchk_view_get.argtypes = [vp, vp]
        L.ctc_fchk_destroy.argtypes = [vp]
        L.ctc_fchk_destroy.restype = None
        L.ctc_molecule_create_from_fchk.argtypes = [C.c_char_p, vp]
        L.ctc_molden_load.argtypes = [C.c_char_p, vp]
        L.ctc_wfn_load.argtypes = [C.c_char_p, vp]
        L.ctc_molecule_create_from_file.argtypes = [C.c_char_p, vp]
        L.ctc_molecule_sync_status.argtypes = [vp, vp]
        L.ctc_molecule_set_wait_limit.argtypes = [vp, i64]
        L.ctc_molecule_esp_info.argtypes = [vp, vp]
    return _lib


def load_fchk(path: str, molden: bool = False, wfn: bool = False) -> dict:
    """Basis (flat layout of synthetic.flatten_basis), atoms and density matrix of an .fchk
    (or, with molden=True, a Molden; with wfn=True, a .wfn/.wfx) file as read by the library's native reader (host only,
    no GPU needed)."""
    h = C.c_void_p()
    if molden:
        check(lib().ctc_molden_load(path.encode(), C.byref(h)), "ctc_molden_load")
    elif wfn:
        check(lib().ctc_wfn_load(path.encode(), C.byref(h)), "ctc_wfn_load")
    else:
        check(lib().ctc_fchk_load(path.encode(), C.byref(h)), "ctc_fchk_load")
    try:
        v = FchkView()
        check(lib().ctc_fchk_view_get(h, C.byref(v)), "ctc_fchk_view_get")
        b = v.basis
        ns = b.nshell

        def arr(ptr, n, ct):
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(n,)).copy()
        nprim = arr(b.nprim, ns, C.c_int32)
        nseg = arr(b.nseg, ns, C.c_int32)
        flat = dict(centers=arr(b.centers, 3 * ns, C.c_double).reshape(ns, 3),
                    shell_atom=arr(b.shell_atom, ns, C.c_int32), nprim=nprim, nseg=nseg,
                    angmoms=arr(b.angmoms, int(nseg.sum()), C.c_int32),
                    exps=arr(b.exps, int(nprim.sum()), C.c_double),
                    coeffs=arr(b.coeffs, int((nseg * nprim).sum()), C.c_double))
        M = v.nbasis
        return dict(flat=flat, coords=arr(v.atom_xyz, 3 * v.natom, C.c_double).reshape(v.natom, 3),
                    charges=arr(v.atom_charges, v.natom, C.c_double),
                    numbers=arr(v.atomic_numbers, v.natom, C.c_int32), nalpha=v.nalpha, nbeta=v.nbeta,
                    D=arr(v.density, M * M, C.c_double).reshape(M, M))
    finally:
        lib().ctc_fchk_destroy(h)


def load_molden(path: str) -> dict:
    return load_fchk(path, molden=True)


def load_wfn(path: str) -> dict:
    """A .wfn or .wfx file through ctc_wfn_load (host only)."""
    return load_fchk(path, wfn=True)


def err() -> str:
    return lib().ctc_last_error().decode()


def check(rc: int, what: str = "call"):
    if rc != 0:
        raise RuntimeError(f"{what} -> {rc}: {err()}")


class Mol:
    """Owns a ctc_molecule built from a flat basis (synthetic.flatten_basis layout)."""

    def __init__(self, flat: dict, coords, charges, D, shell_atom: bool = True):
        self.keep = dict(
            centers=np.ascontiguousarray(flat["centers"], np.float64),
            shell_atom=np.ascontiguousarray(flat["shell_atom"], np.int32),
            nprim=np.ascontiguousarray(flat["nprim"], np.int32),
            nseg=np.ascontiguousarray(flat["nseg"], np.int32),
            angmoms=np.ascontiguousarray(flat["angmoms"], np.int32),
            exps=np.ascontiguousarray(flat["exps"], np.float64),
            coeffs=np.ascontiguousarray(flat["coeffs"], np.float64),
            coords=np.ascontiguousarray(coords, np.float64),
            charges=np.ascontiguousarray(charges, np.float64),
            D=np.ascontiguousarray(D, np.float64))
        k = self.keep
        b = Basis(len(k["nprim"]), k["centers"].ctypes.data,
                  k["shell_atom"].ctypes.data if shell_atom else None, k["nprim"].ctypes.data,
                  k["nseg"].ctypes.data, k["angmoms"].ctypes.data, k["exps"].ctypes.data,
                  k["coeffs"].ctypes.data)
        h = C.c_void_p()
        check(lib().ctc_molecule_create(C.byref(b), len(k["coords"]), k["coords"].ctypes.data,
                                        k["charges"].ctypes.data, k["D"].ctypes.data,
                                        k["D"].shape[0], C.byref(h)), "ctc_molecule_create")
        self.h = h
        self.M = k["D"].shape[0]

    def sync_status(self) -> int:
        """ctc_molecule_sync_status on the legacy default stream: its return code."""
        return lib().ctc_molecule_sync_status(self.h, None)

    def set_wait_limit(self, cycles: int):
        check(lib().ctc_molecule_set_wait_limit(self.h, int(cycles)), "ctc_molecule_set_wait_limit")

    def close(self):
        if self.h:
            lib().ctc_molecule_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- device helpers (torch) ----
    def eval_local(self, points, keys, precision=PREC_FP64, params=(0.5, 1 / 9, 1 / 6, 1.0)):
        import torch
        pts = torch.as_tensor(np.ascontiguousarray(points), dtype=torch.float64, device="cuda")
        n = pts.shape[0]
        outs = {k: torch.full((n * OUT_WIDTH[k],), float("nan"), dtype=torch.float64, device="cuda")
                for k in keys}
        o = Outputs(**{k: outs[k].data_ptr() for k in keys})
        p = Params(*params)
        check(lib().ctc_eval_local(self.h, pts.data_ptr(), n, precision, C.byref(p), C.byref(o),
                                   None), "ctc_eval_local")
        torch.cuda.synchronize()
        res = {}
        for k, t in outs.items():
            a = t.cpu().numpy()
            res[k] = a.reshape(n, 3) if k == "grad" else (a.reshape(n, 3, 3) if k == "hess" else a)
        return res

    def eval_local_host(self, points, keys, precision=PREC_FP64, params=(0.5, 1 / 9, 1 / 6, 1.0)):
        pts = np.ascontiguousarray(points, np.float64)
        n = len(pts)
        outs = {k: np.full(n * OUT_WIDTH[k], np.nan) for k in keys}
        o = Outputs(**{k: outs[k].ctypes.data for k in keys})
        p = Params(*params)
        check(lib().ctc_eval_local_host(self.h, pts.ctypes.data, n, precision, C.byref(p),
                                        C.byref(o)), "ctc_eval_local_host")
        return {k: (a.reshape(n, 3) if k == "grad" else (a.reshape(n, 3, 3) if k == "hess" else a))
                for k, a in outs.items()}

    def eval_cubic(self, origin, axes, shape, keys=("rho",), precision=PREC_FP64, params=None,
                   index=None):
        """Descriptors on the cubic grid; with index (flat grid indices) only those points are
        copied back, reshaped like eval_local's outputs."""
        import torch
        n = int(np.prod(shape))
        outs = {k: torch.full((n * OUT_WIDTH[k],), float("nan"), dtype=torch.float64, device="cuda")
                for k in keys}
        o = Outputs(**{k: outs[k].data_ptr() for k in keys})
        org = np.ascontiguousarray(origin, np.float64)
        ax = np.ascontiguousarray(axes, np.float64)
        sh = np.ascontiguousarray(shape, np.int32)
        p = None if params is None else C.byref(Params(*params))
        check(lib().ctc_eval_cubic(self.h, org.ctypes.data, ax.ctypes.data, sh.ctypes.data,
                                   precision, p, C.byref(o), None), "ctc_eval_cubic")
        torch.cuda.synchronize()
        if index is None:
            return {k: t.cpu().numpy() for k, t in outs.items()}
        idx = torch.as_tensor(np.asarray(index, np.int64), device="cuda")
        res = {}
        for k, t in outs.items():
            w = OUT_WIDTH[k]
            a = t.view(n, w)[idx].cpu().numpy()
            res[k] = a.reshape(-1, 3) if k == "grad" else (a.reshape(-1, 3, 3) if k == "hess" else a.ravel())
        del outs
        return res

    def eval_ao(self, points, deriv):
        import torch
        pts = torch.as_tensor(np.ascontiguousarray(points), dtype=torch.float64, device="cuda")
        n = pts.shape[0]
        nq = {0: 1, 1: 4, 2: 10}[deriv]
        out = torch.full((nq, n, self.M), float("nan"), dtype=torch.float64, device="cuda")
        check(lib().ctc_eval_ao(self.h, pts.data_ptr(), n, deriv, out.data_ptr(), None), "ctc_eval_ao")
        torch.cuda.synchronize()
        return out.cpu().numpy()

    def eval_esp(self, points):
        import torch
        pts = torch.as_tensor(np.ascontiguousarray(points), dtype=torch.float64, device="cuda")
        out = torch.full((pts.shape[0],), float("nan"), dtype=torch.float64, device="cuda")
        check(lib().ctc_eval_esp(self.h, pts.data_ptr(), pts.shape[0], out.data_ptr(), None),
              "ctc_eval_esp")
        torch.cuda.synchronize()
        return out.cpu().numpy()

    def eval_esp_host(self, points):
        pts = np.ascontiguousarray(points, np.float64)
        out = np.full(len(pts), np.nan)
        check(lib().ctc_eval_esp_host(self.h, pts.ctypes.data, len(pts), out.ctypes.data),
              "ctc_eval_esp_host")
        return out

    def adjoint(self, points, v_rho, v_grad=None, want_D=True, want_R=True):
        import torch
        dev = "cuda"
        pts = torch.as_tensor(np.ascontiguousarray(points), dtype=torch.float64, device=dev)
        vr = torch.as_tensor(np.ascontiguousarray(v_rho), dtype=torch.float64, device=dev)
        vg = None if v_grad is None else torch.as_tensor(np.ascontiguousarray(v_grad),
                                                          dtype=torch.float64, device=dev)
        natom = len(self.keep["coords"])
        dD = torch.zeros((self.M, self.M), dtype=torch.float64, device=dev) if want_D else None
        dR = torch.zeros((natom, 3), dtype=torch.float64, device=dev) if want_R else None
        check(lib().ctc_adjoint(self.h, pts.data_ptr(), pts.shape[0], vr.data_ptr(),
                                None if vg is None else vg.data_ptr(),
                                None if dD is None else dD.data_ptr(),
                                None if dR is None else dR.data_ptr(), None), "ctc_adjoint")
        torch.cuda.synchronize()
        return (None if dD is None else dD.cpu().numpy(), None if dR is None else dR.cpu().numpy())
