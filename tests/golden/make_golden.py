"""Generate golden vectors by running the reference's own CUDA drivers.

Needs a GPU and oracle/_ref/libctc_ref.so (``make -C oracle ref``, built from
the reference sources).  Every reference call runs in a fresh process whose
allocator is primed with zeroed memory, because several drivers accumulate
into un-zeroed cudaMalloc buffers (src/evaluate_gradient.cu:1156,1271,1295,
src/evaluate_hessian.cu:1863,1922,2091,2115, src/evaluate_kinetic_dens.cu:90).

    python tests/golden/make_golden.py            # all cases -> tests/golden/<case>.npz
    python tests/golden/make_golden.py --out DIR  # write elsewhere
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import cases  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libctc_ref.so")


def _load():
    lib = C.CDLL(REF_LIB)
    vp, i32, dbl = C.c_void_p, C.c_int, C.c_double
    lib.ref_create.restype = vp
    lib.ref_create.argtypes = [i32, vp, vp, vp, vp, vp, vp, i32, vp, vp, vp, i32]
    lib.ref_last_error.restype = C.c_char_p
    lib.ref_prime_allocator.argtypes = [C.c_size_t]
    for f in ["density", "gradient", "hessian", "laplacian", "tau_pd", "rdg", "shannon",
              "weizsacker", "thomas_fermi", "ao_deriv", "ao_sec_deriv", "ao_laplacian", "esp"]:
        getattr(lib, "ref_" + f).argtypes = [vp, vp, i32, vp]
    lib.ref_tau_general.argtypes = [vp, vp, i32, dbl, vp]
    lib.ref_general_ked.argtypes = [vp, vp, i32, dbl, vp]
    lib.ref_gge.argtypes = [vp, vp, i32, dbl, dbl, vp]
    lib.ref_cubic.argtypes = [vp, vp, vp, vp, vp]
    return lib


def _one(case: str, fn: str, out_path: str) -> None:
    mol, pts = cases.CASES[case]()
    flat = mol.flat()
    lib = _load()
    if lib.ref_prime_allocator(1 << 30) != 0:
        raise RuntimeError(lib.ref_last_error().decode())
    keep = [np.ascontiguousarray(flat[k]) for k in
            ("centers", "nprim", "nseg", "angmoms", "exps", "coeffs")]
    xyz = np.ascontiguousarray(mol.coords)
    chg = np.ascontiguousarray(mol.charges)
    D = np.ascontiguousarray(mol.D)
    M = D.shape[0]
    h = lib.ref_create(len(flat["nprim"]), *[k.ctypes.data for k in keep], len(xyz),
                       xyz.ctypes.data, chg.ctypes.data, D.ctypes.data, M)
    if not h:
        raise RuntimeError(lib.ref_last_error().decode())
    n = len(pts)
    P = pts.ctypes.data
    if fn in ("gradient",):
        out = np.zeros((n, 3))
    elif fn == "hessian":
        out = np.zeros((n, 3, 3))
    elif fn == "ao_deriv":
        out = np.zeros((3, M, n))
    elif fn == "ao_sec_deriv":
        out = np.zeros((6, M, n))
    elif fn == "ao_laplacian":
        out = np.zeros((M, n))
    elif fn == "cubic":
        out = np.zeros(cases.CUBE_SHAPE)
    else:
        out = np.zeros(n)
    O = out.ctypes.data
    if fn == "tau_general":
        rc = lib.ref_tau_general(h, P, n, cases.TAU_ALPHA, O)
    elif fn == "general_ked":
        rc = lib.ref_general_ked(h, P, n, cases.GENERAL_KED_A, O)
    elif fn == "gge":
        rc = lib.ref_gge(h, P, n, cases.GGE_AB[0], cases.GGE_AB[1], O)
    elif fn == "cubic":
        origin, axes = cases.cube_for(mol)
        origin = np.ascontiguousarray(origin)
        axes = np.ascontiguousarray(axes)
        shape = np.ascontiguousarray(np.array(cases.CUBE_SHAPE, dtype=np.int32))
        rc = lib.ref_cubic(h, origin.ctypes.data, axes.ctypes.data, shape.ctypes.data, O)
    else:
        rc = getattr(lib, "ref_" + fn)(h, P, n, O)
    if rc != 0:
        raise RuntimeError(f"{case}/{fn}: {lib.ref_last_error().decode()}")
    np.save(out_path, out)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--one", nargs=3, metavar=("CASE", "FN", "OUT"))
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--cases", nargs="*", default=list(cases.CASES))
    args = ap.parse_args()
    if args.one:
        _one(*args.one)
        return 0
    os.makedirs(args.out, exist_ok=True)
    failures = []
    for case in args.cases:
        mol, pts = cases.CASES[case]()
        flat = mol.flat()
        rec = {f"in_{k}": v for k, v in flat.items()}
        rec.update(in_D=mol.D, in_points=pts, in_coords=mol.coords, in_charges=mol.charges,
                   in_numbers=mol.numbers)
        fns = list(cases.LOCAL_FUNCS)
        if case in cases.ESP_CASES:
            fns.append("esp")
        if case in cases.CUBIC_CASES:
            fns.append("cubic")
            origin, axes = cases.cube_for(mol)
            rec.update(in_cube_origin=origin, in_cube_axes=axes,
                       in_cube_shape=np.array(cases.CUBE_SHAPE))
        with tempfile.TemporaryDirectory() as td:
            for fn in fns:
                path = os.path.join(td, fn + ".npy")
                r = subprocess.run([sys.executable, os.path.abspath(__file__), "--one", case, fn,
                                    path], capture_output=True, text=True, timeout=300)
                if r.returncode != 0 or not os.path.exists(path):
                    failures.append(f"{case}/{fn}: rc={r.returncode} {r.stderr[-400:]}")
                    continue
                rec["ref_" + fn] = np.load(path)
                print(f"{case}/{fn}: ok", flush=True)
        rec.update(meta_tau_alpha=cases.TAU_ALPHA, meta_gge_ab=np.array(cases.GGE_AB),
                   meta_general_ked_a=cases.GENERAL_KED_A)
        np.savez_compressed(os.path.join(args.out, f"{case}.npz"), **rec)
    for f in failures:
        print("FAILED", f)
    return 1 if failures else 0


if __name__ == "__main__":
    sys.exit(main())
