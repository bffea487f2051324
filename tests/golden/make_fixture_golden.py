"""Golden vectors on the reference's own fixture molecules.

The reference's tests evaluate every ``tests/data/*.fchk`` file through density,
gradient, Hessian, Laplacian and kinetic-energy densities
(tests/test_density.py:16-26 and tests/test_electron_density.cu:16-214 of the
reference).  This script records what the reference's CUDA drivers return on
those molecules, in two phases:

  inputs     (any machine holding the reference's fixture files): each file is
             read with this library's native reader (ctc_fchk_load, host only):
             basis, atoms and the density matrix (C occ) C^T; 64 seeded points
             are drawn (40 within ~1 bohr of the atoms, 24 in the padded box);
             everything goes to tests/golden/fixtures/<file>.npz.

  reference  (a GPU box with oracle/_ref/libctc_ref.so built from the reference
             sources): every fixtures/<file>.npz gets the reference's outputs on
             its points -- one fresh process per driver call, as make_golden.py
             does -- and is written to --out.

    python tests/golden/make_fixture_golden.py inputs [--data DIR]
    python tests/golden/make_fixture_golden.py reference --out DIR

DIR defaults to $CTC_REFERENCE/tests/data (CTC_REFERENCE: the reference's
checkout).  Drivers that refuse a molecule (the reference's ESP needs the whole
basis in its constant-memory array and has no g functions) are skipped and
listed in meta_skipped; the ESP is not called at all for bases with g
functions, which the reference's ESP does not support (its kernel stops on a
device-side assert there).
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys
import tempfile
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
FIXDIR = os.path.join(HERE, "fixtures")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, HERE)

TAU_ALPHA = 0.5
FUNCS = ("density", "gradient", "hessian", "laplacian", "tau_pd", "tau_general", "rdg", "esp")


def make_inputs(data_dir: str) -> list[str]:
    import ctc_abi
    os.makedirs(FIXDIR, exist_ok=True)
    written = []
    for path in sorted(glob.glob(os.path.join(data_dir, "*.fchk"))):
        stem = os.path.splitext(os.path.basename(path))[0]
        m = ctc_abi.load_fchk(path)
        rng = np.random.default_rng(zlib.crc32(stem.encode()))
        xyz = m["coords"]
        near = xyz[rng.integers(0, len(xyz), 40)] + rng.normal(0.0, 1.0, (40, 3))
        lo, hi = xyz.min(0) - 3.0, xyz.max(0) + 3.0
        far = rng.uniform(lo, hi, (24, 3))
        pts = np.ascontiguousarray(np.concatenate([near, far]))
        rec = {f"in_{k}": v for k, v in m["flat"].items()}
        rec.update(in_D=m["D"], in_coords=xyz, in_charges=m["charges"], in_numbers=m["numbers"],
                   in_points=pts, meta_source=np.array(os.path.basename(path)),
                   meta_tau_alpha=np.array(TAU_ALPHA))
        out = os.path.join(FIXDIR, stem + ".npz")
        np.savez_compressed(out, **rec)
        written.append(out)
    return written


def _one(inp: str, fn: str, out_path: str) -> None:
    from make_golden import _load
    g = dict(np.load(inp))
    lib = _load()
    if lib.ref_prime_allocator(1 << 30) != 0:
        raise RuntimeError(lib.ref_last_error().decode())
    keep = [np.ascontiguousarray(g["in_" + k]) for k in
            ("centers", "nprim", "nseg", "angmoms", "exps", "coeffs")]
    xyz = np.ascontiguousarray(g["in_coords"])
    chg = np.ascontiguousarray(g["in_charges"])
    D = np.ascontiguousarray(g["in_D"])
    h = lib.ref_create(len(g["in_nprim"]), *[k.ctypes.data for k in keep], len(xyz), xyz.ctypes.data,
                       chg.ctypes.data, D.ctypes.data, D.shape[0])
    if not h:
        raise RuntimeError(lib.ref_last_error().decode())
    pts = np.ascontiguousarray(g["in_points"])
    n = len(pts)
    out = np.zeros((n, 3)) if fn == "gradient" else (np.zeros((n, 3, 3)) if fn == "hessian" else np.zeros(n))
    if fn == "tau_general":
        rc = lib.ref_tau_general(h, pts.ctypes.data, n, TAU_ALPHA, out.ctypes.data)
    else:
        rc = getattr(lib, "ref_" + fn)(h, pts.ctypes.data, n, out.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"{fn}: {lib.ref_last_error().decode()}")
    np.save(out_path, out)


def run_reference(out_dir: str) -> int:
    os.makedirs(out_dir, exist_ok=True)
    failures = 0
    for inp in sorted(glob.glob(os.path.join(FIXDIR, "*.npz"))):
        rec = dict(np.load(inp))
        rec = {k: v for k, v in rec.items() if not k.startswith("ref_")}
        skipped = []
        # The reference's ESP has no g functions (src/evaluate_electrostatic.cu:10135-10137);
        # called on a basis with g shells its kernel stops on a device-side assert, so it is
        # never called for one.
        funcs = [f for f in FUNCS if not (f == "esp" and np.any(np.abs(rec["in_angmoms"]) >= 4))]
        if len(funcs) < len(FUNCS):
            skipped.append("esp: not run, the reference's ESP has no g functions")
        with tempfile.TemporaryDirectory() as td:
            for fn in funcs:
                path = os.path.join(td, fn + ".npy")
                r = subprocess.run([sys.executable, os.path.abspath(__file__), "one", inp, fn, path],
                                   capture_output=True, text=True, timeout=300)
                if r.returncode != 0 or not os.path.exists(path):
                    skipped.append(f"{fn}: {r.stderr.strip().splitlines()[-1] if r.stderr.strip() else r.returncode}")
                    if fn != "esp":
                        failures += 1
                    continue
                rec["ref_" + fn] = np.load(path)
        rec["meta_skipped"] = np.array(skipped if skipped else [""])
        np.savez_compressed(os.path.join(out_dir, os.path.basename(inp)), **rec)
        print(os.path.basename(inp), "ok" if not skipped else f"skipped {skipped}", flush=True)
    return 1 if failures else 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("phase", choices=["inputs", "reference", "one"])
    ap.add_argument("args", nargs="*")
    ap.add_argument("--data", default=os.path.join(os.environ.get("CTC_REFERENCE", "/root/reference"),
                                                   "tests", "data"))
    ap.add_argument("--out", default=FIXDIR)
    a = ap.parse_args()
    if a.phase == "inputs":
        for p in make_inputs(a.data):
            print(p)
        return 0
    if a.phase == "one":
        _one(*a.args)
        return 0
    return run_reference(a.out)


if __name__ == "__main__":
    sys.exit(main())
