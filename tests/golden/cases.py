"""Deterministic inputs of the golden-vector cases.

Each case is a small molecule plus points.  ``make_golden.py`` runs the
reference's own CUDA drivers (oracle/_ref, built from the reference sources)
on these inputs and stores inputs and outputs together in ``<case>.npz``, so
the tests need neither the reference nor this module to read them back.
"""
from __future__ import annotations

import math

import numpy as np

from chemtoolscuda_b200 import synthetic as S


def _shell(rng, center, atom, angmoms, K, emin=0.1, emax=800.0):
    e = np.sort(np.exp(rng.uniform(math.log(emin), math.log(emax), size=K)))[::-1].copy()
    cs = []
    for am in angmoms:
        cs.append(S._normalise_contraction(abs(am), e, rng.standard_normal(K)))
    return S.Shell(center=np.asarray(center, float), atom=atom, angmoms=list(angmoms),
                   exponents=e, coeffs=np.asarray(cs))


def _molecule(rng, coords, numbers, shell_specs, nocc, name):
    shells = [_shell(rng, coords[a], a, am, K) for (a, am, K) in shell_specs]
    M = sum(S.nfunc(a) for s in shells for a in s.angmoms)
    D = S.make_density_matrix(rng, M, nocc)
    return S.SyntheticMolecule(coords=np.asarray(coords, float), numbers=np.asarray(numbers, np.int32),
                               charges=np.asarray(numbers, float), shells=shells, D=D, name=name)


def _points_away(rng, mol, n, pad=3.0, rmin=0.7):
    lo = mol.coords.min(0) - pad
    hi = mol.coords.max(0) + pad
    out = []
    while len(out) < n:
        p = rng.uniform(lo, hi, size=3)
        if np.linalg.norm(mol.coords - p, axis=1).min() > rmin:
            out.append(p)
    return np.ascontiguousarray(np.asarray(out))


def case_allshell():
    """Every segment type the reference evaluates (s p d 5d f 7f g 9g) plus
    generalised s+p and d+5d shells sharing exponents."""
    rng = np.random.default_rng(11)
    coords = np.array([[0.0, 0.0, 0.0], [1.9, 0.4, -0.6], [-0.8, 1.5, 1.1]])
    specs = [(0, [0], 5), (0, [0, 1], 3), (0, [2], 3), (0, [-2], 2), (0, [3], 2), (0, [-3], 2),
             (0, [4], 2), (0, [-4], 1), (1, [0], 4), (1, [1], 3), (1, [2, -2], 2), (1, [3], 1),
             (2, [0], 3), (2, [1], 2), (2, [-4], 2)]
    mol = _molecule(rng, coords, [8, 6, 1], specs, 12, "allshell")
    pts = _points_away(rng, mol, 192, rmin=0.05)
    return mol, pts


def case_c1():
    """The 12-atom synthetic molecule (Cartesian shells up to d, ~120 functions)."""
    mol = S.make_molecule("c1", seed=7)
    rng = np.random.default_rng(12)
    pts = S.random_points(rng, mol, 256)
    return mol, pts


def case_esp():
    """ESP case: every shell type the reference's ESP supports (no g,
    src/evaluate_electrostatic.cu:10135-10137), points kept > 1 bohr from nuclei."""
    rng = np.random.default_rng(13)
    coords = np.array([[0.0, 0.0, 0.0], [2.1, 0.3, 0.2], [-0.7, 1.8, -0.5], [0.4, -1.2, 1.6]])
    specs = [(0, [0], 4), (0, [0, 1], 3), (0, [2], 2), (0, [-2], 2), (0, [3], 1), (0, [-3], 2),
             (1, [0], 3), (1, [1], 2), (1, [-2], 1), (2, [0], 3), (2, [1], 2), (3, [0], 2),
             (3, [1], 1), (3, [2], 2)]
    mol = _molecule(rng, coords, [8, 7, 6, 1], specs, 9, "esp")
    pts = _points_away(rng, mol, 128, rmin=1.0)
    return mol, pts


def case_mixed():
    """Pure g, Cartesian and pure f, Cartesian and pure d, generalised s+p and
    d+5d shells -- every type whose first derivatives the reference gets right
    (its Cartesian-g first derivatives are defective), so every descriptor is
    pinned."""
    rng = np.random.default_rng(14)
    coords = np.array([[0.0, 0.0, 0.0], [1.7, -0.5, 0.9], [-1.1, 1.2, -0.4], [0.6, 1.9, 1.3]])
    specs = [(0, [0], 4), (0, [0, 1], 3), (0, [2], 2), (0, [-3], 2), (0, [-4], 2), (1, [0], 3),
             (1, [1], 2), (1, [2, -2], 2), (1, [3], 2), (1, [-4], 1), (2, [0], 3), (2, [1], 2),
             (2, [-2], 1), (3, [0], 2), (3, [1], 1)]
    mol = _molecule(rng, coords, [8, 6, 7, 1], specs, 14, "mixed")
    pts = _points_away(rng, mol, 192, rmin=0.05)
    return mol, pts


CASES = {"allshell": case_allshell, "c1": case_c1, "esp": case_esp, "mixed": case_mixed}
# Reference calls made for every case; ESP only where the basis has no g shell.
LOCAL_FUNCS = ["density", "gradient", "hessian", "laplacian", "tau_pd", "tau_general", "rdg",
               "shannon", "weizsacker", "thomas_fermi", "gge", "general_ked", "ao_deriv",
               "ao_sec_deriv", "ao_laplacian"]
ESP_CASES = {"c1", "esp"}
CUBIC_CASES = {"c1", "allshell"}
TAU_ALPHA = 0.5
GGE_AB = (0.2, 1.0 / 6.0)
GENERAL_KED_A = 0.3
CUBE_SHAPE = (5, 6, 7)


def cube_for(mol):
    origin = mol.coords.min(0) - 1.5
    axes = np.array([[0.61, 0.0, 0.0], [0.05, 0.55, 0.0], [0.0, -0.03, 0.58]])
    return origin, axes
