"""Seeded synthetic molecules, density matrices and point sets.

The reference reads molecules from Gaussian fchk files through the Python
``iodata`` package (``src/iodata.cpp:15-211``).  The workloads used by the
tests and the benchmark are synthetic, so this module builds them directly in
the reference's data model (``include/contracted_shell.h:39-77``): a list of
contracted shells, each with a centre, shared exponents and one coefficient
vector per segment, where a segment's angular momentum follows the fchk
convention (0 s, 1 p, 2 Cartesian d, -2 pure d, 3/-3 f, 4/-4 g).

The flat array layout returned by :func:`flatten_basis` is the one the C ABI
(``include/chemtools_cuda.h``) takes.  Everything is seeded with
``numpy.random.default_rng`` so every run sees identical inputs.
"""
from __future__ import annotations

from dataclasses import dataclass, field
import math

import numpy as np

# Number of functions per segment, keyed by the fchk angular momentum code
# (``include/contracted_shell.h:10-37``).
NFUNC = {0: 1, 1: 3, 2: 6, -2: 5, 3: 10, -3: 7, 4: 15, -4: 9}


def nfunc(angmom: int) -> int:
    return NFUNC[int(angmom)]


@dataclass
class Shell:
    """One generalised-contraction shell (mirrors ``GeneralizedContractionShell``)."""

    center: np.ndarray            # (3,)
    atom: int                     # index of the atom the shell sits on
    angmoms: list[int]            # one entry per segment
    exponents: np.ndarray         # (K,)
    coeffs: np.ndarray            # (nseg, K), coefficients of normalised primitives


@dataclass
class SyntheticMolecule:
    coords: np.ndarray            # (natom, 3) bohr
    numbers: np.ndarray           # (natom,) atomic numbers
    charges: np.ndarray           # (natom,) nuclear charges used by the ESP
    shells: list[Shell]
    D: np.ndarray                 # (M, M) symmetric one-particle density matrix
    name: str = "synthetic"
    meta: dict = field(default_factory=dict)

    @property
    def nbasis(self) -> int:
        return sum(nfunc(a) for s in self.shells for a in s.angmoms)

    def flat(self) -> dict:
        return flatten_basis(self.shells)


def flatten_basis(shells: list[Shell]) -> dict:
    """Pack shells into the flat arrays the C ABI consumes.

    ``coeffs`` is stored segment-major per shell: shell s with K primitives
    and S segments occupies ``coeffs[off : off + S*K]`` with element
    ``seg * K + k``.
    """
    centers = np.array([s.center for s in shells], dtype=np.float64).reshape(-1, 3)
    atom = np.array([s.atom for s in shells], dtype=np.int32)
    nprim = np.array([len(s.exponents) for s in shells], dtype=np.int32)
    nseg = np.array([len(s.angmoms) for s in shells], dtype=np.int32)
    angmoms = np.array([a for s in shells for a in s.angmoms], dtype=np.int32)
    exps = np.concatenate([np.asarray(s.exponents, np.float64) for s in shells])
    coeffs = np.concatenate([np.asarray(s.coeffs, np.float64).reshape(-1) for s in shells])
    return dict(centers=np.ascontiguousarray(centers), shell_atom=atom, nprim=nprim,
                nseg=nseg, angmoms=angmoms, exps=exps, coeffs=coeffs)


def _dfact(n: int) -> float:
    """(n)!! with (-1)!! = 1."""
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def _normalise_contraction(l: int, exps: np.ndarray, c: np.ndarray) -> np.ndarray:
    """Rescale coefficients of normalised primitives to a unit-norm contraction.

    The overlap of two normalised primitive Gaussians of the same angular
    component is (2 sqrt(a b) / (a + b))^(l + 3/2).
    """
    a = exps[:, None]
    b = exps[None, :]
    S = (2.0 * np.sqrt(a * b) / (a + b)) ** (l + 1.5)
    nrm = float(c @ S @ c)
    return c / math.sqrt(nrm)


def _place_atoms(rng, natom: int, box: float, min_sep: float) -> np.ndarray:
    coords = []
    tries = 0
    while len(coords) < natom:
        tries += 1
        if tries > 2_000_000:
            raise RuntimeError("could not place atoms with the requested separation")
        p = rng.uniform(0.0, box, size=3)
        if coords:
            d = np.linalg.norm(np.asarray(coords) - p, axis=1)
            if d.min() < min_sep:
                continue
        coords.append(p)
    return np.asarray(coords, dtype=np.float64)


# Shell recipes per configuration: element -> list of segment angular momenta
# (one segmented shell per entry).
RECIPES = {
    "c1": {1: [0, 0, 1], 6: [0, 0, 0, 1, 1, 2], 8: [0, 0, 0, 1, 1, 2]},
    "c2": {1: [0, 0, 1], 6: [0, 0, 1, 1, -2], 8: [0, 0, 1, 1, -2, -3]},
    # c3: three p shells on heavy atoms bring 60 atoms to ~800 functions (807 at seed 0)
    "c3": {1: [0, 0, 1], 6: [0, 0, 0, 1, 1, 1, 2], 8: [0, 0, 0, 1, 1, 1, 2]},
    "c4": {1: [0, 0, 1], 6: [0, 0, 1, 1, 2], 8: [0, 0, 1, 1, 2, 4]},
    "c5": {1: [0, 0, 1], 6: [0, 0, 0, 1, 1, 2, 2], 8: [0, 0, 0, 1, 1, 2, 2]},
}


def make_basis(rng, coords, numbers, recipe, kmin=3, kmax=6, emin=0.08, emax=5e3,
               generalised=False) -> list[Shell]:
    """Draw one contracted shell per recipe entry on every atom.

    Exponents are log-uniform in [emin, emax]; coefficients are N(0, 1) and
    then rescaled to unit self-overlap.  With ``generalised=True`` the s and
    p segments of an atom that share a primitive count are merged into one
    generalised-contraction shell (shared exponents), which exercises the
    reference's multi-segment shell layout.
    """
    shells: list[Shell] = []
    for ia, (xyz, z) in enumerate(zip(coords, numbers)):
        for am in recipe[int(z)]:
            K = int(rng.integers(kmin, kmax + 1))
            e = np.sort(np.exp(rng.uniform(math.log(emin), math.log(emax), size=K)))[::-1].copy()
            c = rng.standard_normal(K)
            c = _normalise_contraction(abs(am), e, c)
            if generalised and am == 1 and shells and shells[-1].atom == ia and \
                    shells[-1].angmoms == [0] and len(shells[-1].exponents) == K:
                prev = shells[-1]
                c = _normalise_contraction(1, prev.exponents, rng.standard_normal(K))
                prev.angmoms.append(1)
                prev.coeffs = np.vstack([prev.coeffs, c[None, :]])
                continue
            shells.append(Shell(center=xyz.copy(), atom=ia, angmoms=[am], exponents=e,
                                coeffs=c[None, :]))
    return shells


def make_density_matrix(rng, M: int, nocc: int, device: str | None = None) -> np.ndarray:
    """D = 2 C C^T with C an M x nocc block with orthonormal columns.

    With ``device`` (a torch device string) the QR and the product run there in
    float64 -- the same matrices up to rounding, much faster for M ~ 16 000.
    """
    nocc = min(nocc, M)
    G = rng.standard_normal((M, nocc))
    if device is not None:
        import torch
        Ct, _ = torch.linalg.qr(torch.as_tensor(G, device=device))
        Dt = 2.0 * (Ct @ Ct.T)
        Dt = 0.5 * (Dt + Dt.T)
        return Dt.cpu().numpy()
    C, _ = np.linalg.qr(G)
    D = 2.0 * (C @ C.T)
    return 0.5 * (D + D.T)


def _ao_atom_index(shells: list[Shell]) -> np.ndarray:
    idx = []
    for s in shells:
        for a in s.angmoms:
            idx += [s.atom] * nfunc(a)
    return np.asarray(idx, dtype=np.int64)


def make_molecule(config: str = "c1", seed: int = 0, natom: int | None = None,
                  box: float | None = None, nocc: int | None = None,
                  generalised: bool = False, cutoff: float | None = None,
                  device: str | None = None) -> SyntheticMolecule:
    """Build the synthetic molecule of one benchmark configuration.

    c1: 12 atoms in an 8 bohr box, Cartesian up to d, ~140 functions, 20 occupied.
    c2: 200 atoms in a 25 bohr box, pure d and f, ~2 500 functions, 400 occupied.
    c3: 60 atoms in a 16 bohr box, Cartesian up to d, ~800 functions.
    c4: 1 000 atoms at 0.01 atoms/bohr^3, Cartesian up to g, ~16 000 functions,
        D zeroed beyond 12 bohr between centres.
    c5: 100 atoms in an 18 bohr box, Cartesian up to d, ~1 500 functions.
    """
    defaults = {
        "c1": dict(natom=12, box=8.0, nocc=20),
        "c2": dict(natom=200, box=25.0, nocc=400),
        "c3": dict(natom=60, box=16.0, nocc=120),
        "c4": dict(natom=1000, box=(1000 / 0.01) ** (1 / 3), nocc=2500, cutoff=12.0),
        "c5": dict(natom=100, box=18.0, nocc=200),
    }[config]
    natom = defaults["natom"] if natom is None else natom
    box = defaults["box"] if box is None else box
    nocc = defaults["nocc"] if nocc is None else nocc
    if cutoff is None:
        cutoff = defaults.get("cutoff")
    rng = np.random.default_rng(seed)
    coords = _place_atoms(rng, natom, box, 1.8)
    numbers = rng.choice(np.array([1, 6, 8]), size=natom)
    shells = make_basis(rng, coords, numbers, RECIPES[config], generalised=generalised)
    M = sum(nfunc(a) for s in shells for a in s.angmoms)
    D = make_density_matrix(rng, M, nocc, device=device)
    if cutoff is not None:
        at = _ao_atom_index(shells)
        adist = np.linalg.norm(coords[:, None, :] - coords[None, :, :], axis=-1)
        D[(adist > cutoff)[np.ix_(at, at)]] = 0.0
    return SyntheticMolecule(coords=coords, numbers=numbers.astype(np.int32),
                             charges=numbers.astype(np.float64), shells=shells, D=D,
                             name=config, meta=dict(seed=seed, box=box, nocc=nocc))


def random_points(rng, mol: SyntheticMolecule, n: int, pad: float = 4.0) -> np.ndarray:
    """Points uniform in the molecule's bounding box padded by ``pad`` bohr."""
    lo = mol.coords.min(axis=0) - pad
    hi = mol.coords.max(axis=0) + pad
    return np.ascontiguousarray(rng.uniform(lo, hi, size=(n, 3)))


def cube_grid(mol: SyntheticMolecule, spacing: float, shape: tuple[int, int, int]):
    """Origin and axes of an axis-aligned cube grid centred on the molecule.

    Point (i, j, k) sits at origin + i*axes[0] + j*axes[1] + k*axes[2], k
    fastest (the reference's cubic-grid order, ``src/evaluate_density.cu:433-447``).
    """
    centre = 0.5 * (mol.coords.min(axis=0) + mol.coords.max(axis=0))
    extent = spacing * (np.asarray(shape) - 1)
    origin = centre - 0.5 * extent
    axes = np.eye(3) * spacing
    return origin, axes


def cube_points(origin, axes, shape) -> np.ndarray:
    i, j, k = np.meshgrid(np.arange(shape[0]), np.arange(shape[1]), np.arange(shape[2]),
                          indexing="ij")
    idx = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64)
    return np.ascontiguousarray(origin[None, :] + idx @ np.asarray(axes))


def _fibonacci_sphere(n: int, rng) -> np.ndarray:
    k = np.arange(n) + 0.5
    phi = np.arccos(1.0 - 2.0 * k / n)
    theta = math.pi * (1.0 + 5 ** 0.5) * k + rng.uniform(0, 2 * math.pi)
    return np.stack([np.cos(theta) * np.sin(phi), np.sin(theta) * np.sin(phi), np.cos(phi)], 1)


def surface_points(mol: SyntheticMolecule, seed: int = 0, scales=(1.4, 1.6, 1.8, 2.0),
                   density: float = 20.0, max_points: int | None = None) -> np.ndarray:
    """Points on nested van-der-Waals-like surfaces (ESP workload).

    Radius 2.3 bohr for H and 3.2 bohr otherwise, scaled by each factor in
    ``scales``; ``density`` points per bohr^2 on every atomic sphere; points
    inside another atom's scaled sphere are removed.
    """
    rng = np.random.default_rng(seed)
    rad = np.where(mol.numbers == 1, 2.3, 3.2)
    out = []
    for s in scales:
        R = rad * s
        for ia in range(len(mol.coords)):
            n = max(8, int(round(4 * math.pi * R[ia] ** 2 * density)))
            p = mol.coords[ia] + R[ia] * _fibonacci_sphere(n, rng)
            d = np.linalg.norm(p[:, None, :] - mol.coords[None, :, :], axis=-1)
            inside = d < (R[None, :] - 1e-9)
            inside[:, ia] = False
            out.append(p[~inside.any(axis=1)])
    pts = np.ascontiguousarray(np.concatenate(out))
    if max_points is not None and len(pts) > max_points:
        sel = rng.choice(len(pts), size=max_points, replace=False)
        pts = np.ascontiguousarray(pts[np.sort(sel)])
    return pts


def submolecule(mol: SyntheticMolecule, natom: int, nocc: int, seed: int = 0) -> SyntheticMolecule:
    """The first ``natom`` atoms of ``mol`` with their shells and a fresh density
    matrix D = 2 C C^T of ``nocc`` occupied columns (seeded)."""
    shells = [sh for sh in mol.shells if sh.atom < natom]
    M = sum(nfunc(a) for sh in shells for a in sh.angmoms)
    D = make_density_matrix(np.random.default_rng(seed), M, nocc)
    return SyntheticMolecule(coords=mol.coords[:natom].copy(), numbers=mol.numbers[:natom].copy(),
                             charges=mol.charges[:natom].copy(), shells=shells, D=D,
                             name=f"{mol.name}[:{natom}]", meta=dict(mol.meta, natom=natom, nocc=nocc))


def reference_esp_fit(mol: SyntheticMolecule, limit_bytes: int = 60000) -> int:
    """Largest number of leading atoms whose basis fits the reference's ESP: its
    segmented basis -- per segment x, y, z, K, l and K exponents and K
    coefficients, plus one header double -- must stay below 60 000 bytes of
    constant memory (src/basis_to_gpu.cu:60-120, src/evaluate_electrostatic.cu:10166-10176)."""
    per_atom = np.zeros(len(mol.coords))
    for sh in mol.shells:
        per_atom[sh.atom] += len(sh.angmoms) * (5 + 2 * len(sh.exponents))
    used, k = 1.0, 0
    for a in range(len(mol.coords)):
        if 8 * (used + per_atom[a]) >= limit_bytes:
            break
        used += per_atom[a]
        k = a + 1
    return k


# The ESP workload asks for 1e6 points on the four nested surfaces of the
# 100-atom molecule; at 20 points per bohr^2 those surfaces hold ~277 000
# points, so the workload samples them at the density that gives ~1e6.
ESP_WORKLOAD_DENSITY = 72.2


def esp_workload_points(mol: SyntheticMolecule, seed: int = 0) -> np.ndarray:
    """The ESP workload's ~1e6 surface points (1.4/1.6/1.8/2.0 x radii)."""
    return surface_points(mol, seed=seed, density=ESP_WORKLOAD_DENSITY)


# --- atom-centred quadrature (adjoint workload) -------------------------------------------------

def _becke_weights(points: np.ndarray, coords: np.ndarray, owner: int) -> np.ndarray:
    """Becke fuzzy-cell weight of ``owner`` at each point (3 smoothing steps)."""
    d = np.linalg.norm(points[:, None, :] - coords[None, :, :], axis=-1)  # (n, A)
    R = np.linalg.norm(coords[:, None, :] - coords[None, :, :], axis=-1)
    A = len(coords)
    P = np.ones((len(points), A))
    for i in range(A):
        for j in range(A):
            if i == j:
                continue
            mu = (d[:, i] - d[:, j]) / R[i, j]
            for _ in range(3):
                mu = 1.5 * mu - 0.5 * mu ** 3
            P[:, i] *= 0.5 * (1.0 - mu)
    return P[:, owner] / P.sum(axis=1)


def atom_grid(mol: SyntheticMolecule, nrad: int = 75, ntheta: int = 14, nphi: int = 22,
              rmax_scale: float = 1.0):
    """Atom-centred product grid with Becke partition weights.

    Radial: Gauss-Chebyshev (second kind) on x in (-1, 1) mapped by
    r = (1 + x) / (1 - x) (Becke's map, scaled by ``rmax_scale``).  Angular:
    Gauss-Legendre in cos(theta) times a uniform rule in phi, i.e.
    ntheta * nphi points per shell (14 * 22 = 308 by default).  Returns
    (points (n, 3), weights (n,)).
    """
    i = np.arange(1, nrad + 1)
    x = np.cos(i * math.pi / (nrad + 1))
    wx = math.pi / (nrad + 1) * np.sin(i * math.pi / (nrad + 1)) ** 2 / np.sqrt(1 - x ** 2)
    r = rmax_scale * (1 + x) / (1 - x)
    dr = rmax_scale * 2.0 / (1 - x) ** 2
    wr = wx * dr * r ** 2
    ct, wt = np.polynomial.legendre.leggauss(ntheta)
    ph = 2 * math.pi * (np.arange(nphi) + 0.5) / nphi
    st = np.sqrt(1 - ct ** 2)
    dirs = np.stack([np.outer(st, np.cos(ph)).ravel(), np.outer(st, np.sin(ph)).ravel(),
                     np.repeat(ct, nphi)], axis=1)
    wang = np.repeat(wt, nphi) * (2 * math.pi / nphi)
    pts_all, w_all = [], []
    for ia in range(len(mol.coords)):
        p = mol.coords[ia] + (r[:, None, None] * dirs[None, :, :]).reshape(-1, 3)
        w = (wr[:, None] * wang[None, :]).ravel()
        w = w * _becke_weights(p, mol.coords, ia)
        pts_all.append(p)
        w_all.append(w)
    return np.ascontiguousarray(np.concatenate(pts_all)), np.concatenate(w_all)
