"""Gaussian cube files: write a scalar field on a cubic grid, read one back.

The layout is the one Gaussian's cubegen writes and visualisers read: two
comment lines; the atom count and the grid origin; for each of the three axes
the number of points and the step vector; one line per atom (atomic number,
charge, x, y, z); then the values with the last index running fastest, six per
line.  All lengths in bohr.  The grid order is that of
``Molecule.compute_electron_density_on_cubic_grid`` (point (i, j, k) at
origin + i a0 + j a1 + k a2, k fastest), so its output can be written as is.
"""
from __future__ import annotations

import numpy as np


def write_cube(path: str, values, origin, axes, shape, atom_numbers, atom_coords, atom_charges=None,
               comments=("chemtoolscuda_b200", "scalar field")) -> None:
    values = np.asarray(values, dtype=np.float64).reshape(-1)
    shape = tuple(int(n) for n in shape)
    if values.size != shape[0] * shape[1] * shape[2]:
        raise ValueError(f"{values.size} values for a {shape} grid")
    origin = np.asarray(origin, dtype=np.float64).reshape(3)
    axes = np.asarray(axes, dtype=np.float64).reshape(3, 3)
    nums = np.asarray(atom_numbers).reshape(-1)
    xyz = np.asarray(atom_coords, dtype=np.float64).reshape(-1, 3)
    charges = nums.astype(np.float64) if atom_charges is None else np.asarray(atom_charges, np.float64)
    lines = [str(comments[0])[:80], str(comments[1])[:80],
             f"{len(nums):5d}{origin[0]:12.6f}{origin[1]:12.6f}{origin[2]:12.6f}"]
    for n, a in zip(shape, axes):
        lines.append(f"{n:5d}{a[0]:12.6f}{a[1]:12.6f}{a[2]:12.6f}")
    for z, q, r in zip(nums, charges, xyz):
        lines.append(f"{int(z):5d}{q:12.6f}{r[0]:12.6f}{r[1]:12.6f}{r[2]:12.6f}")
    # rows of the last axis, six values per line, as cubegen writes them
    body = []
    rows = values.reshape(shape[0] * shape[1], shape[2])
    for row in rows:
        for i in range(0, shape[2], 6):
            body.append("".join(f"{v:13.5E}" for v in row[i:i + 6]))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
        fh.write("\n".join(body) + "\n")


def read_cube(path: str) -> dict:
    with open(path) as fh:
        lines = fh.read().splitlines()
    head = lines[2].split()
    natom = abs(int(head[0]))
    origin = np.array([float(v) for v in head[1:4]])
    shape, axes = [], []
    for i in range(3):
        t = lines[3 + i].split()
        shape.append(int(t[0]))
        axes.append([float(v) for v in t[1:4]])
    atoms = [lines[6 + a].split() for a in range(natom)]
    vals = np.array(" ".join(lines[6 + natom:]).split(), dtype=np.float64)
    return dict(origin=origin, axes=np.array(axes), shape=tuple(shape),
                numbers=np.array([int(a[0]) for a in atoms]),
                charges=np.array([float(a[1]) for a in atoms]),
                coords=np.array([[float(v) for v in a[2:5]] for a in atoms]).reshape(-1, 3),
                values=vals.reshape(shape))


def write_density_cube(mol, path: str, origin, axes, shape, precision: str = "fp64") -> np.ndarray:
    """Evaluate the electron density of ``mol`` (a :class:`Molecule`) on the
    cubic grid with the GPU cubic-grid path and write it as a cube file;
    returns the (n0, n1, n2) values written."""
    rho = np.asarray(mol.compute_electron_density_on_cubic_grid(
        np.asarray(origin, np.float64), np.asarray(axes, np.float64),
        np.asarray(shape, np.int32), precision=precision)).reshape(tuple(int(n) for n in shape))
    write_cube(path, rho, origin, axes, shape, mol.numbers, mol.coordinates,
               comments=("chemtoolscuda_b200", f"electron density ({precision})"))
    return rho
