"""B200-native grid evaluation of Gaussian-basis density descriptors.

``chemtools_cuda`` is the pybind11 module with the reference's ``Molecule``
API; the sm_100a kernels behind it live in ``libchemtools_cuda.so`` (C ABI in
``include/chemtools_cuda.h``).  Importing fails loudly when the native library
has not been built (``python chemtoolscuda_b200/build.py``): there is no CPU
fallback.
"""
from __future__ import annotations

import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libchemtools_cuda.so")

try:
    from . import _chemtools_cuda as chemtools_cuda  # noqa: F401
except ImportError as e:  # pragma: no cover - exercised only without a build
    raise ImportError(
        "chemtoolscuda_b200: native extension not built; run `python chemtoolscuda_b200/build.py` "
        f"({e})") from e

Molecule = chemtools_cuda.Molecule


def molecule_from_synthetic(mol, path: str = "") -> "Molecule":
    """Build a :class:`Molecule` from a :class:`synthetic.SyntheticMolecule`."""
    f = mol.flat()
    return Molecule.from_arrays(f["centers"], f["shell_atom"], f["nprim"], f["nseg"], f["angmoms"],
                                f["exps"], f["coeffs"], mol.coords, mol.charges, mol.D,
                                numbers=mol.numbers, path=path)
