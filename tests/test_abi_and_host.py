"""CPU tests: the C ABI library loads and exports every declared symbol, the
pybind11 module exposes the reference's method names, and host-side logic
(synthetic inputs, tables) behaves."""
import ctypes as C
import os

import numpy as np
import pytest

import ctc_abi
from chemtoolscuda_b200 import synthetic as S


def test_library_exports_every_header_symbol():
    syms = ctc_abi.header_symbols()
    assert len(syms) >= 15
    lib = C.CDLL(ctc_abi.LIB)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, f"symbols declared in include/chemtools_cuda.h but not exported: {missing}"


def test_version_and_error_strings_without_gpu():
    L = ctc_abi.lib()
    assert b"sm_100a" in L.ctc_version()
    # invalid arguments are rejected on the host before any CUDA call
    assert L.ctc_eval_local(None, None, 0, 0, None, None, None) == -1
    assert b"null" in L.ctc_last_error()
    assert L.ctc_molecule_create(None, 0, None, None, None, 0, None) == -1


REFERENCE_BOUND = [  # src/pybind.cpp:15-304
    "compute_density", "compute_gradient", "compute_hessian", "compute_laplacian",
    "compute_positive_definite_kinetic_energy_density", "compute_general_kinetic_energy_density",
    "compute_norm_of_vector", "compute_reduced_density_gradient", "compute_weizsacker_ked",
    "compute_thomas_fermi_ked", "compute_general_gradient_expansion_ked",
    "compute_gradient_expansion_ked", "compute_empirical_gradient_expansion_ked",
    "compute_general_ked", "compute_schrodinger_ked", "compute_shannon_information_density",
    "compute_electrostatic_potential", "coordinates", "numbers", "get_file_path"]
README_NAMES = [  # names used by the reference's README and tests
    "compute_electron_density", "compute_electron_density_gradient",
    "compute_electron_density_hessian", "compute_laplacian_electron_density",
    "compute_electron_density_on_cubic_grid", "basis_set_to_constant_memory",
    "compute_local_descriptors"]


def test_python_api_surface():
    from chemtoolscuda_b200 import Molecule
    for name in REFERENCE_BOUND + README_NAMES:
        assert hasattr(Molecule, name), name


def test_synthetic_generator_is_deterministic():
    a = S.make_molecule("c1", seed=3)
    b = S.make_molecule("c1", seed=3)
    np.testing.assert_array_equal(a.coords, b.coords)
    np.testing.assert_array_equal(a.D, b.D)
    fa, fb = a.flat(), b.flat()
    for k in fa:
        np.testing.assert_array_equal(fa[k], fb[k])
    d = np.linalg.norm(a.coords[:, None] - a.coords[None], axis=-1) + np.eye(len(a.coords)) * 99
    assert d.min() >= 1.8
    # D = 2 C C^T with orthonormal C: symmetric, eigenvalues 0 or 2
    w = np.linalg.eigvalsh(a.D)
    assert np.allclose(np.sort(w)[-20:], 2.0) and np.allclose(np.sort(w)[:-20], 0.0, atol=1e-12)


def test_config_sizes():
    sizes = {c: S.make_molecule(c, seed=0).nbasis for c in ("c1", "c3", "c5")}
    assert 100 <= sizes["c1"] <= 200
    assert 500 <= sizes["c3"] <= 1000
    assert 1100 <= sizes["c5"] <= 1900


def test_cube_points_order_matches_reference():
    # point (i, j, k) = origin + i a0 + j a1 + k a2, k fastest (src/evaluate_density.cu:433-447)
    o = np.array([0.1, -0.2, 0.3])
    ax = np.array([[0.5, 0.0, 0.1], [0.0, 0.4, 0.0], [0.05, 0.0, 0.3]])
    p = S.cube_points(o, ax, (2, 3, 4))
    assert p.shape == (24, 3)
    np.testing.assert_allclose(p[1], o + ax[2])
    np.testing.assert_allclose(p[4], o + ax[1])
    np.testing.assert_allclose(p[12], o + ax[0])


def test_becke_partition_of_unity():
    mol = S.make_molecule("c1", seed=0, natom=3, box=4.0)
    rng = np.random.default_rng(0)
    pts = rng.uniform(-2, 6, size=(50, 3))
    w = sum(S._becke_weights(pts, mol.coords, a) for a in range(3))
    np.testing.assert_allclose(w, 1.0, atol=1e-12)


def test_surface_points_outside_other_spheres():
    mol = S.make_molecule("c5", seed=1, natom=6, box=6.0)
    pts = S.surface_points(mol, seed=2, scales=(1.4,), density=2.0)
    rad = np.where(mol.numbers == 1, 2.3, 3.2) * 1.4
    d = np.linalg.norm(pts[:, None] - mol.coords[None], axis=-1)
    assert (d >= rad[None] - 1e-6).all()
