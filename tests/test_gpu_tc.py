"""GPU parity of the tensor-core split path (INT8 tcgen05, 5-digit AO and 4-digit D
operands, exact int32 accumulation) against the FP64 oracle.

Stated tolerance: 1e-8 relative to the per-point sum of absolute terms
(tests/helpers.py) for rho, grad rho, Hessian, Laplacian, tau_PD and
tau_alpha -- the accuracy bound the split path is built to; its measured
error on the 200-atom molecule is ~2e-9."""
import os

import numpy as np
import pytest

import ctc_abi
from helpers import assert_close, term_scales
from oracle import oracle as O
from chemtoolscuda_b200 import synthetic as S

pytestmark = pytest.mark.gpu
TC_RTOL = 1e-8
KEYS = ("rho", "grad", "hess", "lap", "tau_pd", "tau_alpha")


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _cases():
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import cases
    return cases


def _check(mol, pts, keys=KEYS, rtol=TC_RTOL):
    m = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
    got = m.eval_local(pts, keys, ctc_abi.PREC_TC, params=(0.5, 1 / 9, 1 / 6, 1.0))
    ref = O.eval_local(mol.flat(), mol.D, pts, alpha=0.5, keys=tuple(k for k in keys if k in O.LOCAL_KEYS))
    sc = term_scales(mol.flat(), mol.D, pts, alpha=0.5)
    for k in keys:
        assert_close(f"{mol.name}/{k} (tc)", got[k], ref[k], sc[k], rtol, atol=1e-15)
    return got


@pytest.mark.parametrize("case", ["allshell", "c1", "esp", "mixed"])
def test_tc_all_descriptors_vs_oracle(torch_cuda, case):
    mol, pts = _cases().CASES[case]()
    _check(mol, pts)


@pytest.mark.parametrize("case", ["c1", "mixed"])
def test_tc_density_only_variant(torch_cuda, case):
    mol, pts = _cases().CASES[case]()
    _check(mol, pts, keys=("rho", "grad"))


@pytest.mark.parametrize("case", ["allshell", "mixed"])
def test_tc_first_derivative_rows_variant(torch_cuda, case):
    """tau_PD without second-derivative outputs: 32-point tiles of phi and
    grad phi rows over an AO block of value and first derivatives only."""
    mol, pts = _cases().CASES[case]()
    _check(mol, pts, keys=("rho", "grad", "tau_pd"))


def test_tc_density_only_rows(torch_cuda):
    mol, pts = _cases().CASES["allshell"]()
    _check(mol, pts, keys=("rho",))


def test_tc_large_molecule_slice(torch_cuda):
    """60 atoms of the 200-atom generator (pure d and f), cube points."""
    mol = S.make_molecule("c2", seed=4, natom=60, box=14.0, nocc=120)
    origin, axes = S.cube_grid(mol, 0.2, (70, 70, 70))
    rng = np.random.default_rng(3)
    pts = S.cube_points(origin, axes, (70, 70, 70))[rng.choice(70 ** 3, 600, replace=False)]
    _check(mol, pts)


@pytest.mark.parametrize("natom,seed", [(150, 0), (60, 5)])
def test_tc_cartesian_g_cutoff_molecule(torch_cuda, natom, seed):
    """Molecules of the 1000-atom generator at its density (Cartesian up to g,
    D zeroed beyond 12 bohr), points within ~1 bohr of the atoms: AO rows with
    one steep g function and many small entries, the case that needs the
    fifth digit of the A operand (31-bit rows gave 2e-8 here)."""
    mol = S.make_molecule("c4", seed=seed, natom=natom, box=(natom / 0.01) ** (1 / 3))
    rng = np.random.default_rng(seed)
    pts = mol.coords[rng.integers(0, len(mol.coords), 96)] + rng.normal(0, 1.0, (96, 3))
    _check(mol, pts)


def test_tc_matches_fp64_path_on_cube(torch_cuda):
    mol, _ = _cases().CASES["c1"]()
    m = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
    origin, axes = _cases().cube_for(mol)
    shape = (9, 11, 13)
    tc = m.eval_cubic(origin, axes, shape, keys=("rho",), precision=ctc_abi.PREC_TC)
    fp = m.eval_cubic(origin, axes, shape, keys=("rho",), precision=ctc_abi.PREC_FP64)
    pts = S.cube_points(origin, axes, shape)
    sc = term_scales(mol.flat(), mol.D, pts)
    assert_close("cube rho tc vs fp64", tc["rho"], fp["rho"], sc["rho"], TC_RTOL, 1e-15)
