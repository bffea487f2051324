"""GPU parity of the tensor-core split path (INT8 tcgen05, 5-digit AO and 4-digit D
operands, exact int32 accumulation) against the FP64 oracle.

Stated tolerance: 1e-8 relative to the per-point sum of absolute terms
(tests/helpers.py) for every output slot -- rho, grad rho, Hessian, Laplacian,
tau_PD, tau_alpha, the reduced density gradient, Shannon density, Weizsacker,
Thomas-Fermi, general gradient-expansion and general(ish) kinetic-energy
densities -- the accuracy bound the split path is built to.  The ratio-type
outputs (RDG, Shannon, W, TF, GGE) are compared where rho > 1e-10, as the
reference's own tests mask RDG (tests/test_density.py of the reference masks
rho < 1e-12)."""
import os

import numpy as np
import pytest

import ctc_abi
from helpers import assert_close, term_scales
from oracle import oracle as O
from chemtoolscuda_b200 import synthetic as S

pytestmark = pytest.mark.gpu
TC_RTOL = 1e-8
KEYS = ctc_abi.OUT_KEYS
# tau_alpha alpha, gge (a, b), general(ish) KED a
PARAMS = (0.5, 0.2, 1 / 6, 0.3)
MASKED = ("rdg", "shannon", "weizsacker", "thomas_fermi", "gge")


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


def _oracle(mol, pts, keys):
    a, ga, gb, ka = PARAMS
    okeys = tuple(dict.fromkeys(tuple(keys) + ("rho", "grad")))
    ref = O.eval_local(mol.flat(), mol.D, pts, alpha=a, keys=okeys, gge_ab=(ga, gb), ked_a=ka)
    sc = term_scales(mol.flat(), mol.D, pts, alpha=a, gge=(ga, gb), ked_a=ka,
                     ref=dict(ref, rdg=ref.get("rdg", np.ones_like(ref["rho"]))))
    return ref, sc


def _compare(tag, got, ref, sc, keys, rtol=TC_RTOL):
    live = ref["rho"] > 1e-10
    for k in keys:
        assert_close(f"{tag}/{k} (tc)", got[k], ref[k], sc[k], rtol, atol=1e-15,
                     mask=live if k in MASKED else None)


def _check(mol, pts, keys=KEYS, rtol=TC_RTOL):
    m = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
    got = m.eval_local(pts, keys, ctc_abi.PREC_TC, params=PARAMS)
    ref, sc = _oracle(mol, pts, keys)
    _compare(mol.name, got, ref, sc, keys, rtol)
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


def test_tc_headline_configuration_full_size():
    """The benchmark's own step at full size: the 200-atom molecule (pure d and
    f shells, M = 2 655, D = 2 C C^T with 400 occupied columns) on the 215^3
    cube at 0.2 bohr (9 938 375 points), every output slot on the tensor-core
    path through ctc_eval_cubic, checked against the FP64 oracle on 2 000
    sampled grid points (half of them where rho > 1e-4, half anywhere)."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    mol = S.make_molecule("c2", seed=0)
    shape = (215, 215, 215)
    origin, axes = S.cube_grid(mol, 0.2, shape)
    n = int(np.prod(shape))
    m = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
    rng = np.random.default_rng(2024)
    anywhere = rng.choice(n, 4000, replace=False)
    probe = m.eval_cubic(origin, axes, shape, keys=("rho",), precision=ctc_abi.PREC_TC,
                         params=PARAMS, index=anywhere)["rho"]
    dense = anywhere[probe > 1e-4][:1000]
    idx = np.concatenate([dense, anywhere[:2000 - len(dense)]])
    got = m.eval_cubic(origin, axes, shape, keys=KEYS, precision=ctc_abi.PREC_TC, params=PARAMS,
                       index=idx)
    m.close()
    pts = S.cube_points(origin, axes, shape)[idx]
    ref, sc = _oracle(mol, pts, KEYS)
    _compare("c2 headline 215^3", got, ref, sc, KEYS)


@pytest.mark.parametrize("precision", [ctc_abi.PREC_FP64, ctc_abi.PREC_TC], ids=["fp64", "tc"])
def test_capacity_prepass_matches_default_workspace(torch_cuda, precision):
    """A small chunk budget (CTC_CHUNK_BYTES) makes the pipeline size its tile
    workspaces by a count-only screening pass (the largest compact AO set of
    the call) instead of the whole basis; results must not change, on random
    points (Morton tiles) and on a cubic grid."""
    mol = S.make_molecule("c2", seed=4, natom=40, box=12.0, nocc=80)
    rng = np.random.default_rng(8)
    pts = S.random_points(rng, mol, 12000, pad=2.0)
    origin, axes = S.cube_grid(mol, 0.3, (24, 26, 28))
    keys = ("rho", "grad", "hess", "lap", "tau_pd")
    m = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
    base = m.eval_local(pts, keys, precision)
    cbase = m.eval_cubic(origin, axes, (24, 26, 28), keys=keys, precision=precision)
    os.environ["CTC_CHUNK_BYTES"] = str(8 << 20)
    try:
        small = m.eval_local(pts, keys, precision)
        csmall = m.eval_cubic(origin, axes, (24, 26, 28), keys=keys, precision=precision)
    finally:
        del os.environ["CTC_CHUNK_BYTES"]
    assert m.sync_status() == 0
    for k in keys:
        np.testing.assert_allclose(small[k], base[k], rtol=1e-13, atol=1e-16, err_msg=k)
        np.testing.assert_allclose(csmall[k], cbase[k], rtol=1e-13, atol=1e-16, err_msg=k)
    ref, sc = _oracle(mol, pts[:300], keys)
    _compare("prepass", {k: v[:300] for k, v in small.items()}, ref, sc, keys,
             1e-10 if precision == ctc_abi.PREC_FP64 else TC_RTOL)
    m.close()


def test_tc_near_nuclei_headline_molecule(torch_cuda):
    """Points 0.003 - 0.5 bohr from nuclei of the 200-atom benchmark molecule,
    where the tightest functions dominate both operands: AO rows with one steep
    function and D rows whose largest entry is a core element.  With four D
    digits (31 bits) the Hessian reached 2.8e-8 here; five digits keep every
    output within 1e-8."""
    mol = S.make_molecule("c2", seed=0)
    rng = np.random.default_rng(3)
    at = rng.integers(0, len(mol.coords), 300)
    dirs = rng.normal(size=(300, 3))
    dirs /= np.linalg.norm(dirs, axis=1)[:, None]
    r = np.exp(rng.uniform(np.log(0.003), np.log(0.5), 300))
    pts = mol.coords[at] + dirs * r[:, None]
    _check(mol, pts)
