"""The reference's own fixture molecules (its tests/data/*.fchk: atoms H to Kr,
pure f and g shells, CH4, H2O, a QM9 molecule, a 14-atom Cartesian-d
molecule) on the GPU, against what the reference's CUDA drivers returned on
the same molecules and points (tests/golden/fixtures, written by
make_fixture_golden.py) and against the FP64 oracle.

Tolerances: FP64 path 1e-10 relative to the per-point sum of absolute terms
(1e-12 absolute where rho < 1e-12); tensor-core split path 1e-8; RDG where
rho > 1e-10; ESP 1e-10 relative to the sum of the absolute nuclear and
electronic parts (the potential nearly cancels far from a neutral molecule,
where a relative error of |V| alone says nothing), where the reference could
run it."""
import glob
import os

import numpy as np
import pytest

import ctc_abi
from helpers import assert_close, term_scales
from oracle import oracle as O

pytestmark = pytest.mark.gpu
FIXTURES = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "fixtures", "*.npz")))
PAIRS = dict(rho="ref_density", grad="ref_gradient", hess="ref_hessian", lap="ref_laplacian",
             tau_pd="ref_tau_pd", tau_alpha="ref_tau_general", rdg="ref_rdg")


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def esp_scale(g):
    """|nuclear part| + |electronic part| of the reference's ESP at each point."""
    pts = g["in_points"]
    nuc = np.array([(g["in_charges"] / np.linalg.norm(g["in_coords"] - p, axis=1)).sum() for p in pts])
    return np.abs(nuc) + np.abs(nuc - g["ref_esp"])


def _load(path):
    g = dict(np.load(path))
    if "ref_density" not in g:
        pytest.skip(f"{os.path.basename(path)}: reference outputs not generated")
    flat = {k[3:]: g[k] for k in ("in_centers", "in_shell_atom", "in_nprim", "in_nseg",
                                   "in_angmoms", "in_exps", "in_coeffs")}
    return g, flat


@pytest.mark.parametrize("precision,rtol", [(ctc_abi.PREC_FP64, 1e-10), (ctc_abi.PREC_TC, 1e-8)],
                         ids=["fp64", "tc"])
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_fixture_molecule_vs_reference(torch_cuda, path, precision, rtol):
    g, flat = _load(path)
    pts = g["in_points"]
    a = float(g["meta_tau_alpha"])
    keys = tuple(k for k, rk in PAIRS.items() if rk in g)
    m = ctc_abi.Mol(flat, g["in_coords"], g["in_charges"], g["in_D"])
    got = m.eval_local(pts, keys, precision, params=(a, 1 / 9, 1 / 6, 1.0))
    oref = O.eval_local(flat, g["in_D"], pts, alpha=a, keys=keys)
    sc = term_scales(flat, g["in_D"], pts, alpha=a, ref=oref)
    rho = g["ref_density"]
    tiny = rho < 1e-12
    for k in keys:
        ref = g[PAIRS[k]].reshape(got[k].shape)
        if k == "rdg":
            assert_close(f"{k} vs reference", got[k], ref, sc[k], rtol, 1e-15, mask=rho > 1e-10)
            assert_close(f"{k} vs oracle", got[k], oref[k], sc[k], rtol, 1e-15, mask=rho > 1e-10)
            continue
        shp = (-1,) + (1,) * (ref.ndim - 1)
        tol = np.where(tiny.reshape(shp), 0.0, rtol * sc[k]) + np.where(tiny, 1e-12, 1e-15).reshape(shp)
        assert_close(f"{k} vs reference", got[k], ref, tol, 1.0)
        assert_close(f"{k} vs oracle", got[k], oref[k], tol, 1.0)
    if precision == ctc_abi.PREC_FP64 and "ref_esp" in g:
        e = m.eval_esp(pts)
        assert_close("esp vs reference", e, g["ref_esp"], esp_scale(g), 1e-10)
    m.close()
