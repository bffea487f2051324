"""GPU parity: the CUDA path, called through the C ABI, against the FP64 oracle
and against the reference's own outputs (tests/golden/).

Tolerances (relative to the per-point sum of absolute terms, tests/helpers.py):
  * FP64 path: 1e-10 (the reference's own tests use 1e-10 abs for AO/grad/Hessian
    and 1e-8 abs for rho/lap/tau/ESP);
  * AO values and derivatives: 1e-12 relative to max |AO| of the point set.
"""
import os

import numpy as np
import pytest

import ctc_abi
from helpers import assert_close, term_scales
from oracle import oracle as O
from chemtoolscuda_b200 import synthetic as S

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
ALL_KEYS = ("rho", "grad", "hess", "lap", "tau_pd", "tau_alpha", "rdg", "shannon")


def _cases():
    import sys
    sys.path.insert(0, GOLDEN)
    import cases
    return cases


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _mol(mol):
    return ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)


@pytest.mark.parametrize("case", ["allshell", "c1", "esp", "mixed"])
@pytest.mark.parametrize("deriv", [0, 1, 2])
def test_ao_values_and_derivatives(torch_cuda, case, deriv):
    mol, pts = _cases().CASES[case]()
    m = _mol(mol)
    got = m.eval_ao(pts, deriv)
    ref = O.eval_ao(mol.flat(), pts, deriv)
    for q in range(ref.shape[0]):
        scale = np.abs(ref[q]).max()
        assert_close(f"{case} AO q={q}", got[q], ref[q], scale, 1e-12)


@pytest.mark.parametrize("case", ["allshell", "c1", "esp", "mixed"])
def test_local_descriptors_fp64_vs_oracle(torch_cuda, case):
    mol, pts = _cases().CASES[case]()
    m = _mol(mol)
    got = m.eval_local(pts, ALL_KEYS, ctc_abi.PREC_FP64, params=(0.5, 1 / 9, 1 / 6, 1.0))
    ref = O.eval_local(mol.flat(), mol.D, pts, alpha=0.5)
    sc = term_scales(mol.flat(), mol.D, pts, alpha=0.5, ref=ref)
    live = ref["rho"] > 1e-10
    for k in ("rho", "grad", "hess", "lap", "tau_pd", "tau_alpha"):
        s = sc[k] if k != "grad" else sc["grad"]
        assert_close(f"{case}/{k}", got[k], ref[k], s, 1e-10, atol=1e-14)
    for k in ("rdg", "shannon"):
        assert_close(f"{case}/{k}", got[k], ref[k], sc[k], 1e-10, atol=1e-14, mask=live)


def test_every_output_slot_and_host_variant(torch_cuda):
    mol, pts = _cases().CASES["c1"]()
    m = _mol(mol)
    keys = ctc_abi.OUT_KEYS
    prm = (0.3, 0.2, 1 / 6, 0.4)
    dev = m.eval_local(pts, keys, ctc_abi.PREC_FP64, params=prm)
    host = m.eval_local_host(pts, keys, ctc_abi.PREC_FP64, params=prm)
    for k in keys:
        np.testing.assert_array_equal(dev[k], host[k], err_msg=k)
    rho, lap, tau = dev["rho"], dev["lap"], dev["tau_pd"]
    g2 = (dev["grad"] ** 2).sum(1)
    np.testing.assert_allclose(dev["tau_alpha"], tau + 0.3 * lap, rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(dev["general_ked"], tau + (0.4 - 1) / 4 * lap, rtol=1e-13, atol=1e-15)
    w = np.where(8 * rho > 1e-20, g2 / (8 * rho), 1e-20)
    np.testing.assert_allclose(dev["weizsacker"], w, rtol=1e-13)
    tf = 0.3 * (3 * np.pi ** 2) ** (2 / 3) * rho ** (5 / 3)
    np.testing.assert_allclose(dev["thomas_fermi"], tf, rtol=1e-13)
    np.testing.assert_allclose(dev["gge"], tf + 0.2 * w + lap / 6, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(np.trace(dev["hess"], axis1=1, axis2=2), lap, rtol=1e-12, atol=1e-14)
    np.testing.assert_array_equal(dev["hess"], np.transpose(dev["hess"], (0, 2, 1)))
    # every slot, derived densities included, against the FP64 oracle with the same parameters
    ref = O.eval_local(mol.flat(), mol.D, pts, alpha=prm[0], keys=tuple(keys), gge_ab=(prm[1], prm[2]),
                       ked_a=prm[3])
    sc = term_scales(mol.flat(), mol.D, pts, alpha=prm[0], gge=(prm[1], prm[2]), ked_a=prm[3], ref=ref)
    live = ref["rho"] > 1e-10
    for k in keys:
        mask = live if k in ("rdg", "shannon", "weizsacker", "thomas_fermi", "gge") else None
        assert_close(f"{k} vs oracle", dev[k].reshape(ref[k].shape), ref[k], sc[k], 1e-10, 1e-14, mask=mask)


def test_subsets_match_full_pass(torch_cuda):
    """Requesting fewer outputs takes cheaper kernel variants; results agree."""
    mol, pts = _cases().CASES["allshell"]()
    m = _mol(mol)
    full = m.eval_local(pts, ("rho", "grad", "hess"))
    only_rho = m.eval_local(pts, ("rho",))
    rho_grad = m.eval_local(pts, ("rho", "grad"))
    tau = m.eval_local(pts, ("tau_pd",))
    sc = term_scales(mol.flat(), mol.D, pts)
    assert_close("rho", only_rho["rho"], full["rho"], sc["rho"], 1e-13, 1e-16)
    assert_close("grad", rho_grad["grad"], full["grad"], sc["grad"], 1e-13, 1e-16)
    ref = O.eval_local(mol.flat(), mol.D, pts, keys=("tau_pd",))
    assert_close("tau", tau["tau_pd"], ref["tau_pd"], sc["tau_pd"], 1e-10, 1e-14)


def test_cubic_grid_matches_points(torch_cuda):
    mol, _ = _cases().CASES["c1"]()
    m = _mol(mol)
    origin, axes = _cases().cube_for(mol)
    shape = (7, 5, 9)
    got = m.eval_cubic(origin, axes, shape, keys=("rho", "grad"))
    pts = S.cube_points(origin, axes, shape)
    ref = O.eval_local(mol.flat(), mol.D, pts, keys=("rho", "grad"))
    sc = term_scales(mol.flat(), mol.D, pts)
    assert_close("cubic rho", got["rho"], ref["rho"], sc["rho"], 1e-10, 1e-14)
    assert_close("cubic grad", got["grad"].reshape(-1, 3), ref["grad"], sc["grad"], 1e-10, 1e-14)


@pytest.mark.parametrize("precision,rtol", [(ctc_abi.PREC_FP64, 1e-10), (ctc_abi.PREC_TC, 1e-8)])
def test_large_explicit_point_call_matches_cubic_grid(torch_cuda, precision, rtol):
    """Calls of 2^18 points or more pack explicit points sort-tile-recursively
    (three sorts over the points' bounding box; smaller calls use one Morton
    sort): the same cube given as explicit points must reproduce the cubic-grid
    call, and a point sample the oracle."""
    mol, _ = _cases().CASES["c1"]()
    m = _mol(mol)
    origin, axes = _cases().cube_for(mol)
    shape = (72, 66, 60)  # 285 120 points
    keys = ("rho", "grad", "lap")
    cub_ = m.eval_cubic(origin, axes, shape, keys=keys, precision=precision)
    pts = S.cube_points(origin, axes, shape)
    assert len(pts) >= 1 << 18
    got = m.eval_local(pts, keys, precision=precision)
    idx = np.random.default_rng(3).choice(len(pts), 400, replace=False)
    ref = O.eval_local(mol.flat(), mol.D, pts[idx], keys=keys)
    sc = term_scales(mol.flat(), mol.D, pts[idx])
    for k in keys:
        g = got[k].reshape(len(pts), -1)
        c = cub_[k].reshape(len(pts), -1)
        assert_close(f"{k} oracle", g[idx].reshape(ref[k].shape), ref[k], sc[k], rtol, 1e-14)
        np.testing.assert_allclose(g, c, rtol=0, atol=rtol * np.abs(c).max())


@pytest.mark.parametrize("case", ["esp", "c1", "allshell"])
def test_esp_vs_oracle(torch_cuda, case):
    mol, pts = _cases().CASES[case]()
    pts = pts[:64]
    m = _mol(mol)
    got = m.eval_esp(pts)
    host = m.eval_esp_host(pts)
    np.testing.assert_array_equal(got, host)
    ref = O.eval_esp(mol.flat(), mol.D, mol.coords, mol.charges, pts)
    nuc = np.array([(mol.charges / np.linalg.norm(mol.coords - p, axis=1)).sum() for p in pts])
    scale = np.abs(nuc) + np.abs(nuc - ref)
    assert_close(f"{case} esp", got, ref, scale, 1e-10)


def test_edge_cases(torch_cuda):
    mol, pts = _cases().CASES["c1"]()
    m = _mol(mol)
    # zero points: no work, no error
    r = m.eval_local(pts[:0], ("rho",))
    assert r["rho"].shape == (0,)
    # one point; a point far outside the molecule (every AO screened -> rho = 0,
    # RDG takes the reference's masked value 1e-20 * prefactor)
    far = np.array([[1e3, -2e3, 5e2]])
    r = m.eval_local(np.vstack([pts[:1], far]), ("rho", "grad", "rdg", "shannon"))
    assert r["rho"][1] == 0.0 and (r["grad"][1] == 0).all()
    pref = 0.5 / (3 * np.pi ** 2) ** (1 / 3)
    assert r["rdg"][1] == pytest.approx(pref * 1e-20, rel=1e-15)
    ref = O.eval_local(mol.flat(), mol.D, pts[:1], keys=("rho",))
    assert r["rho"][0] == pytest.approx(ref["rho"][0], rel=1e-12)
    # a ragged count that leaves partial tiles everywhere
    n = 129
    rng = np.random.default_rng(5)
    p2 = S.random_points(rng, mol, n)
    got = m.eval_local(p2, ("rho", "hess"))
    ref = O.eval_local(mol.flat(), mol.D, p2, keys=("rho", "hess"))
    sc = term_scales(mol.flat(), mol.D, p2)
    assert_close("ragged rho", got["rho"], ref["rho"], sc["rho"], 1e-10, 1e-14)
    assert_close("ragged hess", got["hess"], ref["hess"], sc["hess"], 1e-10, 1e-14)


@pytest.mark.parametrize("precision,rtol", [(ctc_abi.PREC_FP64, 1e-10), (ctc_abi.PREC_TC, 1e-8)])
def test_degenerate_point_sets(torch_cuda, precision, rtol):
    """Explicit points are packed into tiles by their bounding box (sort by x,
    y, z with cut counts from the box); a set with no extent along one or two
    axes, repeated points, and finite points mixed with non-finite ones must
    give the same outputs as the oracle."""
    mol, pts = _cases().CASES["c1"]()
    m = _mol(mol)
    rng = np.random.default_rng(11)
    c = mol.coords.mean(0)
    u = rng.uniform(-3, 3, size=(700, 2))
    sets = {
        "plane": np.column_stack([c[0] + u[:, 0], c[1] + u[:, 1], np.full(700, c[2] + 0.3)]),
        "line": np.column_stack([np.full(500, c[0] - 0.2), np.full(500, c[1] + 0.1),
                                 c[2] + np.linspace(-4, 4, 500)]),
        "repeated": np.repeat(pts[:3], 50, axis=0),
        "single": pts[:1],
    }
    keys = ("rho", "grad", "hess", "lap")
    for name, p in sets.items():
        got = m.eval_local(p, keys, precision=precision)
        ref = O.eval_local(mol.flat(), mol.D, p, keys=keys)
        sc = term_scales(mol.flat(), mol.D, p)
        for k in keys:
            assert_close(f"{name} {k}", got[k], ref[k], sc[k], rtol, 1e-14)
    # finite points interleaved with non-finite ones: NaN outputs only where the point is
    p = S.random_points(rng, mol, 300)
    bad = rng.choice(300, 40, replace=False)
    p[bad[:20], 0] = np.nan
    p[bad[20:], 2] = np.inf
    got = m.eval_local(p, ("rho", "grad"), precision=precision)
    ok = np.ones(300, bool)
    ok[bad] = False
    assert np.isnan(got["rho"][~ok]).all()
    ref = O.eval_local(mol.flat(), mol.D, p[ok], keys=("rho", "grad"))
    sc = term_scales(mol.flat(), mol.D, p[ok])
    assert_close("mixed rho", got["rho"][ok], ref["rho"], sc["rho"], rtol, 1e-14)
    assert_close("mixed grad", got["grad"][ok], ref["grad"], sc["grad"], rtol, 1e-14)


def test_invalid_basis_rejected(torch_cuda):
    mol, _ = _cases().CASES["c1"]()
    f = mol.flat()
    bad = dict(f)
    bad["angmoms"] = f["angmoms"].copy()
    bad["angmoms"][0] = 5
    with pytest.raises(RuntimeError, match="angular momentum"):
        ctc_abi.Mol(bad, mol.coords, mol.charges, mol.D)
    with pytest.raises(RuntimeError, match="functions"):
        ctc_abi.Mol(f, mol.coords, mol.charges, mol.D[:-1, :-1])


def _golden(case):
    p = os.path.join(GOLDEN, f"{case}.npz")
    if not os.path.exists(p):
        pytest.skip(f"golden vectors {case}.npz not generated")
    return dict(np.load(p))


def _golden_mol(g):
    flat = {k[3:]: g[k] for k in ("in_centers", "in_shell_atom", "in_nprim", "in_nseg",
                                   "in_angmoms", "in_exps", "in_coeffs")}
    return flat, ctc_abi.Mol(flat, g["in_coords"], g["in_charges"], g["in_D"])


REF_PAIRS = dict(rho="ref_density", grad="ref_gradient", hess="ref_hessian", lap="ref_laplacian",
                 tau_pd="ref_tau_pd", tau_alpha="ref_tau_general", rdg="ref_rdg",
                 shannon="ref_shannon", weizsacker="ref_weizsacker",
                 thomas_fermi="ref_thomas_fermi", gge="ref_gge", general_ked="ref_general_ked")
RATIO_KEYS = ("rdg", "shannon", "weizsacker", "thomas_fermi", "gge")


def _vs_reference(case, precision, rtol):
    """Every output slot against what the reference's CUDA drivers returned on the
    same molecule and points: |x - x_ref| <= rtol * (sum of |terms|) where
    rho >= 1e-12 and <= 1e-12 absolute where rho < 1e-12; the ratio-type outputs
    where rho > 1e-10 (their reference values divide by rho)."""
    g = _golden(case)
    flat, m = _golden_mol(g)
    pts = g["in_points"]
    a = float(g["meta_tau_alpha"])
    ga, gb = (float(x) for x in g["meta_gge_ab"])
    ka = float(g["meta_general_ked_a"])
    keys = tuple(k for k, rk in REF_PAIRS.items() if rk in g)
    got = m.eval_local(pts, keys, precision, params=(a, ga, gb, ka))
    oref = O.eval_local(flat, g["in_D"], pts, alpha=a, keys=keys, gge_ab=(ga, gb), ked_a=ka)
    sc = term_scales(flat, g["in_D"], pts, alpha=a, gge=(ga, gb), ked_a=ka, ref=oref)
    rho = g["ref_density"]
    tiny = rho < 1e-12
    for k in keys:
        ref = g[REF_PAIRS[k]].reshape(got[k].shape)
        if k in RATIO_KEYS:
            assert_close(f"{case}/{k} vs reference", got[k], ref, sc[k], rtol, atol=1e-15,
                         mask=rho > 1e-10)
            continue
        scale = np.where(tiny.reshape((-1,) + (1,) * (ref.ndim - 1)), 0.0, rtol * sc[k])
        atol = np.where(tiny, 1e-12, 1e-15).reshape((-1,) + (1,) * (ref.ndim - 1))
        assert_close(f"{case}/{k} vs reference", got[k], ref, scale + atol, 1.0)
    return m, g


@pytest.mark.parametrize("case", ["c1", "esp", "mixed"])
def test_fp64_path_vs_reference_outputs(torch_cuda, case):
    """Directly against what the reference's CUDA drivers returned: 1e-10 relative
    (1e-12 absolute where rho < 1e-12), every output slot."""
    m, g = _vs_reference(case, ctc_abi.PREC_FP64, 1e-10)
    if "ref_esp" in g:
        e = m.eval_esp(g["in_points"])
        assert_close(f"{case}/esp vs reference", e, g["ref_esp"], np.abs(g["ref_esp"]), 1e-10)


@pytest.mark.parametrize("case", ["c1", "esp", "mixed"])
def test_tc_path_vs_reference_outputs(torch_cuda, case):
    """The tensor-core split path against the reference's own outputs at its
    stated 1e-8 (1e-12 absolute where rho < 1e-12), every output slot."""
    _vs_reference(case, ctc_abi.PREC_TC, 1e-8)
