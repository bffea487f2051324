"""GPU tests of the adjoint kernels and the torch.autograd binding.

* dL/dD and dL/dR through the C ABI against the FP64 oracle (1e-10 relative);
* the autograd path on L = sum_g w_g (c1 rho^(4/3) + c2 |grad rho|^2 / rho^(4/3))
  against FP64 central finite differences (h = 1e-5) on 20 random symmetric
  pairs of D entries and all coordinates -- tolerance 1e-6 relative to the largest gradient entry;
* the translational sum rule sum_A dL/dR_A = -sum_g (v_rho grad rho + H v_grad).
"""
import numpy as np
import pytest

import ctc_abi
from oracle import oracle as O
from chemtoolscuda_b200 import synthetic as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _small():
    mol = S.make_molecule("c3", seed=2, natom=5, box=5.0, nocc=10)
    rng = np.random.default_rng(4)
    pts = S.random_points(rng, mol, 700, pad=2.5)
    return mol, pts


@pytest.mark.parametrize("with_grad", [False, True])
def test_adjoint_vs_oracle(torch_cuda, with_grad):
    mol, pts = _small()
    rng = np.random.default_rng(9)
    vr = rng.standard_normal(len(pts))
    vg = rng.standard_normal((len(pts), 3)) if with_grad else None
    m = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
    dD, dR = m.adjoint(pts, vr, vg)
    rD, rR = O.adjoint(mol.flat(), mol.D, len(mol.coords), pts, vr, vg)
    np.testing.assert_allclose(dD, rD, rtol=0, atol=1e-10 * np.abs(rD).max())
    np.testing.assert_allclose(dR, rR, rtol=0, atol=1e-10 * np.abs(rR).max())


def test_adjoint_accumulates_and_handles_no_points(torch_cuda):
    mol, pts = _small()
    m = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
    dD0, dR0 = m.adjoint(pts[:0], np.zeros(0))
    assert np.abs(dD0).max() == 0 and np.abs(dR0).max() == 0


def test_autograd_vs_finite_differences(torch_cuda):
    torch = torch_cuda
    from chemtoolscuda_b200 import molecule_from_synthetic
    from chemtoolscuda_b200.autograd import density_and_gradient, gga_functional
    mol, _ = _small()
    grid, w = S.atom_grid(mol, nrad=20, ntheta=8, nphi=12)
    pts = torch.as_tensor(grid, device="cuda")
    wt = torch.as_tensor(w, device="cuda")
    pm = molecule_from_synthetic(mol)
    D = torch.as_tensor(mol.D, device="cuda").requires_grad_(True)
    R = torch.as_tensor(mol.coords).clone().requires_grad_(True)

    def L(Dm, Rm):
        rho, grad = density_and_gradient(pm, pts, Dm, Rm)
        return gga_functional(rho, grad, wt)

    loss = L(D, R)
    loss.backward()
    gD = D.grad.cpu().numpy()
    gR = R.grad.numpy()
    h = 1e-5
    rng = np.random.default_rng(1)
    M = mol.nbasis
    idx = [(int(a), int(b)) for a, b in rng.integers(0, M, size=(20, 2))]
    fdD = []
    # D stays symmetric under the perturbation (the forward formulas, like the
    # reference's, assume a symmetric density matrix): moving D[a,b] and D[b,a]
    # together measures dL/dD[a,b] + dL/dD[b,a] (once for a == b).
    with torch.no_grad():
        for (a, b) in idx:
            Dp = D.detach().clone()
            Dm = D.detach().clone()
            Dp[a, b] += h
            Dm[a, b] -= h
            if a != b:
                Dp[b, a] += h
                Dm[b, a] -= h
            fdD.append((L(Dp, R.detach()).item() - L(Dm, R.detach()).item()) / (2 * h))
        fdR = np.zeros_like(gR)
        for A in range(len(mol.coords)):
            for j in range(3):
                Rp = R.detach().clone()
                Rp[A, j] += h
                Rm = R.detach().clone()
                Rm[A, j] -= h
                fdR[A, j] = (L(D.detach(), Rp).item() - L(D.detach(), Rm).item()) / (2 * h)
    an = np.array([gD[a, b] + (gD[b, a] if a != b else 0.0) for (a, b) in idx])
    scaleD = max(np.abs(gD).max(), 1e-30)
    assert np.abs(an - np.array(fdD)).max() <= 1e-6 * scaleD, (an, fdD)
    scaleR = max(np.abs(gR).max(), 1e-30)
    assert np.abs(gR - fdR).max() <= 1e-6 * scaleR, (gR, fdR)


def test_translational_sum_rule(torch_cuda):
    mol, pts = _small()
    rng = np.random.default_rng(5)
    vr = rng.standard_normal(len(pts))
    vg = rng.standard_normal((len(pts), 3))
    m = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
    _, dR = m.adjoint(pts, vr, vg, want_D=False)
    loc = m.eval_local(pts, ("grad", "hess"))
    expect = -(vr[:, None] * loc["grad"]).sum(0) - np.einsum("gij,gj->i", loc["hess"], vg)
    np.testing.assert_allclose(dR.sum(0), expect, rtol=1e-9, atol=1e-9 * np.abs(expect).max())


@pytest.mark.parametrize("case", ["c1", "esp", "mixed"])
def test_translational_sum_rule_vs_reference_outputs(torch_cuda, case):
    """sum_A dL/dR_A = -sum_g (v_rho grad rho + H v_grad), the right-hand side
    assembled from the reference's own gradient and Hessian outputs
    (evaluate_electron_density_gradient, src/evaluate_gradient.cu:1197-1422;
    evaluate_electron_density_hessian, src/evaluate_hessian.cu:1906-2307) on
    the same molecule and points (golden vectors).  Every shell sits on an
    atom, so moving all atoms together moves the density rigidly."""
    import os
    g = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", f"{case}.npz")))
    flat = {k[3:]: g[k] for k in ("in_centers", "in_shell_atom", "in_nprim", "in_nseg",
                                   "in_angmoms", "in_exps", "in_coeffs")}
    pts = g["in_points"]
    n = len(pts)
    rng = np.random.default_rng(11)
    vr = rng.standard_normal(n)
    vg = rng.standard_normal((n, 3))
    m = ctc_abi.Mol(flat, g["in_coords"], g["in_charges"], g["in_D"])
    _, dR = m.adjoint(pts, vr, vg, want_D=False)
    grad = g["ref_gradient"].reshape(n, 3)
    hess = g["ref_hessian"].reshape(n, 3, 3)
    expect = -(vr[:, None] * grad).sum(0) - np.einsum("gij,gj->i", hess, vg)
    scale = (np.abs(vr)[:, None] * np.abs(grad)).sum(0) + np.einsum("gij,gj->i", np.abs(hess), np.abs(vg))
    np.testing.assert_array_less(np.abs(dR.sum(0) - expect), 1e-10 * scale + 1e-14)
