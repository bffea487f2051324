"""The native .fchk reader (ctc_fchk_load, host only).

* round trip: a synthetic molecule written in the Gaussian formatted
  checkpoint layout reads back as the same basis arrays, atoms and density
  matrix (restricted closed shell, restricted open shell, unrestricted);
* sp shells become one shell with an s and a p segment;
* errors: missing file, inconsistent basis size;
* the reference's own fixtures (when the reference tree is present): the MO
  density matrix equals the file's "Total SCF Density" and integrates, with the
  FP64 oracle on a Becke grid, to the number of electrons.
"""
import glob
import os

import numpy as np
import pytest

import ctc_abi
from chemtoolscuda_b200 import synthetic as S
from oracle import oracle as O

# the reference checkout holding its fixture files (CTC_REFERENCE); tests that need
# them are skipped where it is absent
REF_DATA = os.path.join(os.environ.get("CTC_REFERENCE", "/root/reference"), "tests", "data")


def _fmt_section(label, kind, values):
    values = np.asarray(values).ravel()
    head = f"{label:<43}{kind}   N={len(values):>12}\n"
    per = 6 if kind == "I" else 5
    body = []
    for i in range(0, len(values), per):
        chunk = values[i:i + per]
        if kind == "I":
            body.append("".join(f"{int(v):12d}" for v in chunk))
        else:
            body.append("".join(f"{float(v):24.16E}" for v in chunk))
    return head + "\n".join(body) + "\n"


def _fmt_scalar(label, kind, value):
    return f"{label:<43}{kind}{int(value):17d}\n" if kind == "I" else f"{label:<43}{kind}{value:27.15E}\n"


def write_fchk(path, mol, nalpha, nbeta, ca, cb=None):
    """Gaussian formatted-checkpoint text for a molecule whose shells have one
    segment each or are s+p pairs (written as sp shells)."""
    f = mol.flat()
    types, coef, pcoef = [], [], []
    ic = 0
    for s in range(len(f["nprim"])):
        K, G = int(f["nprim"][s]), int(f["nseg"][s])
        am = list(f["angmoms"][sum(f["nseg"][:s]):sum(f["nseg"][:s]) + G])
        c = f["coeffs"][ic:ic + G * K]
        ic += G * K
        if G == 1:
            types.append(am[0])
            coef += list(c)
            pcoef += [0.0] * K
        else:
            assert am == [0, 1], "only s+p generalised shells have an fchk form"
            types.append(-1)
            coef += list(c[:K])
            pcoef += list(c[K:])
    M = ca.shape[1]
    out = ["synthetic molecule\n", "SP        RHF                                                         Gen\n",
           _fmt_scalar("Number of atoms", "I", len(mol.coords)),
           _fmt_scalar("Charge", "I", 0), _fmt_scalar("Multiplicity", "I", 1 + nalpha - nbeta),
           _fmt_scalar("Number of electrons", "I", nalpha + nbeta),
           _fmt_scalar("Number of alpha electrons", "I", nalpha),
           _fmt_scalar("Number of beta electrons", "I", nbeta),
           _fmt_scalar("Number of basis functions", "I", M),
           _fmt_section("Atomic numbers", "I", mol.numbers),
           _fmt_section("Nuclear charges", "R", mol.charges),
           _fmt_section("Current cartesian coordinates", "R", mol.coords),
           _fmt_scalar("Number of contracted shells", "I", len(types)),
           _fmt_section("Shell types", "I", types),
           _fmt_section("Number of primitives per shell", "I", f["nprim"]),
           _fmt_section("Shell to atom map", "I", np.asarray(f["shell_atom"]) + 1),
           _fmt_section("Primitive exponents", "R", f["exps"]),
           _fmt_section("Contraction coefficients", "R", coef)]
    if -1 in types:
        out.append(_fmt_section("P(S=P) Contraction coefficients", "R", pcoef))
    out += [_fmt_section("Coordinates of each shell", "R", f["centers"]),
            _fmt_scalar("SCF Energy", "R", -1.0),
            _fmt_section("Alpha MO coefficients", "R", ca)]
    if cb is not None:
        out.append(_fmt_section("Beta MO coefficients", "R", cb))
    with open(path, "w") as fh:
        fh.writelines(out)


def _orbitals(rng, M, nmo):
    q, _ = np.linalg.qr(rng.standard_normal((M, nmo)))
    return np.ascontiguousarray(q.T)  # MO-major


@pytest.mark.parametrize("kind", ["closed", "open", "unrestricted"])
def test_round_trip(tmp_path, kind):
    mol = S.make_molecule("c1", seed=3)
    M = mol.nbasis
    rng = np.random.default_rng(1)
    ca = _orbitals(rng, M, M)
    if kind == "closed":
        na, nb, cb = 7, 7, None
        D = 2 * ca[:7].T @ ca[:7]
    elif kind == "open":
        na, nb, cb = 8, 6, None
        D = 2 * ca[:6].T @ ca[:6] + ca[6:8].T @ ca[6:8]
    else:
        na, nb = 8, 6
        cb = _orbitals(rng, M, M)
        D = ca[:8].T @ ca[:8] + cb[:6].T @ cb[:6]
    p = str(tmp_path / "m.fchk")
    write_fchk(p, mol, na, nb, ca, cb)
    got = ctc_abi.load_fchk(p)
    f = mol.flat()
    for k in ("nprim", "nseg", "angmoms", "shell_atom"):
        np.testing.assert_array_equal(got["flat"][k], f[k], err_msg=k)
    for k in ("centers", "exps", "coeffs"):
        np.testing.assert_allclose(got["flat"][k], f[k], rtol=1e-15, err_msg=k)
    np.testing.assert_allclose(got["coords"], mol.coords, rtol=1e-15)
    np.testing.assert_array_equal(got["numbers"], mol.numbers)
    assert (got["nalpha"], got["nbeta"]) == (na, nb)
    np.testing.assert_allclose(got["D"], D, atol=1e-14)


def test_sp_shells_become_two_segments(tmp_path):
    mol = S.make_molecule("c1", seed=2, generalised=True)
    f = mol.flat()
    # keep only shells the format can hold: single segments and s+p pairs
    ok = True
    off = 0
    for s in range(len(f["nseg"])):
        am = list(f["angmoms"][off:off + f["nseg"][s]])
        off += f["nseg"][s]
        ok &= f["nseg"][s] == 1 or am == [0, 1]
    if not ok or not (f["nseg"] == 2).any():
        pytest.skip("generator gave no pure s+p shells")
    M = mol.nbasis
    ca = _orbitals(np.random.default_rng(3), M, M)
    p = str(tmp_path / "sp.fchk")
    write_fchk(p, mol, 5, 5, ca)
    got = ctc_abi.load_fchk(p)
    np.testing.assert_array_equal(got["flat"]["nseg"], f["nseg"])
    np.testing.assert_array_equal(got["flat"]["angmoms"], f["angmoms"])
    np.testing.assert_allclose(got["flat"]["coeffs"], f["coeffs"], rtol=1e-15)


def test_hand_written_sp_shell(tmp_path):
    text = ("t\nSP RHF Gen\n"
            + _fmt_scalar("Number of atoms", "I", 1) + _fmt_scalar("Number of alpha electrons", "I", 1)
            + _fmt_scalar("Number of beta electrons", "I", 1) + _fmt_scalar("Number of basis functions", "I", 5)
            + _fmt_section("Atomic numbers", "I", [3]) + _fmt_section("Nuclear charges", "R", [3.0])
            + _fmt_section("Current cartesian coordinates", "R", [0.0, 0.0, 0.0])
            + _fmt_section("Shell types", "I", [0, -1]) + _fmt_section("Number of primitives per shell", "I", [1, 2])
            + _fmt_section("Shell to atom map", "I", [1, 1])
            + _fmt_section("Primitive exponents", "R", [16.0, 1.5, 0.3])
            + _fmt_section("Contraction coefficients", "R", [1.0, 0.4, 0.7])
            + _fmt_section("P(S=P) Contraction coefficients", "R", [0.0, 0.2, 0.9])
            + _fmt_section("Coordinates of each shell", "R", [0.0] * 6)
            + _fmt_section("Alpha MO coefficients", "R", np.eye(5)))
    p = tmp_path / "li.fchk"
    p.write_text(text)
    got = ctc_abi.load_fchk(str(p))
    np.testing.assert_array_equal(got["flat"]["nseg"], [1, 2])
    np.testing.assert_array_equal(got["flat"]["angmoms"], [0, 0, 1])
    np.testing.assert_allclose(got["flat"]["coeffs"], [1.0, 0.4, 0.7, 0.2, 0.9])
    np.testing.assert_allclose(got["D"], np.diag([2.0, 0, 0, 0, 0]))


def test_errors(tmp_path):
    with pytest.raises(RuntimeError, match="cannot open"):
        ctc_abi.load_fchk(str(tmp_path / "missing.fchk"))
    mol = S.make_molecule("c1", seed=3)
    ca = _orbitals(np.random.default_rng(1), mol.nbasis, mol.nbasis)
    p = tmp_path / "bad.fchk"
    write_fchk(str(p), mol, 3, 3, ca)
    txt = p.read_text().replace(f"Number of basis functions                  I{mol.nbasis:17d}",
                                f"Number of basis functions                  I{mol.nbasis + 1:17d}")
    p.write_text(txt)
    with pytest.raises(RuntimeError, match="functions"):
        ctc_abi.load_fchk(str(p))


def _total_scf_density(path, M):
    """Lower triangle of the file's 'Total SCF Density' as a full matrix."""
    lines = open(path).read().splitlines()
    for i, line in enumerate(lines):
        if line.startswith("Total SCF Density"):
            n = int(line.split("N=")[1])
            vals = []
            j = i + 1
            while len(vals) < n:
                vals += [float(v) for v in lines[j].split()]
                j += 1
            P = np.zeros((M, M))
            P[np.tril_indices(M)] = vals
            return P + np.tril(P, -1).T
    return None


FIXTURES = sorted(glob.glob(os.path.join(REF_DATA, "*.fchk"))) if os.path.isdir(REF_DATA) else []


@pytest.mark.skipif(not FIXTURES, reason="reference fixtures not present")
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_reference_fixture(path):
    got = ctc_abi.load_fchk(path)
    M = got["D"].shape[0]
    P = _total_scf_density(path, M)
    if P is not None:
        np.testing.assert_allclose(got["D"], P, atol=1e-6 * max(1.0, np.abs(P).max()))
    if M > 200:
        return  # integration below is for the small fixtures
    class _Atoms:  # what atom_grid needs
        coords = got["coords"]
    pts, w = S.atom_grid(_Atoms, nrad=100, ntheta=18, nphi=36)
    rho = O.eval_local(got["flat"], got["D"], pts, keys=("rho",))["rho"]
    nelec = got["nalpha"] + got["nbeta"]
    assert abs((w * rho).sum() - nelec) <= 2e-3 * nelec, ((w * rho).sum(), nelec)


@pytest.mark.gpu
def test_molecule_from_fchk_matches_arrays(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import chemtoolscuda_b200 as ctc
    mol = S.make_molecule("c1", seed=3)
    M = mol.nbasis
    ca = _orbitals(np.random.default_rng(1), M, M)
    p = str(tmp_path / "m.fchk")
    write_fchk(p, mol, 7, 7, ca)
    D = 2 * ca[:7].T @ ca[:7]
    a = ctc.Molecule(p)
    f = mol.flat()
    b = ctc.Molecule.from_arrays(f["centers"], f["shell_atom"], f["nprim"], f["nseg"], f["angmoms"],
                                 f["exps"], f["coeffs"], mol.coords, mol.charges, D)
    pts = S.random_points(np.random.default_rng(2), mol, 500, pad=2.0)
    np.testing.assert_allclose(a.compute_electron_density(pts), b.compute_electron_density(pts),
                               rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(a.compute_electron_density_gradient(pts),
                               b.compute_electron_density_gradient(pts), rtol=1e-11, atol=1e-14)
    np.testing.assert_array_equal(a.numbers, mol.numbers)
    np.testing.assert_allclose(a.coordinates, mol.coords)
    assert a.get_file_path() == p
