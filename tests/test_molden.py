"""The native Molden reader (ctc_molden_load, host only) and Molecule(path) on Molden files.

* the same synthetic molecule written as fchk and as Molden reads back as the
  same basis arrays, atoms and density matrix (Cartesian d, pure d/f with the
  [5D7F] and [5D] flags, sp shells);
* Cartesian g shells: Molden's component order is permuted into the library's;
* unrestricted orbitals (Spin= Beta), coordinates in angstrom, coefficient
  lines with the zeros left out;
* errors: missing file or sections, Slater-type basis, scale factors, unknown
  shell labels, orbital indices out of range;
* on the GPU, Molecule(path.molden) evaluates like Molecule(path.fchk).
"""
import numpy as np
import pytest

import ctc_abi
from chemtoolscuda_b200 import synthetic as S
from test_fchk import _orbitals, write_fchk

BOHR_PER_ANGSTROM = 1.0 / 0.529177210903
LABEL = {0: "s", 1: "p", 2: "d", 3: "f", 4: "g"}
# Molden's Cartesian g components and the library's order (x, y, z exponents)
MOLDEN_G = [(4, 0, 0), (0, 4, 0), (0, 0, 4), (3, 1, 0), (3, 0, 1), (1, 3, 0), (0, 3, 1), (1, 0, 3),
            (0, 1, 3), (2, 2, 0), (2, 0, 2), (0, 2, 2), (2, 1, 1), (1, 2, 1), (1, 1, 2)]
LIB_G = [(0, 0, 4), (0, 1, 3), (0, 2, 2), (0, 3, 1), (0, 4, 0), (1, 0, 3), (1, 1, 2), (1, 2, 1),
         (1, 3, 0), (2, 0, 2), (2, 1, 1), (2, 2, 0), (3, 0, 1), (3, 1, 0), (4, 0, 0)]


def _molden_order(flat):
    """For every function in Molden's order, its index in the library's order."""
    perm, off, ia = [], 0, 0
    for s in range(len(flat["nprim"])):
        for _ in range(int(flat["nseg"][s])):
            t = int(flat["angmoms"][ia])
            ia += 1
            n = S.nfunc(t)
            if t == 4:
                perm += [off + LIB_G.index(c) for c in MOLDEN_G]
            else:
                perm += list(range(off, off + n))
            off += n
    return np.array(perm)


def write_molden(path, mol, orbitals, flags=None, angs=False, sparse=False):
    """Molden text for a molecule whose shells are single segments or s+p pairs.
    orbitals: list of (coefficients in the library's order, occupation, 'Alpha'|'Beta')."""
    f = mol.flat()
    assert np.all(np.diff(f["shell_atom"]) >= 0), "shells must be grouped by atom"
    types = [int(a) for a in f["angmoms"]]
    if flags is None:
        pd, pf, pg = -2 in types, -3 in types, -4 in types
        flags = []
        if pd and pf:
            flags.append("[5D7F]")
        elif pd:
            flags.append("[5D10F]")
        elif pf:
            flags.append("[7F]")
        if pg:
            flags.append("[9G]")
    unit = BOHR_PER_ANGSTROM if angs else 1.0
    out = ["[Molden Format]", "[Title]", "synthetic molecule", "[Atoms] " + ("Angs" if angs else "AU")]
    for a, (z, r) in enumerate(zip(mol.numbers, mol.coords)):
        out.append(f"X{a + 1} {a + 1} {int(z)} {r[0] / unit:.17e} {r[1] / unit:.17e} {r[2] / unit:.17e}")
    out.append("[GTO]")
    ic = ie = ia = 0
    for s in range(len(f["nprim"])):
        a = int(f["shell_atom"][s])
        if s == 0 or int(f["shell_atom"][s - 1]) != a:
            if s:
                out.append("")
            out.append(f"  {a + 1} 0")
        K, G = int(f["nprim"][s]), int(f["nseg"][s])
        am = types[ia:ia + G]
        ia += G
        e = f["exps"][ie:ie + K]
        c = f["coeffs"][ic:ic + G * K].reshape(G, K)
        ie += K
        ic += G * K
        if G == 2:
            assert am == [0, 1]
            out.append(f" sp {K} 1.00")
            out += [f"  {e[k]:.17e} {c[0, k]:.17e} {c[1, k]:.17e}" for k in range(K)]
        else:
            out.append(f" {LABEL[abs(am[0])]} {K} 1.00")
            out += [f"  {e[k]:.17e} {c[0, k]:.17e}" for k in range(K)]
    out.append("")
    out += flags
    out.append("[MO]")
    perm = _molden_order(f)
    for i, (coef, occ, spin) in enumerate(orbitals):
        out += [" Sym= A", f" Ene= {-1.0 + 0.01 * i:.6f}", f" Spin= {spin}", f" Occup= {occ:.6f}"]
        v = np.asarray(coef)[perm]
        for j, x in enumerate(v):
            if sparse and x == 0.0:
                continue
            out.append(f"  {j + 1} {x:.17e}")
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def _closed(ca, nocc):
    return [(ca[i], 2.0 if i < nocc else 0.0, "Alpha") for i in range(len(ca))]


def _compare(got, ref):
    for k in ("nprim", "nseg", "angmoms", "shell_atom"):
        np.testing.assert_array_equal(got["flat"][k], ref["flat"][k], err_msg=k)
    for k in ("centers", "exps", "coeffs"):
        np.testing.assert_allclose(got["flat"][k], ref["flat"][k], rtol=1e-15, atol=1e-300, err_msg=k)
    np.testing.assert_allclose(got["coords"], ref["coords"], rtol=1e-14, atol=1e-14)
    np.testing.assert_array_equal(got["numbers"], ref["numbers"])
    np.testing.assert_allclose(got["D"], ref["D"], atol=1e-13)
    assert (got["nalpha"], got["nbeta"]) == (ref["nalpha"], ref["nbeta"])


@pytest.mark.parametrize("config,natom", [("c1", 12), ("c2", 8)])
def test_same_molecule_as_fchk(tmp_path, config, natom):
    mol = S.make_molecule(config, seed=5, natom=natom, box=8.0, nocc=4)
    M = mol.nbasis
    ca = _orbitals(np.random.default_rng(2), M, M)
    write_fchk(str(tmp_path / "m.fchk"), mol, 6, 6, ca)
    write_molden(str(tmp_path / "m.molden"), mol, _closed(ca, 6))
    _compare(ctc_abi.load_molden(str(tmp_path / "m.molden")), ctc_abi.load_fchk(str(tmp_path / "m.fchk")))


def test_5d_flag_means_pure_d_and_f(tmp_path):
    mol = S.make_molecule("c2", seed=1, natom=6, box=8.0, nocc=4)
    ca = _orbitals(np.random.default_rng(3), mol.nbasis, mol.nbasis)
    write_molden(str(tmp_path / "a.molden"), mol, _closed(ca, 5), flags=["[5D7F]"])
    write_molden(str(tmp_path / "b.molden"), mol, _closed(ca, 5), flags=["[5D]"])
    _compare(ctc_abi.load_molden(str(tmp_path / "b.molden")), ctc_abi.load_molden(str(tmp_path / "a.molden")))


def test_sp_shells(tmp_path):
    mol = S.make_molecule("c1", seed=2, natom=5, box=7.0, nocc=3, generalised=True)
    f = mol.flat()
    off, ok = 0, True
    for s in range(len(f["nseg"])):
        am = list(f["angmoms"][off:off + f["nseg"][s]])
        off += f["nseg"][s]
        ok &= f["nseg"][s] == 1 or am == [0, 1]
    if not ok or not (f["nseg"] == 2).any():
        pytest.skip("generator gave no pure s+p shells")
    ca = _orbitals(np.random.default_rng(4), mol.nbasis, mol.nbasis)
    write_fchk(str(tmp_path / "m.fchk"), mol, 4, 4, ca)
    write_molden(str(tmp_path / "m.molden"), mol, _closed(ca, 4))
    _compare(ctc_abi.load_molden(str(tmp_path / "m.molden")), ctc_abi.load_fchk(str(tmp_path / "m.fchk")))


def test_cartesian_g_order(tmp_path):
    """Cartesian g shells (c4 generator): Molden lists the 15 components in its own order;
    the density matrix must come back in the library's order."""
    mol = S.make_molecule("c4", seed=0, natom=4, box=6.0, nocc=4, cutoff=None)
    assert 4 in [int(a) for a in mol.flat()["angmoms"]], "need a Cartesian g shell"
    M = mol.nbasis
    ca = _orbitals(np.random.default_rng(5), M, M)
    write_molden(str(tmp_path / "g.molden"), mol, _closed(ca, 5))
    got = ctc_abi.load_molden(str(tmp_path / "g.molden"))
    np.testing.assert_allclose(got["D"], 2 * ca[:5].T @ ca[:5], atol=1e-13)
    # and the permutation is not the identity: reading the coefficients without it differs
    perm = _molden_order(mol.flat())
    assert not np.array_equal(perm, np.arange(M))


def test_unrestricted_angstrom_sparse(tmp_path):
    mol = S.make_molecule("c1", seed=7, natom=6, box=7.0, nocc=3)
    M = mol.nbasis
    rng = np.random.default_rng(6)
    ca, cb = _orbitals(rng, M, M), _orbitals(rng, M, M)
    ca[:, ::3] = 0.0  # zeros that a sparse writer leaves out
    orbs = [(ca[i], 1.0 if i < 5 else 0.0, "Alpha") for i in range(M)] + \
           [(cb[i], 1.0 if i < 3 else 0.0, "Beta") for i in range(M)]
    write_molden(str(tmp_path / "u.molden"), mol, orbs, angs=True, sparse=True)
    got = ctc_abi.load_molden(str(tmp_path / "u.molden"))
    np.testing.assert_allclose(got["D"], ca[:5].T @ ca[:5] + cb[:3].T @ cb[:3], atol=1e-13)
    np.testing.assert_allclose(got["coords"], mol.coords, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(got["flat"]["centers"], mol.flat()["centers"], rtol=1e-13, atol=1e-13)
    assert (got["nalpha"], got["nbeta"]) == (5, 3)


def test_errors(tmp_path):
    with pytest.raises(RuntimeError, match="cannot open"):
        ctc_abi.load_molden(str(tmp_path / "missing.molden"))
    mol = S.make_molecule("c1", seed=3, natom=3, box=6.0, nocc=2)
    ca = _orbitals(np.random.default_rng(1), mol.nbasis, mol.nbasis)
    p = tmp_path / "m.molden"
    write_molden(str(p), mol, _closed(ca, 2))
    good = p.read_text()
    cases = {
        "Slater": good.replace("[GTO]", "[STO]"),
        "scale factors": good.replace(" s 3 1.00", " s 3 1.20").replace(" s 4 1.00", " s 4 1.20")
                                  .replace(" s 5 1.00", " s 5 1.20").replace(" s 6 1.00", " s 6 1.20"),
        "not supported": good.replace(" p ", " h ", 1),
        "no \\[MO\\]": good[:good.index("[MO]")],
        "outside": good.rstrip("\n") + f"\n  {mol.nbasis + 5} 1.0\n",
    }
    for msg, text in cases.items():
        p.write_text(text)
        with pytest.raises(RuntimeError, match=msg):
            ctc_abi.load_molden(str(p))
            pytest.fail(f"no error for the {msg!r} case")


@pytest.mark.gpu
def test_molecule_from_molden_matches_fchk(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import chemtoolscuda_b200 as ctc
    mol = S.make_molecule("c4", seed=0, natom=4, box=6.0, nocc=4, cutoff=None)
    M = mol.nbasis
    ca = _orbitals(np.random.default_rng(5), M, M)
    write_fchk(str(tmp_path / "m.fchk"), mol, 5, 5, ca)
    write_molden(str(tmp_path / "m.molden"), mol, _closed(ca, 5))
    a = ctc.Molecule(str(tmp_path / "m.molden"))
    b = ctc.Molecule(str(tmp_path / "m.fchk"))
    pts = S.random_points(np.random.default_rng(2), mol, 400, pad=2.0)
    np.testing.assert_allclose(a.compute_electron_density(pts), b.compute_electron_density(pts),
                               rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(a.compute_electron_density_gradient(pts),
                               b.compute_electron_density_gradient(pts), rtol=1e-11, atol=1e-14)
    np.testing.assert_array_equal(a.numbers, mol.numbers)
