"""The native AIM wavefunction reader (ctc_wfn_load: .wfn and .wfx, host only).

These formats list orbitals over unnormalised primitive Gaussians, so the
reader's basis (one single-primitive Cartesian shell per distinct centre, l
and exponent) differs from the contracted basis the orbitals came from; what
must agree is the density.  The tests write a synthetic molecule's occupied
orbitals in both formats, expanding every contracted function (Cartesian
components, and pure ones through the library's own solid-harmonic tables) into
primitives, read the files back and compare rho and grad rho at random points
with the FP64 oracle against the original contracted molecule.  Errors: g
primitives, unknown types, missing sections.  On the GPU, Molecule(x.wfn)
evaluates like Molecule(x.fchk).
"""
import os
import sys

import numpy as np
import pytest

import ctc_abi
from chemtoolscuda_b200 import synthetic as S
from helpers import assert_close, term_scales
from oracle import oracle as O
from test_fchk import _orbitals, write_fchk

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "chemtoolscuda_b200", "csrc"))
from gen_terms import CART, PURE  # noqa: E402

TYPES = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0),
         (1, 0, 1), (0, 1, 1), (3, 0, 0), (0, 3, 0), (0, 0, 3), (2, 1, 0), (2, 0, 1), (0, 2, 1),
         (1, 2, 0), (1, 0, 2), (0, 1, 2), (1, 1, 1)]  # AIMPAC types 1..20


def _df(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def primitives(mol, C):
    """Expand orbitals C (rows, library's function order) into (centre, type, exponent)
    primitives and per-orbital coefficients on the unnormalised primitives."""
    f = mol.flat()
    prims, index = [], {}
    coef = []  # per primitive: list of (function index, factor)
    fo = ia = ic = ie = 0
    for s in range(len(f["nprim"])):
        K, G = int(f["nprim"][s]), int(f["nseg"][s])
        atom = int(f["shell_atom"][s])
        e = f["exps"][ie:ie + K]
        c = f["coeffs"][ic:ic + G * K].reshape(G, K)
        ie += K
        ic += G * K
        for g in range(G):
            t = int(f["angmoms"][ia])
            ia += 1
            l = abs(t)
            if t >= 0:
                comps = [[(1.0 / np.sqrt(_df(2 * a - 1) * _df(2 * b - 1) * _df(2 * z - 1)), a, b, z)]
                         for (a, b, z) in CART[l]]
            else:
                comps = [[(w / np.sqrt(_df(2 * l - 1)), a, b, z) for (w, a, b, z) in comp] for comp in PURE[l]]
            for k in range(K):
                nrm = (2 * e[k] / np.pi) ** 0.75 * (4 * e[k]) ** (0.5 * l)
                for j, comp in enumerate(comps):
                    for (w, a, b, z) in comp:
                        key = (atom, TYPES.index((a, b, z)) + 1, float(e[k]))
                        if key not in index:
                            index[key] = len(prims)
                            prims.append(key)
                            coef.append([])
                        coef[index[key]].append((fo + j, c[g, k] * nrm * w))
            fo += len(comps)
    P = np.zeros((len(C), len(prims)))
    for p, lst in enumerate(coef):
        for (j, w) in lst:
            P[:, p] += C[:, j] * w
    return prims, P


def write_wfn(path, mol, prims, P, occ):
    out = ["synthetic molecule",
           f"GAUSSIAN {len(P):14d} MOL ORBITALS {len(prims):6d} PRIMITIVES {len(mol.coords):8d} NUCLEI"]
    for a, (q, r) in enumerate(zip(mol.charges, mol.coords)):
        out.append(f"  X{a + 1:<3d} {a + 1:4d}    (CENTRE{a + 1:3d}) {r[0]:.17e} {r[1]:.17e} {r[2]:.17e}  CHARGE = {q:4.1f}")
    for label, vals in (("CENTRE ASSIGNMENTS  ", [p[0] + 1 for p in prims]), ("TYPE ASSIGNMENTS    ", [p[1] for p in prims])):
        for i in range(0, len(vals), 20):
            out.append(label + "".join(f"{v:3d}" for v in vals[i:i + 20]))
    ex = [p[2] for p in prims]
    for i in range(0, len(ex), 5):
        out.append("EXPONENTS " + " ".join(f"{v:.17E}".replace("E", "D") for v in ex[i:i + 5]))
    for i, row in enumerate(P):
        out.append(f"MO{i + 1:5d}     MO 0.0        OCC NO = {occ[i]:13.8f}  ORB. ENERGY = {-1.0:12.6f}")
        for j in range(0, len(row), 5):
            out.append(" ".join(f"{v:.17E}".replace("E", "D") for v in row[j:j + 5]))
    out.append("END DATA")
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def write_wfx(path, mol, prims, P, occ, spins=None):
    def sec(tag, vals):
        return [f"<{tag}>"] + [" ".join(str(v) for v in vals)] + [f"</{tag}>"]
    out = sec("Title", ["synthetic molecule"]) + sec("Keywords", ["GTO"])
    out += sec("Number of Nuclei", [len(mol.coords)]) + sec("Number of Primitives", [len(prims)])
    out += sec("Number of Occupied Molecular Orbitals", [len(P)])
    out += sec("Atomic Numbers", [int(z) for z in mol.numbers])
    out += sec("Nuclear Charges", [f"{q:.17e}" for q in mol.charges])
    out += sec("Nuclear Cartesian Coordinates", [f"{v:.17e}" for v in mol.coords.ravel()])
    out += sec("Primitive Centers", [p[0] + 1 for p in prims]) + sec("Primitive Types", [p[1] for p in prims])
    out += sec("Primitive Exponents", [f"{p[2]:.17e}" for p in prims])
    out += sec("Molecular Orbital Occupation Numbers", [f"{o:.17e}" for o in occ])
    if spins is not None:
        out += ["<Molecular Orbital Spin Types>"] + list(spins) + ["</Molecular Orbital Spin Types>"]
    out.append("<Molecular Orbital Primitive Coefficients>")
    for i, row in enumerate(P):
        out += ["<MO Number>", str(i + 1), "</MO Number>"]
        out += [" ".join(f"{v:.17e}" for v in row[j:j + 4]) for j in range(0, len(row), 4)]
    out.append("</Molecular Orbital Primitive Coefficients>")
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def _check_density(got, mol, D, n=300, seed=9):
    pts = S.random_points(np.random.default_rng(seed), mol, n, pad=2.0)
    ref = O.eval_local(mol.flat(), D, pts, keys=("rho", "grad"))
    val = O.eval_local(got["flat"], got["D"], pts, keys=("rho", "grad"))
    sc = term_scales(mol.flat(), D, pts)
    assert_close("rho", val["rho"], ref["rho"], sc["rho"], 1e-11, atol=1e-15)
    assert_close("grad", val["grad"], ref["grad"], sc["grad"], 1e-11, atol=1e-15)


@pytest.mark.parametrize("fmt", ["wfn", "wfx"])
@pytest.mark.parametrize("config,natom", [("c1", 5), ("c2", 4)])
def test_density_matches_contracted_molecule(tmp_path, fmt, config, natom):
    mol = S.make_molecule(config, seed=3, natom=natom, box=7.0, nocc=4)
    M = mol.nbasis
    C = _orbitals(np.random.default_rng(1), M, M)[:6]
    prims, P = primitives(mol, C)
    path = str(tmp_path / f"m.{fmt}")
    (write_wfn if fmt == "wfn" else write_wfx)(path, mol, prims, P, [2.0] * 6)
    got = ctc_abi.load_wfn(path)
    assert (got["nalpha"], got["nbeta"]) == (6, 6)
    np.testing.assert_array_equal(got["numbers"], mol.numbers)
    np.testing.assert_allclose(got["coords"], mol.coords, rtol=1e-15)
    assert all(n == 1 for n in got["flat"]["nprim"]) and all(a >= 0 for a in got["flat"]["angmoms"])
    _check_density(got, mol, 2 * C.T @ C)


def test_wfx_unrestricted_spins(tmp_path):
    mol = S.make_molecule("c1", seed=4, natom=4, box=6.0, nocc=3)
    M = mol.nbasis
    rng = np.random.default_rng(2)
    Ca, Cb = _orbitals(rng, M, M)[:4], _orbitals(rng, M, M)[:2]
    prims, P = primitives(mol, np.vstack([Ca, Cb]))
    path = str(tmp_path / "u.wfx")
    write_wfx(path, mol, prims, P, [1.0] * 6, spins=["Alpha"] * 4 + ["Beta"] * 2)
    got = ctc_abi.load_wfn(path)
    assert (got["nalpha"], got["nbeta"]) == (4, 2)
    _check_density(got, mol, Ca.T @ Ca + Cb.T @ Cb)


def test_errors(tmp_path):
    with pytest.raises(RuntimeError, match="cannot open"):
        ctc_abi.load_wfn(str(tmp_path / "missing.wfn"))
    mol = S.make_molecule("c1", seed=3, natom=3, box=6.0, nocc=2)
    C = _orbitals(np.random.default_rng(1), mol.nbasis, mol.nbasis)[:2]
    prims, P = primitives(mol, C)
    p = tmp_path / "m.wfn"
    write_wfn(str(p), mol, prims, P, [2.0, 2.0])
    good = p.read_text().splitlines()
    ti = next(i for i, l in enumerate(good) if l.startswith("TYPE ASSIGNMENTS"))
    for msg, newtype in (("g primitives", 21), ("not supported", 40)):
        lines = list(good)
        lines[ti] = lines[ti][:20] + f"{newtype:3d}" + lines[ti][23:]
        p.write_text("\n".join(lines) + "\n")
        with pytest.raises(RuntimeError, match=msg):
            ctc_abi.load_wfn(str(p))
    p.write_text("\n".join(l for l in good if not l.startswith("EXPONENTS")) + "\n")
    with pytest.raises(RuntimeError, match="EXPONENTS"):
        ctc_abi.load_wfn(str(p))
    q = tmp_path / "m.wfx"
    write_wfx(str(q), mol, prims, P, [2.0, 2.0])
    q.write_text(q.read_text().replace("<Primitive Exponents>", "<Other>").replace("</Primitive Exponents>", "</Other>"))
    with pytest.raises(RuntimeError, match="primitive sections"):
        ctc_abi.load_wfn(str(q))


@pytest.mark.gpu
def test_molecule_from_wfn_matches_fchk(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import chemtoolscuda_b200 as ctc
    mol = S.make_molecule("c2", seed=3, natom=4, box=7.0, nocc=4)
    M = mol.nbasis
    ca = _orbitals(np.random.default_rng(1), M, M)
    write_fchk(str(tmp_path / "m.fchk"), mol, 5, 5, ca)
    prims, P = primitives(mol, ca[:5])
    write_wfn(str(tmp_path / "m.wfn"), mol, prims, P, [2.0] * 5)
    a = ctc.Molecule(str(tmp_path / "m.wfn"))
    b = ctc.Molecule(str(tmp_path / "m.fchk"))
    pts = S.random_points(np.random.default_rng(2), mol, 400, pad=2.0)
    ra, rb = a.compute_electron_density(pts), b.compute_electron_density(pts)
    sc = term_scales(mol.flat(), 2 * ca[:5].T @ ca[:5], pts)
    assert_close("rho wfn vs fchk", ra, rb, sc["rho"], 1e-11, atol=1e-15)
    np.testing.assert_array_equal(a.numbers, mol.numbers)
