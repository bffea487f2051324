"""Cube-file writer and reader (chemtoolscuda_b200.cube): round trip of the
header, atoms and values in the grid order of the cubic-grid evaluation."""
import numpy as np
import pytest

from chemtoolscuda_b200 import cube, synthetic as S


def test_round_trip(tmp_path):
    mol = S.make_molecule("c1", seed=0)
    shape = (5, 7, 9)
    origin, axes = S.cube_grid(mol, 0.3, shape)
    vals = np.random.default_rng(0).standard_normal(shape) * 10.0 ** np.random.default_rng(1).integers(-8, 3, shape)
    p = str(tmp_path / "rho.cube")
    cube.write_cube(p, vals, origin, axes, shape, mol.numbers, mol.coords)
    got = cube.read_cube(p)
    assert got["shape"] == shape
    np.testing.assert_allclose(got["origin"], origin, atol=1e-6)
    np.testing.assert_allclose(got["axes"], axes, atol=1e-6)
    np.testing.assert_array_equal(got["numbers"], mol.numbers)
    np.testing.assert_allclose(got["coords"], mol.coords, atol=1e-6)
    np.testing.assert_allclose(got["values"], vals, rtol=1e-5)
    # the last axis runs fastest, six values per line
    body = open(p).read().splitlines()[6 + len(mol.numbers):]
    assert len(body[0].split()) == 6
    assert float(body[0].split()[1]) == float(f"{vals[0, 0, 1]:13.5E}")


@pytest.mark.gpu
def test_density_cube_from_gpu(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import chemtoolscuda_b200 as ctc
    from oracle import oracle as O
    mol = S.make_molecule("c1", seed=0)
    m = ctc.molecule_from_synthetic(mol)
    shape = (6, 5, 7)
    origin, axes = S.cube_grid(mol, 0.5, shape)
    p = str(tmp_path / "rho.cube")
    rho = cube.write_density_cube(m, p, origin, axes, shape)
    ref = O.eval_local(mol.flat(), mol.D, S.cube_points(origin, axes, shape), keys=("rho",))["rho"]
    from helpers import assert_close, term_scales
    sc = term_scales(mol.flat(), mol.D, S.cube_points(origin, axes, shape))["rho"]
    assert_close("cube file rho", rho.reshape(-1), ref, sc, 1e-12, atol=1e-15)
    got = cube.read_cube(p)
    np.testing.assert_allclose(got["values"], rho, rtol=1e-5, atol=1e-300)
