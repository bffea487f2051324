"""Multi-process host logic of the point sharding (chemtoolscuda_b200.sharding)
on CPU: two gloo ranks on 127.0.0.1.

* shard_bounds covers every point exactly once, ragged sizes included;
* max_over_ranks returns the largest per-rank value on every rank;
* sharded_adjoint: each rank runs the adjoint of its own slice (here the FP64
  oracle stands in for the GPU kernels) and the all-reduced dL/dD and dL/dR
  equal the single-process result to rounding;
* sharded_cubic / sharded_points: each rank evaluates its x-slab of one cubic
  grid (or its slice of the points) -- the oracle again standing in for the
  GPU -- and the slabs, in place or gathered, equal the whole grid evaluated
  in one process.
"""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from chemtoolscuda_b200.sharding import shard_bounds

WORLD = 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    from chemtoolscuda_b200 import synthetic as S
    mol = S.make_molecule("c1", seed=5, natom=4, box=5.0, nocc=6)
    rng = np.random.default_rng(8)
    pts = S.random_points(rng, mol, 301, pad=2.0)
    vr = rng.standard_normal(len(pts))
    vg = rng.standard_normal((len(pts), 3))
    return mol, pts, vr, vg


def _oracle_adjoint(mol):
    import torch
    from oracle import oracle as O

    def f(points, v_rho, v_grad):
        dD, dR = O.adjoint(mol.flat(), mol.D, len(mol.coords), points.numpy(), v_rho.numpy(),
                           None if v_grad is None else v_grad.numpy())
        return torch.from_numpy(np.ascontiguousarray(dD)), torch.from_numpy(np.ascontiguousarray(dR))

    return f


def _worker(rank, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    from chemtoolscuda_b200.sharding import max_over_ranks, rank_world, sharded_adjoint
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=WORLD,
                                timeout=datetime.timedelta(seconds=60))
        assert rank_world() == (rank, WORLD)
        mx = max_over_ranks(1.5 + rank)
        mol, pts, vr, vg = _case()
        dD, dR = sharded_adjoint(torch.from_numpy(pts), torch.from_numpy(vr), torch.from_numpy(vg),
                                 adjoint=_oracle_adjoint(mol))
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, mx, dD.numpy(), dR.numpy(), None))
    except Exception as e:  # report to the parent instead of hanging it
        q.put((rank, None, None, None, repr(e)))


GRID_SHAPE = (7, 5, 6)   # 7 x-planes: ragged over 2 ranks


def _grid(mol):
    from chemtoolscuda_b200 import synthetic as S
    return S.cube_grid(mol, 0.45, GRID_SHAPE)


def _oracle_cubic(mol, keys):
    import torch
    from chemtoolscuda_b200 import synthetic as S
    from oracle import oracle as O

    def f(origin, axes, shape):
        pts = S.cube_points(origin, axes, shape)
        r = O.eval_local(mol.flat(), mol.D, pts, keys=keys)
        return {k: torch.from_numpy(np.ascontiguousarray(v)) for k, v in r.items()}

    return f


def _oracle_points(mol, keys):
    import torch
    from oracle import oracle as O

    def f(points):
        r = O.eval_local(mol.flat(), mol.D, points.numpy(), keys=keys)
        return {k: torch.from_numpy(np.ascontiguousarray(v)) for k, v in r.items()}

    return f


def _forward_worker(rank, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    from chemtoolscuda_b200.sharding import sharded_cubic, sharded_points
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=WORLD,
                                timeout=datetime.timedelta(seconds=60))
        mol, pts, _, _ = _case()
        origin, axes = _grid(mol)
        keys = ("rho", "grad")
        lo, hi, own = sharded_cubic(origin, axes, GRID_SHAPE, evaluate=_oracle_cubic(mol, keys), keys=keys)
        _, _, full = sharded_cubic(origin, axes, GRID_SHAPE, evaluate=_oracle_cubic(mol, keys),
                                   keys=keys, gather=True)
        plo, phi, pown = sharded_points(torch.from_numpy(pts), evaluate=_oracle_points(mol, keys), keys=keys)
        _, _, pfull = sharded_points(torch.from_numpy(pts), evaluate=_oracle_points(mol, keys), keys=keys,
                                     gather=True)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, dict(lo=lo, hi=hi, own={k: v.numpy() for k, v in own.items()},
                          full={k: v.numpy() for k, v in full.items()}, plo=plo, phi=phi,
                          pown={k: v.numpy() for k, v in pown.items()},
                          pfull={k: v.numpy() for k, v in pfull.items()}), None))
    except Exception as e:  # report to the parent instead of hanging it
        q.put((rank, None, repr(e)))


def test_two_gloo_ranks_sharded_forward():
    from chemtoolscuda_b200 import synthetic as S
    from oracle import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_forward_worker, args=(r, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    res = {}
    try:
        for _ in range(WORLD):
            rank, r, err = q.get(timeout=240)
            assert err is None, f"rank {rank}: {err}"
            res[rank] = r
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    mol, pts, _, _ = _case()
    origin, axes = _grid(mol)
    keys = ("rho", "grad")
    whole = O.eval_local(mol.flat(), mol.D, S.cube_points(origin, axes, GRID_SHAPE), keys=keys)
    wp = O.eval_local(mol.flat(), mol.D, pts, keys=keys)
    plane = GRID_SHAPE[1] * GRID_SHAPE[2]
    covered = []
    for rank in range(WORLD):
        r = res[rank]
        assert (r["lo"], r["hi"]) == shard_bounds(GRID_SHAPE[0], rank, WORLD)
        covered.extend(range(r["lo"], r["hi"]))
        for k in keys:
            np.testing.assert_allclose(r["own"][k], whole[k][r["lo"] * plane:r["hi"] * plane],
                                       rtol=1e-13, atol=1e-16)
            np.testing.assert_allclose(r["full"][k], whole[k], rtol=1e-13, atol=1e-16)
            np.testing.assert_allclose(r["pown"][k], wp[k][r["plo"]:r["phi"]], rtol=1e-13, atol=1e-16)
            np.testing.assert_allclose(r["pfull"][k], wp[k], rtol=1e-13, atol=1e-16)
    assert covered == list(range(GRID_SHAPE[0]))


@pytest.mark.parametrize("n", [0, 1, 2, 7, 301, 1000])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_bounds_partition(n, world):
    seen = []
    for r in range(world):
        lo, hi = shard_bounds(n, r, world)
        assert 0 <= lo <= hi <= n
        assert hi - lo in (n // world, n // world + 1)
        seen.extend(range(lo, hi))
    assert seen == list(range(n))


def test_shard_bounds_rejects_bad_rank():
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)
    with pytest.raises(ValueError):
        shard_bounds(-1, 0, 1)


def test_two_gloo_ranks_adjoint_and_timing_reduction():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    res = {}
    try:
        for _ in range(WORLD):
            rank, mx, dD, dR, err = q.get(timeout=240)
            assert err is None, f"rank {rank}: {err}"
            res[rank] = (mx, dD, dR)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    from oracle import oracle as O
    mol, pts, vr, vg = _case()
    rD, rR = O.adjoint(mol.flat(), mol.D, len(mol.coords), pts, vr, vg)
    for rank in range(WORLD):
        mx, dD, dR = res[rank]
        assert mx == 1.5 + (WORLD - 1)
        np.testing.assert_allclose(dD, rD, rtol=0, atol=1e-12 * np.abs(rD).max())
        np.testing.assert_allclose(dR, rR, rtol=0, atol=1e-12 * np.abs(rR).max())
