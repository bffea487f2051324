"""Multi-process host logic of the point sharding (chemtoolscuda_b200.sharding)
on CPU: two gloo ranks on 127.0.0.1.

* shard_bounds covers every point exactly once, ragged sizes included;
* max_over_ranks returns the largest per-rank value on every rank;
* sharded_adjoint: each rank runs the adjoint of its own slice (here the FP64
  oracle stands in for the GPU kernels) and the all-reduced dL/dD and dL/dR
  equal the single-process result to rounding.
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
