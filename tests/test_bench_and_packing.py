"""CPU checks of two pieces of host-side logic that the GPU tests only reach
indirectly:

* bench.py's parity measure (largest error over a point sample relative to the
  sum of absolute terms, with the test suite's absolute floor) and its DRAM
  traffic scaling (per-tile figure x tiles per launch);
* the cut counts of the sort-tile-recursive packing of explicit points
  (chemtoolscuda_b200/csrc/ctc_tiles.cuh, str_shape): restated here, they must
  keep every group id below the key bits the radix sorts use (2 P for P tiles),
  give whole tiles per slab and column, and near-cubic tiles for box-shaped
  point sets."""
import importlib.util
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod
    spec.loader.exec_module(mod)
    return mod


def test_sample_errors_use_the_absolute_floor(bench):
    got = {"rho": np.array([1.0, 2.0 + 1e-9, 0.0])}
    ref = {"rho": np.array([1.0, 2.0, 5e-15])}
    scale = {"rho": np.array([1.0, 2.0, 1e-20])}
    err = bench._sample_errors(got, ref, scale, ("rho",))["rho"]
    # point 1: (1e-9 - 1e-14) / 2; point 2: below the 1e-14 floor -> 0
    assert err == pytest.approx((1e-9 - 1e-14) / 2.0, rel=1e-6)


def test_profile_traffic_scales_per_tile_bytes(bench):
    per_tile = bench.profile_traffic("tc_tile_kernel", 1.0)
    assert per_tile is not None and per_tile > 1e6
    assert bench.profile_traffic("tc_tile_kernel", 1863.5) == pytest.approx(per_tile * 1863.5)
    assert bench.profile_traffic("no_such_kernel", 10.0) is None


def str_shape(L, P, TP):
    """Restatement of str_shape (ctc_tiles.cuh): slabs along x, columns along y."""
    Lmax = max(L) if max(L) > 0 else 1.0
    L = [max(x, 1e-3 * Lmax) for x in L]
    a = (L[0] * L[1] * L[2] / P) ** (1.0 / 3.0)
    sx = int(min(max(round(L[0] / a), 1.0), P))
    Tsl = (P + sx - 1) // sx
    sy = int(min(max(round(L[1] / a), 1.0), Tsl))
    Tcol = (Tsl + sy - 1) // sy
    sy = (Tsl + Tcol - 1) // Tcol
    return Tsl * TP, Tcol * TP, sy


@pytest.mark.parametrize("seed", range(5))
def test_str_group_ids_fit_the_sort_bits(seed):
    rng = np.random.default_rng(seed)
    for _ in range(2000):
        TP = int(rng.choice([32, 128]))
        n = int(rng.integers(1, 3_000_000))
        P = (n + TP - 1) // TP
        L = list(rng.uniform(0, 60, 3) * (rng.random(3) > 0.1))  # some flat or linear sets
        Sx, Scol, c = str_shape(L, P, TP)
        assert Sx % TP == 0 and Scol % TP == 0, "slabs and columns hold whole tiles"
        last = n - 1
        g1 = last // Sx
        g2 = (last // Sx) * c + (last % Sx) // Scol
        gbits = (2 * P).bit_length()
        assert g1 < 2 ** gbits and g2 < 2 ** gbits


def test_str_tiles_of_a_uniform_box_are_near_cubic():
    """A uniform grid of points in a box: slab and column counts follow the box's
    aspect ratio, so a tile spans about the same number of points per axis."""
    for dims in [(215, 215, 215), (23, 215, 215), (96, 40, 200)]:
        n = int(np.prod(dims))
        TP = 32
        P = (n + TP - 1) // TP
        L = [d - 1.0 for d in dims]
        Sx, Scol, c = str_shape(L, P, TP)
        per_plane = dims[1] * dims[2]
        x_thick = Sx / per_plane                 # grid planes per slab
        y_rows = Scol / (x_thick * dims[2])       # grid rows per column
        z_run = TP / (x_thick * y_rows)           # points along z per tile
        edges = np.array([x_thick, y_rows, z_run])
        assert edges.max() / edges.min() < 1.6, (dims, edges)
        assert abs(math.prod(edges) - TP) < 1e-6 * TP
