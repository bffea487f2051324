"""GPU test of ctc_eval_local_noalloc, the FP64 local-descriptor entry point
that takes its scratch from a fixed array inside the library instead of
allocating device memory.

Two calls in a row (different point sets, so the second call runs over the
first call's leftover scratch contents) are each checked against
ctc_eval_local on the same points, at the FP64 tolerance of the parity tests:
1e-10 relative to the per-point sum of absolute terms (tests/helpers.py).
The point counts span several chunks of tiles.  The file is named to be
collected last; it passes alone in a fresh process as well.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import ctc_abi
from helpers import assert_close, term_scales

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
KEYS = ctc_abi.OUT_KEYS
PARAMS = (0.5, 1 / 9, 1 / 6, 1.0)


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _lib():
    L = ctc_abi.lib()
    L.ctc_eval_local_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                         C.c_void_p, C.c_void_p]
    return L


def _noalloc(torch, m, pts, keys=KEYS):
    d = torch.as_tensor(np.ascontiguousarray(pts), dtype=torch.float64, device="cuda")
    n = d.shape[0]
    outs = {k: torch.full((n * ctc_abi.OUT_WIDTH[k],), float("nan"), dtype=torch.float64,
                          device="cuda") for k in keys}
    o = ctc_abi.Outputs(**{k: outs[k].data_ptr() for k in keys})
    p = ctc_abi.Params(*PARAMS)
    ctc_abi.check(_lib().ctc_eval_local_noalloc(m.h, d.data_ptr(), n, C.byref(p), C.byref(o), None),
                  "ctc_eval_local_noalloc")
    torch.cuda.synchronize()
    res = {}
    for k, t in outs.items():
        a = t.cpu().numpy()
        res[k] = a.reshape(n, 3) if k == "grad" else (a.reshape(n, 3, 3) if k == "hess" else a)
    return res


def _compare(name, mol, pts, got, want):
    sc = term_scales(mol.flat(), mol.D, pts, alpha=PARAMS[0], ref=want)
    live = want["rho"] > 1e-10
    for k in ("rho", "grad", "hess", "lap", "tau_pd", "tau_alpha"):
        assert_close(f"{name}/{k}", got[k], want[k], sc[k], 1e-10, atol=1e-14)
    for k in ("rdg", "shannon", "weizsacker", "thomas_fermi", "gge"):
        assert_close(f"{name}/{k}", got[k], want[k], sc[k], 1e-10, atol=1e-14, mask=live)
    assert_close(f"{name}/general_ked", got["general_ked"], want["general_ked"],
                 sc["general_ked"], 1e-10, atol=1e-14)


def test_noalloc_matches_eval_local_on_two_calls(torch_cuda):
    sys.path.insert(0, GOLDEN)
    import cases
    from chemtoolscuda_b200 import synthetic as S
    mol, pts1 = cases.CASES["c1"]()
    rng = np.random.default_rng(11)
    pts1 = np.concatenate([pts1, S.random_points(rng, mol, 6000 - len(pts1), pad=3.0)])
    pts2 = S.random_points(np.random.default_rng(12), mol, 4321, pad=2.0)
    m = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
    try:
        got1 = _noalloc(torch_cuda, m, pts1)
        got2 = _noalloc(torch_cuda, m, pts2)
        want1 = m.eval_local(pts1, KEYS, ctc_abi.PREC_FP64, params=PARAMS)
        want2 = m.eval_local(pts2, KEYS, ctc_abi.PREC_FP64, params=PARAMS)
        _compare("call 1", mol, pts1, got1, want1)
        _compare("call 2", mol, pts2, got2, want2)
        # and against the FP64 oracle directly, on a sample of the second call
        from oracle import oracle as O
        idx = np.random.default_rng(13).choice(len(pts2), 300, replace=False)
        ref = O.eval_local(mol.flat(), mol.D, pts2[idx], alpha=PARAMS[0], keys=tuple(KEYS),
                           gge_ab=(PARAMS[1], PARAMS[2]), ked_a=PARAMS[3])
        _compare("oracle", mol, pts2[idx], {k: v[idx] for k, v in got2.items()}, ref)
    finally:
        m.close()


def test_noalloc_rejects_more_points_than_its_scratch_holds(torch_cuda):
    sys.path.insert(0, GOLDEN)
    import cases
    mol, pts = cases.CASES["c1"]()
    m = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
    try:
        d = torch_cuda.as_tensor(pts, dtype=torch_cuda.float64, device="cuda")
        rho = torch_cuda.empty(len(pts), dtype=torch_cuda.float64, device="cuda")
        o = ctc_abi.Outputs(rho=rho.data_ptr())
        # the count is checked on the host before anything runs on the device
        rc = _lib().ctc_eval_local_noalloc(m.h, d.data_ptr(), (1 << 20) + 1, None, C.byref(o), None)
        assert rc == -1
        assert "maximum of 1048576" in ctc_abi.err()
    finally:
        m.close()
