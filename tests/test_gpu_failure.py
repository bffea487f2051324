"""Failure paths on the GPU, made to happen without faulting anything.

* A bounded wait of the tensor-core pipeline that runs out: the molecule's
  wait limit is cut to one SM cycle, so the kernel's waits give up at once.
  The kernel must stop, wait for its own copies in flight, free its tensor
  memory and record CTC_ERR_DEVICE, which ctc_molecule_sync_status (or the
  next call on the molecule) reports; with the limit restored the molecule
  gives correct results again.
* Points with NaN or infinite coordinates: NaN in every output of those
  points, the other points unaffected.
* A scratch allocation that fails: CTC_SCRATCH_LIMIT_BYTES makes the
  molecule's scratch allocation fail as if the device were out of memory;
  the call returns CTC_ERR_NOMEM and the next call works.
* A second device, when one is visible (skipped otherwise): kernels whose
  shared-memory limit is a per-device attribute must run there too.

The reference has none of these paths: its drivers turn a cudaError_t into a
C++ exception (include/cuda_utils.cuh:55-60)."""
import os

import numpy as np
import pytest

import ctc_abi
from helpers import assert_close, term_scales
from oracle import oracle as O

pytestmark = pytest.mark.gpu
KEYS = ("rho", "grad", "hess", "lap", "tau_pd", "tau_alpha")


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _case(name="mixed"):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import cases
    return cases.CASES[name]()


def _check(mol, pts, got, rtol):
    ref = O.eval_local(mol.flat(), mol.D, pts, alpha=0.5, keys=KEYS)
    sc = term_scales(mol.flat(), mol.D, pts, alpha=0.5)
    for k in KEYS:
        assert_close(k, got[k], ref[k], sc[k], rtol, atol=1e-15)


def test_tc_wait_timeout_is_reported_and_the_molecule_recovers(torch_cuda):
    mol, pts = _case()
    m = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
    assert m.sync_status() == 0
    m.set_wait_limit(1)
    m.eval_local(pts, KEYS, ctc_abi.PREC_TC)          # stream-ordered: returns CTC_OK
    assert m.sync_status() == -5, "a one-cycle wait limit must run out"
    assert "bounded wait" in ctc_abi.err()
    assert m.sync_status() == 0                       # reporting clears the record
    # the next call reports an earlier call's failure once its copy has landed
    m.eval_local(pts, KEYS, ctc_abi.PREC_TC)
    m.set_wait_limit(0)
    with pytest.raises(RuntimeError, match="earlier call"):
        m.eval_local(pts, KEYS, ctc_abi.PREC_TC)
    # default limit: correct results, nothing recorded
    got = m.eval_local(pts, KEYS, ctc_abi.PREC_TC)
    assert m.sync_status() == 0
    _check(mol, pts, got, 1e-8)
    m.close()


@pytest.mark.parametrize("precision,rtol", [(ctc_abi.PREC_FP64, 1e-10), (ctc_abi.PREC_TC, 1e-8)])
def test_non_finite_points(torch_cuda, precision, rtol):
    mol, pts = _case()
    bad = pts.copy()
    rows = [3, 17, 40, len(pts) - 1]
    bad[rows[0], 0] = np.nan
    bad[rows[1], 1] = np.inf
    bad[rows[2], 2] = -np.inf
    bad[rows[3]] = np.nan
    m = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
    keys = ctc_abi.OUT_KEYS
    got = m.eval_local(bad, keys, precision)
    for k in keys:
        assert np.isnan(got[k][rows]).all(), f"{k}: non-finite points must give NaN"
    ok = np.setdiff1d(np.arange(len(pts)), rows)
    _check(mol, pts[ok], {k: got[k][ok] for k in KEYS}, rtol)
    m.close()


def test_scratch_allocation_failure_and_recovery(torch_cuda):
    mol, pts = _case()
    m = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
    os.environ["CTC_SCRATCH_LIMIT_BYTES"] = "4096"
    try:
        with pytest.raises(RuntimeError, match="-4: .*CTC_SCRATCH_LIMIT_BYTES"):
            m.eval_local(pts, KEYS, ctc_abi.PREC_FP64)
    finally:
        del os.environ["CTC_SCRATCH_LIMIT_BYTES"]
    got = m.eval_local(pts, KEYS, ctc_abi.PREC_FP64)
    _check(mol, pts, got, 1e-10)
    m.close()


def test_second_device(torch_cuda):
    """Every kernel configured per device: FP64, tensor-core and no-allocation
    paths on device 1 after device 0 has used them."""
    torch = torch_cuda
    if torch.cuda.device_count() < 2:
        pytest.skip("one visible device")
    mol, pts = _case()
    m0 = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
    m0.eval_local(pts, KEYS, ctc_abi.PREC_TC)
    m0.close()
    with torch.cuda.device(1):
        m1 = ctc_abi.Mol(mol.flat(), mol.coords, mol.charges, mol.D)
        for prec, rtol in ((ctc_abi.PREC_FP64, 1e-10), (ctc_abi.PREC_TC, 1e-8)):
            _check(mol, pts, m1.eval_local(pts, KEYS, prec), rtol)
        m1.close()
