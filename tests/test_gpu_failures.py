"""Failure paths, made on the host (nothing here faults, traps or hangs a GPU):

* cancellation (src/cancel.rs:22-63): the cancel word set between calls makes
  the next synchronising call fail with WQC_ERR_CANCELLED, and a reset state
  works again;
* a corrupted input site (NaN) gives an error status, not a wrong result
  (the non-finite check of needs_f64_fallback, svd_guard.rs:59-61);
* the memory budget refusal (ensure_mps_workspace_budget, mps.rs:36-48): a
  state larger than the device fails with WQC_ERR_OOM before allocating.
"""
import numpy as np
import pytest

import wqc_cuda as W
from wqc_cuda import circuits as C

pytestmark = pytest.mark.gpu


def test_cancel_between_calls_then_reset(cuda_ctx):
    gates = C.gates_array(C.random_layers(12, 6, seed=8))
    m = W.CudaMps(12, 16, ctx=cuda_ctx)
    m.apply_gates(gates)
    m.cancel()
    with pytest.raises(W.WqcCudaError) as e:
        m.synchronize()
    assert e.value.code == W.ERR_CANCELLED and "cancelled" in str(e.value)
    m.reset()
    m.apply_gates(gates)
    ref = W.CudaMps(12, 16, ctx=cuda_ctx)
    ref.apply_gates(gates)
    assert m.amplitude_zero() == ref.amplitude_zero()


def test_nan_site_gives_an_error_not_a_result(cuda_ctx):
    m = W.CudaMps(4, 4, ctx=cuda_ctx)
    m.apply_gates(C.gates_array([C.g1(C.H, q) for q in range(4)] + [C.g2(C.CNOT, 0, 1), C.g2(C.CNOT, 2, 3)]))
    s = m.site(1)
    s[0, 0, 0] = np.nan
    m.set_site(1, s)
    m.apply_gates(C.gates_array([C.g2(C.CNOT, 1, 2)]))
    with pytest.raises(W.WqcCudaError) as e:
        m.synchronize()
    assert e.value.code == W.ERR_SVD_FAILED and "non-finite" in str(e.value)
    m.reset()  # the next request starts clean
    m.apply_gates(C.gates_array([C.g1(C.X, 3)]))
    assert abs(m.amplitude_zero()) < 1e-15


def test_state_beyond_device_memory_is_refused(cuda_ctx):
    n = 100_000  # 100000 * 256^2 * 32 B = 210 GB of sites alone
    with pytest.raises(W.WqcCudaError) as e:
        W.CudaMps(n, 256, ctx=cuda_ctx)
    assert e.value.code == W.ERR_OOM and "Insufficient memory" in str(e.value)
    # EngineError::InsufficientMemory { required, available } gets both counts
    # through wqc_cuda_last_oom.
    assert e.value.required >= W.workspace_bytes(n, 256) > e.value.available > 0
    assert W.last_oom() == (e.value.required, e.value.available)
    m = W.CudaMps(4, 4, ctx=cuda_ctx)  # the context is still usable
    m.apply_gates(C.gates_array([C.g1(C.H, 0)]))
    assert abs(m.amplitude_zero() - 2 ** -0.5) < 1e-12


def test_uploaded_sites_that_do_not_chain_are_refused(cuda_ctx):
    """An upload whose bonds disagree with its neighbours' is refused by the
    next call that computes on the state, instead of giving wrong results."""
    m = W.CudaMps(4, 8, ctx=cuda_ctx)
    rng = np.random.default_rng(3)
    m.set_site(1, rng.normal(size=(1, 2, 4)) + 0j)  # site 2 still has left bond 1
    with pytest.raises(W.WqcCudaError) as e:
        m.apply_gates(C.gates_array([C.g2(C.CNOT, 0, 1)]))
    assert e.value.code == W.ERR_INVALID and "do not chain" in str(e.value)
    m.set_site(2, rng.normal(size=(4, 2, 1)) + 0j)  # now 1 x 2 x 4 | 4 x 2 x 1 closes the chain
    m.apply_gates(C.gates_array([C.g2(C.CNOT, 0, 1)]))
    assert np.isfinite(m.amplitude_zero())
