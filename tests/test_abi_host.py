"""CPU checks of the drop-in boundary and the host logic (no device work).

* libwqc_cuda.so loads and exports every entry point include/*.h declares;
* without a device, opening a context fails with WQC_ERR_NO_DEVICE instead
  of crashing or falling back to the CPU;
* the Python bindings pass their arguments through ctypes to the library,
  which rejects a null state before any device work;
* the host scheduler expands gates into the reference's split sequence and
  keeps every site's operations in program order;
* the circuit generators match their stated shapes.
"""
import os
import re

import numpy as np
import pytest

import wqc_cuda as W
from wqc_cuda import circuits as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        names |= set(re.findall(r"^WQC_API\s+[\w\s\*]+?\b(wqc_\w+)\s*\(", text, flags=re.M))
    return names


def test_library_exports_every_declared_entry_point():
    names = declared_entry_points()
    assert len(names) >= 30
    lib = W.lib()
    for name in sorted(names):
        assert hasattr(lib, name), f"{name} is declared in include/ but not exported"
    assert set(W.EXPORTS) == names


def test_open_without_device_reports_no_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import ctypes

    h = ctypes.c_void_p()
    rc = W.lib().wqc_cuda_open(-1, ctypes.byref(h))
    assert rc == W.ERR_NO_DEVICE
    assert W.lib().wqc_cuda_last_error()


def test_bindings_reach_the_library_with_a_null_state():
    """Every binding that takes a state handle passes its arguments through
    ctypes to the library, which rejects a null handle before any device
    work: this checks the Python side of the boundary without a GPU."""
    fake = W.CudaMps.__new__(W.CudaMps)
    fake._h = None
    fake.n = 4
    calls = [
        lambda: fake.sample([0, 2], 3, 7),
        lambda: fake.sample_counts([(0, 0)], 1, 3, 7),
        lambda: fake.expectation(["ZZZZ"], [1.0]),
        lambda: fake.set_merge(W.MERGE_TC_INT8),
    ]
    for call in calls:
        with pytest.raises(W.WqcCudaError) as e:
            call()
        assert e.value.code == W.ERR_INVALID and "null" in str(e.value)
    with pytest.raises(W.WqcCudaError) as e:
        fake.sample_counts([(4, 0)], 1, 3, 7)  # checked on the host, as compute_outcome_probabilities does
    assert e.value.code == W.ERR_QUBIT_OUT_OF_RANGE
    with pytest.raises(W.WqcCudaError) as e:
        fake.sample_counts([(0, 2)], 2, 3, 7)
    assert e.value.code == W.ERR_INVALID and "classical bit index 2" in str(e.value)


def test_tensor_core_gemms_reject_a_null_context_before_device_work():
    """wqc_tc_zgemm and wqc_tc_zgemm_int8 check their arguments on the host:
    a null context is refused without touching a device."""
    import numpy as np

    from wqc_cuda import tc as T

    class NoCtx:
        _h = None

    a, b = np.ones((3, 2), dtype=complex), np.ones((2, 4), dtype=complex)
    for form in ("tf32x3", "int8"):
        with pytest.raises(W.WqcCudaError) as e:
            T.zgemm(a, b, ctx=NoCtx(), form=form)
        assert e.value.code == W.ERR_INVALID and "null" in str(e.value)
    with pytest.raises(ValueError):
        T.zgemm(a, b, ctx=NoCtx(), form="fp16")


def test_workspace_bytes_matches_reference_formula():
    assert W.workspace_bytes(100, 128) == 52_428_800  # mps.rs:1870-1889
    assert W.workspace_bytes(50, 128) == 50 * 128 * 128 * 32


def test_schedule_matches_reference_split_sequence_and_keeps_site_order():
    for gates, n in ((C.config0().gates, 16), (C.config1(n=30, depth=12).gates, 30),
                     (C.gates_array(C.large_chi(n=24, depth=20)), 24)):
        site, level, nlevels = W.schedule(n, gates)
        assert len(site) == C.split_plan(gates)
        # splits of one level are disjoint
        for L in range(nlevels):
            s = site[level == L]
            touched = np.concatenate([s, s + 1])
            assert len(set(touched.tolist())) == len(touched)
        # each site sees its splits at strictly increasing levels, in program order
        last = np.full(n, -1)
        for p, L in zip(site, level):
            assert L > last[p] and L > last[p + 1]
            last[p] = last[p + 1] = L


def test_schedule_routes_long_range_gates_with_swaps():
    """mps.rs:353-375: CNOT(0, 3) is swaps at 2, 1, the gate at 0, swaps at 1, 2."""
    site, level, _ = W.schedule(4, C.gates_array([C.g2(C.CNOT, 0, 3)]))
    assert site.tolist() == [2, 1, 0, 1, 2]
    assert level.tolist() == [0, 1, 2, 3, 4]
    site, _, _ = W.schedule(3, C.gates_array([C.g3(0, 1, 2)]))
    assert len(site) == 10  # 6 CNOTs, the two CNOT(0, 2) routed over site 1


def test_schedule_rejects_bad_gates():
    with pytest.raises(W.WqcCudaError) as e:
        W.schedule(4, C.gates_array([C.g2(C.CNOT, 0, 4)]))
    assert e.value.code == W.ERR_QUBIT_OUT_OF_RANGE
    with pytest.raises(W.WqcCudaError):
        W.schedule(4, C.gates_array([C.g2(C.CZ, 2, 2)]))


def test_generators_have_the_stated_shapes():
    w0 = C.config0()
    assert (w0.n, w0.chi) == (16, 32)
    assert int(np.sum(np.isin(w0.gates["kind"], [C.CNOT]))) == 10 * 8 + 10 * 7
    w1 = C.config1()
    assert (w1.n, w1.chi) == (50, 128)
    k = w1.gates["kind"]
    assert int(np.sum(np.isin(k, list(C.ONE_QUBIT)))) == 50 * 40
    d = np.abs(w1.gates["q0"] - w1.gates["q1"])[np.isin(k, [C.CNOT, C.CZ])]
    assert d.min() == 1 and d.max() <= 8 and int(np.sum(d > 1)) == 5 * 40
    slices = C.config2_slices(16)
    assert all(20 <= s.n <= 60 and s.chi in (16, 32, 64, 128) for s in slices)
    g, pidx, params = C.hea_ansatz()
    assert len(params) == 512 and int(np.sum(pidx >= 0)) == 512
    labels, coeffs = C.zz_x_observable(32)
    assert len(labels) == 63 and all(len(x) == 32 for x in labels)


def test_cuda_request_without_device_fails():
    """A `cuda` request without a device is reported as unavailable and no
    state is built: there is no CPU fallback (engine_status.rs:40-84)."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    st = W.probe_tn_engine_status("cuda")
    assert st["active"] == "unavailable" and "CUDA device not found" in st["note"]
    with pytest.raises(W.WqcCudaError) as e:
        W.CudaMps(4, 8)
    assert e.value.code == W.ERR_NO_DEVICE


def test_oom_byte_counts_start_at_zero():
    """wqc_cuda_last_oom is exported and reports (0, 0) before any OOM on
    this thread."""
    import threading

    out = []
    t = threading.Thread(target=lambda: out.append(W.last_oom()))
    t.start()
    t.join()
    assert out == [(0, 0)]


def test_pauli_labels_are_checked_before_the_c_abi():
    """The C ABI reads nterms * width label bytes and 2 * nterms doubles; the
    binding refuses short labels and short coefficient arrays first."""
    fake = W.CudaMps.__new__(W.CudaMps)
    fake._h = None
    fake.n = 4
    with pytest.raises(ValueError, match="characters"):
        fake.expectation(["ZZZ"], [1.0])
    with pytest.raises(ValueError, match="coefficients"):
        fake.expectation(["ZZZZ", "XXXX"], [1.0])
    with pytest.raises(ValueError, match="characters"):
        W.expectation_pauli_noalloc(0, 8, [2, 2, 1], ["ZZ"], [1.0])
    with pytest.raises(ValueError, match="coefficients"):
        W.expectation_pauli_noalloc(0, 8, [2, 2, 1], ["ZZZ"], [])
