"""Python binding of the `WQC_TN_BACKEND=cuda` MPS backend (libwqc_cuda.so).

``CudaMps`` mirrors the reference's ``MpsState`` (src/tn/mps.rs:55-781):
the same operations under the same names, all executed by the sm_100a
kernels behind the C ABI in include/wqc_cuda.h.  There is no CPU fallback:
importing this module fails when the shared library is missing, and every
call raises ``WqcCudaError`` when the device reports an error.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

from .circuits import GATE_DTYPE, SPLIT_INFO_DTYPE, gates_array  # noqa: F401

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "libwqc_cuda.so")

OK = 0
ERR_INVALID = 1
ERR_OOM = 2
ERR_TRUNCATION_REJECTED = 3
ERR_SVD_FAILED = 4
ERR_CANCELLED = 5
ERR_DEVICE_TIMEOUT = 6
ERR_CUDA = 7
ERR_NO_DEVICE = 8
ERR_QUBIT_OUT_OF_RANGE = 9
ERR_INVALID_QUBIT_COUNT = 10

PRECISION_FP64 = 0
PRECISION_FP32 = 1
PRECISION_TF32X3 = 2
MERGE_FFMA = 0
MERGE_TC_INT8 = 1
OVERLAP_ENV_LIMIT = 256  # mps.rs:1443-1448 (the STARK witness limit)
SPLIT_RULE_REFERENCE = 0
SPLIT_RULE_EXACT = 1

# Exported entry points of include/wqc_cuda.h (checked by the ABI tests).
EXPORTS = (
    "wqc_cuda_last_error", "wqc_cuda_open", "wqc_cuda_close", "wqc_cuda_device_info", "wqc_mps_workspace_bytes",
    "wqc_mps_create", "wqc_mps_destroy", "wqc_mps_apply_gates", "wqc_mps_apply_gates_adjoint", "wqc_mps_apply_1q",
    "wqc_mps_apply_2q", "wqc_mps_apply_2q_routed", "wqc_mps_apply_layer", "wqc_mps_synchronize", "wqc_mps_cancel",
    "wqc_mps_amplitude_zero", "wqc_mps_site_amplitudes", "wqc_mps_bond_dims", "wqc_mps_download_site",
    "wqc_mps_upload_site", "wqc_mps_expectation_pauli", "wqc_mps_set_split_rule", "wqc_mps_split_count", "wqc_mps_split_records",
    "wqc_mps_peak_vram_bytes", "wqc_mps_backend_label", "wqc_mps_set_profiling", "wqc_mps_kernel_stats",
    "wqc_mps_reset_stats", "wqc_mps_stream", "wqc_schedule_gates", "wqc_mps_reset", "wqc_mps_debug_workspace",
    "wqc_batch_create", "wqc_batch_apply_gates", "wqc_batch_amplitudes", "wqc_batch_slice_times",
    "wqc_expectation_pauli_noalloc", "wqc_batch_expectation_pauli", "wqc_mps_sample",
    "wqc_mps_overlap", "wqc_cuda_last_oom", "wqc_mps_site_amplitudes_many", "wqc_mps_to_dense",
    "wqc_adjoint_forward", "wqc_adjoint_backward", "wqc_adjoint_destroy", "wqc_cuda_autotune",
    "wqc_exact_create", "wqc_exact_destroy", "wqc_exact_validate", "wqc_exact_measured_peak", "wqc_exact_contract",
    "wqc_exact_cancel", "wqc_exact_last_stats", "wqc_exact_set_tile_bits",
    "wqc_network_create", "wqc_network_destroy", "wqc_network_validate", "wqc_network_measured_peak",
    "wqc_network_contract", "wqc_network_cancel", "wqc_network_last_stats", "wqc_tc_zgemm", "wqc_tc_zgemm_int8", "wqc_mps_set_merge",
)

KERNEL_KINDS = ("jacobi_svd", "merge_gate", "range_finder", "one_qubit", "cut_absorb")


class WqcCudaError(RuntimeError):
    """A failing C ABI call.  For WQC_ERR_OOM, ``required`` and ``available``
    carry the byte counts of EngineError::InsufficientMemory (src/engine.rs:72)."""

    def __init__(self, code: int, message: str, required: int = 0, available: int = 0):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.required = required
        self.available = available


class KernelStats(ctypes.Structure):
    _fields_ = [
        ("launches", ctypes.c_uint64 * 5),
        ("milliseconds", ctypes.c_double * 5),
        ("total_launches", ctypes.c_uint64),
        ("h2d_bytes", ctypes.c_uint64),
        ("d2h_bytes", ctypes.c_uint64),
        ("jacobi_tasks", ctypes.c_uint64),
        ("jacobi_sweeps", ctypes.c_uint64),
        ("jacobi_sweeps_first", ctypes.c_uint64),
    ]


def build() -> str:
    """Compile libwqc_cuda.so in place for sm_100a."""
    subprocess.run(["make", "-s", "-C", _PKG], check=True)
    return LIB_PATH


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built (run make -C {_PKG}); the cuda backend has no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        P, I, U32, U8, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint8, ctypes.POINTER(ctypes.c_double)
        L.wqc_cuda_last_error.restype = ctypes.c_char_p
        L.wqc_cuda_last_oom.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
        L.wqc_cuda_last_oom.restype = None
        L.wqc_cuda_open.argtypes = [I, ctypes.POINTER(P)]
        L.wqc_cuda_close.argtypes = [P]
        L.wqc_cuda_autotune.argtypes = [P, ctypes.c_char_p, ctypes.c_double, ctypes.POINTER(U32)]
        L.wqc_cuda_device_info.argtypes = [P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                           ctypes.POINTER(ctypes.c_int32)]
        L.wqc_mps_workspace_bytes.argtypes = [U32, U32]
        L.wqc_mps_workspace_bytes.restype = ctypes.c_uint64
        L.wqc_mps_create.argtypes = [P, U32, U32, ctypes.c_int32, U8, ctypes.POINTER(P)]
        L.wqc_mps_destroy.argtypes = [P]
        L.wqc_mps_reset.argtypes = [P]
        L.wqc_mps_apply_gates.argtypes = [P, P, U32]
        L.wqc_mps_apply_gates_adjoint.argtypes = [P, P, U32]
        L.wqc_mps_apply_1q.argtypes = [P, U32, D]
        L.wqc_mps_apply_2q.argtypes = [P, U32, D, U8, P]
        L.wqc_mps_apply_2q_routed.argtypes = [P, U32, U32, D]
        L.wqc_mps_apply_layer.argtypes = [P, P, U32]
        L.wqc_mps_set_split_rule.argtypes = [P, ctypes.c_int32]
        L.wqc_mps_set_merge.argtypes = [P, ctypes.c_int32]
        L.wqc_mps_synchronize.argtypes = [P]
        L.wqc_mps_cancel.argtypes = [P]
        L.wqc_mps_cancel.restype = None
        L.wqc_mps_amplitude_zero.argtypes = [P, D]
        L.wqc_mps_site_amplitudes.argtypes = [P, U32, D]
        L.wqc_mps_site_amplitudes_many.argtypes = [P, ctypes.POINTER(U32), U32, D]
        L.wqc_mps_to_dense.argtypes = [P, ctypes.c_int32, D]
        L.wqc_adjoint_forward.argtypes = [P, P, U32, ctypes.POINTER(U32), U32, ctypes.POINTER(P)]
        L.wqc_adjoint_backward.argtypes = [P, ctypes.c_char_p, D, U32, D, D]
        L.wqc_adjoint_destroy.argtypes = [P]
        L.wqc_adjoint_destroy.restype = None
        L.wqc_mps_bond_dims.argtypes = [P, ctypes.POINTER(U32)]
        L.wqc_mps_download_site.argtypes = [P, U32, ctypes.POINTER(U32), ctypes.POINTER(U32), D]
        L.wqc_mps_upload_site.argtypes = [P, U32, U32, U32, D]
        L.wqc_mps_expectation_pauli.argtypes = [P, ctypes.c_char_p, D, U32, D]
        L.wqc_mps_overlap.argtypes = [P, P, U32, D]
        L.wqc_mps_sample.argtypes = [P, ctypes.POINTER(U32), U32, U32, ctypes.c_uint64,
                                     ctypes.POINTER(ctypes.c_uint64)]
        L.wqc_mps_split_count.argtypes = [P]
        L.wqc_mps_split_count.restype = U32
        L.wqc_mps_split_records.argtypes = [P, P, U32, ctypes.POINTER(U32)]
        L.wqc_mps_peak_vram_bytes.argtypes = [P]
        L.wqc_mps_peak_vram_bytes.restype = ctypes.c_uint64
        L.wqc_mps_backend_label.argtypes = [P]
        L.wqc_mps_backend_label.restype = ctypes.c_char_p
        L.wqc_mps_set_profiling.argtypes = [P, ctypes.c_int32]
        L.wqc_mps_kernel_stats.argtypes = [P, ctypes.POINTER(KernelStats)]
        L.wqc_mps_reset_stats.argtypes = [P]
        L.wqc_mps_reset_stats.restype = None
        L.wqc_schedule_gates.argtypes = [U32, P, U32, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                         U32, ctypes.POINTER(U32), ctypes.POINTER(U32)]
        L.wqc_mps_debug_workspace.argtypes = [P, U32, ctypes.c_int32, P, ctypes.c_uint64]
        L.wqc_batch_create.argtypes = [P, U32, ctypes.POINTER(U32), ctypes.POINTER(U32), ctypes.c_int32, U32,
                                       ctypes.POINTER(P)]
        L.wqc_batch_apply_gates.argtypes = [P, P, ctypes.POINTER(U32)]
        L.wqc_batch_amplitudes.argtypes = [P, D]
        L.wqc_batch_slice_times.argtypes = [P, D]
        L.wqc_batch_expectation_pauli.argtypes = [P, ctypes.c_char_p, D, U32, D]
        L.wqc_mps_stream.argtypes = [P]
        L.wqc_mps_stream.restype = P
        L.wqc_expectation_pauli_noalloc.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(U32), U32, ctypes.c_char_p, D,
                                                    U32, P, D]
        _LIB = L
    return _LIB


def last_oom():
    """(required, available) bytes of the last WQC_ERR_OOM on this thread."""
    req, avail = ctypes.c_uint64(), ctypes.c_uint64()
    lib().wqc_cuda_last_oom(ctypes.byref(req), ctypes.byref(avail))
    return req.value, avail.value


def _check(rc: int) -> None:
    if rc != OK:
        msg = lib().wqc_cuda_last_error().decode()
        if rc == ERR_OOM:
            raise WqcCudaError(rc, msg, *last_oom())
        raise WqcCudaError(rc, msg)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _c128(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex128)


def _pauli_args(labels, coeffs, width: int):
    """Labels joined for the C ABI and coefficients as complex128, after the
    checks the C side cannot make: it reads nterms * width label bytes and
    2 * nterms doubles, so a short label or a short coefficient array would
    be read past its end."""
    labels = list(labels)
    c = _c128(coeffs).reshape(-1)
    if len(c) != len(labels):
        raise ValueError(f"{len(labels)} Pauli labels but {len(c)} coefficients")
    for i, lab in enumerate(labels):
        if len(lab) != width:
            raise ValueError(f"Pauli label {i} has {len(lab)} characters; the register has {width} qubits")
    return "".join(labels).encode(), c


class Context:
    """The process-wide device context (engine_status.rs:27 shared device)."""

    _shared = None

    def __init__(self, device: int = -1):
        h = ctypes.c_void_p()
        _check(lib().wqc_cuda_open(device, ctypes.byref(h)))
        self._h = h

    @classmethod
    def shared(cls) -> "Context":
        if cls._shared is None:
            cls._shared = Context()
        return cls._shared

    def autotune(self, cache_path: str | None = None, budget_seconds: float = 0.0) -> int:
        """Measured Jacobi cluster sizes for this device (wqc_cuda_autotune),
        loaded from the fingerprinted cache when it matches; the number of
        tuned shapes."""
        n = ctypes.c_uint32()
        _check(lib().wqc_cuda_autotune(self._h, cache_path.encode() if cache_path else None, float(budget_seconds),
                                       ctypes.byref(n)))
        return n.value

    def device_info(self):
        tot, fr, sm = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_int32()
        _check(lib().wqc_cuda_device_info(self._h, ctypes.byref(tot), ctypes.byref(fr), ctypes.byref(sm)))
        return {"total_bytes": tot.value, "free_bytes": fr.value, "sm_count": sm.value}


def probe_tn_engine_status(requested: str = "cuda") -> dict:
    """The backend probe of src/tn/engine_status.rs:40-84 for a `cuda`
    request: active "cuda" when a context opens, else "unavailable" with the
    reason.  There is no CPU fallback, so a state cannot be built then."""
    if requested != "cuda":
        return {"requested": requested, "active": requested, "note": None}
    try:
        Context.shared()
    except WqcCudaError as e:
        return {"requested": "cuda", "active": "unavailable", "note": f"CUDA device not found: {e}"}
    return {"requested": "cuda", "active": "cuda", "note": None}


def schedule(n: int, gates: np.ndarray):
    """Host-only: (left site per split, level per split, number of levels)
    of the schedule wqc_mps_apply_gates uses; needs no device."""
    g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
    ns, nl = ctypes.c_uint32(), ctypes.c_uint32()
    _check(lib().wqc_schedule_gates(n, g.ctypes.data, len(g), None, None, 0, ctypes.byref(ns), ctypes.byref(nl)))
    site = np.zeros(ns.value, dtype=np.int32)
    level = np.zeros(ns.value, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int32)
    _check(lib().wqc_schedule_gates(n, g.ctypes.data, len(g), site.ctypes.data_as(ip), level.ctypes.data_as(ip),
                                    ns.value, ctypes.byref(ns), ctypes.byref(nl)))
    return site, level, nl.value


def workspace_bytes(n: int, chi: int) -> int:
    return int(lib().wqc_mps_workspace_bytes(n, chi))


class CudaMps:
    """MpsState on the device: try_new_with_bond (mps.rs:82-126)."""

    def __init__(self, n: int, chi: int, reject_truncation: bool = False, ctx: Context | None = None,
                 precision: int = PRECISION_FP64):
        self.ctx = ctx or Context.shared()
        self.n = n
        self.chi = chi
        h = ctypes.c_void_p()
        _check(lib().wqc_mps_create(self.ctx._h, n, chi, precision, int(reject_truncation), ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().wqc_mps_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def reset(self) -> None:
        """Back to |0...0> with the split records cleared (keeps device memory)."""
        _check(lib().wqc_mps_reset(self._h))

    # --- gate application (mps.rs:278-375, 520-565, 621-677) -----------------
    def apply_gates(self, gates: np.ndarray) -> None:
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        _check(lib().wqc_mps_apply_gates(self._h, g.ctypes.data, len(g)))

    def apply_gate(self, gate) -> None:
        self.apply_gates(gates_array([gate]) if isinstance(gate, tuple) else np.atleast_1d(gate))

    def apply_gates_adjoint(self, gates: np.ndarray) -> None:
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        _check(lib().wqc_mps_apply_gates_adjoint(self._h, g.ctypes.data, len(g)))

    def apply_one_qubit(self, site: int, u) -> None:
        _check(lib().wqc_mps_apply_1q(self._h, site, _dp(_c128(u).reshape(-1).view(np.float64))))

    def apply_two_qubit_at_positions(self, p: int, q: int, u, ctrl_is_first: bool, want_info: bool = False):
        if q != p + 1:
            raise WqcCudaError(ERR_INVALID, "two-site apply needs adjacent positions")
        info = np.zeros(1, dtype=SPLIT_INFO_DTYPE)
        _check(lib().wqc_mps_apply_2q(self._h, p, _dp(_c128(u).reshape(-1).view(np.float64)), int(ctrl_is_first),
                                      info.ctypes.data if want_info else None))
        return info[0] if want_info else None

    def apply_two_qubit_gate(self, ctrl: int, tgt: int, u) -> None:
        _check(lib().wqc_mps_apply_2q_routed(self._h, ctrl, tgt, _dp(_c128(u).reshape(-1).view(np.float64))))

    def apply_adjacent_disjoint_gates(self, gates: np.ndarray) -> None:
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        _check(lib().wqc_mps_apply_layer(self._h, g.ctypes.data, len(g)))

    # sweep-tree hooks (mps.rs:621-655)
    def apply_unary_at(self, site: int, gate) -> None:
        """gate: (kind, angle) or a C.g1 tuple (kind, qubit, 0, 0, angle); the
        qubit is replaced by `site` (the tree's wire-to-site mapping)."""
        angle = gate[1] if len(gate) == 2 else (gate[-1] if len(gate) > 2 else 0.0)
        self.apply_gate((gate[0], site, 0, 0, float(angle)))

    def apply_tdg_at(self, site: int) -> None:
        r = 0.70710678118654752440
        self.apply_one_qubit(site, np.array([[1, 0], [0, complex(r, -r)]]))

    def apply_swap_at(self, site: int) -> None:
        self.apply_two_qubit_at_positions(site, site + 1, SWAP4, True)

    def apply_pair_at(self, site: int, kind: int, ctrl_on_left: bool) -> None:
        from .circuits import CNOT
        self.apply_two_qubit_at_positions(site, site + 1, CNOT4 if kind == CNOT else CZ4, ctrl_on_left)

    def apply_cnot_at(self, site: int, ctrl_on_left: bool) -> None:
        self.apply_two_qubit_at_positions(site, site + 1, CNOT4, ctrl_on_left)

    # --- reads ---------------------------------------------------------------
    def set_split_rule(self, rule: int) -> None:
        _check(lib().wqc_mps_set_split_rule(self._h, rule))

    def set_merge(self, merge: int) -> None:
        """MERGE_FFMA (FP64 FMA tiles) or MERGE_TC_INT8 (int8 digit slices on
        the tcgen05 tensor cores, FP64-level) for the merges that follow."""
        _check(lib().wqc_mps_set_merge(self._h, merge))

    def synchronize(self) -> None:
        _check(lib().wqc_mps_synchronize(self._h))

    def cancel(self) -> None:
        lib().wqc_mps_cancel(self._h)

    def amplitude_at_compact_zero(self) -> complex:
        out = np.zeros(2)
        _check(lib().wqc_mps_amplitude_zero(self._h, _dp(out)))
        return complex(out[0], out[1])

    amplitude_zero = amplitude_at_compact_zero

    def site_amplitudes(self, target: int):
        out = np.zeros(4)
        _check(lib().wqc_mps_site_amplitudes(self._h, target, _dp(out)))
        return complex(out[0], out[1]), complex(out[2], out[3])

    def site_amplitudes_many(self, targets) -> np.ndarray:
        """(a0, a1) of every target in one call: shape (len(targets), 2)."""
        t = np.ascontiguousarray(targets, dtype=np.uint32)
        out = np.zeros((len(t), 2), dtype=np.complex128)
        _check(lib().wqc_mps_site_amplitudes_many(self._h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                                  len(t), _dp(out.view(np.float64))))
        return out

    def control_probability(self, control: int) -> float:
        _, a1 = self.site_amplitudes(control)
        return a1.real * a1.real + a1.imag * a1.imag

    def bond_dims(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.uint32)
        _check(lib().wqc_mps_bond_dims(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))))
        return out.astype(np.int32)

    def site(self, i: int) -> np.ndarray:
        l, r = ctypes.c_uint32(), ctypes.c_uint32()
        _check(lib().wqc_mps_download_site(self._h, i, ctypes.byref(l), ctypes.byref(r), None))
        out = np.zeros((l.value, 2, r.value), dtype=np.complex128)
        _check(lib().wqc_mps_download_site(self._h, i, ctypes.byref(l), ctypes.byref(r), _dp(out.view(np.float64))))
        return out

    def set_site(self, i: int, t: np.ndarray) -> None:
        t = _c128(t)
        _check(lib().wqc_mps_upload_site(self._h, i, t.shape[0], t.shape[2], _dp(t.view(np.float64))))

    def to_dense_state(self) -> np.ndarray:
        """to_dense_state (mps.rs:742-780) on the device: the 2^N vector,
        qubit q is bit q, site entries with |x|^2 < 1e-30 skipped."""
        out = np.zeros(1 << self.n, dtype=np.complex128)
        _check(lib().wqc_mps_to_dense(self._h, 0, _dp(out.view(np.float64))))
        return out

    def contract_to_statevector(self) -> np.ndarray:
        """contract_to_statevector (mps.rs:215-260) on the device (N <= 20)."""
        out = np.zeros(1 << min(self.n, 20), dtype=np.complex128)
        _check(lib().wqc_mps_to_dense(self._h, 1, _dp(out.view(np.float64))))
        return out

    def expectation(self, labels, coeffs) -> complex:
        joined, c = _pauli_args(labels, coeffs, self.n)
        out = np.zeros(2)
        _check(lib().wqc_mps_expectation_pauli(self._h, joined, _dp(c.view(np.float64)), len(labels), _dp(out)))
        return complex(out[0], out[1])

    def overlap(self, bra: "CudaMps", env_limit: int = OVERLAP_ENV_LIMIT) -> complex:
        """<bra|self> (overlap, mps.rs:1423-1474), computed on the device;
        env_limit 0 lifts the reference's cap on the environment."""
        out = np.zeros(2)
        _check(lib().wqc_mps_overlap(self._h, bra._h, int(env_limit), _dp(out)))
        return complex(out[0], out[1])

    def sample(self, qubits, shots: int, seed: int) -> np.ndarray:
        """`shots` draws of the listed (distinct) qubits from |<b|psi>|^2:
        element k, bit j is the outcome of qubits[j] in shot k."""
        q = np.ascontiguousarray(qubits, dtype=np.uint32)
        out = np.zeros(int(shots), dtype=np.uint64)
        _check(lib().wqc_mps_sample(self._h, q.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), len(q), int(shots),
                                    int(seed) & 0xFFFFFFFFFFFFFFFF,
                                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        return out

    def sample_counts(self, measures, classical_bit_count: int, shots: int, seed: int) -> dict:
        """Counts keyed like the reference's outcome_key (src/sample.rs:133-156):
        measures are (qubit, cbit) pairs applied in order, the key has
        classical_bit_count characters with cbit 0 rightmost."""
        if classical_bit_count <= 0:
            raise WqcCudaError(ERR_INVALID, "classical_bit_count must be > 0 for sample_counts")
        for q, c in measures:
            if q >= self.n:
                raise WqcCudaError(ERR_QUBIT_OUT_OF_RANGE, f"qubit {q} out of range (limit {self.n})")
            if c >= classical_bit_count:
                raise WqcCudaError(ERR_INVALID, f"classical bit index {c} out of bounds (limit: {classical_bit_count})")
        qubits = sorted({int(q) for q, _ in measures})
        col = {q: j for j, q in enumerate(qubits)}
        draws = self.sample(qubits, shots, seed)
        counts: dict = {}
        for b in np.unique(draws):
            bits = [0] * classical_bit_count
            for q, c in measures:
                bits[c] = int(b >> np.uint64(col[q])) & 1
            key = "".join(str(bits[classical_bit_count - 1 - i]) for i in range(classical_bit_count))
            counts[key] = counts.get(key, 0) + int(np.count_nonzero(draws == b))
        return counts

    def split_count(self) -> int:
        return int(lib().wqc_mps_split_count(self._h))

    def split_records(self) -> np.ndarray:
        k = lib().wqc_mps_split_count(self._h)
        out = np.zeros(k, dtype=SPLIT_INFO_DTYPE)
        w = ctypes.c_uint32()
        _check(lib().wqc_mps_split_records(self._h, out.ctypes.data if k else None, k, ctypes.byref(w)))
        return out[: w.value]

    def peak_vram_bytes(self) -> int:
        return int(lib().wqc_mps_peak_vram_bytes(self._h))

    def backend_label(self) -> str:
        return lib().wqc_mps_backend_label(self._h).decode()

    def set_profiling(self, on: bool) -> None:
        _check(lib().wqc_mps_set_profiling(self._h, int(on)))

    def kernel_stats(self) -> dict:
        st = KernelStats()
        _check(lib().wqc_mps_kernel_stats(self._h, ctypes.byref(st)))
        return {
            "launches": {k: int(st.launches[i]) for i, k in enumerate(KERNEL_KINDS)},
            "milliseconds": {k: float(st.milliseconds[i]) for i, k in enumerate(KERNEL_KINDS)},
            "total_launches": int(st.total_launches),
            "h2d_bytes": int(st.h2d_bytes),
            "d2h_bytes": int(st.d2h_bytes),
            "jacobi_tasks": int(st.jacobi_tasks),
            "jacobi_sweeps": int(st.jacobi_sweeps),
            "jacobi_sweeps_first": int(st.jacobi_sweeps_first),
        }

    def reset_stats(self) -> None:
        lib().wqc_mps_reset_stats(self._h)

    def debug_workspace(self, slot: int, which: int, count: int, dtype=np.complex128) -> np.ndarray:
        """Copy of one split-workspace buffer (see wqc_mps_debug_workspace)."""
        out = np.zeros(count, dtype=dtype)
        _check(lib().wqc_mps_debug_workspace(self._h, slot, which, out.ctypes.data, out.nbytes))
        return out

    def stream(self) -> int:
        return int(lib().wqc_mps_stream(self._h) or 0)


def expectation_pauli_noalloc(sites_ptr: int, site_stride: int, bond_dims, labels, coeffs, stream: int = 0) -> complex:
    """Sum_t coeff_t <psi|P_t|psi> for an MPS in the caller's own device memory
    (wqc_expectation_pauli_noalloc): the call allocates no device memory.
    sites_ptr is a device address on the current device holding
    len(bond_dims) sites of site_stride complex128 values each, site q laid
    out [l][2][r]; stream is a cudaStream_t handle (0 = legacy default)."""
    dims = np.ascontiguousarray(bond_dims, dtype=np.uint32)
    joined, c = _pauli_args(labels, coeffs, len(dims))
    out = np.zeros(2)
    _check(lib().wqc_expectation_pauli_noalloc(sites_ptr or None, site_stride,
                                               dims.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), len(dims),
                                               joined, _dp(c.view(np.float64)), len(labels), stream or None,
                                               _dp(out)))
    return complex(out[0], out[1])


class Adjoint:
    """The differentiation form's forward/backward op pair
    (wqc_adjoint_forward / wqc_adjoint_backward) on a single state: the
    forward runs `gates` from |0...0> keeping checkpoints at the gate
    indices `checkpoints`; backward(labels, coeffs) returns (f, df/dangle
    per gate) by the reverse sweep."""

    def __init__(self, mps: "CudaMps", gates: np.ndarray, checkpoints=()):
        self.mps = mps
        self.gates = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        cps = np.ascontiguousarray(checkpoints, dtype=np.uint32)
        h = ctypes.c_void_p()
        _check(lib().wqc_adjoint_forward(mps._h, self.gates.ctypes.data, len(self.gates),
                                         cps.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), len(cps),
                                         ctypes.byref(h)))
        self._h = h

    def backward(self, labels, coeffs):
        joined, c = _pauli_args(labels, coeffs, self.mps.n)
        value = np.zeros(2)
        grad = np.zeros(max(len(self.gates), 1))
        _check(lib().wqc_adjoint_backward(self._h, joined, _dp(c.view(np.float64)), len(labels), _dp(value),
                                          _dp(grad)))
        return float(value[0]), grad[: len(self.gates)]

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().wqc_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def adjoint_gradient(n: int, chi: int, gates: np.ndarray, pidx: np.ndarray, labels, coeffs, checkpoints=(),
                     ctx: Context | None = None):
    """(f, df/dparams) by the adjoint: per-gate derivatives summed over the
    gate instances of each parameter (pidx[i] = parameter of gate i, or -1)."""
    m = CudaMps(n, chi, ctx=ctx)
    adj = Adjoint(m, gates, checkpoints)
    try:
        f, g = adj.backward(labels, coeffs)
    finally:
        adj.close()
        m.close()
    pidx = np.asarray(pidx)
    grad = np.zeros(int(pidx.max()) + 1 if pidx.size and pidx.max() >= 0 else 0)
    for i, p in enumerate(pidx):
        if p >= 0:
            grad[p] += g[i]
    return f, grad


class CudaBatch(CudaMps):
    """Many independent slices in one device state (wqc_batch_create): their
    splits share waves; each slice keeps its own MpsState semantics."""

    def __init__(self, qubits, chis, ctx: Context | None = None, max_concurrent_splits: int = 0,
                 precision: int = PRECISION_FP64):
        self.ctx = ctx or Context.shared()
        self.qubits = np.ascontiguousarray(qubits, dtype=np.uint32)
        self.chis = np.ascontiguousarray(chis, dtype=np.uint32)
        self.n = int(self.qubits.sum())
        self.chi = int(self.chis.max())
        self.first_site = np.concatenate([[0], np.cumsum(self.qubits)[:-1]]).astype(np.int64)
        u32 = ctypes.POINTER(ctypes.c_uint32)
        h = ctypes.c_void_p()
        _check(lib().wqc_batch_create(self.ctx._h, len(self.qubits), self.qubits.ctypes.data_as(u32),
                                      self.chis.ctypes.data_as(u32), precision, max_concurrent_splits,
                                      ctypes.byref(h)))
        self._h = h

    def apply_slices(self, gate_lists) -> None:
        """gate_lists[s] are slice s's gates (qubits local to the slice)."""
        lens = [len(g) for g in gate_lists]
        offsets = np.zeros(len(lens) + 1, dtype=np.uint32)
        offsets[1:] = np.cumsum(lens)
        allg = np.ascontiguousarray(np.concatenate(gate_lists) if sum(lens) else np.zeros(0, GATE_DTYPE),
                                    dtype=GATE_DTYPE)
        _check(lib().wqc_batch_apply_gates(self._h, allg.ctypes.data if len(allg) else None,
                                           offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))))

    def amplitudes(self) -> np.ndarray:
        out = np.zeros(len(self.qubits), dtype=np.complex128)
        _check(lib().wqc_batch_amplitudes(self._h, _dp(out.view(np.float64))))
        return out

    def expectations(self, labels, coeffs) -> np.ndarray:
        """The Pauli sum on every slice (wqc_batch_expectation_pauli)."""
        joined, c = _pauli_args(labels, coeffs, int(self.qubits[0]) if len(self.qubits) else 0)
        out = np.zeros(len(self.qubits), dtype=np.complex128)
        _check(lib().wqc_batch_expectation_pauli(self._h, joined, _dp(c.view(np.float64)), len(labels),
                                                 _dp(out.view(np.float64))))
        return out

    def slice_times_ms(self) -> np.ndarray:
        out = np.zeros(len(self.qubits))
        _check(lib().wqc_batch_slice_times(self._h, _dp(out)))
        return out

    def slice_records(self):
        """Split records of each slice (left_site local to the slice), in order."""
        rec = self.split_records()
        site = rec["left_site"].astype(np.int64)
        sl = np.searchsorted(self.first_site, site, side="right") - 1
        out = []
        for s in range(len(self.qubits)):
            r = rec[sl == s].copy()
            r["left_site"] -= self.first_site[s]
            out.append(r)
        return out


def _mat4(entries) -> np.ndarray:
    m = np.zeros((2, 2, 2, 2), dtype=np.complex128)
    for idx, v in entries:
        m[idx] = v
    return m


# Mat4 [c_out][t_out][c_in][t_in] (src/tn/gates.rs:68-104)
CNOT4 = _mat4([((0, 0, 0, 0), 1), ((0, 1, 0, 1), 1), ((1, 0, 1, 1), 1), ((1, 1, 1, 0), 1)])
CZ4 = _mat4([((0, 0, 0, 0), 1), ((0, 1, 0, 1), 1), ((1, 0, 1, 0), 1), ((1, 1, 1, 1), -1)])
SWAP4 = _mat4([((0, 0, 0, 0), 1), ((0, 1, 1, 0), 1), ((1, 0, 0, 1), 1), ((1, 1, 1, 1), 1)])


def run(n: int, chi: int, gates: np.ndarray, ctx: Context | None = None, rule: int = SPLIT_RULE_REFERENCE,
        merge: int | None = None) -> CudaMps:
    """A state with the gates applied; `merge` (MERGE_*) overrides the
    default merge (int8 digit slices on the tensor cores for single states)."""
    m = CudaMps(n, chi, ctx=ctx)
    m.set_split_rule(rule)
    if merge is not None:
        m.set_merge(merge)
    m.apply_gates(gates)
    return m


def bra_unitary_gates(second_half: np.ndarray):
    """The adjoint of `second_half` in reverse as plain gates (mps.rs:1393-1421):
    rotations negated, S^H = S Z, T^H = T T T Z, the rest self-inverse; None
    when a MEASURE, RESET or IF is present."""
    from . import circuits as C

    out = []
    for g in np.asarray(second_half, dtype=GATE_DTYPE)[::-1]:
        k = int(g["kind"])
        if k in (C.MEASURE, C.RESET, C.IF):
            return None
        if k in (C.RX, C.RY, C.RZ):
            h = g.copy()
            h["angle"] = -g["angle"]
            out.append(h)
        elif k == C.S:
            z = g.copy()
            z["kind"] = C.Z
            out += [g, z]
        elif k == C.T:
            z = g.copy()
            z["kind"] = C.Z
            out += [g, g, g, z]
        else:
            out.append(g)
    return np.array(out, dtype=GATE_DTYPE)


def contract_time_split(n: int, gates: np.ndarray, split: int, max_bond: int, ctx: Context | None = None) -> complex:
    """contract_time_split (mps.rs:1241-1249, 1358-1384): the ket runs the first
    `split` gates, the bra the adjoint of the rest, both rejecting truncation,
    and the result is their overlap under the reference's environment cap."""
    gates = np.asarray(gates, dtype=GATE_DTYPE)
    if split > len(gates):
        raise WqcCudaError(ERR_INVALID, "time-split index past the gate list")
    ket = CudaMps(n, max_bond, reject_truncation=True, ctx=ctx)
    ket.apply_gates(gates[:split])
    bra = CudaMps(n, max_bond, reject_truncation=True, ctx=ctx)
    seq = bra_unitary_gates(gates[split:])
    if seq is not None:
        bra.apply_gates(seq)
    else:
        bra.apply_gates_adjoint(gates[split:][::-1].copy())
    return ket.overlap(bra)


def svd_flops(rows: int, cols: int) -> float:
    """Algorithmic complex SVD flops (Golub-Van Loan count for S, thin U, V, x4 for complex)."""
    p, q = min(rows, cols), max(rows, cols)
    return 4.0 * (14.0 * q * p * p + 8.0 * p ** 3)


def split_flops(rec) -> float:
    """Algorithmic flops of one split's SVD stage from its record (the exact
    SVD, or the range finder's products, QR and projected SVD)."""
    rows, cols, ell, path = int(rec["rows"]), int(rec["cols"]), int(rec["ell"]), int(rec["path"])
    if path == 1:
        return 8.0 * (3 * rows * cols * ell + ell * rows * cols) + 4.0 * (4 * rows * ell * ell) + svd_flops(ell, cols)
    f = svd_flops(rows, cols)
    if path == 2:
        f += 8.0 * (3 * rows * cols * ell + ell * rows * cols) + 4.0 * (4 * rows * ell * ell) + svd_flops(ell, cols)
    return f


__all__ = ["CudaMps", "CudaBatch", "Context", "Adjoint", "adjoint_gradient", "WqcCudaError", "lib", "build", "run", "workspace_bytes", "split_flops",
           "svd_flops", "CNOT4", "CZ4", "SWAP4", "EXPORTS", "KERNEL_KINDS", "math"]
