"""ORACLE — test infrastructure only.

ctypes binding of the FP64 C++ restatement of wqc-core's CPU MPS path
(oracle/mps_oracle.cpp).  Only tests, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` import this module; the cuda backend never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

GATE_DTYPE = np.dtype(
    [("kind", "<i4"), ("q0", "<i4"), ("q1", "<i4"), ("q2", "<i4"), ("angle", "<f8")], align=True
)
SPLIT_INFO_DTYPE = np.dtype(
    [("left_site", "<i4"), ("rows", "<i4"), ("cols", "<i4"), ("ell", "<i4"), ("path", "<i4"),
     ("chi", "<i4"), ("discarded_weight", "<f8")],
    align=True,
)


def build() -> str:
    """Compile liboracle.so in place (make) and return its path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        I = ctypes.c_int
        D = ctypes.POINTER(ctypes.c_double)
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_mps_create.argtypes = [I, I, I, ctypes.POINTER(P)]
        L.oracle_mps_destroy.argtypes = [P]
        for name in ("oracle_mps_apply_gates", "oracle_mps_apply_call_sequence", "oracle_mps_apply_layer"):
            getattr(L, name).argtypes = [P, P, I]
        L.oracle_mps_set_split_rule.argtypes = [P, I]
        L.oracle_mps_apply_1q.argtypes = [P, I, D]
        L.oracle_mps_apply_2q.argtypes = [P, I, I, D]
        L.oracle_mps_apply_2q_at.argtypes = [P, I, D, I]
        L.oracle_mps_amplitude_zero.argtypes = [P, D]
        L.oracle_mps_site_amplitudes.argtypes = [P, I, D]
        L.oracle_mps_bond_dims.argtypes = [P, ctypes.POINTER(I)]
        L.oracle_mps_num_records.argtypes = [P]
        L.oracle_mps_records.argtypes = [P, P, I]
        L.oracle_mps_dense.argtypes = [P, D]
        L.oracle_mps_statevector.argtypes = [P, D]
        L.oracle_mps_site.argtypes = [P, I, ctypes.POINTER(I), ctypes.POINTER(I), D]
        L.oracle_mps_set_site.argtypes = [P, I, I, I, D]
        L.oracle_mps_expectation_pauli.argtypes = [P, ctypes.c_char_p, D, I, D]
        L.oracle_time_split.argtypes = [I, P, I, I, I, D]
        L.oracle_checked_svd.argtypes = [I, I, D, D, D, D, ctypes.POINTER(I)]
        L.oracle_gk_svd.argtypes = [I, I, D, D, D, D]
        L.oracle_jacobi_svd.argtypes = [I, I, D, D, D, D]
        L.oracle_thin_q.argtypes = [I, I, D, D]
        L.oracle_rsvd_sites.argtypes = [I, I, I, I, I, I, D, ctypes.POINTER(I), D, D]
        L.oracle_retained_chi.argtypes = [D, I, I, I, I]
        L.oracle_needs_f64_fallback.argtypes = [D, I, I]
        L.oracle_rsvd_worth.argtypes = [I, I, I]
        L.oracle_jacobi_pairs.argtypes = [I, ctypes.POINTER(ctypes.c_uint32)]
        L.oracle_mix_seed.argtypes = [ctypes.c_uint64] * 3
        L.oracle_mix_seed.restype = ctypes.c_uint64
        L.oracle_rademacher.argtypes = [I, I, ctypes.c_uint64, D]
        L.oracle_svd_counters.argtypes = [ctypes.POINTER(I), ctypes.POINTER(I)]
        L.oracle_set_primary_svd.argtypes = [I]
        L.oracle_snap.argtypes = [ctypes.c_double]
        L.oracle_snap.restype = ctypes.c_double
        L.oracle_mps_workspace_bytes.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.oracle_mps_workspace_bytes.restype = ctypes.c_uint64
        _LIB = L
    return _LIB


class OracleError(RuntimeError):
    pass


def _check(rc: int) -> None:
    if rc != 0:
        raise OracleError(lib().oracle_last_error().decode())


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _c128(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex128)


class OracleMps:
    """The reference's MpsState, on the CPU in FP64."""

    def __init__(self, n: int, chi: int, reject_truncation: bool = False):
        self.n = n
        self.chi = chi
        h = ctypes.c_void_p()
        _check(lib().oracle_mps_create(n, chi, int(reject_truncation), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_mps_destroy(self._h)
            self._h = None

    def set_split_rule(self, rule: int) -> None:
        """0: the reference rule (exact or range finder); 1: exact SVD on every split."""
        lib().oracle_mps_set_split_rule(self._h, rule)

    def apply_gates(self, gates: np.ndarray) -> None:
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        _check(lib().oracle_mps_apply_gates(self._h, g.ctypes.data, len(g)))

    def apply_call_sequence(self, gates: np.ndarray) -> None:
        """The MpsState calls src/tn/trace.rs:55-187 makes for this gate list."""
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        _check(lib().oracle_mps_apply_call_sequence(self._h, g.ctypes.data, len(g)))

    def apply_layer(self, gates: np.ndarray) -> None:
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        _check(lib().oracle_mps_apply_layer(self._h, g.ctypes.data, len(g)))

    def apply_1q(self, site: int, u) -> None:
        _check(lib().oracle_mps_apply_1q(self._h, site, _dp(_c128(u).view(np.float64))))

    def apply_2q(self, ctrl: int, tgt: int, u) -> None:
        _check(lib().oracle_mps_apply_2q(self._h, ctrl, tgt, _dp(_c128(u).view(np.float64))))

    def apply_2q_at(self, left: int, u, ctrl_is_first: bool) -> None:
        _check(lib().oracle_mps_apply_2q_at(self._h, left, _dp(_c128(u).view(np.float64)), int(ctrl_is_first)))

    def amplitude_zero(self) -> complex:
        out = np.zeros(2)
        _check(lib().oracle_mps_amplitude_zero(self._h, _dp(out)))
        return complex(out[0], out[1])

    def site_amplitudes(self, target: int):
        out = np.zeros(4)
        _check(lib().oracle_mps_site_amplitudes(self._h, target, _dp(out)))
        return complex(out[0], out[1]), complex(out[2], out[3])

    def bond_dims(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.int32)
        _check(lib().oracle_mps_bond_dims(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return out

    def records(self) -> np.ndarray:
        k = lib().oracle_mps_num_records(self._h)
        out = np.zeros(k, dtype=SPLIT_INFO_DTYPE)
        lib().oracle_mps_records(self._h, out.ctypes.data, k)
        return out

    def dense(self) -> np.ndarray:
        out = np.zeros(1 << self.n, dtype=np.complex128)
        _check(lib().oracle_mps_dense(self._h, _dp(out.view(np.float64))))
        return out

    def statevector(self) -> np.ndarray:
        out = np.zeros(1 << self.n, dtype=np.complex128)
        _check(lib().oracle_mps_statevector(self._h, _dp(out.view(np.float64))))
        return out

    def site(self, i: int) -> np.ndarray:
        l, r = ctypes.c_int(), ctypes.c_int()
        _check(lib().oracle_mps_site(self._h, i, ctypes.byref(l), ctypes.byref(r), None))
        out = np.zeros((l.value, 2, r.value), dtype=np.complex128)
        _check(lib().oracle_mps_site(self._h, i, ctypes.byref(l), ctypes.byref(r), _dp(out.view(np.float64))))
        return out

    def set_site(self, i: int, t: np.ndarray) -> None:
        t = _c128(t)
        _check(lib().oracle_mps_set_site(self._h, i, t.shape[0], t.shape[2], _dp(t.view(np.float64))))

    def expectation(self, labels, coeffs) -> complex:
        joined = "".join(labels).encode()
        c = _c128(coeffs)
        out = np.zeros(2)
        _check(lib().oracle_mps_expectation_pauli(self._h, joined, _dp(c.view(np.float64)), len(labels), _dp(out)))
        return complex(out[0], out[1])


def run(n: int, chi: int, gates: np.ndarray, call_sequence: bool = False, rule: int = 0) -> OracleMps:
    m = OracleMps(n, chi)
    m.set_split_rule(rule)
    if call_sequence:
        m.apply_call_sequence(gates)
    else:
        m.apply_gates(gates)
    return m


def self_drift(n: int, chi: int, gates: np.ndarray, rule: int = 0, call_sequence: bool = False) -> np.ndarray:
    """Per-split |discarded weight| difference between two oracle runs of the
    same circuit, one with its Golub-Kahan SVD (the reference's primary) and
    one with its Jacobi SVD as primary: how far two FP64 SVDs of the same
    matrices drift apart once truncation carries their rounding on.  Kept
    chi, paths and shapes must agree between the two."""
    runs = []
    for primary in (0, 1):
        set_primary_svd(primary)
        try:
            runs.append(run(n, chi, gates, call_sequence=call_sequence, rule=rule).records())
        finally:
            set_primary_svd(0)
    if not all(np.array_equal(runs[0][k], runs[1][k]) for k in ("rows", "cols", "path", "chi")):
        raise OracleError("the oracle's two SVDs disagree in a kept chi or path")
    return np.abs(runs[0]["discarded_weight"] - runs[1]["discarded_weight"])


def time_split(n: int, gates: np.ndarray, split: int, max_bond: int) -> complex:
    g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
    out = np.zeros(2)
    _check(lib().oracle_time_split(n, g.ctypes.data, len(g), split, max_bond, _dp(out)))
    return complex(out[0], out[1])


def _svd_call(fn, a, with_route=False):
    a = _c128(a)
    m, n = a.shape
    k = min(m, n)
    s = np.zeros(k)
    u = np.zeros((m, k), dtype=np.complex128)
    vt = np.zeros((k, n), dtype=np.complex128)
    args = [m, n, _dp(a.view(np.float64)), _dp(s), _dp(u.view(np.float64)), _dp(vt.view(np.float64))]
    route = ctypes.c_int(-1)
    if with_route:
        args.append(ctypes.byref(route))
    _check(fn(*args))
    return (u, s, vt, route.value) if with_route else (u, s, vt)


def checked_svd(a):
    """svd_guard.rs:91-139; returns (U, s, V^H, route) with route 0/1/2 =
    primary / transpose retry / Jacobi."""
    return _svd_call(lib().oracle_checked_svd, a, with_route=True)


def gk_svd(a):
    return _svd_call(lib().oracle_gk_svd, a)


def jacobi_svd(a):
    return _svd_call(lib().oracle_jacobi_svd, a)


def thin_q(a) -> np.ndarray:
    a = _c128(a)
    m, n = a.shape
    q = np.zeros((m, min(m, n)), dtype=np.complex128)
    _check(lib().oracle_thin_q(m, n, _dp(a.view(np.float64)), _dp(q.view(np.float64))))
    return q


def rsvd_sites(mat, ell, dl, dr, max_bond):
    mat = _c128(mat)
    rows, cols = mat.shape
    chi = ctypes.c_int(0)
    left = np.zeros((dl, 2, max_bond), dtype=np.complex128)
    right = np.zeros((max_bond, 2, dr), dtype=np.complex128)
    rc = lib().oracle_rsvd_sites(rows, cols, ell, dl, dr, max_bond, _dp(mat.view(np.float64)), ctypes.byref(chi),
                                 _dp(left.view(np.float64)), _dp(right.view(np.float64)))
    if rc == 2:
        return None
    _check(rc)
    c = chi.value
    left = left.reshape(-1)[: dl * 2 * c].reshape(dl, 2, c)
    right = right.reshape(-1)[: c * 2 * dr].reshape(c, 2, dr)
    return left, right


def retained_chi(values, max_bond, rows, cols) -> int:
    v = np.ascontiguousarray(values, dtype=np.float64)
    return lib().oracle_retained_chi(_dp(v), len(v), max_bond, rows, cols)


def needs_f64_fallback(values, chi) -> bool:
    v = np.ascontiguousarray(values, dtype=np.float64)
    return bool(lib().oracle_needs_f64_fallback(_dp(v), len(v), chi))


def rsvd_worth(rows, cols, ell) -> bool:
    return bool(lib().oracle_rsvd_worth(rows, cols, ell))


def jacobi_pairs(cols: int) -> np.ndarray:
    out = np.zeros((cols - 1) * cols, dtype=np.uint32)
    lib().oracle_jacobi_pairs(cols, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    return out


def mix_seed(rows, cols, ell) -> int:
    return int(lib().oracle_mix_seed(rows, cols, ell))


def rademacher(cols, ell, salt) -> np.ndarray:
    out = np.zeros(cols * ell, dtype=np.complex128)
    lib().oracle_rademacher(cols, ell, salt, _dp(out.view(np.float64)))
    return out.reshape(cols, ell)


def svd_counters():
    r, j = ctypes.c_int(), ctypes.c_int()
    lib().oracle_svd_counters(ctypes.byref(r), ctypes.byref(j))
    return r.value, j.value


def set_primary_svd(mode: int) -> None:
    """0: Golub-Kahan primary (nalgebra's family), 1: svd_guard.rs Jacobi as primary."""
    lib().oracle_set_primary_svd(mode)


def snap(x: float) -> float:
    return lib().oracle_snap(x)


def mps_workspace_bytes(n: int, chi: int) -> int:
    return int(lib().oracle_mps_workspace_bytes(n, chi))
