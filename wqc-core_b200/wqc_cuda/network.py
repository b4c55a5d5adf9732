"""Network contraction trees on the device (src/tn/network.rs) through the
``wqc_network_*`` entry points of include/wqc_cuda.h.

Trees are given in the reference's JSON form with ``"kind": "network"``
(src/tn/tree.rs ``ContractionTree``): nodes ``{"op": "contract", "left":
{"ket0": 0}, "right": {"gate": 3}}`` whose references are ket0, bra0, gate,
control, target or node.  ``contract_network`` returns <0...0|U|0...0> as the
reference's function of that name does (network.rs:145-160); failures raise
``WqcCudaError`` with the reference's message.
"""
from __future__ import annotations

import ctypes

from . import Context, _check, lib
from .exact import _gates, _order, _TreeArgs


class NetworkStats(ctypes.Structure):
    _fields_ = [
        ("nodes", ctypes.c_uint32),
        ("permutes", ctypes.c_uint32),
        ("gemms", ctypes.c_uint32),
        ("launches", ctypes.c_uint32),
        ("device_ms", ctypes.c_double),
        ("permute_ms", ctypes.c_double),
        ("gemm_ms", ctypes.c_double),
        ("permute_bytes", ctypes.c_uint64),
        ("gemm_flops", ctypes.c_double),
        ("arena_bytes", ctypes.c_uint64),
        ("small", ctypes.c_uint32),
    ]


def _bind(L):
    if getattr(L, "_network_bound", False):
        return L
    P, U32, U64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
    from .exact import _Tree

    T = ctypes.POINTER(_Tree)
    L.wqc_network_create.argtypes = [P, ctypes.POINTER(P)]
    L.wqc_network_destroy.argtypes = [P]
    L.wqc_network_destroy.restype = None
    L.wqc_network_cancel.argtypes = [P]
    L.wqc_network_cancel.restype = None
    L.wqc_network_validate.argtypes = [U32, P, U32, T, P, U32]
    L.wqc_network_measured_peak.argtypes = [U32, P, U32, T, ctypes.POINTER(U64)]
    L.wqc_network_contract.argtypes = [P, U32, P, U32, T, P, U32, P]
    L.wqc_network_last_stats.argtypes = [P, ctypes.POINTER(NetworkStats)]
    L._network_bound = True
    return L


def validate(n: int, gates, tree, mps_site_order=None) -> None:
    """network::validate (network.rs:128-143): the walk and the declared peak."""
    L = _bind(lib())
    g = _gates(gates)
    t = _TreeArgs(tree)
    ptr, ln, keep = _order(mps_site_order)  # noqa: F841 (keep holds the buffer)
    _check(L.wqc_network_validate(n, g.ctypes.data if len(g) else None, len(g), ctypes.byref(t.struct), ptr, ln))


def measured_peak(n: int, gates, tree) -> int:
    """network.rs:162-169: the walk's peak (the declared peak is not read)."""
    L = _bind(lib())
    g = _gates(gates)
    t = _TreeArgs(tree, peak=False)
    out = ctypes.c_uint64()
    _check(L.wqc_network_measured_peak(n, g.ctypes.data if len(g) else None, len(g), ctypes.byref(t.struct),
                                       ctypes.byref(out)))
    return out.value


class NetworkContractor:
    """A network-tree executor on one device: its own stream, cuBLAS handle
    and device arena, reused across calls."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or Context.shared()
        L = _bind(lib())
        h = ctypes.c_void_p()
        _check(L.wqc_network_create(self.ctx._h, ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().wqc_network_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def cancel(self) -> None:
        lib().wqc_network_cancel(self._h)

    def contract(self, n: int, gates, tree, mps_site_order=None) -> complex:
        L = _bind(lib())
        g = _gates(gates)
        t = _TreeArgs(tree)
        out = (ctypes.c_double * 2)()
        ptr, ln, keep = _order(mps_site_order)  # noqa: F841
        _check(L.wqc_network_contract(self._h, n, g.ctypes.data if len(g) else None, len(g), ctypes.byref(t.struct),
                                      ptr, ln, out))
        return complex(out[0], out[1])

    def stats(self) -> dict:
        s = NetworkStats()
        _check(lib().wqc_network_last_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in NetworkStats._fields_}


_SHARED = None


def contract_network(n: int, gates, tree, mps_site_order=None) -> complex:
    """contract_network (network.rs:145-160) on the shared device."""
    global _SHARED
    if _SHARED is None:
        _SHARED = NetworkContractor()
    return _SHARED.contract(n, gates, tree, mps_site_order)
