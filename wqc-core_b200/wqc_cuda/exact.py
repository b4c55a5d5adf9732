"""Exact contraction trees on the device (src/tn/exact.rs) through the
``wqc_exact_*`` entry points of include/wqc_cuda.h.

Trees are given in the reference's JSON form (src/tn/tree.rs
``ContractionTree``, serde): a dict ``{"nodes": [{"op": "contract", "left":
{"ket0": 0}, "right": {"gate": 0}}, ...], "peak_bytes": P, "site_order":
[...]}`` or its JSON text.  ``contract_exact_at`` returns the amplitude of one
basis vector, as the reference's function of that name does
(exact.rs:70-85); ``ExactContractor.contract`` also takes a list of basis
vectors and contracts the tree once for all of them.  Failures raise
``WqcCudaError`` with the reference's message.
"""
from __future__ import annotations

import ctypes
import json

import numpy as np

from . import Context, _check, lib
from .circuits import GATE_DTYPE

REF_KINDS = {"ket0": 0, "gate": 1, "node": 2, "left": 3, "right": 4, "bra0": 5, "control": 6, "target": 7}
TREE_NODE_DTYPE = np.dtype([("op", "<i4"), ("lkind", "<i4"), ("lindex", "<u4"), ("rkind", "<i4"),
                            ("rindex", "<u4")])


class _Tree(ctypes.Structure):
    _fields_ = [
        ("nodes", ctypes.c_void_p),
        ("node_count", ctypes.c_uint32),
        ("site_order", ctypes.c_void_p),
        ("site_order_len", ctypes.c_uint32),
        ("has_peak", ctypes.c_int32),
        ("peak_bytes", ctypes.c_uint64),
        ("kind", ctypes.c_int32),
    ]


class ExactStats(ctypes.Structure):
    _fields_ = [
        ("launches", ctypes.c_uint32),
        ("passes", ctypes.c_uint32),
        ("outer_products", ctypes.c_uint32),
        ("gates", ctypes.c_uint32),
        ("device_ms", ctypes.c_double),
        ("pass_ms", ctypes.c_double),
        ("pass_bytes", ctypes.c_uint64),
        ("bytes_moved", ctypes.c_uint64),
        ("arena_bytes", ctypes.c_uint64),
        ("exchanges", ctypes.c_uint32),
    ]


def _bind(L):
    if getattr(L, "_exact_bound", False):
        return L
    P, U32, U64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
    T = ctypes.POINTER(_Tree)
    L.wqc_exact_create.argtypes = [P, ctypes.POINTER(P)]
    L.wqc_exact_destroy.argtypes = [P]
    L.wqc_exact_destroy.restype = None
    L.wqc_exact_cancel.argtypes = [P]
    L.wqc_exact_cancel.restype = None
    L.wqc_exact_validate.argtypes = [U32, P, U32, T, P, U32]
    L.wqc_exact_measured_peak.argtypes = [U32, P, U32, T, ctypes.POINTER(U64)]
    L.wqc_exact_contract.argtypes = [P, U32, P, U32, T, P, U32, P, U32, P]
    L.wqc_exact_last_stats.argtypes = [P, ctypes.POINTER(ExactStats)]
    L.wqc_exact_set_tile_bits.argtypes = [P, ctypes.c_int32]
    L._exact_bound = True
    return L


def _ref(r) -> tuple[int, int]:
    if isinstance(r, dict):
        if len(r) != 1:
            raise ValueError(f"tensor reference {r!r} needs exactly one key")
        (name, index), = r.items()
        return REF_KINDS[name], int(index)
    kind, index = r
    return int(kind), int(index)


def tree_nodes(nodes) -> np.ndarray:
    """The nodes as the C ABI's wqc_tree_node records.  A node is a dict of
    the reference's JSON form (op "contract" is 0; any other op is a sweep
    step and is passed on as such) or a (left, right) pair of references."""
    rows = []
    for node in nodes:
        op = 0
        if isinstance(node, dict):
            op = 0 if node.get("op", "contract") == "contract" else 1
            left, right = node.get("left", node.get("tensor", {"ket0": 0})), node.get("right", {"ket0": 0})
        else:
            left, right = node
        rows.append((op, *_ref(left), *_ref(right)))
    return np.array(rows, dtype=TREE_NODE_DTYPE) if rows else np.zeros(0, dtype=TREE_NODE_DTYPE)


class _TreeArgs:
    """Keeps the arrays a wqc_tree points at alive for one call."""

    def __init__(self, tree, peak=True):
        if isinstance(tree, (str, bytes)):
            tree = json.loads(tree)
        self.nodes = tree_nodes(tree.get("nodes", []))
        self.site_order = np.ascontiguousarray(tree.get("site_order", []) or [], dtype=np.uint32)
        pb = tree.get("peak_bytes") if peak else None
        kind = tree.get("kind")
        if kind not in (None, "network"):
            raise ValueError(f"unknown contraction tree kind {kind!r}")
        self.struct = _Tree(
            self.nodes.ctypes.data if len(self.nodes) else None, len(self.nodes),
            self.site_order.ctypes.data if len(self.site_order) else None, len(self.site_order),
            0 if pb is None else 1, 0 if pb is None else int(pb), 1 if kind == "network" else 0)


def _gates(gates) -> np.ndarray:
    return np.ascontiguousarray(gates, dtype=GATE_DTYPE)


def _order(mps_site_order):
    if mps_site_order is None:
        return None, 0, None
    a = np.ascontiguousarray(mps_site_order, dtype=np.uint64)
    keep = a if len(a) else np.zeros(1, dtype=np.uint64)  # Some(&[]) still passes a pointer
    return keep.ctypes.data, len(a), keep


def validate(n: int, gates, tree, mps_site_order=None) -> None:
    """exact::validate (exact.rs:48-58): declared peak and tree shape."""
    L = _bind(lib())
    g = _gates(gates)
    t = _TreeArgs(tree)
    ptr, ln, keep = _order(mps_site_order)  # noqa: F841 (keep holds the buffer)
    _check(L.wqc_exact_validate(n, g.ctypes.data if len(g) else None, len(g), ctypes.byref(t.struct), ptr, ln))


def measured_peak(n: int, gates, tree) -> int:
    """The walk's peak without evaluating (exact.rs:650-658)."""
    L = _bind(lib())
    g = _gates(gates)
    t = _TreeArgs(tree, peak=False)
    out = ctypes.c_uint64()
    _check(L.wqc_exact_measured_peak(n, g.ctypes.data if len(g) else None, len(g), ctypes.byref(t.struct),
                                     ctypes.byref(out)))
    return out.value


def is_contraction_client_error(code: int, message: str) -> bool:
    """tree.rs:213-230: failures that are the caller's tree (HTTP 400)."""
    from . import ERR_INVALID, ERR_INVALID_QUBIT_COUNT, ERR_QUBIT_OUT_OF_RANGE

    if code in (ERR_INVALID_QUBIT_COUNT, ERR_QUBIT_OUT_OF_RANGE):
        return True
    if code != ERR_INVALID:
        return False
    return message.startswith(("contraction tree", "contraction_tree", "exact contraction", "mps sweep",
                               "mps_site_order", "gate ", "gates ", "tensors share", "qubit index exceeds",
                               "IF value"))


class ExactContractor:
    """An exact-tree executor on one device: its own stream and a device arena
    for the live tensors, reused across calls."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or Context.shared()
        L = _bind(lib())
        h = ctypes.c_void_p()
        _check(L.wqc_exact_create(self.ctx._h, ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().wqc_exact_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def cancel(self) -> None:
        lib().wqc_exact_cancel(self._h)

    def set_tile_bits(self, bits: int) -> None:
        """Register tiles of 2^bits amplitudes (12 or 13) for states of 12 or
        more legs; results do not depend on it."""
        _check(lib().wqc_exact_set_tile_bits(self._h, bits))

    def contract(self, n: int, gates, tree, bits=0, mps_site_order=None):
        """Amplitude(s) of basis vector(s) `bits` (bit q = wire q): a complex
        for one int, an array for a sequence."""
        L = _bind(lib())
        g = _gates(gates)
        t = _TreeArgs(tree)
        scalar = np.isscalar(bits)
        b = np.ascontiguousarray(np.atleast_1d(np.asarray(bits, dtype=np.uint64)))
        out = np.zeros(2 * len(b), dtype=np.float64)
        ptr, ln, keep = _order(mps_site_order)  # noqa: F841
        _check(L.wqc_exact_contract(self._h, n, g.ctypes.data if len(g) else None, len(g), ctypes.byref(t.struct),
                                    ptr, ln, b.ctypes.data if len(b) else None, len(b), out.ctypes.data))
        amps = out[0::2] + 1j * out[1::2]
        return complex(amps[0]) if scalar else amps

    def stats(self) -> dict:
        s = ExactStats()
        _check(lib().wqc_exact_last_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in ExactStats._fields_}


_SHARED = None


def contract_exact_at(n: int, gates, tree, bits: int = 0, mps_site_order=None) -> complex:
    """contract_exact_at (exact.rs:70-85) on the shared device."""
    global _SHARED
    if _SHARED is None:
        _SHARED = ExactContractor()
    return _SHARED.contract(n, gates, tree, int(bits), mps_site_order)


def contract_exact(n: int, gates, tree, mps_site_order=None) -> complex:
    """contract_exact (exact.rs:60-68): the amplitude of |0...0>."""
    return contract_exact_at(n, gates, tree, 0, mps_site_order)
