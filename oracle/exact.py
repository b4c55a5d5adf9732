"""ORACLE — test infrastructure only.

A restatement of the reference's exact contraction of a `Contract` tree
(src/tn/exact.rs:60-560), the checker of the device version
(wqc_exact_contract).  The walk (validation, circuit order, live bytes,
peak) is Python; the dense kernels (outer product, gate in place) are the C
loops of exact_oracle.cpp in liboracle.so, compiled without floating-point
contraction so that every amplitude carries the reference's rounding; numpy
versions of the two kernels (apply_in_place_numpy, outer_numpy) check them.
A state tensor is a dense array over its open wires
(sorted; wire at position p is bit p of the index).  A node consumes two
operands: a gate applied in place to a state that holds all its wires, or
two states with no wire in common joined by an outer product.  Gates are
consumed in circuit order; the peak of the live tensors' bytes is walked
and must equal the tree's declared peak; the amplitude of one basis vector
is the product of the live tensors' components.

Nodes are (left, right) pairs of references (kind, index) with kind
KET0 = 0 (index: wire), GATE = 1 (index: gate), NODE = 2 (index: node).
"""
from __future__ import annotations

import ctypes

import numpy as np

import dense as D
import oracle as _O

KET0, GATE, NODE = 0, 1, 2
MAX_OPEN_LEGS = 26  # exact.rs:25
MAX_PEAK_BYTES = 1 << 30  # exact.rs:27
UNITARY = (D.H, D.X, D.Y, D.Z, D.S, D.T, D.RX, D.RY, D.RZ, D.CNOT, D.CZ, D.CCNOT)


class ExactError(RuntimeError):
    pass


def gate_wires(g):
    k = int(g["kind"])
    if k in (D.CNOT, D.CZ):
        return [int(g["q0"]), int(g["q1"])]
    if k == D.CCNOT:
        return [int(g["q0"]), int(g["q1"]), int(g["q2"])]
    return [int(g["q0"])]


def _cmat(kind):
    """The 4x4 matrix m[co][to][ci][ti] of CNOT or CZ (src/tn/gates.rs)."""
    m = np.zeros((2, 2, 2, 2), dtype=np.complex128)
    m[0, 0, 0, 0] = m[0, 1, 0, 1] = 1
    if kind == D.CNOT:
        m[1, 0, 1, 1] = m[1, 1, 1, 0] = 1
    else:
        m[1, 0, 1, 0] = 1
        m[1, 1, 1, 1] = -1
    return m


def _bind():
    L = _O.lib()
    if not getattr(L, "_exact_bound", False):
        P, U = ctypes.c_void_p, ctypes.c_uint32
        L.oracle_exact_outer.argtypes = [P, U, P, P, U, P, P]
        L.oracle_exact_outer.restype = None
        L.oracle_exact_apply_1q.argtypes = [P, U, U, P]
        L.oracle_exact_apply_1q.restype = None
        L.oracle_exact_apply_2q.argtypes = [P, U, U, U, P]
        L.oracle_exact_apply_2q.restype = None
        L.oracle_exact_apply_ccnot.argtypes = [P, U, U, U, U]
        L.oracle_exact_apply_ccnot.restype = None
        L._exact_bound = True
    return L


def apply_in_place(data, wires, g):
    """exact.rs:482-560, by the C loops of exact_oracle.cpp (the reference's
    operation order, per-operation rounding)."""
    L = _bind()
    k = int(g["kind"])
    pos = {w: i for i, w in enumerate(wires)}
    legs = len(wires)
    assert data.dtype == np.complex128 and data.flags.c_contiguous and len(data) == 1 << legs
    if k in (D.CNOT, D.CZ):
        m = np.ascontiguousarray(_cmat(k))
        L.oracle_exact_apply_2q(data.ctypes.data, legs, pos[int(g["q0"])], pos[int(g["q1"])], m.ctypes.data)
    elif k == D.CCNOT:
        L.oracle_exact_apply_ccnot(data.ctypes.data, legs, pos[int(g["q0"])], pos[int(g["q1"])], pos[int(g["q2"])])
    else:
        u = np.ascontiguousarray(D.unary(k, float(g["angle"])), dtype=np.complex128)
        L.oracle_exact_apply_1q(data.ctypes.data, legs, pos[int(g["q0"])], u.ctypes.data)
    return data


def apply_in_place_numpy(data, wires, g):
    """exact.rs:490-560 in numpy (permutations for CNOT/CZ/CCNOT): a second
    restatement the C loops are checked against."""
    k = int(g["kind"])
    pos = {w: i for i, w in enumerate(wires)}
    idx = np.arange(len(data))
    if k in (D.CNOT, D.CZ):
        c, t = (1 << pos[int(g["q0"])]), (1 << pos[int(g["q1"])])
        base = idx[((idx & c) == 0) & ((idx & t) == 0)]
        v00, v10, v01, v11 = data[base].copy(), data[base | c].copy(), data[base | t].copy(), data[base | c | t].copy()
        if k == D.CNOT:  # control set: target flips
            data[base | c], data[base | c | t] = v11, v10
        else:
            data[base | c | t] = -v11
        return data
    if k == D.CCNOT:
        m1, m2, mt = (1 << pos[int(g["q0"])]), (1 << pos[int(g["q1"])]), (1 << pos[int(g["q2"])])
        sel = idx[((idx & m1) != 0) & ((idx & m2) != 0) & ((idx & mt) == 0)]
        a, b = data[sel].copy(), data[sel | mt].copy()
        data[sel], data[sel | mt] = b, a
        return data
    bit = 1 << pos[int(g["q0"])]
    u = D.unary(k, float(g["angle"]))
    lo = idx[(idx & bit) == 0]
    v0, v1 = data[lo].copy(), data[lo | bit].copy()
    data[lo] = u[0, 0] * v0 + u[0, 1] * v1
    data[lo | bit] = u[1, 0] * v0 + u[1, 1] * v1
    return data


def outer(lw, ld, rw, rd):
    """exact.rs:444-488: sorted union of the wires, product at scattered
    bits, by the C loop of exact_oracle.cpp."""
    if set(lw) & set(rw):
        raise ExactError("tensors share a wire")
    wires = sorted(lw + rw)
    if len(wires) > MAX_OPEN_LEGS:
        raise ExactError("contraction tree tensor exceeds 26 legs")
    lp = np.array([wires.index(w) for w in lw], dtype=np.uint32)
    rp = np.array([wires.index(w) for w in rw], dtype=np.uint32)
    ld = np.ascontiguousarray(ld, dtype=np.complex128)
    rd = np.ascontiguousarray(rd, dtype=np.complex128)
    data = np.empty(1 << len(wires), dtype=np.complex128)
    _bind().oracle_exact_outer(ld.ctypes.data, len(lw), lp.ctypes.data, rd.ctypes.data, len(rw), rp.ctypes.data,
                               data.ctypes.data)
    return wires, data


def outer_numpy(lw, ld, rw, rd):
    """exact.rs:444-488 in numpy, the check of the C loop."""
    wires = sorted(lw + rw)
    lp = [wires.index(w) for w in lw]
    rp = [wires.index(w) for w in rw]

    def scatter(i, pos):
        out = np.zeros_like(i)
        for b, p in enumerate(pos):
            out |= ((i >> b) & 1) << p
        return out

    li = scatter(np.arange(len(ld)), lp)
    ri = scatter(np.arange(len(rd)), rp)
    data = np.zeros(1 << len(wires), dtype=np.complex128)
    data[(li[:, None] | ri[None, :]).ravel()] = (ld[:, None] * rd[None, :]).ravel()
    return wires, data


def contract(n, gates, nodes, peak_bytes, bits=0):
    """contract_exact_at (exact.rs:70-85): (peak, amplitude of basis vector
    `bits`), or ExactError with the reference's message."""
    if peak_bytes is None:
        raise ExactError("exact contraction tree requires a peak")
    if peak_bytes > MAX_PEAK_BYTES:
        raise ExactError("contraction tree peak exceeds 1 GiB")
    peak, amp = walk(n, gates, nodes, bits, True)
    if peak_bytes != peak:
        raise ExactError("contraction tree peak does not match")
    return peak, amp


def measured_peak(n, gates, nodes):
    """exact.rs:650-658: the walk's peak without evaluating."""
    return walk(n, gates, nodes, 0, False)[0]


def walk(n, gates, nodes, bits=0, evaluate=True):
    """walk + sample (exact.rs:136-231)."""
    unitary = [i for i, g in enumerate(gates) if int(g["kind"]) in UNITARY]
    live = {}
    consumed_nodes = set()
    consumed_gate = set()
    consumed_ket = set()
    next_gate = 0
    peak = 0

    def occupied(t):
        return 0 if t[0] == "gate" else 16 << len(t[1])

    def materialize(ref):
        nonlocal next_gate
        if ref in live:
            return
        kind, i = ref
        if kind == KET0:
            if i >= n:
                raise ExactError(f"Qubit index {i} out of bounds (limit: {n})")
            if i in consumed_ket:
                raise ExactError("contraction tree reuses a tensor")
            consumed_ket.add(i)
            live[ref] = ("state", [i], np.array([1.0, 0.0], dtype=np.complex128))
        elif kind == GATE:
            if i >= len(gates):
                raise ExactError("contraction tree gate is missing")
            if int(gates[i]["kind"]) not in UNITARY:
                raise ExactError(f"gate {i} is not a contraction leaf")
            expected = next((u for u in unitary if u >= next_gate), None)
            if expected is None or i != expected:
                raise ExactError("gates are out of circuit order")
            next_gate = i + 1
            if i in consumed_gate:
                raise ExactError("contraction tree reuses a tensor")
            consumed_gate.add(i)
            live[ref] = ("gate", i)
        else:
            if i in consumed_nodes:
                raise ExactError("contraction tree reuses a tensor")
            raise ExactError("contraction tree tensor is not ready")

    def take(ref):
        if ref not in live:
            raise ExactError("contraction tree tensor is not ready")
        t = live.pop(ref)
        if ref[0] == NODE:
            if ref[1] in consumed_nodes:
                raise ExactError("contraction tree reuses a tensor")
            consumed_nodes.add(ref[1])
        return t

    for index, (left, right) in enumerate(nodes):
        materialize(left)
        materialize(right)
        lt, rt = take(left), take(right)
        allocating = lt[0] == "state" and rt[0] == "state"
        inputs = occupied(lt) + occupied(rt)
        if lt[0] == "gate" or rt[0] == "gate":
            gt, st = (lt, rt) if lt[0] == "gate" else (rt, lt)
            if st[0] != "state":
                raise ExactError("exact contraction does not contract two gates")
            g = gates[gt[1]]
            if any(w not in st[1] for w in gate_wires(g)):
                raise ExactError("gate wires are not open")
            result = ("state", st[1], apply_in_place(st[2], st[1], g) if evaluate else None)
        else:
            if set(lt[1]) & set(rt[1]):
                raise ExactError("tensors share a wire")
            if len(lt[1]) + len(rt[1]) > MAX_OPEN_LEGS:
                raise ExactError("contraction tree tensor exceeds 26 legs")
            if evaluate:
                w, d = outer(lt[1], lt[2], rt[1], rt[2])
            else:
                w, d = sorted(lt[1] + rt[1]), None
            result = ("state", w, d)
        during = sum(occupied(t) for t in live.values()) + inputs + (occupied(result) if allocating else 0)
        if during > MAX_PEAK_BYTES:
            raise ExactError("contraction tree peak exceeds 1 GiB")
        peak = max(peak, during)
        live[(NODE, index)] = result
    for i in unitary:
        if i not in consumed_gate:
            raise ExactError("gate was not contracted")
    if not evaluate:
        return peak, 0j
    amp = 1.0 + 0.0j
    covered = set()
    for key in sorted(live):  # the reference's BTreeMap order: Ket < Gate < Node, then index
        t = live[key]
        if t[0] == "gate":
            raise ExactError("gate was not contracted")
        covered |= set(t[1])
        idx = sum(1 << p for p, w in enumerate(t[1]) if w < 64 and (bits >> w) & 1)
        c = complex(t[2][idx])
        # num_complex's product, one rounding per operation (Python floats)
        amp = complex(amp.real * c.real - amp.imag * c.imag, amp.real * c.imag + amp.imag * c.real)
    if any(w < 64 and (bits >> w) & 1 and w not in covered for w in range(n)):
        amp = 0j
    return peak, amp

