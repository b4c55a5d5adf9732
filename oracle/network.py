"""ORACLE — test infrastructure only.

A numpy restatement of the reference's network contraction
(src/tn/network.rs:1-790), the checker of the device version
(wqc_network_contract).  <0...0|U|0...0> of a circuit as one tensor
network: wire w starts at a ket0(w) leaf and ends at a bra0(w) leaf; unitary
gate i is a gate(i) leaf with an input and an output leg per wire (or, for
CNOT and CZ, two halves joined by a bond edge).  A node contracts two tensors
over the edges they share; the result's legs are the right operand's free
legs (low bits), then the left's.  Leg p of a tensor is bit p of its index.
The walk, the byte accounting (live results, both inputs, the larger of the
result and each reordered copy) and every failure message follow
network.rs:183-282, 591-664.  The contraction itself is numpy's matmul, not
the reference's matrixmultiply GEMM, so results agree to rounding.

Nodes are (left, right) pairs of references (kind, index) with the kinds of
the C ABI: KET0 0, GATE 1, NODE 2, LEFT 3, RIGHT 4, BRA0 5, CONTROL 6,
TARGET 7.
"""
from __future__ import annotations

import numpy as np

import dense as D
import exact as OX

KET0, GATE, NODE, LEFT, RIGHT, BRA0, CONTROL, TARGET = range(8)
MAX_OPEN_LEGS = 26
MAX_PEAK_BYTES = 1 << 30
UNITARY = OX.UNITARY
WHOLE, HALF_C, HALF_T = 1, 2, 4
HALVES = HALF_C | HALF_T


class NetworkError(RuntimeError):
    pass


def build(n, gates):
    """Network::build (network.rs:62-96): (bra edges, gate legs or None,
    wire_edges)."""
    current = list(range(n))
    nxt = n
    legs_of = []
    for g in gates:
        if int(g["kind"]) not in UNITARY:
            legs_of.append(None)
            continue
        wires = OX.gate_wires(g)
        legs = [current[w] for w in wires]
        for w in wires:
            current[w] = nxt
            legs.append(nxt)
            nxt += 1
        legs_of.append(legs)
    return current, legs_of, nxt


def gate_tensor(g):
    """network.rs:431-445: entry input | output << m is <output|U|input>,
    columns by exact.rs's apply_in_place over the gate's own wires."""
    wires = OX.gate_wires(g)
    m = len(wires)
    dim = 1 << m
    data = np.zeros(dim * dim, dtype=np.complex128)
    for inp in range(dim):
        col = np.zeros(dim, dtype=np.complex128)
        col[inp] = 1
        OX.apply_in_place(col, wires, g)
        for out in range(dim):
            data[inp | (out << m)] = col[out]
    return data


def half_tensor(half, target_is_z):
    """network.rs:371-392: entry input | output << 1 | bond << 2."""
    out = np.zeros(8, dtype=np.complex128)
    for index in range(8):
        inp, outp, bond = index & 1, (index >> 1) & 1, index >> 2
        if half == 0:
            v = float(inp == outp == bond)
        elif bond == 0:
            v = float(inp == outp)
        elif target_is_z:
            v = 0.0 if inp != outp else (-1.0 if inp == 1 else 1.0)
        else:
            v = float(inp != outp)
        out[index] = v
    return out


def permute(data, frm, to):
    """Reorder legs `frm` into `to` (leg p is bit p)."""
    if list(frm) == list(to):
        return data
    L = len(frm)
    # numpy axes run from the most significant bit: axis a is bit L-1-a
    t = data.reshape([2] * L)
    axes = [L - 1 - list(frm).index(to[L - 1 - a]) for a in range(L)]
    return np.ascontiguousarray(np.transpose(t, axes)).reshape(-1)


def contract_pair(left, right, evaluate):
    """network.rs:591-664: (result, working bytes)."""
    llegs, ldata = left
    rlegs, rdata = right
    shared = [l for l in llegs if l in rlegs]
    lfree = [l for l in llegs if l not in shared]
    rfree = [l for l in rlegs if l not in shared]
    legs = rfree + lfree
    if len(legs) > MAX_OPEN_LEGS:
        raise NetworkError("contraction tree tensor exceeds 26 legs")
    lorder, rorder = shared + lfree, shared + rfree
    working = 16 << len(legs)
    if llegs != lorder:
        working = max(working, 16 << len(llegs))
    if rlegs != rorder:
        working = max(working, 16 << len(rlegs))
    data = None
    if evaluate:
        a = permute(ldata, llegs, lorder).reshape(1 << len(lfree), 1 << len(shared))
        b = permute(rdata, rlegs, rorder).reshape(1 << len(rfree), 1 << len(shared))
        data = (a @ b.T).reshape(-1)
    return (legs, data), working


def walk(n, gates, nodes, evaluate=True):
    """walk (network.rs:183-248): (peak, amplitude)."""
    if n == 0:
        raise NetworkError("Invalid qubit count: 0. Max limit is 40.")
    bra, gate_legs, wire_edges = build(n, gates)
    ket_used = [False] * n
    bra_used = [False] * n
    gate_used = [0] * len(gates)
    live = {}
    live_bytes = 0
    peak = 0

    def mark(used, w):
        if w >= n:
            raise NetworkError(f"Qubit index {w} out of bounds (limit: {n})")
        if used[w]:
            raise NetworkError("contraction tree reuses a tensor")
        used[w] = True

    def take_gate(i, part):
        used = gate_used[i]
        if used & part:
            raise NetworkError("contraction tree reuses a tensor")
        if used != 0 and (used | part) & WHOLE:
            raise NetworkError("contraction tree mixes a gate and its halves")
        gate_used[i] = used | part

    def take(ref, index):
        nonlocal live_bytes
        kind, i = ref
        if kind == NODE:
            if i >= index:
                raise NetworkError("contraction tree tensor is not ready")
            if i not in live:
                raise NetworkError("contraction tree reuses a tensor")
            t = live.pop(i)
            live_bytes -= 16 << len(t[0])
            return t
        if kind == KET0:
            mark(ket_used, i)
            return [i], np.array([1, 0], dtype=np.complex128)
        if kind == BRA0:
            mark(bra_used, i)
            return [bra[i]], np.array([1, 0], dtype=np.complex128)
        if kind == GATE:
            if i >= len(gates):
                raise NetworkError("contraction tree gate is missing")
            if gate_legs[i] is None:
                raise NetworkError(f"gate {i} is not a contraction leaf")
            take_gate(i, WHOLE)
            return list(gate_legs[i]), gate_tensor(gates[i]) if evaluate else None
        if kind in (CONTROL, TARGET):
            if i >= len(gates):
                raise NetworkError("contraction tree gate is missing")
            k = int(gates[i]["kind"])
            if k not in (D.CNOT, D.CZ):
                raise NetworkError(f"gate {i} has no halves")
            half = 0 if kind == CONTROL else 1
            take_gate(i, HALF_C if half == 0 else HALF_T)
            legs = gate_legs[i]
            return [legs[half], legs[2 + half], wire_edges + i], half_tensor(half, k == D.CZ)
        raise NetworkError("contraction tree network has no split")

    for index, (left, right) in enumerate(nodes):
        lt = take(left, index)
        rt = take(right, index)
        inputs = (16 << len(lt[0])) + (16 << len(rt[0]))
        result, working = contract_pair(lt, rt, evaluate)
        during = live_bytes + inputs + working
        if during > MAX_PEAK_BYTES:
            raise NetworkError("contraction tree peak exceeds 1 GiB")
        peak = max(peak, during)
        live_bytes += 16 << len(result[0])
        live[index] = result
    if not all(ket_used) or not all(bra_used) or any(
            gate_legs[i] is not None and gate_used[i] not in (WHOLE, HALVES) for i in range(len(gates))):
        raise NetworkError("contraction tree leaves a leaf out")
    if len(live) != 1 or next(iter(live.values()))[0]:
        raise NetworkError("contraction tree does not end in one scalar")
    root = next(iter(live.values()))
    return peak, complex(root[1][0]) if evaluate else 0j


def contract(n, gates, nodes, peak_bytes):
    """contract_network (network.rs:145-160): (peak, amplitude)."""
    if peak_bytes is None:
        raise NetworkError("contraction tree requires a peak")
    if peak_bytes > MAX_PEAK_BYTES:
        raise NetworkError("contraction tree peak exceeds 1 GiB")
    peak, amp = walk(n, gates, nodes, True)
    if peak != peak_bytes:
        raise NetworkError("contraction tree peak does not match")
    return peak, amp


def measured_peak(n, gates, nodes):
    """network.rs:162-169."""
    return walk(n, gates, nodes, False)[0]
