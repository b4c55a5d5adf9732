"""The greedy exact-contraction planner (src/tn/plan.rs:1-284).

The reference keeps this planner as the test double of its orchestrator's
``PlanGreedyContraction``: gates stay in circuit order; a gate is applied
once every wire it touches sits on one state; joins of those states pick the
fewest result legs, then the younger origin gate, then the smaller minimum
wire, then the smaller maximum wire, then the earlier gate argument.  The
declared peak counts both inputs and the result during an outer product.
Trees come out in the reference's JSON form (tree.rs ``ContractionTree``):
``{"nodes": [{"op": "contract", "left": {"ket0": 0}, "right": {"gate": 0}},
...], "peak_bytes": P}``.
"""
from __future__ import annotations

import json

from .circuits import CCNOT, CNOT, CZ, IF, MEASURE, RESET

MAX_QUBITS = 4096  # plan.rs:16
MAX_GATES = 100_000  # plan.rs:17
MAX_LEGS = 26  # plan.rs:18
MAX_PEAK = 1 << 30  # plan.rs:19
_U64_MAX = (1 << 64) - 1


def _leg_bytes(legs: int) -> int:
    return 16 << legs


def _unitary_wires(g, n: int):
    """tree.rs:460-493: None for MEASURE/RESET/IF, the wires otherwise;
    False when the gate is invalid (a wire out of range or repeated)."""
    kind = int(g["kind"])
    if kind in (MEASURE, RESET, IF):
        return None
    if kind in (CNOT, CZ):
        wires = [int(g["q0"]), int(g["q1"])]
    elif kind == CCNOT:
        wires = [int(g["q0"]), int(g["q1"]), int(g["q2"])]
    else:
        wires = [int(g["q0"])]
    if any(w < 0 or w >= n for w in wires) or len(set(wires)) != len(wires):
        return False
    return wires


class _Slot:
    __slots__ = ("wires", "node", "gate", "alive")

    def __init__(self, wires, node=None, gate=None):
        self.wires = wires
        self.node = node
        self.gate = gate
        self.alive = True


def _younger(a, b):
    if a is not None and b is not None:
        return min(a, b)
    return a if a is not None else b


def _ref(slot: _Slot) -> dict:
    return {"node": slot.node} if slot.node is not None else {"ket0": slot.wires[0]}


class _Plan:
    def __init__(self, n: int):
        self.slots: list[_Slot] = []
        self.at = [None] * n
        self.nodes: list[dict] = []
        self.peak = 0
        self.alive_bytes = 0

    def ensure(self, wire: int) -> int:
        if self.at[wire] is not None:
            return self.at[wire]
        self.slots.append(_Slot([wire]))
        self.alive_bytes += _leg_bytes(1)
        self.at[wire] = len(self.slots) - 1
        return self.at[wire]

    def others(self, skip) -> int:
        return self.alive_bytes - sum(_leg_bytes(len(self.slots[i].wires)) for i in set(skip) if self.slots[i].alive)

    def pair_key(self, a_id: int, b_id: int, pos: dict):
        a, b = self.slots[a_id], self.slots[b_id]
        min_w = min(a.wires[0], b.wires[0])
        max_w = max(a.wires[-1], b.wires[-1])
        pa, pb = pos[a_id], pos[b_id]
        earlier, later = (pa, pb) if pa < pb else (pb, pa)
        origin = _younger(a.gate, b.gate)
        return (len(a.wires) + len(b.wires), _U64_MAX if origin is None else origin, min_w, max_w, earlier, later)

    def join(self, a_id: int, b_id: int):
        if self.slots[b_id].wires[0] < self.slots[a_id].wires[0]:
            a_id, b_id = b_id, a_id
        a, b = self.slots[a_id], self.slots[b_id]
        legs = len(a.wires) + len(b.wires)
        if legs > MAX_LEGS:
            return None
        during = self.others([a_id, b_id]) + _leg_bytes(len(a.wires)) + _leg_bytes(len(b.wires)) + _leg_bytes(legs)
        if during > MAX_PEAK:
            return None
        self.peak = max(self.peak, during)
        index = len(self.nodes)
        self.nodes.append({"op": "contract", "left": _ref(a), "right": _ref(b)})
        a.alive = b.alive = False
        self.alive_bytes -= _leg_bytes(len(a.wires)) + _leg_bytes(len(b.wires))
        slot = _Slot(sorted(a.wires + b.wires), node=index, gate=_younger(a.gate, b.gate))
        self.slots.append(slot)
        self.alive_bytes += _leg_bytes(legs)
        sid = len(self.slots) - 1
        for w in slot.wires:
            self.at[w] = sid
        return sid

    def apply(self, sid: int, gate_index: int) -> bool:
        slot = self.slots[sid]
        during = self.others([sid]) + _leg_bytes(len(slot.wires))
        if during > MAX_PEAK:
            return False
        self.peak = max(self.peak, during)
        index = len(self.nodes)
        self.nodes.append({"op": "contract", "left": _ref(slot), "right": {"gate": gate_index}})
        slot.node = index
        slot.gate = _younger(slot.gate, gate_index)
        return True

    def contract_gate(self, wires, gate_index: int) -> bool:
        ids, pos = [], {}
        for arg, wire in enumerate(wires):
            sid = self.ensure(wire)
            if sid not in pos:
                pos[sid] = arg
                ids.append(sid)
        while len(ids) > 1:
            best_i, best_j = 0, 1
            best = self.pair_key(ids[0], ids[1], pos)
            for i in range(len(ids)):
                for j in range(i + 1, len(ids)):
                    key = self.pair_key(ids[i], ids[j], pos)
                    if key < best:
                        best, best_i, best_j = key, i, j
            earlier = min(pos[ids[best_i]], pos[ids[best_j]])
            merged = self.join(ids[best_i], ids[best_j])
            if merged is None:
                return False
            pos[merged] = earlier
            lo, hi = sorted((best_i, best_j))
            del ids[hi]
            del ids[lo]
            ids.append(merged)
        return self.apply(ids[0], gate_index)


def plan_greedy(n: int, gates):
    """plan_greedy (plan.rs:21-44): the tree, or None when the circuit has no
    tree within 26 legs and 1 GiB (or is past the planner's caps)."""
    if n == 0 or n > MAX_QUBITS or len(gates) > MAX_GATES:
        return None
    plan = _Plan(n)
    for index, g in enumerate(gates):
        wires = _unitary_wires(g, n)
        if wires is False:
            return None
        if wires is None:
            continue
        if not plan.contract_gate(wires, index):
            return None
    return {"nodes": plan.nodes, "peak_bytes": plan.peak}


def tree_json(tree: dict) -> str:
    """The tree as the reference serialises it (serde_json, no spaces)."""
    out = {}
    if tree.get("kind") is not None:
        out["kind"] = tree["kind"]
    if tree.get("site_order"):
        out["site_order"] = list(tree["site_order"])
    out["nodes"] = tree["nodes"]
    if tree.get("peak_bytes") is not None:
        out["peak_bytes"] = tree["peak_bytes"]
    return json.dumps(out, separators=(",", ":"))
