"""Network contraction trees for a circuit: the leaves of its tensor network
(src/tn/network.rs:55-120) and the plain greedy pass of the reference's
orchestrator (network.rs:914-972, the tree its ``PlanNetworkContraction``
returns when the search stops at once): among the pairs of live tensors that
share an edge, contract the one whose result grows least, |result| - |left|
- |right| in amplitudes, then the smaller tensor ids (leaves take ids in
canonical order -- ket0, unitary gates, bra0 -- and node i takes leaves + i);
scalars join last, smallest ids first.  The declared peak is the walk's
(``wqc_network_measured_peak``), absent when the tree is over budget.
"""
from __future__ import annotations

from .circuits import CCNOT, CNOT, CZ, IF, MEASURE, RESET


def _wires(g):
    k = int(g["kind"])
    if k in (CNOT, CZ):
        return [int(g["q0"]), int(g["q1"])]
    if k == CCNOT:
        return [int(g["q0"]), int(g["q1"]), int(g["q2"])]
    return [int(g["q0"])]


def build(n: int, gates):
    """Network::build (network.rs:62-96): (bra edge per wire, legs per gate
    -- inputs then outputs in the gate's wire order, None if not unitary --,
    wire_edges).  Edge w leaves ket0(w); the bond of gate i is wire_edges + i."""
    current = list(range(n))
    nxt = n
    legs_of = []
    for g in gates:
        if int(g["kind"]) in (MEASURE, RESET, IF):
            legs_of.append(None)
            continue
        wires = _wires(g)
        legs = [current[w] for w in wires]
        for w in wires:
            current[w] = nxt
            legs.append(nxt)
            nxt += 1
        legs_of.append(legs)
    return current, legs_of, nxt


def leaves(n: int, gates):
    """Leaves in canonical order: ket0, unitary gates, bra0 (network.rs:807-822)."""
    bra, legs_of, _ = build(n, gates)
    out = [({"ket0": w}, [w]) for w in range(n)]
    out += [({"gate": i}, list(legs)) for i, legs in enumerate(legs_of) if legs is not None]
    out += [({"bra0": w}, [bra[w]]) for w in range(n)]
    return out


def split_leaves(n: int, gates):
    """``leaves`` with every CNOT and CZ as its control half, then its target
    (network.rs:824-846): each half has its wire's input, output and the bond."""
    _, legs_of, wire_edges = build(n, gates)
    out = []
    for ref, legs in leaves(n, gates):
        i = ref.get("gate")
        if i is not None and int(gates[i]["kind"]) in (CNOT, CZ):
            g = legs_of[i]
            out.append(({"control": i}, [g[0], g[2], wire_edges + i]))
            out.append(({"target": i}, [g[1], g[3], wire_edges + i]))
        else:
            out.append((ref, legs))
    return out


def _symmetric_difference(a, b):
    sa, sb = set(a), set(b)
    return [l for l in b if l not in sa] + [l for l in a if l not in sb]


def greedy_tree_of(n: int, gates, live) -> dict:
    """network.rs:918-972 over the given leaves."""
    slots = [(ref, list(legs)) for ref, legs in live]
    owners: dict[int, list[int]] = {}
    for sid, (_, legs) in enumerate(slots):
        for leg in legs:
            owners.setdefault(leg, []).append(sid)
    sets = [set(legs) for _, legs in slots]
    nodes = []
    alive = len(slots)
    while alive > 1:
        best = None
        for edge in sorted(owners):
            pair = owners[edge]
            i, j = min(pair[0], pair[1]), max(pair[0], pair[1])
            a, b = sets[i], sets[j]
            common = len(a & b)
            legs = len(a) + len(b) - 2 * common
            cost = (1 << legs) - (1 << len(a)) - (1 << len(b))
            if best is None or (cost, i, j) < best:
                best = (cost, i, j)
        if best is not None:
            _, i, j = best
        else:
            live_ids = [sid for sid, s in enumerate(slots) if s is not None]
            i, j = live_ids[0], live_ids[1]
        left, a = slots[i]
        right, b = slots[j]
        slots[i] = slots[j] = None
        legs = _symmetric_difference(a, b)
        keep = set(legs)
        new_id = len(slots)
        for leg in a + b:
            if leg in keep:
                owners[leg] = [new_id if o in (i, j) else o for o in owners[leg]]
            else:
                owners.pop(leg, None)
        nodes.append({"op": "contract", "left": left, "right": right})
        slots.append(({"node": len(nodes) - 1}, legs))
        sets.append(set(legs))
        alive -= 1
    return finish(n, gates, nodes)


def finish(n: int, gates, nodes) -> dict:
    """The tree with its measured peak, or no peak when the walk fails (over
    budget) -- network.rs:854-866."""
    from . import WqcCudaError
    from .network import measured_peak

    tree = {"kind": "network", "nodes": nodes}
    try:
        tree["peak_bytes"] = measured_peak(n, gates, tree)
    except WqcCudaError:
        pass
    return tree


def greedy_tree(n: int, gates) -> dict:
    return greedy_tree_of(n, gates, leaves(n, gates))


def greedy_split_tree(n: int, gates) -> dict:
    return greedy_tree_of(n, gates, split_leaves(n, gates))
