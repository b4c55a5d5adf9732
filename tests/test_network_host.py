"""Network contraction trees, host side (no GPU).

* The oracle (oracle/network.py) against the dense statevector and the known
  answers of the reference's tests (src/tn/network.rs:1038-1760): any
  contraction order, whole gates and gate halves, the orchestrator's trees
  (fixture JSON, tree hash, the three searched 4x4 grid trees), peaks and
  rejections.
* The greedy planner (wqc_cuda.network_plan) against the reference's JSON
  text and SHA3 pin.
* The C ABI's host walk (wqc_network_validate, wqc_network_measured_peak)
  against the oracle on planned and on mutated trees.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import dense as D
import network as ON
from wqc_cuda import ERR_INVALID, WqcCudaError
from wqc_cuda import circuits as C
from wqc_cuda import exact as XE
from wqc_cuda import exact_plan as EP
from wqc_cuda import network as N
from wqc_cuda import network_plan as NP

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KIND = {"ket0": ON.KET0, "gate": ON.GATE, "node": ON.NODE, "left": ON.LEFT, "right": ON.RIGHT, "bra0": ON.BRA0,
        "control": ON.CONTROL, "target": ON.TARGET}


def onodes(tree):
    out = []
    for nd in tree["nodes"]:
        (lk, li), = nd["left"].items()
        (rk, ri), = nd["right"].items()
        out.append(((KIND[lk], li), (KIND[rk], ri)))
    return out


def node(left, right):
    return {"op": "contract", "left": left, "right": right}


def dense_zero(n, gates):
    d = D.Dense(n)
    d.apply_gates([g for g in gates if int(g["kind"]) < C.MEASURE])
    return d.state[0]


def oracle_amp(n, gates, tree):
    return ON.contract(n, gates, onodes(tree), tree.get("peak_bytes"))[1]


def lcg_circuit(n, count, seed):
    """network.rs:986-1020: the reference's seeded random circuit."""
    state = [seed]

    def nxt(bound):
        state[0] = (state[0] * 6364136223846793005 + 1442695040888963407) & (2 ** 64 - 1)
        return (state[0] >> 33) % bound

    gates = []
    for _ in range(count):
        a = nxt(n)
        b = (a + 1 + nxt(n - 1)) % n
        theta = nxt(1000) * 0.00731 + 0.1
        k = nxt(12)
        if k <= 5:
            gates.append(C.g1(k, a))
        elif k <= 8:
            gates.append(C.g1(k, a, theta))
        elif k == 9:
            gates.append(C.g2(C.CNOT, a, b))
        elif k == 10:
            gates.append(C.g2(C.CZ, a, b))
        elif n >= 3:
            c = next(c for c in range(n) if c != a and c != b)
            gates.append(C.g3(a, b, c))
        else:
            gates.append(C.g2(C.CNOT, a, b))
    return C.gates_array(gates)


def random_tree_of(n, gates, live, seed):
    """network.rs:872-912: any order, a neighbour sharing an edge when there
    is one."""
    mask = 2 ** 64 - 1
    state = [(seed * 6364136223846793005 + 1442695040888963407) & mask]

    def nxt(bound):
        state[0] = (state[0] * 6364136223846793005 + 1442695040888963407) & mask
        return (state[0] >> 33) % bound

    live = [(r, list(l)) for r, l in live]
    nodes = []
    while len(live) > 1:
        i = nxt(len(live))
        nb = [j for j in range(len(live)) if j != i and any(l in live[i][1] for l in live[j][1])]
        j = (i + 1 + nxt(len(live) - 1)) % len(live) if not nb else nb[nxt(len(nb))]
        hi, lo = max(i, j), min(i, j)
        b = live.pop(hi)
        a = live.pop(lo)
        legs = [l for l in b[1] if l not in a[1]] + [l for l in a[1] if l not in b[1]]
        nodes.append(node(a[0], b[0]))
        live.append(({"node": len(nodes) - 1}, legs))
    return NP.finish(n, gates, nodes)


def ghz_far():
    ghz = C.gates_array([C.g1(C.H, 0)] + [C.g2(C.CNOT, q, q + 1) for q in range(4)])
    far = C.gates_array([C.g1(C.H, 0), C.g2(C.CNOT, 0, 4), C.g1(C.RY, 4, 0.4), C.g2(C.CZ, 4, 1)])
    return [(5, ghz), (5, far)] + [(6, lcg_circuit(6, 40, s)) for s in range(6)]


# --- oracle and planner against network.rs's tests ----------------------------

def test_any_order_matches_dense():
    for n, gates in ghz_far():
        expected = dense_zero(n, gates)
        for seed in range(8):
            tree = random_tree_of(n, gates, NP.leaves(n, gates), seed)
            assert abs(oracle_amp(n, gates, tree) - expected) < 1e-9
        assert abs(oracle_amp(n, gates, NP.greedy_tree(n, gates)) - expected) < 1e-9


FIXTURE_JSON = ('{"kind":"network","nodes":[{"op":"contract","left":{"ket0":1},"right":{"gate":3}},{"op":"contract",'
                '"left":{"bra0":0},"right":{"node":0}},{"op":"contract","left":{"gate":1},"right":{"node":1}},'
                '{"op":"contract","left":{"ket0":2},"right":{"node":2}},{"op":"contract","left":{"bra0":2},"right":'
                '{"node":3}},{"op":"contract","left":{"ket0":0},"right":{"gate":0}},{"op":"contract","left":{"gate":4},'
                '"right":{"bra0":1}},{"op":"contract","left":{"node":4},"right":{"node":5}},{"op":"contract","left":'
                '{"ket0":3},"right":{"bra0":3}},{"op":"contract","left":{"node":6},"right":{"node":7}},{"op":"contract",'
                '"left":{"node":8},"right":{"node":9}}],"peak_bytes":2080}')


def fixture_gates():
    return C.gates_array([C.g1(C.H, 0), C.g2(C.CNOT, 0, 2), (C.MEASURE, 1, 0, 0, 0.0), C.g3(0, 2, 1),
                          C.g1(C.RZ, 1, 0.4)])


def test_orchestrator_fixture_is_the_greedy_tree():
    gates = fixture_gates()
    tree = NP.greedy_tree(4, gates)
    assert EP.tree_json(tree) == FIXTURE_JSON
    expected = dense_zero(4, gates)
    assert abs(expected) > 0.1
    assert abs(oracle_amp(4, gates, json.loads(FIXTURE_JSON)) - expected) < 1e-9


def test_brickwork_tree_hash_matches_the_greedy():
    tree = NP.greedy_tree(6, C.ry_rz_cnot_brickwork(6, 3))
    assert hashlib.sha3_256(EP.tree_json(tree).encode()).hexdigest() == \
        "dccaf420f62676fdc7f589aa8791dd29ecd145c68a9af661dabfd443429aa2c1"


GRIDS = {"network_grid_4x4_d12.json": None, "network_grid_4x4_d12_split.json": 843776,
         "network_grid_4x4_d12_bisect.json": 262144}


def load_grid(name):
    with open(os.path.join(GOLDEN, name), "rb") as f:
        return f.read()


def test_orchestrator_grid_trees():
    gates = C.grid(4, 12)
    expected = dense_zero(16, gates)
    assert abs(expected) > 0.1
    import importlib.util

    spec = importlib.util.spec_from_file_location("copy_network_fixtures",
                                                  os.path.join(GOLDEN, "copy_network_fixtures.py"))
    fx = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(fx)
    PINS = fx.PINS
    for name, peak in GRIDS.items():
        text = load_grid(name)
        assert hashlib.sha3_256(text).hexdigest() == PINS[name]
        tree = json.loads(text)
        if peak is not None:
            assert tree["peak_bytes"] == peak
            assert EP.tree_json(tree) == text.decode()
            assert '{"control":' in text.decode()
        else:
            assert tree["nodes"] != NP.greedy_tree(16, gates)["nodes"]  # a searched tree
        N.validate(16, gates, tree)
        assert ON.measured_peak(16, gates, onodes(tree)) == tree["peak_bytes"]
        assert abs(oracle_amp(16, gates, tree) - expected) < 1e-9


def test_untouched_wire_and_skipped_ops_close_with_one():
    gates = C.gates_array([C.g1(C.H, 0), (C.MEASURE, 0, 0, 0, 0.0), (C.IF, 1, 0, 0, 0.0), C.g2(C.CNOT, 0, 2)])
    tree = NP.greedy_tree(4, gates)
    assert abs(oracle_amp(4, gates, tree) - dense_zero(4, gates)) < 1e-9
    one = {"kind": "network", "nodes": [node({"ket0": 0}, {"bra0": 0})], "peak_bytes": 32 + 32 + 16}
    N.validate(1, C.gates_array([]), one)
    assert abs(oracle_amp(1, C.gates_array([]), one) - 1) < 1e-15


def test_split_gates_match_dense():
    circuits = [(5, C.ry_rz_cnot_brickwork(5, 4)), (4, C.grid(2, 6))]
    circuits += [(6, lcg_circuit(6, 40, s)) for s in range(6)]
    circuits.append((3, C.gates_array([C.g1(C.H, 0), C.g1(C.H, 2), C.g2(C.CZ, 2, 0), C.g2(C.CNOT, 0, 2),
                                       C.g2(C.CZ, 0, 1)])))
    for n, gates in circuits:
        expected = dense_zero(n, gates)
        for seed in range(8):
            tree = random_tree_of(n, gates, NP.split_leaves(n, gates), seed)
            assert abs(oracle_amp(n, gates, tree) - expected) < 1e-9
        assert abs(oracle_amp(n, gates, NP.greedy_split_tree(n, gates)) - expected) < 1e-9


def test_split_and_whole_gates_mix():
    n = 4
    gates = C.ry_rz_cnot_brickwork(n, 3)
    whole = next(i for i, g in enumerate(gates) if int(g["kind"]) == C.CNOT)
    _, legs_of, _ = NP.build(n, gates)
    live = []
    for ref, legs in NP.split_leaves(n, gates):
        if ref.get("target") == whole:
            continue
        if ref.get("control") == whole:
            live.append(({"gate": whole}, legs_of[whole]))
        else:
            live.append((ref, legs))
    tree = random_tree_of(n, gates, live, 3)
    assert abs(oracle_amp(n, gates, tree) - dense_zero(n, gates)) < 1e-9


def test_split_tree_names_the_halves():
    gates = C.gates_array([C.g1(C.H, 0), C.g2(C.CNOT, 0, 1)])
    nodes = [node({"control": 1}, {"target": 1}), node({"ket0": 0}, {"gate": 0}), node({"node": 1}, {"node": 0}),
             node({"ket0": 1}, {"node": 2}), node({"bra0": 0}, {"node": 3}), node({"bra0": 1}, {"node": 4})]
    tree = NP.finish(2, gates, nodes)
    _, legs_of, wire_edges = NP.build(2, gates)
    assert [legs_of[1][0], legs_of[1][2], wire_edges + 1] == [2, 3, 6]
    assert [legs_of[1][1], legs_of[1][3], wire_edges + 1] == [1, 4, 6]
    assert EP.tree_json(tree).startswith('{"kind":"network","nodes":[{"op":"contract","left":{"control":1},'
                                         '"right":{"target":1}}')
    assert abs(oracle_amp(2, gates, tree) - dense_zero(2, gates)) < 1e-9


def test_outer_products_keep_their_order_and_reordered_copy_counts():
    gates = C.gates_array([C.g1(C.RY, 0, 0.3), C.g1(C.RY, 1, 0.5)])
    tree = NP.finish(2, gates, [node({"ket0": 0}, {"gate": 0}), node({"node": 0}, {"ket0": 1}),
                                node({"node": 1}, {"gate": 1}), node({"node": 2}, {"bra0": 0}),
                                node({"node": 3}, {"bra0": 1})])
    assert abs(oracle_amp(2, gates, tree) - dense_zero(2, gates)) < 1e-9
    cnot = C.gates_array([C.g2(C.CNOT, 0, 1)])
    tree = NP.finish(2, cnot, [node({"gate": 0}, {"ket0": 1}), node({"node": 0}, {"ket0": 0}),
                               node({"node": 1}, {"bra0": 0}), node({"node": 2}, {"bra0": 1})])
    assert tree["peak_bytes"] == 544
    assert abs(oracle_amp(2, cnot, tree) - 1) < 1e-15


def err(fn, *a):
    with pytest.raises(WqcCudaError) as e:
        fn(*a)
    return str(e.value).split("] ", 1)[1]


def test_bad_trees_are_rejected():
    n = 3
    gates = C.gates_array([C.g1(C.H, 0), C.g2(C.CNOT, 0, 1), C.g3(0, 1, 2)])
    good = NP.greedy_tree(n, gates)
    N.validate(n, gates, good)

    def check(tree, needle):
        msg = err(N.validate, n, gates, tree)
        assert needle in msg, msg
        assert XE.is_contraction_client_error(ERR_INVALID, msg)
        if tree.get("peak_bytes") is not None:
            with pytest.raises(ON.NetworkError, match=needle):
                ON.contract(n, gates, onodes(tree), tree["peak_bytes"])

    check(dict(good, peak_bytes=good["peak_bytes"] + 16), "does not match")
    check(dict(good, peak_bytes=None), "requires a peak")
    check(dict(good, nodes=good["nodes"][:-1]), "one scalar")
    check(dict(good, nodes=good["nodes"][:1]), "leaves a leaf out")
    check(dict(good, nodes=good["nodes"] + [node(good["nodes"][0]["left"], {"node": len(good["nodes"]) - 1})]),
          "reuses a tensor")
    check(dict(good, nodes=[node({"node": 0}, {"ket0": 0})] + good["nodes"][1:]), "not ready")
    assert "parent wire" in err(N.validate, n, gates, dict(good, site_order=[2, 1, 0]))
    assert "no split" in err(N.validate, n, gates, dict(good, nodes=[node({"left": 0}, {"ket0": 0})] + good["nodes"][1:]))
    assert err(N.validate, n, gates, dict(good, kind=None)) == "contraction tree is not a network"
    assert "sweep steps" in err(N.validate, n, gates, dict(good, nodes=[{"op": "site", "tensor": {"ket0": 0},
                                                                          "gate": 0}]))


def test_bad_split_trees_are_rejected():
    n = 3
    gates = C.gates_array([C.g1(C.H, 0), C.g2(C.CNOT, 0, 1), C.g3(0, 1, 2)])
    good = NP.greedy_split_tree(n, gates)
    N.validate(n, gates, good)

    def replace(frm, to):
        t = json.loads(json.dumps(good))
        for nd in t["nodes"]:
            for side in ("left", "right"):
                if nd[side] == frm:
                    nd[side] = to
        return t

    for frm, to, needle in (({"target": 1}, {"gate": 1}, "mixes a gate and its halves"),
                            ({"target": 1}, {"control": 1}, "reuses a tensor"),
                            ({"target": 1}, {"control": 0}, "gate 0 has no halves"),
                            ({"target": 1}, {"target": 2}, "gate 2 has no halves"),
                            ({"target": 1}, {"target": 9}, "gate is missing")):
        t = replace(frm, to)
        assert needle in err(N.validate, n, gates, t)
        with pytest.raises(ON.NetworkError, match=needle):
            ON.contract(n, gates, onodes(t), t["peak_bytes"])
    at = next(i for i, nd in enumerate(good["nodes"]) if {"target": 1} in (nd["left"], nd["right"]))
    assert "leaves a leaf out" in err(N.validate, n, gates, dict(good, nodes=good["nodes"][:at]))


def test_over_budget_and_wide_joins_are_rejected():
    gates = C.gates_array([C.g1(C.H, 0)])
    tree = NP.greedy_tree(3, gates)
    assert "peak exceeds 1 GiB" in err(N.validate, 3, gates, dict(tree, peak_bytes=(1 << 30) + 1))
    nodes = []
    for start in (0, 25):
        acc = {"ket0": start}
        for w in range(start + 1, start + 25):
            nodes.append(node(acc, {"ket0": w}))
            acc = {"node": len(nodes) - 1}
    big = {"kind": "network", "nodes": nodes, "peak_bytes": 0}
    assert "peak exceeds 1 GiB" in err(N.validate, 50, C.gates_array([]), big)
    with pytest.raises(ON.NetworkError, match="peak exceeds 1 GiB"):
        ON.measured_peak(50, C.gates_array([]), onodes(big))
    nodes = []
    acc = {"ket0": 0}
    for w in range(1, 27):
        nodes.append(node(acc, {"ket0": w}))
        acc = {"node": len(nodes) - 1}
    assert "exceeds" in err(N.validate, 27, C.gates_array([]), {"kind": "network", "nodes": nodes, "peak_bytes": 0})


def test_brickwork_50q_depth_8_fits():
    gates = C.ry_rz_cnot_brickwork(50, 8)
    tree = NP.greedy_tree(50, gates)
    assert tree["peak_bytes"] <= 1 << 30
    assert N.measured_peak(50, gates, tree) == ON.measured_peak(50, gates, onodes(tree)) == tree["peak_bytes"]


def c_outcome(n, gates, tree):
    try:
        return ("ok", N.measured_peak(n, gates, tree))
    except WqcCudaError as e:
        return ("err", str(e).split("] ", 1)[1])


def o_outcome(n, gates, tree):
    try:
        return ("ok", ON.measured_peak(n, gates, onodes(tree)))
    except ON.NetworkError as e:
        return ("err", str(e))


def test_c_walk_matches_the_oracle_on_planned_and_mutated_trees():
    rng = np.random.default_rng(99)
    checked = errors = 0
    names = ["ket0", "gate", "node", "bra0", "control", "target"]
    for trial in range(120):
        n = int(rng.integers(2, 7))
        gates = lcg_circuit(n, int(rng.integers(1, 16)), int(rng.integers(0, 1 << 30)))
        base = NP.greedy_split_tree(n, gates) if trial % 2 else NP.greedy_tree(n, gates)
        cases = [base]
        for _ in range(4):
            nodes = json.loads(json.dumps(base["nodes"]))
            i = int(rng.integers(0, len(nodes)))
            k = int(rng.integers(0, 4))
            if k == 0 and len(nodes) > 1:
                j = int(rng.integers(0, len(nodes)))
                nodes[i], nodes[j] = nodes[j], nodes[i]
            elif k == 1:
                side = "left" if rng.random() < 0.5 else "right"
                nodes[i][side] = {str(rng.choice(names)): int(rng.integers(0, max(n, len(gates), len(nodes))))}
            elif k == 2:
                del nodes[i]
            else:
                nodes.insert(i, nodes[i])
            cases.append({"kind": "network", "nodes": nodes})
        for t in cases:
            c, o = c_outcome(n, gates, t), o_outcome(n, gates, t)
            assert c == o, (trial, t, c, o)
            checked += 1
            errors += c[0] == "err"
    assert errors > 100 and checked - errors > 100
