"""Exact contraction trees, host side (no GPU).

* The oracle (oracle/exact.py) against the known answers of the reference's
  own tests: src/tn/exact.rs:726-916 and src/tn/plan.rs:274-519.
* The planner (wqc_cuda.exact_plan) against plan.rs's expected trees, JSON
  text and peaks.
* The C ABI's host walk (wqc_exact_validate, wqc_exact_measured_peak)
  against the oracle on planned and on mutated trees: the same peak, or the
  same failure with the same message.
"""
import json

import numpy as np
import pytest

import dense as D
import exact as OX
from wqc_cuda import ERR_INVALID, ERR_INVALID_QUBIT_COUNT, ERR_QUBIT_OUT_OF_RANGE, WqcCudaError
from wqc_cuda import circuits as C
from wqc_cuda import exact as X
from wqc_cuda import exact_plan as P

KIND = {"ket0": OX.KET0, "gate": OX.GATE, "node": OX.NODE}


def oracle_nodes(tree):
    out = []
    for node in tree["nodes"]:
        (lk, li), = node["left"].items()
        (rk, ri), = node["right"].items()
        out.append(((KIND[lk], li), (KIND[rk], ri)))
    return out


def node(left, right):
    return {"op": "contract", "left": left, "right": right}


def star_tree(n):
    """exact.rs:678-703, unmeasured."""
    nodes = [node({"ket0": 0}, {"gate": 0})]
    for q in range(1, n):
        nodes.append(node({"node": len(nodes) - 1}, {"ket0": q}))
        nodes.append(node({"node": len(nodes) - 1}, {"gate": q}))
    return {"nodes": nodes}


def star_peak(n):
    return 32 if n <= 1 else (16 << (n - 1)) + (16 << 1) + (16 << n)


def dense(n, gates):
    d = D.Dense(n)
    d.apply_gates(gates)
    return d.state


def measured(n, gates, tree):
    t = dict(tree)
    t["peak_bytes"] = OX.measured_peak(n, gates, oracle_nodes(tree))
    return t


def oracle_amp(n, gates, tree, bits=0):
    return OX.contract(n, gates, oracle_nodes(tree), tree.get("peak_bytes"), bits)[1]


# --- the oracle against exact.rs's tests ------------------------------------

def test_oracle_star_16_leaf_ones():
    n = 16
    gates = C.star(n)
    tree = measured(n, gates, star_tree(n))
    assert tree["peak_bytes"] == star_peak(n)
    d = dense(n, gates)
    ones = (1 << n) - 1
    assert abs(d[ones]) > 0.1
    assert abs(oracle_amp(n, gates, tree, ones) - d[ones]) < 1e-8
    assert abs(oracle_amp(n, gates, tree, 0) - d[0]) < 1e-8


def test_oracle_ccnot_and_cz():
    n = 4
    gates = C.gates_array([C.g1(C.X, 0), C.g1(C.X, 1), C.g3(0, 1, 2), C.g1(C.X, 3), C.g2(C.CZ, 2, 3)])
    nodes = [node({"ket0": 0}, {"ket0": 1}), node({"node": 0}, {"ket0": 2}), node({"node": 1}, {"ket0": 3})]
    for g in range(len(gates)):
        nodes.append(node({"node": len(nodes) - 1}, {"gate": g}))
    tree = measured(n, gates, {"nodes": nodes})
    assert tree["peak_bytes"] == (16 << 3) + (16 << 1) + (16 << 4)
    d = dense(n, gates)
    assert abs(d[0b1111]) > 0.5
    assert abs(oracle_amp(n, gates, tree, 0b1111) - d[0b1111]) < 1e-8


def test_oracle_rejections():
    gates = C.gates_array([C.g1(C.H, 0), C.g1(C.X, 0)])
    with pytest.raises(OX.ExactError, match="circuit order"):
        OX.contract(1, gates, [((OX.KET0, 0), (OX.GATE, 1))], 0)
    g3 = C.star(3)
    nodes = oracle_nodes(star_tree(3))
    with pytest.raises(OX.ExactError, match="exceeds 1 GiB"):
        OX.contract(3, g3, nodes, OX.MAX_PEAK_BYTES + 1)
    with pytest.raises(OX.ExactError, match="does not match"):
        OX.contract(3, g3, nodes, 1)
    with pytest.raises(OX.ExactError, match="exceeds 1 GiB"):
        OX.measured_peak(26, C.star(26), oracle_nodes(star_tree(26)))
    with pytest.raises(OX.ExactError, match="exceeds 26 legs"):
        OX.contract(27, C.gates_array([]), oracle_nodes(join_past_26_legs()), 0)


def test_oracle_untouched_wire_stays_ket0():
    gates = C.gates_array([C.g1(C.H, 0)])
    tree = measured(3, gates, {"nodes": [node({"ket0": 0}, {"gate": 0})]})
    assert abs(oracle_amp(3, gates, tree, 0) - dense(3, gates)[0]) < 1e-8
    assert oracle_amp(3, gates, tree, 0b100) == 0


def join_wires(wires, nodes):
    acc = {"ket0": wires[0]}
    for w in wires[1:]:
        nodes.append(node(acc, {"ket0": w}))
        acc = {"node": len(nodes) - 1}
    return acc


def join_past_26_legs():
    """exact.rs:944-967: 14 and 13 wires, a 27-leg product."""
    nodes = []
    left = join_wires(list(range(0, 14)), nodes)
    right = join_wires(list(range(14, 27)), nodes)
    nodes.append(node(left, right))
    return {"nodes": nodes, "peak_bytes": 0}


# --- the planner against plan.rs's tests -------------------------------------

CHAIN_JSON = ('{"nodes":[{"op":"contract","left":{"ket0":0},"right":{"gate":0}},{"op":"contract","left":{"node":0},'
              '"right":{"ket0":1}},{"op":"contract","left":{"node":1},"right":{"gate":1}},{"op":"contract","left":'
              '{"node":2},"right":{"ket0":2}},{"op":"contract","left":{"node":3},"right":{"gate":2}}],"peak_bytes":224}')


def test_plan_chain_json_and_amplitudes():
    gates = C.gates_array([C.g1(C.H, 0), C.g2(C.CNOT, 0, 1), C.g2(C.CNOT, 1, 2)])
    tree = P.plan_greedy(3, gates)
    assert P.tree_json(tree) == CHAIN_JSON
    d = dense(3, gates)
    for bits in (0, 0b101, 0b111):
        assert abs(oracle_amp(3, gates, tree, bits) - d[bits]) < 1e-8


def test_plan_younger_gate_wins_and_ccnot():
    gates = C.gates_array([C.g1(C.H, 5), C.g1(C.H, 0), C.g1(C.H, 1), C.g3(5, 0, 1)])
    tree = P.plan_greedy(6, gates)
    assert tree["nodes"] == [
        node({"ket0": 5}, {"gate": 0}), node({"ket0": 0}, {"gate": 1}), node({"ket0": 1}, {"gate": 2}),
        node({"node": 1}, {"node": 0}), node({"node": 3}, {"node": 2}), node({"node": 4}, {"gate": 3}),
    ]
    bits = (1 << 5) | 1 | 2
    assert abs(oracle_amp(6, gates, tree, bits) - dense(6, gates)[bits]) < 1e-8


def interior_gates(cc):
    return C.gates_array([C.g2(C.CNOT, 0, 5), C.g2(C.CNOT, 1, 2), C.g2(C.CNOT, 3, 4), C.g3(*cc)])


def test_plan_interior_pair_follows_the_gate_arguments():
    early, late, first = (P.plan_greedy(6, interior_gates(c)) for c in ((0, 1, 3), (0, 3, 1), (1, 3, 0)))
    assert len(early["nodes"]) == 9
    assert early["nodes"][6] == node({"node": 1}, {"node": 3})
    assert late["nodes"][6] == node({"node": 1}, {"node": 5})
    assert early["nodes"][6] == first["nodes"][6]
    assert early["peak_bytes"] == 1344 == late["peak_bytes"]
    ea = oracle_amp(6, interior_gates((0, 1, 3)), early)
    la = oracle_amp(6, interior_gates((0, 3, 1)), late)
    assert abs(ea - la) < 1e-8 and abs(ea - dense(6, interior_gates((0, 1, 3)))[0]) < 1e-8


def test_plan_measure_keeps_the_following_gate_index():
    gates = C.gates_array([C.g1(C.H, 0), (C.MEASURE, 0, 0, 0, 0.0), C.g2(C.CNOT, 0, 1)])
    tree = P.plan_greedy(2, gates)
    seen = [nd["right"]["gate"] for nd in tree["nodes"] if "gate" in nd["right"]]
    assert seen == [0, 2] and tree["peak_bytes"] == 128
    assert abs(oracle_amp(2, gates, tree) - dense(2, gates)[0]) < 1e-8


def test_plan_brickwork_16_depth_8():
    gates = C.ry_cnot_brickwork(16, 8)
    tree = P.plan_greedy(16, gates)
    assert tree["peak_bytes"] == (16 << 14) + (16 << 2) + (16 << 16)
    d = dense(16, gates)
    assert abs(d[0]) > 1e-3
    for bits in (0, 0b1010_1010_1010_1010):
        assert abs(oracle_amp(16, gates, tree, bits) - d[bits]) < 1e-8
    assert P.plan_greedy(50, C.ry_cnot_brickwork(50, 8)) is None


def test_plan_stars_and_caps():
    tree = P.plan_greedy(16, C.star(16))
    assert tree["peak_bytes"] == star_peak(16)
    ones = (1 << 16) - 1
    assert abs(oracle_amp(16, C.star(16), tree, ones) - dense(16, C.star(16))[ones]) < 1e-8
    assert P.plan_greedy(25, C.star(25))["peak_bytes"] == star_peak(25)
    assert P.plan_greedy(26, C.star(26)) is None
    assert P.plan_greedy(40, C.star(40)) is None
    assert P.plan_greedy(P.MAX_QUBITS + 1, C.gates_array([C.g1(C.H, 0)])) is None
    many = np.zeros(P.MAX_GATES + 1, dtype=C.GATE_DTYPE)  # H(0) records
    assert P.plan_greedy(1, many) is None
    assert len(P.plan_greedy(1, many[:P.MAX_GATES])["nodes"]) == P.MAX_GATES
    assert P.plan_greedy(2, C.gates_array([C.g2(C.CNOT, 0, 0)])) is None
    assert P.plan_greedy(3, C.gates_array([C.g1(C.H, 3)])) is None


def test_plan_local_gates_on_50_qubits():
    gates = C.gates_array([C.g1(C.H, q) for q in range(50)])
    tree = P.plan_greedy(50, gates)
    assert tree["peak_bytes"] == 50 * 32 and len(tree["nodes"]) == 50
    assert abs(oracle_amp(50, gates, tree) - 2.0 ** -25) < 1e-8


# --- the C ABI's host walk against the oracle ----------------------------------

def c_outcome(n, gates, tree):
    try:
        return ("ok", X.measured_peak(n, gates, tree))
    except WqcCudaError as e:
        return ("err", str(e).split("] ", 1)[1])


def o_outcome(n, gates, tree):
    try:
        return ("ok", OX.measured_peak(n, gates, oracle_nodes(tree)))
    except OX.ExactError as e:
        return ("err", str(e))


def random_circuit(rng, n, count):
    out = []
    for _ in range(count):
        r = rng.random()
        if r < 0.5:
            out.append(C.g1(int(rng.integers(0, 9)), int(rng.integers(0, n)), float(rng.normal())))
        elif r < 0.9 or n < 3:
            a, b = rng.choice(n, 2, replace=False)
            out.append(C.g2(int(rng.choice([C.CNOT, C.CZ])), int(a), int(b)))
        else:
            a, b, c = rng.choice(n, 3, replace=False)
            out.append(C.g3(int(a), int(b), int(c)))
    return C.gates_array(out)


def mutate(rng, tree, n, gate_count):
    nodes = json.loads(json.dumps(tree["nodes"]))
    k = int(rng.integers(0, 5))
    i = int(rng.integers(0, len(nodes)))
    if k == 0 and len(nodes) > 1:
        j = int(rng.integers(0, len(nodes)))
        nodes[i], nodes[j] = nodes[j], nodes[i]
    elif k == 1:
        side = "left" if rng.random() < 0.5 else "right"
        (name, idx), = nodes[i][side].items()
        nodes[i][side] = {name: max(0, idx + int(rng.choice([-1, 1])))}
    elif k == 2:
        side = "left" if rng.random() < 0.5 else "right"
        name = str(rng.choice(["ket0", "gate", "node"]))
        nodes[i][side] = {name: int(rng.integers(0, max(n, gate_count, len(nodes))))}
    elif k == 3:
        del nodes[i]
    else:
        nodes.insert(i, nodes[i])
    return {"nodes": nodes}


def test_c_walk_matches_the_oracle_on_planned_and_mutated_trees():
    rng = np.random.default_rng(20261204)
    checked = errors = 0
    for trial in range(150):
        n = int(rng.integers(2, 8))
        gates = random_circuit(rng, n, int(rng.integers(1, 14)))
        tree = P.plan_greedy(n, gates)
        assert tree is not None
        cases = [tree] + [mutate(rng, tree, n, len(gates)) for _ in range(4)]
        for t in cases:
            c, o = c_outcome(n, gates, t), o_outcome(n, gates, t)
            assert c == o, (trial, t, c, o)
            checked += 1
            errors += c[0] == "err"
    assert errors > 100 and checked - errors > 150  # both branches exercised


def test_c_walk_known_peaks():
    for n in (1, 2, 3, 10, 16, 25):
        assert X.measured_peak(n, C.star(n), star_tree(n)) == star_peak(n)
    gates = C.ry_cnot_brickwork(16, 8)
    assert X.measured_peak(16, gates, P.plan_greedy(16, gates)) == (16 << 14) + (16 << 2) + (16 << 16)
    gates = C.ry_cnot_brickwork(25, 4)
    tree = P.plan_greedy(25, gates)
    assert X.measured_peak(25, gates, tree) == tree["peak_bytes"] == OX.measured_peak(25, gates, oracle_nodes(tree))


def err_of(fn, *a, **k):
    with pytest.raises(WqcCudaError) as e:
        fn(*a, **k)
    return e.value.code, str(e.value).split("] ", 1)[1]


def test_c_validate_rejections():
    g3 = C.star(3)
    t = measured(3, g3, star_tree(3))
    X.validate(3, g3, t)
    assert err_of(X.validate, 3, g3, dict(t, peak_bytes=None)) == (ERR_INVALID, "exact contraction tree requires a peak")
    assert err_of(X.validate, 3, g3, dict(t, peak_bytes=(1 << 30) + 1))[1] == "contraction tree peak exceeds 1 GiB"
    g2 = C.star(2)
    t2 = measured(2, g2, star_tree(2))
    assert "parent wire" in err_of(X.validate, 2, g2, dict(t2, site_order=[1, 0]))[1]
    X.validate(2, g2, dict(t2, site_order=[0, 1]))  # the identity is no order
    assert err_of(X.validate, 2, g2, t2, mps_site_order=[1, 0])[1] == "mps_site_order does not match the contraction tree"
    X.validate(2, g2, t2, mps_site_order=[])
    assert err_of(X.validate, 2, g2, t2, mps_site_order=[0])[1] == "mps_site_order length 1 != qubit_count 2"
    code, msg = err_of(X.validate, 2, g2, t2, mps_site_order=[0, 0])
    assert msg == "mps_site_order is not a permutation (duplicate logical 0)"
    assert err_of(X.validate, 2, g2, t2, mps_site_order=[0, 5])[0] == ERR_QUBIT_OUT_OF_RANGE
    assert err_of(X.validate, 0, C.gates_array([]), {"nodes": [], "peak_bytes": 0})[0] == ERR_INVALID_QUBIT_COUNT
    assert err_of(X.validate, 1, C.gates_array([C.g1(C.H, 3)]), {"nodes": [], "peak_bytes": 0})[0] == \
        ERR_QUBIT_OUT_OF_RANGE


def test_c_walk_rejections():
    assert err_of(X.measured_peak, 26, C.star(26), star_tree(26))[1] == "contraction tree peak exceeds 1 GiB"
    assert err_of(X.measured_peak, 27, C.gates_array([]), join_past_26_legs())[1] == \
        "contraction tree tensor exceeds 26 legs"
    gates = C.gates_array([C.g1(C.H, 0), C.g1(C.X, 0)])
    code, msg = err_of(X.measured_peak, 1, gates, {"nodes": [node({"ket0": 0}, {"gate": 1})]})
    assert msg == "gates are out of circuit order" and X.is_contraction_client_error(code, msg)
    for ref, text in (({"left": 0}, "exact contraction has no split"), ({"right": 0}, "exact contraction has no split"),
                      ({"bra0": 0}, "exact contraction has no bra0"),
                      ({"control": 0}, "exact contraction has no gate halves"),
                      ({"target": 0}, "exact contraction has no gate halves")):
        assert err_of(X.measured_peak, 1, gates, {"nodes": [node({"ket0": 0}, ref)]})[1] == text
    sweep = {"nodes": [{"op": "site", "tensor": {"ket0": 0}, "gate": 0}]}
    assert err_of(X.measured_peak, 1, gates, sweep)[1] == "contraction tree mixes sweep steps and exact contractions"
    two = C.gates_array([C.g2(C.CNOT, 0, 1)])
    assert err_of(X.measured_peak, 2, two, {"nodes": [node({"ket0": 0}, {"gate": 0})]})[1] == "gate wires are not open"
    assert err_of(X.measured_peak, 2, two, {"nodes": []})[1] == "gate was not contracted"
    assert err_of(X.measured_peak, 2, two, {"nodes": [node({"ket0": 0}, {"ket0": 0})]})[1] == \
        "contraction tree tensor is not ready"
    assert err_of(X.measured_peak, 2, two, {"nodes": [node({"ket0": 3}, {"ket0": 0})]}) == \
        (ERR_QUBIT_OUT_OF_RANGE, "Qubit index 3 out of bounds (limit: 2)")
    assert not X.is_contraction_client_error(ERR_INVALID, "mps bond exceeded chi")


def test_oracle_c_kernels_match_the_numpy_restatement():
    rng = np.random.default_rng(3)
    for legs in (1, 2, 3, 5, 9):
        wires = sorted(int(w) for w in rng.choice(40, legs, replace=False))
        for kind in range(12):
            if (kind in (C.CNOT, C.CZ) and legs < 2) or (kind == C.CCNOT and legs < 3):
                continue
            q = [wires[int(i)] for i in rng.choice(legs, 3 if legs >= 3 else legs, replace=False)]
            g = C.gates_array([(kind, q[0], q[1] if legs > 1 else 0, q[2] if legs > 2 else 0, float(rng.normal()))])[0]
            data = rng.normal(size=1 << legs) + 1j * rng.normal(size=1 << legs)
            a = OX.apply_in_place(data.copy(), wires, g)
            b = OX.apply_in_place_numpy(data.copy(), wires, g)
            assert np.max(np.abs(a - b)) <= 4e-16 * np.max(np.abs(data)), (legs, kind)
        lw = sorted(int(w) for w in rng.choice(20, 3, replace=False))
        rw = sorted(int(w) for w in set(range(20, 20 + legs)))
        ld = rng.normal(size=8) + 1j * rng.normal(size=8)
        rd = rng.normal(size=1 << legs) + 1j * rng.normal(size=1 << legs)
        wa, a = OX.outer(lw, ld, rw, rd)
        wb, b = OX.outer_numpy(lw, ld, rw, rd)
        assert wa == wb and np.max(np.abs(a - b)) <= 1e-15 * np.max(np.abs(a))
