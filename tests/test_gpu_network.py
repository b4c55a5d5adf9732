"""Network contraction trees on the device (wqc_network_contract) against the
oracle (oracle/network.py, the reference's walk restated), the dense
statevector, the reference's own trees, and the two other device paths.

Tolerances: the device contracts with cuBLAS ZGEMM, the oracle with numpy's
matmul; both sum in their own order, so amplitudes agree to rounding:
1e-12 absolute against the oracle, and the reference's own 1e-9 against
the dense statevector (network.rs:982-984).
"""
import json

import numpy as np
import pytest

from wqc_cuda import ERR_CANCELLED, ERR_INVALID, WqcCudaError
from wqc_cuda import circuits as C
from wqc_cuda import exact as XE
from wqc_cuda import exact_plan as EP
from wqc_cuda import network as N
from wqc_cuda import network_plan as NP

from test_network_host import (FIXTURE_JSON, GRIDS, dense_zero, fixture_gates, ghz_far, lcg_circuit, load_grid, node, oracle_amp,
                               random_tree_of)

pytestmark = pytest.mark.gpu
ORACLE_TOL = 1e-12
DENSE_TOL = 1e-9


@pytest.fixture(scope="module")
def net(cuda_ctx):
    e = N.NetworkContractor(cuda_ctx)
    yield e
    e.close()


def check(net, n, gates, tree, expected=None):
    got = net.contract(n, gates, tree)
    assert abs(got - oracle_amp(n, gates, tree)) < ORACLE_TOL
    if expected is None:
        expected = dense_zero(n, gates)
    assert abs(got - expected) < DENSE_TOL
    return got


def test_any_order_and_greedy(net):
    for n, gates in ghz_far():
        expected = dense_zero(n, gates)
        for seed in range(8):
            check(net, n, gates, random_tree_of(n, gates, NP.leaves(n, gates), seed), expected)
            check(net, n, gates, random_tree_of(n, gates, NP.split_leaves(n, gates), seed), expected)
        check(net, n, gates, NP.greedy_tree(n, gates), expected)
        check(net, n, gates, NP.greedy_split_tree(n, gates), expected)


def test_orchestrator_trees(net):
    gates = fixture_gates()
    check(net, 4, gates, json.loads(FIXTURE_JSON))
    grid = C.grid(4, 12)
    expected = dense_zero(16, grid)
    for name in GRIDS:
        tree = json.loads(load_grid(name))
        check(net, 16, grid, tree, expected)
        st = net.stats()
        assert st["gemms"] + st["small"] == len(tree["nodes"]) and st["launches"] >= st["gemms"]


def test_skipped_ops_outer_products_and_reordered_copies(net):
    gates = C.gates_array([C.g1(C.H, 0), (C.MEASURE, 0, 0, 0, 0.0), (C.IF, 1, 0, 0, 0.0), C.g2(C.CNOT, 0, 2)])
    check(net, 4, gates, NP.greedy_tree(4, gates))
    one = {"kind": "network", "nodes": [node({"ket0": 0}, {"bra0": 0})], "peak_bytes": 80}
    assert net.contract(1, C.gates_array([]), one) == 1
    ry = C.gates_array([C.g1(C.RY, 0, 0.3), C.g1(C.RY, 1, 0.5)])
    check(net, 2, ry, NP.finish(2, ry, [node({"ket0": 0}, {"gate": 0}), node({"node": 0}, {"ket0": 1}),
                                        node({"node": 1}, {"gate": 1}), node({"node": 2}, {"bra0": 0}),
                                        node({"node": 3}, {"bra0": 1})]))
    cnot = C.gates_array([C.g2(C.CNOT, 0, 1)])
    t = NP.finish(2, cnot, [node({"gate": 0}, {"ket0": 1}), node({"node": 0}, {"ket0": 0}),
                            node({"node": 1}, {"bra0": 0}), node({"node": 2}, {"bra0": 1})])
    assert t["peak_bytes"] == 544 and abs(net.contract(2, cnot, t) - 1) < 1e-15


def test_split_gates(net):
    circuits = [(5, C.ry_rz_cnot_brickwork(5, 4)), (4, C.grid(2, 6))] + [(6, lcg_circuit(6, 40, s)) for s in range(6)]
    for n, gates in circuits:
        expected = dense_zero(n, gates)
        for seed in range(4):
            check(net, n, gates, random_tree_of(n, gates, NP.split_leaves(n, gates), seed), expected)
        check(net, n, gates, NP.greedy_split_tree(n, gates), expected)


def test_far_20q_matches_dense_and_the_exact_tree(net, cuda_ctx):
    n = 20
    gates = list(C.ry_rz_cnot_brickwork(n, 3))
    gates += list(C.gates_array([C.g2(C.CNOT, 0, 19), C.g3(3, 11, 17), C.g2(C.CZ, 14, 5), C.g1(C.RX, 19, 0.23),
                                 C.g2(C.CNOT, 17, 2)]))
    gates += [g for g in lcg_circuit(n, 30, 7) if int(g["kind"]) not in (C.X, C.Y, C.CCNOT)]
    gates = C.gates_array([(int(g["kind"]), int(g["q0"]), int(g["q1"]), int(g["q2"]), float(g["angle"]))
                           for g in gates])
    tree = NP.greedy_tree(n, gates)
    got = check(net, n, gates, tree)
    ex = XE.ExactContractor(cuda_ctx)
    state = ex.contract(n, gates, EP.plan_greedy(n, gates), 0)
    ex.close()
    assert abs(got - state) < DENSE_TOL


def test_brickwork_50q_depth_8_matches_the_mps(net, cuda_ctx):
    """network.rs:1758-1782: the network amplitude against the MPS at an
    exact bond (chi 256 holds the 50-qubit depth-8 brickwork exactly)."""
    import wqc_cuda as W

    n = 50
    gates = C.ry_rz_cnot_brickwork(n, 8)
    tree = NP.greedy_tree(n, gates)
    got = net.contract(n, gates, tree)
    assert abs(got - oracle_amp(n, gates, tree)) < ORACLE_TOL
    m = W.CudaMps(n, 256, ctx=cuda_ctx)
    m.apply_gates(gates)
    assert abs(got - m.amplitude_at_compact_zero()) < DENSE_TOL
    m.close()


def test_grid_5x5_depth_12_against_the_oracle(net):
    """A GEMM-heavy tree: 25 qubits, 769 nodes, 290 GFLOP, peak 554 MB."""
    n = 25
    gates = C.grid(5, 12)
    tree = NP.greedy_tree(n, gates)
    got = net.contract(n, gates, tree)
    ref = oracle_amp(n, gates, tree)
    assert abs(got - ref) < ORACLE_TOL, (got, ref)
    st = net.stats()
    assert st["gemm_flops"] > 2e11 and st["gemm_ms"] > 0
    assert st["small"] > 700 and st["launches"] < 200  # the small joins run level-batched


def test_failures_come_before_device_work_and_cancel(net):
    n = 3
    gates = C.gates_array([C.g1(C.H, 0), C.g2(C.CNOT, 0, 1), C.g3(0, 1, 2)])
    good = NP.greedy_tree(n, gates)
    for tree, needle in ((dict(good, peak_bytes=good["peak_bytes"] + 16), "does not match"),
                         (dict(good, peak_bytes=None), "requires a peak"),
                         (dict(good, nodes=good["nodes"][:-1]), "one scalar"),
                         (dict(good, kind=None), "is not a network")):
        with pytest.raises(WqcCudaError, match=needle) as e:
            net.contract(n, gates, tree)
        assert e.value.code == ERR_INVALID
    net.cancel()
    with pytest.raises(WqcCudaError) as e:
        net.contract(n, gates, good)
    assert e.value.code == ERR_CANCELLED
    check(net, n, gates, good)
    assert abs(N.contract_network(n, gates, good) - dense_zero(n, gates)) < DENSE_TOL
