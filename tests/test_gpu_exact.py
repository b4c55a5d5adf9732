"""Exact contraction trees on the device (wqc_exact_contract) against the
oracle (oracle/exact.py, the reference's walk restated), the dense
statevector, and the known answers of src/tn/exact.rs and src/tn/plan.rs.

Tolerances: the device computes every amplitude with the reference's
operations in the reference's order (complex products and sums without
fused multiply-adds), as the oracle's C loops do, so against the oracle the
amplitudes must be equal (tolerance 0).  Against the dense statevector
(another operation order) 1e-11 absolute on a normalised state.  At 25
qubits, where the oracle takes too long, a circuit followed by its inverse
must return |0...0> to 1e-11.
"""
import numpy as np
import pytest

import dense as D
import exact as OX
from wqc_cuda import ERR_CANCELLED, ERR_INVALID, WqcCudaError
from wqc_cuda import circuits as C
from wqc_cuda import exact as X
from wqc_cuda import exact_plan as P

from test_exact_host import (join_past_26_legs, measured, node, oracle_amp, oracle_nodes, random_circuit,
                             star_peak, star_tree)

pytestmark = pytest.mark.gpu
ORACLE_TOL = 0.0
DENSE_TOL = 1e-11


@pytest.fixture(scope="module")
def ex(cuda_ctx):
    e = X.ExactContractor(cuda_ctx)
    yield e
    e.close()


def dense(n, gates):
    d = D.Dense(n)
    d.apply_gates(gates)
    return d.state


def test_star_16_leaf_ones(ex):
    n = 16
    gates = C.star(n)
    tree = measured(n, gates, star_tree(n))
    ones = (1 << n) - 1
    got = ex.contract(n, gates, tree, [0, ones, 5])
    d = dense(n, gates)
    assert np.max(np.abs(got - d[[0, ones, 5]])) < 1e-12
    st = ex.stats()
    assert st["gates"] == n and st["outer_products"] == n - 1 and st["launches"] >= st["passes"] + st["outer_products"]


def test_ccnot_cz_and_untouched_wire(ex):
    gates = C.gates_array([C.g1(C.X, 0), C.g1(C.X, 1), C.g3(0, 1, 2), C.g1(C.X, 3), C.g2(C.CZ, 2, 3)])
    nodes = [node({"ket0": 0}, {"ket0": 1}), node({"node": 0}, {"ket0": 2}), node({"node": 1}, {"ket0": 3})]
    for g in range(len(gates)):
        nodes.append(node({"node": len(nodes) - 1}, {"gate": g}))
    tree = measured(4, gates, {"nodes": nodes})
    assert abs(ex.contract(4, gates, tree, 0b1111, mps_site_order=[]) - dense(4, gates)[0b1111]) < 1e-15
    h = C.gates_array([C.g1(C.H, 0)])
    t = measured(3, h, {"nodes": [node({"ket0": 0}, {"gate": 0})]})
    amps = ex.contract(3, h, t, [0, 1, 0b100, 0b101])
    assert np.allclose(amps, [2 ** -0.5, 2 ** -0.5, 0, 0], atol=1e-15, rtol=0)


def test_plan_rs_known_answers(ex):
    cases = [
        (3, C.gates_array([C.g1(C.H, 0), C.g2(C.CNOT, 0, 1), C.g2(C.CNOT, 1, 2)]), [0, 0b101, 0b111]),
        (6, C.gates_array([C.g1(C.H, 5), C.g1(C.H, 0), C.g1(C.H, 1), C.g3(5, 0, 1)]), [(1 << 5) | 3, 0, 63]),
        (6, C.gates_array([C.g2(C.CNOT, 0, 5), C.g2(C.CNOT, 1, 2), C.g2(C.CNOT, 3, 4), C.g3(0, 3, 1)]), [0, 1, 33]),
        (2, C.gates_array([C.g1(C.H, 0), (C.MEASURE, 0, 0, 0, 0.0), C.g2(C.CNOT, 0, 1)]), [0, 3]),
        (16, C.ry_cnot_brickwork(16, 8), [0, 0b1010_1010_1010_1010, 12345]),
        (16, C.star(16), [0, (1 << 16) - 1]),
    ]
    for n, gates, bits in cases:
        tree = P.plan_greedy(n, gates)
        got = ex.contract(n, gates, tree, bits)
        d = dense(n, gates)
        assert np.max(np.abs(got - d[bits])) < DENSE_TOL, (n, bits)
        for b, a in zip(bits, got):
            assert abs(a - oracle_amp(n, gates, tree, b)) <= ORACLE_TOL, (n, b)
    gates = C.gates_array([C.g1(C.H, q) for q in range(50)])
    assert abs(ex.contract(50, gates, P.plan_greedy(50, gates)) - 2.0 ** -25) < 1e-15


def test_random_circuits_against_the_oracle(ex):
    rng = np.random.default_rng(7)
    worst = 0.0
    for trial in range(40):
        n = int(rng.integers(2, 13))
        gates = random_circuit(rng, n, int(rng.integers(1, 60)))
        tree = P.plan_greedy(n, gates)
        bits = [int(b) for b in rng.integers(0, 1 << n, size=4)]
        got = ex.contract(n, gates, tree, bits)
        for b, a in zip(bits, got):
            worst = max(worst, abs(a - oracle_amp(n, gates, tree, b)))
        full = ex.contract(n, gates, tree, np.arange(1 << n))
        assert np.max(np.abs(full - dense(n, gates))) < DENSE_TOL, trial
    assert worst <= ORACLE_TOL, worst


def test_wide_pass_trees_against_dense(ex):
    """Tensors past 12 legs: several passes per gate queue, blocks of 4096
    amplitudes gathered from scattered positions."""
    for n, depth in ((18, 6), (20, 5)):
        gates = C.ry_cnot_brickwork(n, depth)
        extra = C.gates_array([C.g3(0, n - 1, n // 2), C.g2(C.CZ, n - 1, 1), C.g1(C.T, n - 2), C.g2(C.CNOT, 13, 2)])
        gates = np.concatenate([gates, extra])
        tree = P.plan_greedy(n, gates)
        rng = np.random.default_rng(n)
        bits = rng.integers(0, 1 << n, size=2048)
        got = ex.contract(n, gates, tree, bits)
        d = dense(n, gates)
        assert np.max(np.abs(got - d[bits])) < DENSE_TOL
        assert ex.stats()["passes"] > 1
    # one amplitude against the oracle's own walk (same operation order)
    n, gates = 18, C.ry_cnot_brickwork(18, 6)
    tree = P.plan_greedy(n, gates)
    assert abs(ex.contract(n, gates, tree, 77) - oracle_amp(n, gates, tree, 77)) <= ORACLE_TOL


@pytest.mark.parametrize("tile", [12, 13])
def test_register_tiles_every_gate_kind(cuda_ctx, tile):
    """States past the tile size with every gate kind: targets on lane,
    register and warp bits (exchanges), controls and diagonal bits inside and
    outside the tile, exact gates moved past others; equal to the oracle."""
    ex = X.ExactContractor(cuda_ctx)
    ex.set_tile_bits(tile)
    rng = np.random.default_rng(tile)
    for n in (tile, 15, 17):
        gates = random_circuit(rng, n, 320)
        tree = P.plan_greedy(n, gates)
        bits = rng.integers(0, 1 << n, size=256)
        got = ex.contract(n, gates, tree, bits)
        st = ex.stats()
        assert st["exchanges"] > 0 and st["gates"] == len(gates)
        assert np.max(np.abs(got - dense(n, gates)[bits])) < DENSE_TOL, n
        for b, a in zip(bits[:3], got[:3]):
            assert a == oracle_amp(n, gates, tree, int(b)), (n, int(b))
    with pytest.raises(WqcCudaError, match="12 or 13"):
        ex.set_tile_bits(11)
    ex.close()


def inverse(gates):
    inv = gates[::-1].copy()
    for g in inv:
        if int(g["kind"]) in (C.RX, C.RY, C.RZ):
            g["angle"] = -g["angle"]
    return inv


def test_brickwork_25_equals_the_oracle_at_full_width(ex):
    """The widest state the 1 GiB peak admits, against the oracle's own walk
    (its C loops take ~10 s on the 2^25-amplitude state): equal amplitudes."""
    n = 25
    gates = C.ry_cnot_brickwork(n, 3)
    tree = P.plan_greedy(n, gates)
    bits = 0b1011001110001111000011111
    got = ex.contract(n, gates, tree, bits)
    assert ex.stats()["pass_bytes"] > 0  # passes over the full 25-leg state ran
    assert got == oracle_amp(n, gates, tree, bits)


def test_brickwork_25_then_inverse_returns_zero(ex):
    n = 25
    fwd = C.ry_cnot_brickwork(n, 12)
    gates = np.concatenate([fwd, inverse(fwd)])
    tree = P.plan_greedy(n, gates)
    assert tree["peak_bytes"] <= 1 << 30
    amps = ex.contract(n, gates, tree, [0, 1, (1 << n) - 1, 123456])
    assert abs(amps[0] - 1.0) < DENSE_TOL and np.max(np.abs(amps[1:])) < DENSE_TOL
    st = ex.stats()
    assert st["gates"] == len(gates) and st["pass_bytes"] > 0 and st["pass_ms"] > 0


def test_failures_come_before_device_work(ex):
    g3 = C.star(3)
    t = measured(3, g3, star_tree(3))
    with pytest.raises(WqcCudaError, match="does not match"):
        ex.contract(3, g3, dict(t, peak_bytes=1))
    with pytest.raises(WqcCudaError, match="requires a peak"):
        ex.contract(3, g3, dict(t, peak_bytes=None))
    with pytest.raises(WqcCudaError, match="exceeds 26 legs"):
        ex.contract(27, C.gates_array([]), join_past_26_legs())
    with pytest.raises(WqcCudaError, match="circuit order") as e:
        ex.contract(1, C.gates_array([C.g1(C.H, 0), C.g1(C.X, 0)]), {"nodes": [node({"ket0": 0}, {"gate": 1})],
                                                                     "peak_bytes": 0})
    assert e.value.code == ERR_INVALID and X.is_contraction_client_error(e.value.code, str(e.value).split("] ", 1)[1])
    # the executor still works after the failures
    assert abs(ex.contract(3, g3, t, 7) - 2 ** -0.5) < 1e-15
    assert t["peak_bytes"] == star_peak(3)


def test_cancel_stops_the_next_launch(ex):
    gates = C.ry_cnot_brickwork(12, 4)
    tree = P.plan_greedy(12, gates)
    ex.cancel()
    with pytest.raises(WqcCudaError) as e:
        ex.contract(12, gates, tree, 0)
    assert e.value.code == ERR_CANCELLED
    assert abs(ex.contract(12, gates, tree, 0) - dense(12, gates)[0]) < DENSE_TOL


def test_module_level_calls(cuda_ctx):
    gates = C.star(5)
    tree = P.plan_greedy(5, gates)
    assert abs(X.contract_exact(5, gates, tree) - 2 ** -0.5) < 1e-15
    assert abs(X.contract_exact_at(5, gates, P.tree_json(tree), 31) - 2 ** -0.5) < 1e-15
    assert OX.measured_peak(5, gates, oracle_nodes(tree)) == tree["peak_bytes"]
