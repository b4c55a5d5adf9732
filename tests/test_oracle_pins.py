"""Pins of the FP64 oracle against the reference's own tests and values.

Each test restates a reference unit test (file:line in its docstring) and
checks the oracle against it, so the oracle the GPU parity tests rely on is
itself anchored to the reference.  CPU only.
"""
import hashlib
import math

import numpy as np
import pytest

import dense as D
import oracle as O
from wqc_cuda import circuits as C


def exact_bond_dim(n):  # gates.rs:131-134
    return 1 << (min(n, 20) // 2 + 1)


def max_diff(n, gates, chi=128):  # mps.rs:1906-1918
    m = O.run(n, chi, gates)
    d = D.Dense(n)
    d.apply_gates(gates)
    return np.abs(m.dense() - d.state).max()


def test_h_amplitude():
    """mps.rs:1482-1493."""
    m = O.run(1, exact_bond_dim(1), C.gates_array([C.g1(C.H, 0)]))
    a = m.amplitude_zero()
    assert abs(a.real - 1 / math.sqrt(2)) < 1e-8 and abs(a.imag) < 1e-8


def test_h_ccnot_exact_bond_matches_dense():
    """mps.rs:1495-1513 and contract.rs:37-46."""
    g = C.gates_array([C.g1(C.H, 0), C.g3(0, 1, 2)])
    m = O.run(3, exact_bond_dim(3), g)
    assert abs(m.dense()[0] - 1 / math.sqrt(2)) < 1e-6
    assert abs(m.amplitude_zero().real - 1 / math.sqrt(2)) < 1e-5


def test_nonadjacent_two_qubit_gates_match_dense():
    """mps.rs:1515-1540."""
    g = C.gates_array([C.g1(C.H, 0), C.g1(C.H, 1), C.g2(C.CNOT, 0, 2), C.g2(C.CZ, 3, 1), C.g2(C.CNOT, 2, 0)])
    assert max_diff(4, g, exact_bond_dim(4)) < 1e-8


def random_circuit(rng, n, depth):
    gl = []
    for _ in range(depth):
        k = rng.random()
        q = int(rng.integers(0, n))
        others = [w for w in range(n) if w != q]
        if n >= 3 and k < 0.08:
            c2 = int(rng.choice(others))
            t = int(rng.choice([w for w in others if w != c2]))
            gl.append(C.g3(q, c2, t))
        elif n >= 2 and k < 0.35:
            t = int(rng.choice(others))
            gl.append(C.g2(C.CNOT if rng.random() < 0.5 else C.CZ, q, t))
        elif k < 0.65:
            gl.append(C.g1((C.RX, C.RY, C.RZ)[int(rng.integers(0, 3))], q, rng.uniform(-7, 7)))
        else:
            gl.append(C.g1((C.H, C.X, C.Y, C.Z, C.S, C.T)[int(rng.integers(0, 6))], q))
    return C.gates_array(gl)


def test_random_circuits_match_dense():
    """mps.rs:1920-1972: 300 seeded random circuits on 1-6 qubits with every
    gate type, 1e-9.  The reference draws them with rand's StdRng; the same
    distribution is drawn here with numpy's PCG64 from the same seed value."""
    rng = np.random.default_rng(0x5EED_2026_1128)
    for case in range(300):
        n = int(rng.integers(1, 7))
        g = random_circuit(rng, n, int(rng.integers(1, 25)))
        assert max_diff(n, g) < 1e-9, f"case {case}"


def spread(n, phase):  # mps.rs:1897-1904
    out = []
    for q in range(n):
        out.append(C.g1(C.RY, q, 0.3 + 0.4 * q + phase))
        out.append(C.g1(C.RZ, q, 0.7 - 0.2 * q + phase))
    return out


def test_ccnot_matches_dense_in_every_order():
    """mps.rs:1974-1994."""
    for n in range(3, 6):
        for c1 in range(n):
            for c2 in range(n):
                for t in range(n):
                    if len({c1, c2, t}) < 3:
                        continue
                    g = C.gates_array(spread(n, 0.1) + [C.g3(c1, c2, t)] + spread(n, -0.25))
                    assert max_diff(n, g) < 1e-10


def test_checked_svd_reproduces_the_matrix_nalgebra_got_wrong():
    """mps.rs:1996-2028."""
    m = np.array([[4.1435686496782016e-16, -1.597611177955782e-16j],
                  [-0.35975005528623j, 0.9330487113337411]])
    u, s, vt, _ = O.checked_svd(m)
    assert abs(s[0] - 1.0) < 1e-12
    assert np.abs((u * s) @ vt - m).max() < 1e-12


def test_jacobi_reproduces_tall_wide_and_rank_deficient():
    """mps.rs:2030-2065."""
    def entry(r, c, k):
        t = (r * 7 + c * 3) * 0.37 + k
        return complex(math.sin(t), math.cos(1.3 * t))
    for rows, cols in ((4, 4), (6, 3), (3, 6), (8, 8)):
        full = np.array([[entry(r, c, 0.0) for c in range(cols)] for r in range(rows)])
        rank1 = np.array([[entry(r, 0, 0.2) * entry(0, c, 0.9) for c in range(cols)] for r in range(rows)])
        for m in (full, rank1):
            u, s, vt = O.jacobi_svd(m)
            assert np.all(s[:-1] >= s[1:])
            k = len(s)
            assert np.abs((u[:, :k] * s) @ vt[:k] - m).max() < 1e-12


def test_brickwork_matches_dense():
    """mps.rs:2067-2099 (6q x 6 and 8q x 8, 1e-9)."""
    for n, depth in ((6, 6), (8, 8)):
        g = []
        for layer in range(depth):
            for q in range(n):
                g.append(C.g1(C.RY, q, 0.17 + 0.03 * (q + layer)))
                g.append(C.g1(C.RZ, q, 0.4 - 0.05 * q))
            for q in range(layer % 2, n - 1, 2):
                g.append(C.g2(C.CNOT, q, q + 1))
        assert max_diff(n, C.gates_array(g)) < 1e-9


def test_exact_zero_through_rank_one_split():
    """mps.rs:2101-2113."""
    g = C.gates_array([C.g1(C.X, 0), C.g2(C.CZ, 1, 0), C.g1(C.RX, 1, -0.736), C.g2(C.CZ, 1, 0),
                       C.g2(C.CNOT, 0, 1), C.g2(C.CZ, 1, 0)])
    assert max_diff(2, g) < 1e-12


def test_rsvd_recovers_gapped_rank4():
    """mps.rs:1795-1854: rank-4 32x24 with sigma 8, 4, 2, 1 rebuilds to 1e-6."""
    rows, cols, ell, dl, dr = 32, 24, 8, 16, 12
    u_raw = np.array([[complex(math.sin(r * 3 + c * 5), math.cos((r + c) * 0.3)) for c in range(4)]
                      for r in range(rows)])
    v_raw = np.array([[complex(math.cos(r * 7 + c * 11), math.sin((r * 2 + c) * 0.2)) for c in range(4)]
                      for r in range(cols)])
    uq, vq = O.thin_q(u_raw), O.thin_q(v_raw)
    mat = (uq * np.array([8.0, 4.0, 2.0, 1.0])) @ vq.conj().T
    left, right = O.rsvd_sites(mat, ell, dl, dr, 4)
    assert left.shape[2] == 4
    rebuilt = np.einsum("asg,gtb->astb", left, right).reshape(rows, cols)
    assert np.abs(rebuilt - mat).max() < 1e-6


def test_disjoint_adjacent_layer_matches_sequential():
    """mps.rs:1772-1793."""
    prep = C.gates_array([C.g1(C.H, 0), C.g1(C.H, 2), C.g1(C.RY, 1, 0.3), C.g1(C.RY, 3, 0.7)])
    layer = C.gates_array([C.g2(C.CNOT, 0, 1), C.g2(C.CZ, 3, 2)])
    seq = O.OracleMps(4, exact_bond_dim(4))
    seq.apply_gates(np.concatenate([prep, layer]))
    bat = O.OracleMps(4, exact_bond_dim(4))
    bat.apply_gates(prep)
    bat.apply_layer(layer)
    assert np.abs(seq.dense() - bat.dense()).max() < 1e-8


def ry_cnot_brickwork(n, depth):  # mps.rs:1542-1559
    g, split = [], 0
    for layer in range(depth):
        if layer == depth // 2:
            split = len(g)
        for q in range(n):
            g.append(C.g1(C.RY, q, 0.17 + 0.01 * (q + layer)))
        for q in range(layer % 2, n - 1, 2):
            g.append(C.g2(C.CNOT, q, q + 1))
    return C.gates_array(g), split


def test_brickwork_16q_depth_16_chi_256_matches_dense():
    """tree.rs:1143-1155: chi 256 keeps the 16-qubit sweep exact."""
    g, _ = ry_cnot_brickwork(16, 16)
    m = O.run(16, 256, g)
    d = D.Dense(16)
    d.apply_gates(g)
    assert abs(m.amplitude_zero() - d.state[0]) < 1e-8
    assert np.all(m.records()["path"] == 0)


def test_time_split_matches_dense_and_rejects_truncation():
    """mps.rs:1561-1597 and 1649-1680."""
    g = C.gates_array([C.g1(C.H, 0), C.g1(C.S, 0), C.g1(C.RZ, 0, 0.4)])
    d = D.Dense(1)
    d.apply_gates(g)
    assert abs(O.time_split(1, g, 2, 128) - d.state[0]) < 1e-8
    g, split = ry_cnot_brickwork(16, 16)
    d = D.Dense(16)
    d.apply_gates(g)
    assert abs(O.time_split(16, g, split, 128) - d.state[0]) < 1e-8
    with pytest.raises(O.OracleError):
        O.time_split(16, g, len(g), 128)
    g8, _ = ry_cnot_brickwork(16, 8)
    g8 = np.concatenate([g8, C.gates_array([C.g2(C.CNOT, 0, 15)])])
    with pytest.raises(O.OracleError, match="mps bond exceeded chi"):
        O.time_split(16, g8, len(g8), 16)
    g6, _ = ry_cnot_brickwork(16, 6)
    g6 = np.concatenate([g6, C.gates_array([C.g2(C.CNOT, 0, 15)])])
    d = D.Dense(16)
    d.apply_gates(g6)
    assert abs(O.time_split(16, g6, len(g6), 16) - d.state[0]) < 1e-8


@pytest.mark.parametrize("n", [50, 100])
def test_product_amplitude_at_50_and_100_qubits(n):
    """contract.rs:216-230."""
    m = O.run(n, 128, C.gates_array([C.g1(C.H, 0)]))
    a = m.amplitude_zero()
    assert abs(a.real - 1 / math.sqrt(2)) < 1e-8 and abs(a.imag) < 1e-8


def test_workspace_bytes():
    """mps.rs:1870-1889."""
    assert O.mps_workspace_bytes(100, 128) == 52_428_800


def test_truncation_rule_cases():
    """svd_guard.rs:289-342."""
    values = [1.0 - 0.4 * i / 7.0 for i in range(8)]
    chi = O.retained_chi(values, 8, 8, 8)
    assert chi == 8 and not O.needs_f64_fallback(values, chi)
    values = [1.0, 0.5, 1e-12 * 1.5]
    assert O.needs_f64_fallback(values, O.retained_chi(values, 8, 8, 8))
    values = [1.0, 1.0 - 1e-8, 0.2]
    chi = O.retained_chi(values, 8, 8, 8)
    assert chi == 3 and not O.needs_f64_fallback(values, chi)
    assert O.needs_f64_fallback([1.0, 0.5, 0.5 * (1.0 - 1e-4)], 2)
    pairs = O.jacobi_pairs(6).reshape(5, 3, 2)
    seen = set()
    for step in pairs:
        assert len({int(x) for x in step.reshape(-1)}) == 6
        seen |= {tuple(sorted((int(a), int(b)))) for a, b in step}
    assert len(seen) == 15
    assert O.retained_chi([], 8, 8, 8) == 0
    assert O.retained_chi([1e-13, 1e-14], 8, 8, 8) == 1


def test_range_finder_rule_and_seed():
    """mps.rs:929-935, 951-954, 1103-1122: the switch and the exact Omega bits."""
    assert O.rsvd_worth(160, 160, 160) and not O.rsvd_worth(160, 160, 159)
    assert O.mix_seed(256, 256, 144) == ((256 * 0x9E37 + 256) * 0x9E37 + 144)
    om = O.rademacher(4, 3, 12345)
    state, scale, want = 12345 | 1, 1 / math.sqrt(4), []
    for _ in range(12):
        state = (state * 6364136223846793005 + 1) % (1 << 64)
        want.append(complex(scale if state & 0x100 == 0 else -scale, scale if state & 0x200 == 0 else -scale))
    assert np.array_equal(om.reshape(-1), np.array(want))


def test_rademacher_rank_is_48():
    """The reference's test matrix takes bits 8 and 9 of a mod-2^64 LCG, which
    repeat with period 1024: Omega has rank 48 at every range-finder shape, so
    the range finder is only well determined on splits of rank <= 48."""
    for rows, cols, ell in ((192, 192, 112), (256, 256, 144), (512, 512, 272)):
        sv = np.linalg.svd(O.rademacher(cols, ell, O.mix_seed(rows, cols, ell)), compute_uv=False)
        assert int(np.sum(sv > sv[0] * 1e-12)) == 48


def _expect_dense(n, gates, label):
    d = D.Dense(n)
    d.apply_gates(C.gates_array(gates))
    return D.pauli_expectation(d.state, label)


def test_pauli_expectation_semantics():
    """expectation.rs:291-466 on both the dense formula and the oracle's MPS
    transfer-matrix expectation."""
    cases = [
        (1, [], "Z", 1.0),
        (1, [C.g1(C.H, 0), C.g1(C.S, 0)], "Y", 1.0),
        (1, [C.g1(C.H, 0), C.g1(C.S, 0), C.g1(C.Z, 0)], "Y", -1.0),
        (2, [C.g1(C.H, 0), C.g1(C.S, 0), C.g2(C.CNOT, 0, 1)], "XY", 1.0),
        (2, [C.g1(C.H, 0), C.g1(C.S, 0), C.g2(C.CNOT, 0, 1)], "YX", 1.0),
        (2, [C.g1(C.H, 0), C.g2(C.CNOT, 0, 1)], "YY", -1.0),
        (1, [C.g1(C.H, 0)], "Z", 0.0),
        (2, [C.g1(C.H, 0), C.g2(C.CNOT, 0, 1)], "ZZ", 1.0),
    ]
    for n, gates, label, want in cases:
        assert abs(_expect_dense(n, gates, label) - want) < 1e-9
        m = O.run(n, 4, C.gates_array(gates) if gates else C.gates_array([C.g1(C.Z, 0)]))
        got = m.expectation([label], [1.0])
        assert abs(got.real - want) < 1e-9 and abs(got.imag) < 1e-12
    m = O.run(2, 4, C.gates_array([C.g1(C.H, 0), C.g2(C.CNOT, 0, 1)]))
    assert abs(m.expectation(["ZZ", "II"], [0.5, 0.5]) - 1.0) < 1e-12


def test_mps_expectation_matches_dense_on_random_state():
    n = 10
    g = C.gates_array(C.ry_rz_brickwork(n, 6, seed=9))
    m = O.run(n, 64, g)
    d = D.Dense(n)
    d.apply_gates(g)
    labels, coeffs = C.zz_x_observable(n)
    want = sum(c * D.pauli_expectation(d.state, lab) for lab, c in zip(labels, coeffs))
    assert abs(m.expectation(labels, coeffs) - want) < 1e-10


def test_amplitude_snap_and_hash():
    """engine.rs:25-64 and the golden hash at engine.rs:924-934."""
    assert O.snap(0.4999999701976776) == 0.5 and O.snap(-0.4999999701976776) == -0.5
    assert O.snap(0.5000000000000001) == 0.5
    body = '{"real":0.7071067811865475,"imag":0.0}'
    assert hashlib.sha3_256(body.encode()).hexdigest() == \
        "ee10cd493b1b6773f6e947b471b3fc8c94009eac7ac09d189e64ead838dfc0d5"


def test_statevector_projection_limits():
    """mps.rs:1856-1868."""
    with pytest.raises(O.OracleError):
        O.OracleMps(0, 8)
    O.OracleMps(41, 8)
    m = O.OracleMps(21, 4)
    with pytest.raises(O.OracleError, match="qubit_count <= 20"):
        m.statevector()


def test_call_sequence_folds_rotations_and_batches_layers():
    """trace.rs:99-154: same-axis rotation runs apply as one net gate; at
    N > 16 a run of disjoint adjacent CNOT/CZ is one layer.  Both give the
    sequential result."""
    n = 18
    g = []
    for q in range(n):
        g += [C.g1(C.RY, q, 0.3), C.g1(C.RY, q, 0.2 + 0.01 * q)]
    g += [C.g2(C.CNOT, q, q + 1) for q in range(0, n - 1, 2)]
    g += [C.g1(C.RZ, 3, 2 * math.pi), C.g1(C.H, 1), C.g1(C.H, 1)]
    g = C.gates_array(g)
    a = O.run(n, 16, g).amplitude_zero()
    b = O.run(n, 16, g, call_sequence=True).amplitude_zero()
    assert abs(a - b) < 1e-12


def test_oracle_drift_under_a_change_of_svd():
    """Two FP64 SVDs of the same matrices -- the oracle's Golub-Kahan (the
    reference's primary, nalgebra's family) and its svd_guard.rs Jacobi as
    primary -- agree to rounding on one split, but a long truncating run
    carries the difference into every later cut.  On the deepest slice of the
    batching test (43 qubits, 1008 splits at chi 32) the kept chi and paths
    stay identical while the per-split discarded weights drift apart far
    beyond 1e-12: the drift the device's Jacobi shows against the oracle on
    such runs is rounding of this kind, and the GPU tests bound it by this
    drift measured on the oracle itself."""
    s = C.config2_slices(12, seed=99)[1]
    chi = min(s.chi, 32)
    runs = []
    for primary in (0, 1):
        O.set_primary_svd(primary)
        try:
            runs.append(O.run(s.n, chi, s.gates).records())
        finally:
            O.set_primary_svd(0)
    a, b = runs
    assert len(a) == len(b) > 1000
    for k in ("left_site", "rows", "cols", "path", "chi"):
        assert np.array_equal(a[k], b[k]), k
    d = np.abs(a["discarded_weight"] - b["discarded_weight"])
    assert d[:150].max() <= 1e-12  # early splits agree to the per-split tolerance
    assert 1e-11 < d.max() < 1e-6  # the tail drifts, by rounding amplified through the cuts


def test_numpy_adjoint_matches_central_differences():
    """oracle/adjoint.py, the checker of the device adjoint: its forward is
    the oracle's (same value) and its reverse sweep through truncating
    splits matches central differences of its own forward to 1e-8."""
    import adjoint as A

    for n, layers, chi in ((6, 3, 3), (8, 2, 64)):
        gates, pidx, _ = C.hea_ansatz(n, layers, seed=5)
        labels, coeffs = C.zz_x_observable(n)
        f, g = A.gradient(n, chi, gates, labels, coeffs)
        assert abs(f - O.run(n, chi, gates).expectation(labels, coeffs).real) <= 1e-12
        h = 1e-5
        for i in np.nonzero(pidx >= 0)[0][::5]:
            gp, gm = gates.copy(), gates.copy()
            gp["angle"][i] += h
            gm["angle"][i] -= h
            fd = (A.value(n, chi, gp, labels, coeffs) - A.value(n, chi, gm, labels, coeffs)) / (2 * h)
            assert abs(g[i] - fd) <= 1e-8
