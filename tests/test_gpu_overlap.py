"""The time split's overlap on the device (wqc_mps_overlap) and the time split
built on it (contract_time_split, src/tn/mps.rs:1241-1249, 1358-1474),
against the oracle's restatement of the same path and the dense simulator:
values within 1e-10, the reference's errors (environment above 256 entries,
rejected truncation, mismatched registers) with its messages."""
import numpy as np
import pytest

import dense as D
import oracle as O
import wqc_cuda as W
from wqc_cuda import circuits as C

pytestmark = pytest.mark.gpu


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


def test_overlap_matches_dense_inner_product(cuda_ctx):
    n = 10
    ga = C.gates_array(C.random_layers(n, 5, seed=31))
    gb = C.gates_array(C.random_layers(n, 5, seed=32))
    ket = W.CudaMps(n, 64, ctx=cuda_ctx)
    ket.apply_gates(ga)
    bra = W.CudaMps(n, 64, ctx=cuda_ctx)
    bra.apply_gates(gb)
    da, db = D.Dense(n), D.Dense(n)
    da.apply_gates(ga)
    db.apply_gates(gb)
    want = np.vdot(db.state, da.state)  # <bra|ket>
    got = ket.overlap(bra, env_limit=0)
    assert abs(got - want) < 1e-10 * max(1.0, abs(want)), (got, want)
    norm = ket.overlap(ket, env_limit=0)
    assert abs(norm - 1.0) < 1e-10
    env = int(np.max(ket.bond_dims().astype(np.int64) * bra.bond_dims()))
    if env > 256:  # the reference's cap applies by default
        with pytest.raises(W.WqcCudaError) as e:
            ket.overlap(bra)
        assert e.value.code == W.ERR_INVALID and "exceeds 256" in str(e.value)
    else:
        assert ket.overlap(bra) == got


def test_time_split_matches_oracle_and_dense(cuda_ctx):
    """mps.rs:1561-1597: the 16-qubit brickwork split in the middle."""
    g = C.gates_array([C.g1(C.H, 0), C.g1(C.S, 0), C.g1(C.RZ, 0, 0.4)])
    d = D.Dense(1)
    d.apply_gates(g)
    got = W.contract_time_split(1, g, 2, 128, ctx=cuda_ctx)
    assert abs(got - d.state[0]) < 1e-12
    assert abs(got - O.time_split(1, g, 2, 128)) < 1e-12
    g, split = ry_cnot_brickwork(16, 16)
    d = D.Dense(16)
    d.apply_gates(g)
    got = W.contract_time_split(16, g, split, 128, ctx=cuda_ctx)
    ref = O.time_split(16, g, split, 128)
    assert abs(got - ref) < 1e-10 * max(abs(ref), 1e-3), (got, ref)
    assert abs(got - d.state[0]) < 1e-8
    # S and T in the second half take the S Z / T T T Z adjoint sequences.
    g2 = C.gates_array([C.g1(C.H, q) for q in range(4)] + [C.g2(C.CNOT, 0, 1), C.g1(C.T, 1), C.g1(C.S, 2),
                                                            C.g2(C.CZ, 2, 3), C.g1(C.T, 3), C.g1(C.RX, 0, 0.3)])
    d = D.Dense(4)
    d.apply_gates(g2)
    for split in (0, 3, 6, len(g2)):
        got = W.contract_time_split(4, g2, split, 16, ctx=cuda_ctx)
        assert abs(got - d.state[0]) < 1e-12, split
        assert abs(got - O.time_split(4, g2, split, 16)) < 1e-12, split


def test_time_split_errors_match_the_reference(cuda_ctx):
    g, _ = ry_cnot_brickwork(16, 16)
    with pytest.raises(W.WqcCudaError) as e:  # the whole circuit in the ket: bond 256 needed at chi 128
        W.contract_time_split(16, g, len(g), 128, ctx=cuda_ctx)
    assert e.value.code == W.ERR_TRUNCATION_REJECTED and "mps bond exceeded chi" in str(e.value)
    with pytest.raises(O.OracleError, match="mps bond exceeded chi"):
        O.time_split(16, g, len(g), 128)
    g20 = C.gates_array(C.random_layers(10, 20, seed=41))  # both halves reach bond 32: environment 1024
    with pytest.raises(W.WqcCudaError) as e:
        W.contract_time_split(10, g20, len(g20) // 2, 64, ctx=cuda_ctx)
    assert e.value.code == W.ERR_INVALID and "mps overlap environment exceeds 256" in str(e.value)
    with pytest.raises(O.OracleError, match="mps overlap environment exceeds 256"):
        O.time_split(10, g20, len(g20) // 2, 64)
    g8, _ = ry_cnot_brickwork(16, 8)
    g8 = np.concatenate([g8, C.gates_array([C.g2(C.CNOT, 0, 15)])])
    with pytest.raises(W.WqcCudaError) as e:
        W.contract_time_split(16, g8, len(g8), 16, ctx=cuda_ctx)
    assert e.value.code == W.ERR_TRUNCATION_REJECTED
    with pytest.raises(W.WqcCudaError) as e:
        W.contract_time_split(16, g8, len(g8) + 1, 16, ctx=cuda_ctx)
    assert "past the gate list" in str(e.value)
    a = W.CudaMps(3, 4, ctx=cuda_ctx)
    b = W.CudaMps(4, 4, ctx=cuda_ctx)
    with pytest.raises(W.WqcCudaError) as e:
        a.overlap(b)
    assert e.value.code == W.ERR_INVALID and "mismatched register" in str(e.value)
