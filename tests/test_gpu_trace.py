"""The production call patterns of the reference, through the C ABI, against
the oracle:

* the trace loop (src/tn/trace.rs:55-187): rotation and H folding, disjoint
  layers at N > 16, and before every traced step the control probabilities
  and first-time target amplitudes (resolve_pre_amps, trace.rs:375-411) --
  every read, every split record and the final amplitude;
* the trace feeders' cached environments: reads interleaved with every kind
  of operation (1q gates, splits, routed gates, uploads, reset) must equal a
  from-scratch contraction by the oracle;
* the sweep-tree route (Live::replay, src/tn/tree.rs:704-788): the MpsState
  hooks apply_unary_at / apply_tdg_at / apply_swap_at / apply_pair_at /
  apply_cnot_at (mps.rs:621-655), with wires moved by SWAPs, against the
  oracle's same calls and the dense simulator on the logical wires;
* the dense state on the device (to_dense_state, contract_to_statevector,
  mps.rs:215-260, 742-780) against the dense simulator and the oracle.

Reads are compared relative to the largest read of the run (the all-ones
environments sum amplitudes of very different sizes); records bit-exact in
shape, path and kept chi, discarded weights within 1e-12.
"""
import numpy as np
import pytest

import dense as D
import oracle as O
import wqc_cuda as W
from wqc_cuda import circuits as C
from wqc_cuda import trace_replay as TR

pytestmark = pytest.mark.gpu

READ_RTOL = 1e-10


class OracleState:
    """The oracle behind the interface trace_replay drives."""

    def __init__(self, n, chi):
        self.m = O.OracleMps(n, chi)

    def apply_gates(self, g):
        self.m.apply_gates(g)

    def apply_adjacent_disjoint_gates(self, g):
        self.m.apply_layer(g)

    def site_amplitudes_many(self, targets):
        return np.array([self.m.site_amplitudes(int(t)) for t in targets], dtype=np.complex128)


def assert_records_equal(got, ref, drift=None):
    """Shapes, paths and kept chi bit-exact; discarded weights within 1e-12
    plus ten times the oracle's own drift between two FP64 SVDs."""
    assert len(got) == len(ref)
    for k in ("left_site", "rows", "cols", "ell", "path", "chi"):
        assert np.array_equal(got[k], ref[k]), k
    tol = 1e-12 * np.maximum(1.0, np.abs(ref["discarded_weight"]))
    if drift is not None:
        tol = tol + 10.0 * np.maximum.accumulate(drift)
    assert np.all(np.abs(got["discarded_weight"] - ref["discarded_weight"]) <= tol)


def trace_workload(n=24, depth=12, seed=31):
    """The random-layer generator plus what the trace loop folds: same-axis
    rotation runs (one of them a full turn), an H pair and an odd H run."""
    g = C.random_layers(n, depth, seed)
    g += [C.g1(C.RY, 3, 0.4), C.g1(C.RY, 3, 0.5), C.g1(C.RZ, 5, np.pi), C.g1(C.RZ, 5, np.pi)]
    g += [C.g1(C.H, 7), C.g1(C.H, 7), C.g1(C.H, 8), C.g1(C.H, 8), C.g1(C.H, 8)]
    g += [C.g2(C.CZ, q, q + 1) for q in range(0, n - 1, 2)] + [C.g3(2, 3, 4)]
    return C.gates_array(g)


def test_trace_loop_reads_and_splits_match_oracle(cuda_ctx):
    n, chi = 24, 32
    gates = trace_workload(n)
    kinds = [s[0] for s in TR.steps(n, gates)]
    assert "layer" in kinds and "net" in kinds and "silent" in kinds
    m = W.CudaMps(n, chi, ctx=cuda_ctx)
    o = OracleState(n, chi)
    got = TR.replay(m, n, gates)
    ref = TR.replay(o, n, gates)
    assert len(got) == len(ref) > 0
    scale = max(np.abs(r[1]).max() for r in ref)
    for (tg, ag), (tr, ar) in zip(got, ref):
        assert np.array_equal(tg, tr)
        assert np.abs(ag - ar).max() <= READ_RTOL * scale, (tg, ag, ar)
    drift = O.self_drift(n, chi, gates, call_sequence=True)
    assert_records_equal(m.split_records(), o.m.records(), drift)
    # the oracle's own restatement of the call sequence gives the same splits
    assert_records_equal(o.m.records(), O.run(n, chi, gates, call_sequence=True).records())
    a, b = m.amplitude_zero(), o.m.amplitude_zero()
    assert abs(a - b) <= 1e-10 * max(abs(b), 2.0 ** (-n / 2))


def test_cached_environments_follow_every_operation(cuda_ctx):
    """Reads interleaved with 1q gates, adjacent and routed splits, a CCNOT,
    an upload and a reset: each read equals the oracle's from-scratch
    contraction (the cache recomputes exactly what operations touched)."""
    n, chi = 20, 16
    rng = np.random.default_rng(5)
    m = W.CudaMps(n, chi, ctx=cuda_ctx)
    o = O.OracleMps(n, chi)
    ops = C.random_layers(n, 6, seed=17)
    scale = 0.0
    for i, g in enumerate(ops):
        arr = C.gates_array([g])
        m.apply_gates(arr)
        o.apply_gates(arr)
        if i % 7 == 0:
            targets = sorted(set(int(t) for t in rng.integers(0, n, size=3)))
            got = m.site_amplitudes_many(targets)
            ref = np.array([o.site_amplitudes(t) for t in targets])
            scale = max(scale, np.abs(ref).max())
            assert np.abs(got - ref).max() <= READ_RTOL * scale, (i, targets)
    # an upload (each side scales its own site 9: the two gauges differ)
    m.set_site(9, 0.5 * m.site(9))
    o.set_site(9, 0.5 * o.site(9))
    for t in (0, 9, n - 1):
        assert np.abs(np.array(m.site_amplitudes(t)) - np.array(o.site_amplitudes(t))).max() <= READ_RTOL * scale
    m.apply_gates(C.gates_array([C.g3(4, 12, 8)]))
    o.apply_gates(C.gates_array([C.g3(4, 12, 8)]))
    got = m.site_amplitudes_many(list(range(n)))
    ref = np.array([o.site_amplitudes(t) for t in range(n)])
    assert np.abs(got - ref).max() <= READ_RTOL * max(scale, np.abs(ref).max())
    m.reset()
    a0, a1 = m.site_amplitudes(11)
    assert abs(a0 - 1) < 1e-15 and abs(a1) < 1e-15


def test_sweep_tree_hooks_match_oracle_and_dense(cuda_ctx):
    """A sweep-tree replay: Site / CcnotH / CcnotT / CcnotTdg nodes through
    apply_unary_at and apply_tdg_at, Swap nodes through apply_swap_at (which
    exchange the wires of two sites), Pair and CcnotCnot nodes through
    apply_pair_at and apply_cnot_at with the control on either side."""
    n, chi = 10, 64
    rng = np.random.default_rng(2026)
    m = W.CudaMps(n, chi, ctx=cuda_ctx)
    o = O.OracleMps(n, chi)
    d = D.Dense(n)
    wire_at = list(range(n))  # wire held by each site
    r2 = 0.70710678118654752440
    tdg = np.array([[1, 0], [0, complex(r2, -r2)]])
    for _ in range(160):
        node = int(rng.integers(0, 6))
        if node <= 1:  # Site or CcnotH / CcnotT
            s = int(rng.integers(0, n))
            kind = int(rng.choice([C.H, C.T, C.RX, C.RY, C.RZ, C.S, C.X]))
            ang = float(rng.uniform(0, 2 * np.pi))
            m.apply_unary_at(s, (kind, ang))
            o.apply_1q(s, D.unary(kind, ang))
            d.apply_unary(wire_at[s], D.unary(kind, ang))
        elif node == 2:  # CcnotTdg
            s = int(rng.integers(0, n))
            m.apply_tdg_at(s)
            o.apply_1q(s, tdg)
            d.apply_unary(wire_at[s], tdg)
        elif node == 3:  # Swap
            s = int(rng.integers(0, n - 1))
            m.apply_swap_at(s)
            o.apply_2q_at(s, W.SWAP4, True)
            wire_at[s], wire_at[s + 1] = wire_at[s + 1], wire_at[s]
        else:  # Pair (CNOT or CZ) / CcnotCnot
            s = int(rng.integers(0, n - 1))
            left = bool(rng.integers(0, 2))
            kind = C.CNOT if node == 5 else int(rng.choice([C.CNOT, C.CZ]))
            if node == 5:
                m.apply_cnot_at(s, left)
            else:
                m.apply_pair_at(s, kind, left)
            o.apply_2q_at(s, W.CNOT4 if kind == C.CNOT else W.CZ4, left)
            c, t = (wire_at[s], wire_at[s + 1]) if left else (wire_at[s + 1], wire_at[s])
            d.apply_controlled(c, t, D.unary(C.X if kind == C.CNOT else C.Z))
    assert_records_equal(m.split_records(), o.records())
    got = m.to_dense_state()
    assert np.abs(got - o.dense()).max() < 1e-10
    # physical basis index: bit s is the wire held by site s
    idx = np.arange(1 << n)
    logical = np.zeros_like(idx)
    for s in range(n):
        logical |= ((idx >> s) & 1) << wire_at[s]
    assert np.abs(got - d.state[logical]).max() < 1e-9


def test_dense_state_on_device(cuda_ctx):
    n = 12
    g = C.gates_array(C.random_layers(n, 6, seed=4))
    m = W.run(n, 8, g, ctx=cuda_ctx)  # truncating: to_dense_state of the truncated MPS
    o = O.run(n, 8, g)
    assert np.abs(m.to_dense_state() - o.dense()).max() < 1e-12
    assert np.abs(m.contract_to_statevector() - o.statevector()).max() < 1e-12
    m = W.run(n, 64, g, ctx=cuda_ctx)
    dd = D.Dense(n)
    dd.apply_gates(g)
    assert np.abs(m.to_dense_state() - dd.state).max() < 1e-10
    big = W.CudaMps(21, 4, ctx=cuda_ctx)
    with pytest.raises(W.WqcCudaError, match="qubit_count <= 20"):
        big.contract_to_statevector()
    assert abs(big.to_dense_state()[0] - 1.0) < 1e-15
