"""CPU checks of the host-side helpers above the C ABI (no device work):

* bra_unitary_gates restates bra_unitary_gates / adjoint_gate_sequence
  (src/tn/mps.rs:1393-1421): applied after a circuit on the dense simulator
  it returns |0...0>, and it gives up on MEASURE / RESET / IF;
* sample_counts forms the reference's Qiskit-order keys (outcome_key,
  src/sample.rs:133-156) from packed draws: measures apply in order, several
  measures of one qubit land in their own classical bits, cbit 0 is the
  rightmost character, and unmeasured classical bits read 0.
"""
import numpy as np
import pytest

import dense as D
import wqc_cuda as W
from wqc_cuda import circuits as C


def random_gate_list(rng, n, count):
    out = []
    for _ in range(count):
        k = int(rng.integers(0, 4))
        q = int(rng.integers(0, n))
        if k == 0:
            out.append(C.g1(int(rng.choice([C.H, C.X, C.Y, C.Z, C.S, C.T])), q))
        elif k == 1:
            out.append(C.g1(int(rng.choice([C.RX, C.RY, C.RZ])), q, float(rng.uniform(-3, 3))))
        elif k == 2:
            out.append(C.g2(int(rng.choice([C.CNOT, C.CZ])), q, (q + 1 + int(rng.integers(0, n - 1))) % n))
        else:
            out.append(C.g3(0, 1, 2))
    return C.gates_array(out)


def test_bra_unitary_gates_inverts_the_second_half():
    rng = np.random.default_rng(0xB4A)
    for _ in range(25):
        n = 4
        g = random_gate_list(rng, n, 18)
        d = D.Dense(n)
        d.apply_gates(g)
        d.apply_gates(W.bra_unitary_gates(g))
        assert abs(abs(d.state[0]) - 1.0) < 1e-12
    g = C.gates_array([C.g1(C.H, 0), C.g1(C.MEASURE, 0)])
    assert W.bra_unitary_gates(g) is None


class _FakeDraws(W.CudaMps):
    """A CudaMps whose draws are given, to test the key construction alone."""

    def __init__(self, n, draws):  # no device state
        self.n = n
        self._h = None
        self._draws = np.asarray(draws, dtype=np.uint64)
        self.asked = None

    def sample(self, qubits, shots, seed):
        self.asked = list(qubits)
        return self._draws[:shots]


def test_sample_counts_builds_the_reference_keys():
    # qubits asked in ascending order: bit 0 = qubit 0, bit 1 = qubit 2
    m = _FakeDraws(3, [0b00, 0b01, 0b10, 0b11, 0b01])
    counts = m.sample_counts([(2, 0), (0, 2), (0, 1)], 4, 5, seed=1)
    assert m.asked == [0, 2]
    # draw 0b01: qubit 0 = 1, qubit 2 = 0 -> cbits (0: q2=0, 1: q0=1, 2: q0=1, 3: 0) -> "0110"
    assert counts == {"0000": 1, "0110": 2, "0001": 1, "0111": 1}
    assert sum(counts.values()) == 5
    # a later measure into the same classical bit wins, as in outcome_key
    m2 = _FakeDraws(2, [0b10])
    assert m2.sample_counts([(0, 0), (1, 0)], 1, 1, seed=0) == {"1": 1}


def test_trace_replay_steps_follow_the_oracle_call_sequence():
    """wqc_cuda/trace_replay.py folds the gate list as trace.rs does (H runs,
    rotation runs with the full-turn rule, disjoint layers above 16 qubits):
    driven on the oracle it leaves the same state and split records as the
    oracle's own restatement of the call sequence, and it reads each
    control's probability and each target's amplitudes at most as the
    reference's resolve_pre_amps does."""
    import math

    import oracle as O
    from wqc_cuda import trace_replay as TR

    class OracleState:
        def __init__(self, n, chi):
            self.m = O.OracleMps(n, chi)

        def apply_gates(self, g):
            self.m.apply_gates(g)

        def apply_adjacent_disjoint_gates(self, g):
            self.m.apply_layer(g)

        def site_amplitudes_many(self, targets):
            return np.array([self.m.site_amplitudes(int(t)) for t in targets], dtype=np.complex128)

    n, chi = 18, 8
    g = C.random_layers(n, 4, seed=3)
    g += [C.g1(C.RZ, 2, math.pi), C.g1(C.RZ, 2, math.pi), C.g1(C.RY, 4, 0.2), C.g1(C.RY, 4, 0.3)]
    g += [C.g1(C.H, 6), C.g1(C.H, 6), C.g1(C.H, 7)] + [C.g2(C.CZ, q, q + 1) for q in range(0, n - 1, 2)]
    gates = C.gates_array(g)
    kinds = [k for k, _, _ in TR.steps(n, gates)]
    assert {"layer", "net", "silent", "one"} <= set(kinds)
    st = OracleState(n, chi)
    reads = TR.replay(st, n, gates)
    ref = O.run(n, chi, gates, call_sequence=True)
    a, b = st.m.records(), ref.records()
    assert len(a) == len(b) and np.array_equal(a["chi"], b["chi"])
    assert abs(st.m.amplitude_zero() - ref.amplitude_zero()) <= 1e-12 * max(1.0, abs(ref.amplitude_zero()))
    # each qubit's amplitudes are read once as a target; controls at every 2q gate
    targets_seen = [int(t) for tg, _ in reads for t in tg]
    n2q = int(np.isin(gates["kind"], [C.CNOT, C.CZ]).sum()) + 2 * int((gates["kind"] == C.CCNOT).sum())
    assert len(targets_seen) <= n2q + n
