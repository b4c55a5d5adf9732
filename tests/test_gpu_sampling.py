"""Shot sampling from the MPS on the device (wqc_mps_sample).

The reference samples terminal measurements from the dense statevector
(src/sample.rs:85-131, 192-211), so only up to 20 qubits, and draws with
rand's StdRng.  The device samples the same distribution from the MPS with
its own deterministic stream (SplitMix64 keyed by seed, shot and qubit), so
parity is checked three ways:

* draw for draw against a numpy restatement of the same site-by-site
  sampler run on the state's own sites (downloaded from the device) with
  the same stream: every shot must agree;
* in distribution against the dense statevector of the oracle's dense
  simulator (total variation within the sampling noise);
* on the reference's own sampling tests: the Bell state gives only "00" and
  "11" with Qiskit-order keys (src/sample.rs:226-250), and a 32-qubit GHZ
  state, beyond the reference's dense limit, only all-zeros and all-ones.
"""
import numpy as np
import pytest

import dense as D
import wqc_cuda as W
from wqc_cuda import circuits as C

pytestmark = pytest.mark.gpu

M64 = (1 << 64) - 1


def splitmix64(z: int) -> int:
    z = (z + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def uniform(seed: int, shot: int, q: int) -> float:
    key = splitmix64(seed ^ splitmix64(shot))
    return (splitmix64((key + q) & M64) >> 11) * 2.0 ** -53


def numpy_sampler(sites, qubits, shots, seed):
    """The device's algorithm restated: right environments, then site-by-site
    conditional draws with v normalised after each site."""
    n = len(sites)
    env = [None] * (n + 1)
    env[n] = np.ones((1, 1), complex)
    for q in range(n - 1, 0, -1):
        a = sites[q]
        env[q] = sum(a[:, s, :] @ env[q + 1] @ a[:, s, :].conj().T for s in range(2))
    col = {q: j for j, q in enumerate(qubits)}
    out = np.zeros(shots, dtype=np.uint64)
    for k in range(shots):
        v = np.ones(1, complex)
        bits = 0
        for q in range(n):
            a = sites[q]
            w = [v @ a[:, s, :] for s in range(2)]
            p = [max(float(np.real(w[s] @ env[q + 1] @ w[s].conj())), 0.0) for s in range(2)]
            u = uniform(seed, k, q)
            s = 1 if (p[0] + p[1] > 0 and u * (p[0] + p[1]) >= p[0]) else 0
            v = w[s] / np.sqrt(p[s]) if p[s] > 0 else w[s]
            if s and q in col:
                bits |= 1 << col[q]
        out[k] = bits
    return out


def test_draws_match_the_restated_sampler_shot_for_shot(cuda_ctx):
    n = 10
    gates = C.gates_array(C.random_layers(n, 8, seed=21))
    m = W.CudaMps(n, 16, ctx=cuda_ctx)  # bond 16 < 32: the state is truncated
    m.apply_gates(gates)
    qubits = [7, 0, 3, 9, 4]
    seed = 0xC0FFEE
    got = m.sample(qubits, 400, seed)
    want = numpy_sampler([m.site(q) for q in range(n)], qubits, 400, seed)
    assert np.array_equal(got, want)
    assert np.array_equal(m.sample(qubits, 400, seed), got)  # deterministic for a seed
    assert not np.array_equal(m.sample(qubits, 400, seed + 1), got)


def test_distribution_matches_dense_statevector(cuda_ctx):
    n = 10
    gates = C.gates_array(C.random_layers(n, 6, seed=3))
    m = W.CudaMps(n, 64, ctx=cuda_ctx)  # no truncation at 10 qubits
    m.apply_gates(gates)
    d = D.Dense(n)
    d.apply_gates(gates)
    p = np.abs(d.state) ** 2
    p /= p.sum()
    shots = 40000
    draws = m.sample(list(range(n)), shots, 12345).astype(np.int64)  # bit q = qubit q = dense index bit q
    freq = np.bincount(draws, minlength=1 << n) / shots
    tv = 0.5 * np.abs(freq - p).sum()
    # E[TV] <= 0.5 sum sqrt(p (1-p) / shots) <= 0.5 sqrt(2^n / shots) = 0.08; a random-circuit
    # distribution is far from uniform, so the expected value is well below that.
    noise = 0.5 * np.sum(np.sqrt(p * (1 - p) / shots))
    assert tv < 1.5 * noise + 0.01, (tv, noise)
    # Marginal of a subset: qubits (2, 5) against the dense marginal.
    sub = m.sample([2, 5], shots, 777).astype(np.int64)
    idx = np.arange(1 << n)
    marg = np.zeros(4)
    np.add.at(marg, ((idx >> 2) & 1) | (((idx >> 5) & 1) << 1), p)
    fsub = np.bincount(sub, minlength=4) / shots
    assert np.abs(fsub - marg).max() < 5 * np.sqrt(0.25 / shots) + 1e-3, (fsub, marg)


def test_bell_state_counts_use_qiskit_keys(cuda_ctx):
    """src/sample.rs:226-250: H(0), CNOT(0, 1), 1024 shots: only "00" and "11"."""
    m = W.CudaMps(2, 2, ctx=cuda_ctx)
    m.apply_gates(C.gates_array([C.g1(C.H, 0), C.g2(C.CNOT, 0, 1)]))
    counts = m.sample_counts([(0, 0), (1, 1)], 2, 1024, 42)
    assert sum(counts.values()) == 1024
    assert set(counts) == {"00", "11"}
    assert 400 < counts["00"] < 624
    # X(0) then measuring qubit 0 into cbit 1 of a 3-bit register: key "010".
    m2 = W.CudaMps(2, 2, ctx=cuda_ctx)
    m2.apply_gates(C.gates_array([C.g1(C.X, 0)]))
    assert m2.sample_counts([(0, 1)], 3, 64, 1) == {"010": 64}


def test_ghz_beyond_the_dense_limit(cuda_ctx):
    n = 32
    gl = [C.g1(C.H, 0)] + [C.g2(C.CNOT, q, q + 1) for q in range(n - 1)]
    m = W.CudaMps(n, 4, ctx=cuda_ctx)
    m.apply_gates(C.gates_array(gl))
    draws = m.sample(list(range(n)), 2000, 5)
    ones = np.uint64((1 << n) - 1)
    assert np.all((draws == 0) | (draws == ones))
    frac = np.count_nonzero(draws == 0) / 2000
    assert 0.44 < frac < 0.56, frac


def test_sampling_argument_errors(cuda_ctx):
    m = W.CudaMps(3, 4, ctx=cuda_ctx)
    with pytest.raises(W.WqcCudaError) as e:
        m.sample([0, 0], 4, 1)
    assert e.value.code == W.ERR_INVALID
    with pytest.raises(W.WqcCudaError) as e:
        m.sample([3], 4, 1)
    assert e.value.code == W.ERR_QUBIT_OUT_OF_RANGE
    assert m.sample([0, 1], 0, 1).size == 0
    with pytest.raises(W.WqcCudaError) as e:  # an index past 2^31 must not wrap negative
        m.sample([2 ** 31], 4, 1)
    assert e.value.code == W.ERR_QUBIT_OUT_OF_RANGE
    with pytest.raises(W.WqcCudaError) as e:
        m.site(2 ** 31)
    assert e.value.code == W.ERR_QUBIT_OUT_OF_RANGE
    b = W.CudaBatch([3, 4], [4, 4], ctx=cuda_ctx)
    with pytest.raises(W.WqcCudaError) as e:
        b.sample([0], 4, 1)
    assert e.value.code == W.ERR_INVALID
