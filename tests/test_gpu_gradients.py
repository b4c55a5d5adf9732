"""Parameter-shift gradients on the batching form (wqc_cuda.gradients),
through wqc_batch_expectation_pauli.

Without truncation the shift rule is the exact gradient: it must equal the
dense statevector's own shift-rule gradient to 1e-9.  With truncation it
must equal the FP64 oracle run on every shifted circuit (what a parameter-
shift run of the reference's CPU path gives at the same chi) to 1e-10."""
import math

import numpy as np
import pytest

import dense as D
import oracle as O
import wqc_cuda as W
from wqc_cuda import circuits as C
from wqc_cuda import gradients as G

pytestmark = pytest.mark.gpu


def dense_value(n, gates, labels, coeffs):
    d = D.Dense(n)
    d.apply_gates(gates)
    return sum(c.real * D.pauli_expectation(d.state, lab) for lab, c in zip(labels, coeffs))


def test_batch_expectations_equal_single_state_ones(cuda_ctx):
    gates, _, _ = C.hea_ansatz(8, 2, seed=3)
    labels, coeffs = C.zz_x_observable(8)
    b = W.CudaBatch([8, 8], [16, 16], ctx=cuda_ctx)
    b.apply_slices([gates, gates[: len(gates) // 2]])
    got = b.expectations(labels, coeffs)
    for s, g in enumerate((gates, gates[: len(gates) // 2])):
        m = W.CudaMps(8, 16, ctx=cuda_ctx)
        m.set_merge(W.MERGE_FFMA)  # the batch's merges: bit for bit only on the same merge path
        m.apply_gates(g)
        assert got[s] == m.expectation(labels, coeffs)


def test_parameter_shift_equals_dense_gradient_without_truncation(cuda_ctx):
    n = 6
    gates, pidx, _ = C.hea_ansatz(n, 2, seed=5)
    labels, coeffs = C.zz_x_observable(n)
    f, grad = G.parameter_shift(n, 64, gates, pidx, labels, coeffs, ctx=cuda_ctx)
    assert abs(f - dense_value(n, gates, labels, coeffs)) <= 1e-10
    want = np.zeros_like(grad)
    for i in np.nonzero(pidx >= 0)[0]:
        gp, gm = gates.copy(), gates.copy()
        gp["angle"][i] += math.pi / 2
        gm["angle"][i] -= math.pi / 2
        want[pidx[i]] += 0.5 * (dense_value(n, gp, labels, coeffs) - dense_value(n, gm, labels, coeffs))
    assert np.abs(grad - want).max() <= 1e-9
    # and the shift rule is the derivative: central difference h = 1e-4 (config 3's check)
    h = 1e-4
    for j in (0, 7, 23):
        i = int(np.nonzero(pidx == j)[0][0])
        gp, gm = gates.copy(), gates.copy()
        gp["angle"][i] += h
        gm["angle"][i] -= h
        fd = (dense_value(n, gp, labels, coeffs) - dense_value(n, gm, labels, coeffs)) / (2 * h)
        assert abs(grad[j] - fd) <= 1e-6


def test_parameter_shift_matches_oracle_with_truncation(cuda_ctx):
    n, chi = 10, 4
    gates, pidx, _ = C.hea_ansatz(n, 3, seed=8)
    labels, coeffs = C.zz_x_observable(n)
    f, grad = G.parameter_shift(n, chi, gates, pidx, labels, coeffs, ctx=cuda_ctx)
    lists, owner = G.shifted_circuits(gates, pidx)
    vals = []
    for g in lists:
        o = O.run(n, chi, g)
        assert max(o.bond_dims()) <= chi
        vals.append(o.expectation(labels, coeffs).real)
    want = np.zeros_like(grad)
    for k, p in enumerate(owner):
        want[p] += 0.5 * (vals[1 + 2 * k] - vals[2 + 2 * k])
    assert abs(f - vals[0]) <= 1e-10 * max(1.0, abs(vals[0]))
    assert np.abs(grad - want).max() <= 1e-10 * max(1.0, np.abs(want).max())
