"""The differentiation form's adjoint (wqc_adjoint_forward / _backward)
through the C ABI:

* against the numpy restatement of the same reverse sweep (oracle/adjoint.py,
  itself pinned to central differences on the CPU) on truncating circuits:
  every per-gate derivative;
* against central differences of the device's own forward (h = 1e-4), with
  routed long-range CNOTs and a CCNOT in the circuit;
* against the parameter-shift rule where nothing is truncated (the two are
  then the same derivative);
* on the 32-qubit, 8-layer ansatz at chi 64 with checkpoints every 2
  layers: the value and 16 derivatives against central differences, and the
  distance to the oracle's parameter-shift estimate, which through the
  truncating splits is not the derivative of the truncated map.
"""
import os

import numpy as np
import pytest

import adjoint as A
import wqc_cuda as W
from wqc_cuda import circuits as C
from wqc_cuda import gradients as G

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def device_value(n, chi, gates, labels, coeffs, ctx):
    m = W.CudaMps(n, chi, ctx=ctx)
    m.set_split_rule(W.SPLIT_RULE_EXACT)
    m.apply_gates(gates)
    v = m.expectation(labels, coeffs).real
    m.close()
    return v


def central_differences(n, chi, gates, idx, labels, coeffs, ctx, h=1e-4):
    out = []
    for i in idx:
        gp, gm = gates.copy(), gates.copy()
        gp["angle"][i] += h
        gm["angle"][i] -= h
        out.append((device_value(n, chi, gp, labels, coeffs, ctx) - device_value(n, chi, gm, labels, coeffs, ctx))
                   / (2 * h))
    return np.array(out)


@pytest.mark.parametrize("n,layers,chi", [(8, 3, 4), (10, 4, 8), (8, 2, 64)])
def test_adjoint_matches_numpy_reverse_sweep(cuda_ctx, n, layers, chi):
    gates, pidx, _ = C.hea_ansatz(n, layers, seed=n + layers)
    labels, coeffs = C.zz_x_observable(n)
    m = W.CudaMps(n, chi, ctx=cuda_ctx)
    adj = W.Adjoint(m, gates, C.hea_checkpoints(n, layers, 1))
    f, g = adj.backward(labels, coeffs)
    fr, gr = A.gradient(n, chi, gates, labels, coeffs)
    assert abs(f - fr) <= 1e-11
    assert np.abs(g - gr).max() <= 1e-9 * max(1.0, np.abs(gr).max())
    # a second observable on the same forward
    f2, g2 = adj.backward(["Z" * n], [1.0])
    fr2, gr2 = A.gradient(n, chi, gates, ["Z" * n], [1.0])
    assert abs(f2 - fr2) <= 1e-11 and np.abs(g2 - gr2).max() <= 1e-9 * max(1.0, np.abs(gr2).max())


def test_adjoint_with_routed_gates_matches_central_differences(cuda_ctx):
    n, chi = 10, 8
    rng = np.random.default_rng(77)
    g = []
    for layer in range(5):
        for q in range(n):
            g.append(C.g1((C.RX, C.RY, C.RZ)[int(rng.integers(0, 3))], q, rng.uniform(0, 2 * np.pi)))
        for q in range(layer % 2, n - 1, 2):
            g.append(C.g2(C.CNOT if rng.random() < 0.5 else C.CZ, q, q + 1))
        a = int(rng.integers(0, n - 4))
        g.append(C.g2(C.CNOT, a + 4, a))
    g.insert(25, C.g3(2, 6, 4))
    g.append(C.g1(C.T, 3))
    gates = C.gates_array(g)
    labels = ["".join(rng.choice(list("IXYZ"), size=n)) for _ in range(6)]
    coeffs = rng.normal(size=6) + 0.3j
    m = W.CudaMps(n, chi, ctx=cuda_ctx)
    adj = W.Adjoint(m, gates, [20, 44, 71])
    f, grad = adj.backward(labels, coeffs)
    assert abs(f - device_value(n, chi, gates, labels, coeffs, cuda_ctx)) <= 1e-11
    rot = np.nonzero(np.isin(gates["kind"], [C.RX, C.RY, C.RZ]))[0]
    pick = rot[np.linspace(0, len(rot) - 1, 12).astype(int)]
    fd = central_differences(n, chi, gates, pick, labels, coeffs, cuda_ctx)
    assert np.abs(grad[pick] - fd).max() <= 1e-6 * max(1.0, np.abs(fd).max())
    assert np.all(grad[np.isin(gates["kind"], [C.CNOT, C.CZ, C.CCNOT, C.T])] == 0.0)


def test_adjoint_equals_parameter_shift_without_truncation(cuda_ctx):
    n, layers, chi = 10, 4, 32  # 2^5 = 32: no split truncates
    gates, pidx, _ = C.hea_ansatz(n, layers, seed=3)
    labels, coeffs = C.zz_x_observable(n)
    f, g = W.adjoint_gradient(n, chi, gates, pidx, labels, coeffs, C.hea_checkpoints(n, layers), ctx=cuda_ctx)
    fs, gs = G.parameter_shift(n, chi, gates, pidx, labels, coeffs, ctx=cuda_ctx)
    assert abs(f - fs) <= 1e-11
    assert np.abs(g - gs).max() <= 1e-10


def test_config3_adjoint_against_differences_and_shift(cuda_ctx):
    fx = np.load(os.path.join(GOLDEN, "config3_hea.npz"))
    n, layers, chi = int(fx["n"]), int(fx["layers"]), int(fx["chi"])
    gates, pidx, _ = C.hea_ansatz(n, layers)
    labels, coeffs = C.zz_x_observable(n)
    f, grad = W.adjoint_gradient(n, chi, gates, pidx, labels, coeffs, C.hea_checkpoints(n, layers, 2), ctx=cuda_ctx)
    assert abs(f - float(fx["value"])) <= 1e-10
    params = fx["params"]
    inst = np.array([int(np.nonzero(pidx == p)[0][0]) for p in params])
    fd = central_differences(n, chi, gates, inst, labels, coeffs, cuda_ctx)
    assert np.abs(grad[params] - fd).max() <= 1e-6
    # the shift rule applied to truncated evaluations is not the truncated
    # map's derivative; at chi 64 they differ by the truncation's effect
    assert np.abs(grad[params] - fx["shift_grad"]).max() <= 1e-3
