"""Gradients of a Pauli-sum expectation by the parameter-shift rule, on the
batching form.

For a rotation exp(-i theta P / 2) (RX, RY, RZ: src/tn/gates.rs:10-66) the
derivative of f = <psi|O|psi> is [f(theta + pi/2) - f(theta - pi/2)] / 2.
Every parametrised gate instance gives two shifted circuits; all of them,
plus the unshifted one, run as slices of one batch state, and
wqc_batch_expectation_pauli evaluates O on every slice.  Gradients of
parameters shared by several gate instances are summed over the instances.
Through truncating splits this is the shift rule applied to the truncated
evaluations (what a parameter-shift run of the reference's CPU path gives at
the same chi), not the derivative of the truncated map.
"""
from __future__ import annotations

import math

import numpy as np

from . import CudaBatch, Context, PRECISION_FP64


def shifted_circuits(gates: np.ndarray, pidx: np.ndarray):
    """[unshifted, +pi/2 on instance 0, -pi/2 on instance 0, ...] and the
    parameter index of each instance."""
    inst = np.nonzero(pidx >= 0)[0]
    lists = [gates]
    for i in inst:
        for sgn in (1.0, -1.0):
            g = gates.copy()
            g["angle"][i] += sgn * math.pi / 2.0
            lists.append(g)
    return lists, pidx[inst]


def parameter_shift(n: int, chi: int, gates: np.ndarray, pidx: np.ndarray, labels, coeffs,
                    ctx: Context | None = None, precision: int = PRECISION_FP64):
    """(f, df/dparams): f = Re sum_t coeff_t <psi|P_t|psi> at the given angles."""
    lists, owner = shifted_circuits(gates, pidx)
    b = CudaBatch([n] * len(lists), [chi] * len(lists), ctx=ctx, precision=precision)
    try:
        b.apply_slices(lists)
        vals = b.expectations(labels, coeffs).real
    finally:
        b.close()
    grad = np.zeros(int(pidx.max()) + 1 if pidx.size and pidx.max() >= 0 else 0)
    for k, p in enumerate(owner):
        grad[p] += 0.5 * (vals[1 + 2 * k] - vals[2 + 2 * k])
    return float(vals[0]), grad
