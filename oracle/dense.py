"""ORACLE — test infrastructure only.

Dense 2^N statevector restating the reference's test oracle
(src/tn/dense.rs:12-170) and Pauli expectations (src/expectation.rs:98-167).
Qubit q is bit q of the basis index.  Used to pin the FP64 MPS oracle.
"""
from __future__ import annotations

import math

import numpy as np

H, X, Y, Z, S, T, RX, RY, RZ, CNOT, CZ, CCNOT, MEASURE, RESET, IF = range(15)


def unary(kind: int, theta: float = 0.0) -> np.ndarray:
    """gates.rs:10-66 (row = output amplitude, column = input)."""
    if kind == H:
        k = 1.0 / math.sqrt(2.0)
        return np.array([[k, k], [k, -k]], dtype=complex)
    if kind == X:
        return np.array([[0, 1], [1, 0]], dtype=complex)
    if kind == Y:
        return np.array([[0, -1j], [1j, 0]], dtype=complex)
    if kind == Z:
        return np.array([[1, 0], [0, -1]], dtype=complex)
    if kind == S:
        return np.array([[1, 0], [0, 1j]], dtype=complex)
    if kind == T:
        r = 0.70710678118654752440
        return np.array([[1, 0], [0, complex(r, r)]], dtype=complex)
    s, c = math.sin(theta / 2.0), math.cos(theta / 2.0)
    if kind == RX:
        return np.array([[c, -1j * s], [-1j * s, c]], dtype=complex)
    if kind == RY:
        return np.array([[c, -s], [s, c]], dtype=complex)
    if kind == RZ:
        return np.array([[complex(c, -s), 0], [0, complex(c, s)]], dtype=complex)
    raise ValueError(kind)


class Dense:
    def __init__(self, n: int):
        if n <= 0 or n > 26:
            raise ValueError("dense oracle holds 1..26 qubits")
        self.n = n
        self.state = np.zeros(1 << n, dtype=np.complex128)
        self.state[0] = 1.0

    def _view(self, q: int):
        # axes ordered from the most significant bit; qubit q is axis n-1-q
        return self.state.reshape([2] * self.n), self.n - 1 - q

    def apply_unary(self, q: int, u: np.ndarray) -> None:
        st, ax = self._view(q)
        st = np.moveaxis(st, ax, 0)
        v0, v1 = st[0].copy(), st[1].copy()
        st[0] = u[0, 0] * v0 + u[0, 1] * v1
        st[1] = u[1, 0] * v0 + u[1, 1] * v1

    def apply_controlled(self, c: int, t: int, u: np.ndarray) -> None:
        idx = np.arange(1 << self.n)
        sel = ((idx >> c) & 1 == 1) & ((idx >> t) & 1 == 0)
        i0 = idx[sel]
        i1 = i0 | (1 << t)
        v0, v1 = self.state[i0].copy(), self.state[i1].copy()
        self.state[i0] = u[0, 0] * v0 + u[0, 1] * v1
        self.state[i1] = u[1, 0] * v0 + u[1, 1] * v1

    def apply_gate(self, g) -> None:
        kind = int(g["kind"])
        if kind in (H, X, Y, Z, S, T, RX, RY, RZ):
            self.apply_unary(int(g["q0"]), unary(kind, float(g["angle"])))
        elif kind == CNOT:
            self.apply_controlled(int(g["q0"]), int(g["q1"]), unary(X))
        elif kind == CZ:
            self.apply_controlled(int(g["q0"]), int(g["q1"]), unary(Z))
        elif kind == CCNOT:
            c1, c2, t = int(g["q0"]), int(g["q1"]), int(g["q2"])
            idx = np.arange(1 << self.n)
            sel = ((idx >> c1) & 1 == 1) & ((idx >> c2) & 1 == 1) & ((idx >> t) & 1 == 0)
            i0 = idx[sel]
            i1 = i0 | (1 << t)
            self.state[i0], self.state[i1] = self.state[i1].copy(), self.state[i0].copy()

    def apply_gates(self, gates) -> None:
        for g in gates:
            self.apply_gate(g)


def pauli_expectation(state: np.ndarray, label: str) -> float:
    """expectation.rs:140-167: label character n-1-q acts on qubit q."""
    n = len(label)
    idx = np.arange(1 << n)
    j = idx.copy()
    phase = np.ones(1 << n, dtype=complex)
    for q in range(n):
        ch = label[n - 1 - q]
        bit = (idx >> q) & 1
        if ch == "Z":
            phase *= np.where(bit == 1, -1.0, 1.0)
        elif ch == "X":
            j ^= 1 << q
        elif ch == "Y":
            j ^= 1 << q
            phase *= np.where(bit == 0, 1j, -1j)
        elif ch != "I":
            raise ValueError(ch)
    return float(np.sum(np.conj(state[j]) * phase * state).real)
