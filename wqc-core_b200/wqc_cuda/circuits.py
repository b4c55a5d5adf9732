"""Gate records and seeded synthetic circuits for the MPS workloads.

A gate is one ``wqc_gate`` record (include/wqc_types.h): ``kind`` in the order
of the reference's ``Gate`` enum (src/engine.rs), three qubit operands and an
angle.  The generators build the five workload shapes the backend is measured
on; each is seeded with numpy's PCG64 so a circuit is reproducible from
(generator, seed).  They are synthetic stand-ins: the reference ships no
circuit files for these shapes.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

H, X, Y, Z, S, T, RX, RY, RZ, CNOT, CZ, CCNOT, MEASURE, RESET, IF = range(15)
ONE_QUBIT = (H, X, Y, Z, S, T, RX, RY, RZ)
NAMES = ["H", "X", "Y", "Z", "S", "T", "RX", "RY", "RZ", "CNOT", "CZ", "CCNOT", "MEASURE", "RESET", "IF"]

GATE_DTYPE = np.dtype(
    [("kind", "<i4"), ("q0", "<i4"), ("q1", "<i4"), ("q2", "<i4"), ("angle", "<f8")], align=True
)
assert GATE_DTYPE.itemsize == 24

SPLIT_INFO_DTYPE = np.dtype(
    [
        ("left_site", "<i4"),
        ("rows", "<i4"),
        ("cols", "<i4"),
        ("ell", "<i4"),
        ("path", "<i4"),
        ("chi", "<i4"),
        ("discarded_weight", "<f8"),
    ],
    align=True,
)
assert SPLIT_INFO_DTYPE.itemsize == 32


def gates_array(gates) -> np.ndarray:
    """Pack a list of (kind, q0, q1, q2, angle) tuples into wqc_gate records."""
    arr = np.zeros(len(gates), dtype=GATE_DTYPE)
    for i, g in enumerate(gates):
        kind = g[0]
        qs = list(g[1:-1]) if len(g) > 2 else [g[1]]
        angle = g[-1] if len(g) > 2 else 0.0
        arr[i]["kind"] = kind
        for j, q in enumerate(qs[:3]):
            arr[i][f"q{j}"] = q
        arr[i]["angle"] = angle
    return arr


def g1(kind: int, q: int, angle: float = 0.0):
    return (kind, q, 0, 0, float(angle))


def g2(kind: int, c: int, t: int):
    return (kind, c, t, 0, 0.0)


def g3(c1: int, c2: int, t: int):
    return (CCNOT, c1, c2, t, 0.0)


@dataclass
class Workload:
    name: str
    n: int
    chi: int
    gates: np.ndarray
    seed: int

    @property
    def logical_two_qubit(self) -> int:
        k = self.gates["kind"]
        return int(np.count_nonzero((k == CNOT) | (k == CZ)) + np.count_nonzero(k == CCNOT))

    def layer_starts(self) -> list:
        """Gate index where each layer begins: every generator opens a layer
        with a one-qubit gate on qubit 0."""
        k, q0 = self.gates["kind"], self.gates["q0"]
        first = np.isin(k, ONE_QUBIT) & (q0 == 0)
        return [i for i in range(len(k)) if first[i] and (i == 0 or not first[i - 1])]


def ry_rz_brickwork(n: int, depth: int, seed: int) -> list:
    """RY(theta) and RZ(phi) on every qubit (angles U[0, 2pi)), then CNOT on
    even pairs (0-1, 2-3, ...) on even layers and odd pairs on odd layers."""
    rng = np.random.Generator(np.random.PCG64(seed))
    gates = []
    for layer in range(depth):
        for q in range(n):
            gates.append(g1(RY, q, rng.uniform(0.0, 2.0 * math.pi)))
            gates.append(g1(RZ, q, rng.uniform(0.0, 2.0 * math.pi)))
        for q in range(layer % 2, n - 1, 2):
            gates.append(g2(CNOT, q, q + 1))
    return gates


def config0(seed: int = 20261203) -> Workload:
    """16 qubits, depth 20 RY/RZ + alternating CNOT brickwork, chi_max = 32."""
    return Workload("brickwork16_d20_chi32", 16, 32, gates_array(ry_rz_brickwork(16, 20, seed)), seed)


def random_layers(n: int, depth: int, seed: int, long_range_frac: float = 0.1) -> list:
    """Per layer each qubit gets one of {H, T, S, RX, RY, RZ} (angles U[0, 2pi));
    then CZ or CNOT (50/50, random orientation) on the alternating even/odd
    nearest-neighbour pairs; then round(frac * n) extra CNOTs at distance
    U{2..8}, which the executor routes with SWAPs."""
    rng = np.random.Generator(np.random.PCG64(seed))
    gates = []
    extra = int(round(long_range_frac * n))
    for layer in range(depth):
        for q in range(n):
            k = int(rng.integers(0, 6))
            kind = (H, T, S, RX, RY, RZ)[k]
            ang = rng.uniform(0.0, 2.0 * math.pi) if kind in (RX, RY, RZ) else 0.0
            gates.append(g1(kind, q, ang))
        for q in range(layer % 2, n - 1, 2):
            kind = CZ if rng.integers(0, 2) == 0 else CNOT
            if rng.integers(0, 2) == 0:
                gates.append(g2(kind, q, q + 1))
            else:
                gates.append(g2(kind, q + 1, q))
        for _ in range(extra):
            d = int(rng.integers(2, 9))
            lo = int(rng.integers(0, n - d))
            hi = lo + d
            if rng.integers(0, 2) == 0:
                gates.append(g2(CNOT, lo, hi))
            else:
                gates.append(g2(CNOT, hi, lo))
    return gates


def config1(n: int = 50, depth: int = 40, chi: int = 128, seed: int = 20261204) -> Workload:
    """50 qubits, depth 40 random 1q layer + CZ/CNOT brickwork + 10% long-range CNOTs, chi_max = 128."""
    return Workload(f"random{n}_d{depth}_chi{chi}", n, chi, gates_array(random_layers(n, depth, seed)), seed)


def config2_slices(count: int = 512, seed: int = 20261205):
    """Independent slices: width U[20, 60], depth U[10, 50], chi_max from {16, 32, 64, 128},
    each a RY/RZ + CNOT brickwork with its own seed."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(count):
        n = int(rng.integers(20, 61))
        depth = int(rng.integers(10, 51))
        chi = int((16, 32, 64, 128)[int(rng.integers(0, 4))])
        s = int(rng.integers(0, 2**62))
        out.append(Workload(f"slice{i}", n, chi, gates_array(ry_rz_brickwork(n, depth, s)), s))
    return out


def hea_ansatz(n: int = 32, layers: int = 8, seed: int = 20261206):
    """Hardware-efficient ansatz: per layer RY(theta) then RZ(theta') on every qubit,
    then a CZ ladder 0-1, 1-2, ..., (n-2)-(n-1).  Returns (gates, parameter index per gate or -1)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    params = rng.uniform(0.0, 2.0 * math.pi, size=2 * n * layers)
    gates, pidx = [], []
    p = 0
    for _ in range(layers):
        for q in range(n):
            gates.append(g1(RY, q, params[p])); pidx.append(p); p += 1
            gates.append(g1(RZ, q, params[p])); pidx.append(p); p += 1
        for q in range(n - 1):
            gates.append(g2(CZ, q, q + 1)); pidx.append(-1)
    return gates_array(gates), np.array(pidx, dtype=np.int64), params


def hea_checkpoints(n: int, layers: int, every: int = 2) -> np.ndarray:
    """Gate indices of the first gate of every `every`-th layer of
    hea_ansatz(n, layers) after the first (the adjoint's checkpoints)."""
    per_layer = 2 * n + (n - 1)
    return np.array([L * per_layer for L in range(every, layers, every)], dtype=np.uint32)


def zz_x_observable(n: int):
    """sum_i Z_i Z_{i+1} + 0.5 sum_i X_i as (labels, coefficients); label
    character n-1-q acts on qubit q."""
    labels, coeffs = [], []
    for i in range(n - 1):
        lab = ["I"] * n
        lab[n - 1 - i] = "Z"
        lab[n - 1 - (i + 1)] = "Z"
        labels.append("".join(lab)); coeffs.append(1.0)
    for i in range(n):
        lab = ["I"] * n
        lab[n - 1 - i] = "X"
        labels.append("".join(lab)); coeffs.append(0.5)
    return labels, np.array(coeffs, dtype=np.complex128)


def large_chi(n: int = 100, depth: int = 100, seed: int = 20261207) -> list:
    """Blocks RZ.RY.RZ on both qubits, CNOT, RY on both, CNOT, RZ.RY.RZ on both,
    on alternating even/odd nearest-neighbour pairs; every 10th layer adds a
    CCNOT on a random adjacent triple and an H layer."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ang = lambda: rng.uniform(0.0, 2.0 * math.pi)  # noqa: E731
    gates = []
    for layer in range(depth):
        for q in range(layer % 2, n - 1, 2):
            for w in (q, q + 1):
                gates += [g1(RZ, w, ang()), g1(RY, w, ang()), g1(RZ, w, ang())]
            gates.append(g2(CNOT, q, q + 1))
            gates += [g1(RY, q, ang()), g1(RY, q + 1, ang())]
            gates.append(g2(CNOT, q, q + 1))
            for w in (q, q + 1):
                gates += [g1(RZ, w, ang()), g1(RY, w, ang()), g1(RZ, w, ang())]
        if layer % 10 == 9:
            a = int(rng.integers(0, n - 2))
            gates.append(g3(a, a + 1, a + 2))
            gates += [g1(H, q) for q in range(n)]
    return gates


def config4(depth: int = 100, seed: int = 20261207) -> Workload:
    """100 qubits, depth 100 blocks (large_chi), chi_max = 256: theta up to 512 x 512."""
    return Workload(f"blocks100_d{depth}_chi256", 100, 256, gates_array(large_chi(100, depth, seed)), seed)


def split_plan(gates: np.ndarray) -> int:
    """Number of two-site splits the reference performs for this gate list
    (SWAP routing at mps.rs:353-375, CCNOT as 6 CNOTs at mps.rs:657-677)."""
    total = 0
    for g in gates:
        k = int(g["kind"])
        if k in (CNOT, CZ):
            d = abs(int(g["q0"]) - int(g["q1"]))
            total += 1 + 2 * (d - 1)
        elif k == CCNOT:
            c1, c2, t = int(g["q0"]), int(g["q1"]), int(g["q2"])
            for a, b in ((c2, t), (c1, t), (c2, t), (c1, t), (c1, c2), (c1, c2)):
                total += 1 + 2 * (abs(a - b) - 1)
    return total


def ry_cnot_brickwork(n: int, depth: int) -> np.ndarray:
    """Layers of RY(0.17 + 0.01 (q + layer)) on every qubit, then CNOT on
    alternating neighbour pairs (the exact-tree workload of
    src/tn/plan.rs:396-410)."""
    gates = []
    for layer in range(depth):
        for q in range(n):
            gates.append(g1(RY, q, 0.17 + 0.01 * (q + layer)))
        for q in range(layer % 2, n - 1, 2):
            gates.append(g2(CNOT, q, q + 1))
    return gates_array(gates)


def star(n: int) -> np.ndarray:
    """H on qubit 0, then CNOT(0, q) for every other qubit (a GHZ star,
    src/tn/exact.rs:668-676)."""
    return gates_array([g1(H, 0)] + [g2(CNOT, 0, q) for q in range(1, n)])


def ry_rz_cnot_brickwork(n: int, depth: int) -> np.ndarray:
    """Layers of RY(0.17 + 0.013 (q + 3 layer)) and RZ(0.31 + 0.007 (2q + layer))
    on every qubit, then CNOT on alternating neighbour pairs (the network-tree
    workload of src/tn/network.rs:1022-1036)."""
    gates = []
    for layer in range(depth):
        for q in range(n):
            gates.append(g1(RY, q, 0.17 + 0.013 * (q + 3 * layer)))
            gates.append(g1(RZ, q, 0.31 + 0.007 * (2 * q + layer)))
        for q in range(layer % 2, n - 1, 2):
            gates.append(g2(CNOT, q, q + 1))
    return gates_array(gates)


def grid(side: int, depth: int) -> np.ndarray:
    """RY(0.17) and RZ(0.31) on every qubit of a side x side grid, then CNOTs
    on alternating pairs, two layers along rows and two along columns (the
    orchestrator's grid circuit, src/tn/network.rs:1114-1139)."""
    gates = []
    at = lambda row, col: row * side + col  # noqa: E731
    for layer in range(depth):
        for q in range(side * side):
            gates.append(g1(RY, q, 0.17))
            gates.append(g1(RZ, q, 0.31))
        if layer % 4 < 2:
            for row in range(side):
                for col in range(layer % 2, side - 1, 2):
                    gates.append(g2(CNOT, at(row, col), at(row, col + 1)))
        else:
            for row in range(layer % 2, side - 1, 2):
                for col in range(side):
                    gates.append(g2(CNOT, at(row, col), at(row + 1, col)))
    return gates_array(gates)
