"""The MpsState call pattern of the reference's trace loop, for registers of
more than 16 qubits (src/tn/trace.rs:55-187, 264-411, 619-657).

``execute_with_trace_using`` walks the gate list in steps:

* a run of H on one qubit: the even part applied silently, an odd remainder
  as one traced H (trace.rs:78-97);
* a run of same-axis rotations on one qubit: one net-angle gate, or, when
  the angles add to a full turn, every gate applied with no trace row
  (trace.rs:99-129, 203-230);
* above 16 qubits, a run of at least two qubit-disjoint adjacent CNOT/CZ:
  one ``apply_adjacent_disjoint_gates`` call (trace.rs:135-154, 243-262);
* any other gate on its own.

Before each traced step it reads the state: the control probability of
every control of the step's gates (``control_probability``, trace.rs:649-656)
and, the first time a qubit is a step's logical target, that target's
``site_amplitudes`` (``resolve_pre_amps``, trace.rs:375-411); later rows of
that target reuse the post amplitudes the AIR formulas give, with no read.
A disjoint layer reads for every gate of the layer before it applies any
(``emit_disjoint_layer``, trace.rs:264-315).  The reads of one step are one
``site_amplitudes_many`` call here: the state does not change between them.

The trace rows themselves (Mersenne-31 AIR values, STARK) stay with the
caller; what this module reproduces is the sequence of state operations and
reads that the backend serves.  Registers of at most 16 qubits sample a
dense slice instead (trace.rs:391-400), which this module does not model.
"""
from __future__ import annotations

import math

import numpy as np

from .circuits import CCNOT, CNOT, CZ, GATE_DTYPE, H, IF, MEASURE, RESET, RX, RY, RZ

_SKIP = (MEASURE, RESET, IF)
_TAU = 2.0 * math.pi


def _identity_rotation(angle_sum: float) -> bool:
    """trace.rs:317-320."""
    reduced = math.fmod(angle_sum, _TAU)
    if reduced < 0:
        reduced += _TAU
    return abs(reduced) < 1e-9 or abs(_TAU - reduced) < 1e-9


def _disjoint_len(gates, i: int) -> int:
    """adjacent_disjoint_len (trace.rs:243-262)."""
    seen = set()
    n = 0
    for g in gates[i:]:
        k = int(g["kind"])
        if k not in (CNOT, CZ):
            break
        c, t = int(g["q0"]), int(g["q1"])
        if abs(c - t) != 1:
            break
        lo, hi = min(c, t), max(c, t)
        if lo in seen or hi in seen:
            break
        seen.update((lo, hi))
        n += 1
    return n if n >= 2 else 0


def steps(n: int, gates):
    """The steps of execute_with_trace_using for this gate list: tuples
    (kind, gate records to apply, gate records traced), kind in 'silent',
    'one', 'net', 'layer'."""
    gates = np.asarray(gates, dtype=GATE_DTYPE)
    out = []
    i = 0
    while i < len(gates):
        g = gates[i]
        k = int(g["kind"])
        if k in _SKIP:
            i += 1
            continue
        if k == H:
            run = 1
            while i + run < len(gates) and int(gates[i + run]["kind"]) == H and gates[i + run]["q0"] == g["q0"]:
                run += 1
            silent = run - run % 2
            if silent:
                out.append(("silent", gates[i:i + silent], gates[0:0]))
            if run % 2:
                out.append(("one", gates[i + silent:i + run], gates[i + silent:i + run]))
            i += run
            continue
        if k in (RX, RY, RZ):
            run, total = 1, float(g["angle"])
            while i + run < len(gates) and int(gates[i + run]["kind"]) == k and gates[i + run]["q0"] == g["q0"]:
                total += float(gates[i + run]["angle"])
                run += 1
            if _identity_rotation(total):
                out.append(("silent", gates[i:i + run], gates[0:0]))
            else:
                net = gates[i:i + 1].copy()
                net["angle"] = total
                out.append(("net", net, net))
            i += run
            continue
        layer = _disjoint_len(gates, i) if n > 16 else 0
        if layer >= 2:
            out.append(("layer", gates[i:i + layer], gates[i:i + layer]))
            i += layer
            continue
        out.append(("one", gates[i:i + 1], gates[i:i + 1]))
        i += 1
    return out


def _controls(g):
    k = int(g["kind"])
    if k in (CNOT, CZ):
        return [int(g["q0"])]
    if k == CCNOT:
        return [int(g["q0"]), int(g["q1"])]
    return []


def _target(g) -> int:
    k = int(g["kind"])
    if k in (CNOT, CZ):
        return int(g["q1"])
    if k == CCNOT:
        return int(g["q2"])
    return int(g["q0"])


def replay(state, n: int, gates):
    """Run the trace loop's state operations and reads on `state` (a CudaMps,
    or any object with apply_gates, apply_adjacent_disjoint_gates and
    site_amplitudes_many).  Returns the reads in order: one (targets,
    amplitudes) pair per step that reads, amplitudes of shape
    (len(targets), 2) holding (a0, a1) of each target; the control
    probability of a control c is |a1|^2 of its entry."""
    if n <= 16:
        raise ValueError("registers of at most 16 qubits sample a dense slice (trace.rs:391-400)")
    seen = set()
    reads = []
    for kind, apply, traced in steps(n, gates):
        targets = []
        for g in traced:
            targets += _controls(g)
            t = _target(g)
            if t not in seen:
                targets.append(t)
                seen.add(t)
        if targets:
            reads.append((np.array(targets, dtype=np.uint32), state.site_amplitudes_many(targets)))
        if kind == "layer":
            state.apply_adjacent_disjoint_gates(apply)
        else:
            state.apply_gates(apply)
    return reads
