"""Benchmark of the cuda MPS backend: two-site applies per second.

The workload is the 50-qubit, depth-40 random circuit at chi_max 128 (random
1q layer, CZ/CNOT brickwork, 10% long-range CNOTs routed with SWAPs) in the
plain FP64 form with the reference's split rule, from |0...0> to
<0...0|psi>.  The metric counts every merge + gate + split (SWAPs and
CCNOT-internal CNOTs included), the unit the reference's cost is made of.

Both arms time the same gates.  The first 10 layers (the bonds grow to
chi_max there) run untimed; the rest of the circuit (gates 795..3180, 2089
of its 2804 splits, all at the saturated shapes) is the timed range.  The
CUDA arm times the whole range in every step, each from the prefix state
(rerun untimed), with CUDA events on the state's stream (`value`) and with
the wall clock around the C ABI calls, plan upload and result read included
(`e2e`).  `--impl reference` runs the same prefix and then the same range on
the FP64 CPU restatement of the reference path, one independent replica per
host core, cut into K consecutive windows so that one pass of the range is
spread over its K steps.  The whole circuit from |0...0> is reported beside
the range (`whole_circuit`), and the same circuit under the exact split
rule, checked against the committed oracle fixture, as `exact_rule`.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]

With N > 1 (torchrun, one rank per GPU) every rank runs its own replica: a
single circuit is a chain of dependent splits and does not shard, so the
scaling is weak and there is no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "wqc-core_b200"))

import numpy as np  # noqa: E402

from wqc_cuda import circuits as C  # noqa: E402

METRIC = "2q-gate applies/s"
UNIT = "2q applies/s"


def workload(name: str, depth: int = 0):
    if name == "config0":
        w = C.config0()
    elif name == "config4":
        w = C.config4(depth or 100)
    else:
        w = C.config1(depth=depth or 40)
    return w


def timed_windows(w, skip_layers: int, k: int):
    """(g0, windows): the first `skip_layers` layers end at gate g0 and run
    untimed; gates g0.. are cut into k consecutive windows of about equal
    gate count, one per timed step."""
    starts = w.layer_starts()
    g0 = starts[skip_layers] if 0 < skip_layers < len(starts) else 0
    k = max(1, min(k, len(w.gates) - g0))
    edges = np.linspace(g0, len(w.gates), k + 1).round().astype(int)
    return g0, [(int(edges[i]), int(edges[i + 1])) for i in range(k)]


def workload_config(w, rule: str, g0: int, windows) -> dict:
    """The workload; `windows` are the reference arm's K windows of the
    timed range (the CUDA arm times the whole range in each step)."""
    timed = w.gates[g0:]
    return {
        "workload": f"{w.name}: {w.n} qubits, chi_max {w.chi}, plain FP64 (complex128), split rule {rule}",
        "qubits": w.n,
        "chi_max": w.chi,
        "gates": int(len(w.gates)),
        "logical_2q_gates": w.logical_two_qubit,
        "splits_per_circuit": C.split_plan(w.gates),
        "timed_gates": [g0, int(len(w.gates))],
        "timed_splits": C.split_plan(timed),
        "steps_are": f"the timed range is gates {g0}..{len(w.gates)}, after an untimed prefix of gates 0..{g0} "
                     f"(the layers in which the bonds grow to chi_max); the CUDA arm times the whole range in each "
                     f"step from the prefix state, the reference arm spreads one pass of the range over its steps "
                     f"as {len(windows)} consecutive windows",
        "seed": w.seed,
        "split_rule": rule,
        "l2": "flushed between steps (256 MiB device write outside the timed events)",
        "parallelism": "replicas (one circuit per GPU)",
    }


# ---------------------------------------------------------------------------
# CPU leg: the oracle (FP64 restatement of the reference CPU path)
# ---------------------------------------------------------------------------
def oracle_windows(w, g0: int, windows, threads: int, budget_s: float = 0.0):
    """The CPU restatement on `threads` independent replicas (one thread
    each): gates 0..g0 untimed, then the windows in order, each timed with its
    closing <0...0|psi> read.  With budget_s > 0 a replica stops after the
    window that crosses the budget.  Returns (splits of the timed windows
    over all replicas, the slowest replica's timed seconds, windows done by
    replica 0)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    O.lib()
    done = [0] * threads
    secs = [0.0] * threads
    wins = [0] * threads
    barrier = threading.Barrier(threads)

    def worker(t):
        m = O.OracleMps(w.n, w.chi)
        if g0:
            m.apply_gates(w.gates[:g0])
        m.amplitude_zero()
        before = len(m.records())
        barrier.wait()
        for a, b in windows:
            t0 = time.perf_counter()
            m.apply_gates(w.gates[a:b])
            m.amplitude_zero()
            secs[t] += time.perf_counter() - t0
            wins[t] += 1
            if budget_s > 0 and secs[t] >= budget_s:
                break
        done[t] = len(m.records()) - before

    ths = [threading.Thread(target=worker, args=(t,)) for t in range(threads)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    return sum(done), max(secs), wins[0]


SATURATED_LAYERS = {"config1": 10, "config0": 4}


def oracle_batch_sample(slices, budget_s: float, threads: int):
    """CPU leg of the batching form: thread t runs slice t from |0...0> on the
    oracle, gate chunk by gate chunk, until `budget_s` seconds; returns (splits
    done by all threads, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    O.lib()
    done = [0] * threads
    secs = [0.0] * threads
    barrier = threading.Barrier(threads)

    def worker(t):
        s = slices[t % len(slices)]
        m = O.OracleMps(s.n, s.chi)
        barrier.wait()
        t0 = time.perf_counter()
        i = 0
        while i < len(s.gates) and time.perf_counter() - t0 < budget_s:
            m.apply_gates(s.gates[i:i + 16])
            i += 16
        secs[t] = time.perf_counter() - t0
        done[t] = len(m.records())

    ths = [threading.Thread(target=worker, args=(t,)) for t in range(threads)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    return sum(done), max(secs)


def precision_leg(W, torch, ctx, w, rule, steps: int, flush, fp64_value: float) -> dict:
    """The precision form (WQC_PRECISION_FP32: complex64 Jacobi sweeps with
    the accumulated V as each SVD's first phase, V made orthonormal in FP64,
    X V in FP64, FP64 sweeps to finish) on the whole headline circuit, and
    its error against FP64: on the 16-qubit chi 32 brickwork against the
    plain form (itself within 1e-12 of the FP64 oracle there), and on the
    headline circuit under the exact rule against the oracle's fixture."""
    m = W.CudaMps(w.n, w.chi, ctx=ctx, precision=W.PRECISION_FP32)
    m.set_split_rule(rule)
    stream = torch.cuda.ExternalStream(m.stream())
    total_ms, splits = 0.0, 0
    for k in range(steps + 1):
        m.reset()
        if k == 1:
            m.reset_stats()
        flush.fill_(float(np.random.random()))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m.apply_gates(w.gates)
        m.amplitude_at_compact_zero()
        e1.record(stream)
        e1.synchronize()
        if k > 0:  # the first pass is a warm-up
            total_ms += e0.elapsed_time(e1)
            splits += m.split_count()
    st = m.kernel_stats()
    m.close()
    value = splits / (total_ms * 1e-3)
    w0 = C.config0()
    amps = []
    for prec in (W.PRECISION_FP64, W.PRECISION_FP32):
        m0 = W.CudaMps(w0.n, w0.chi, ctx=ctx, precision=prec)
        m0.apply_gates(w0.gates)
        amps.append(m0.amplitude_at_compact_zero())
        m0.close()
    out = {
        "form": "each SVD: complex64 Jacobi sweeps (FP32 dot products and updates, FP64 rotation parameters and "
                "tests) carrying X V and V, then V orthonormalised (two Newton-Schulz steps), X V formed and FP64 "
                "sweeps to finish; sites, merge, range finder, sort and cut FP64",
        "value": value,
        "unit": UNIT,
        "steps": steps,
        "workload": "whole circuit from |0...0>, same as whole_circuit of the plain form",
        "speedup_vs_fp64": value / fp64_value,
        "sweeps_per_svd_first_phase": st["jacobi_sweeps_first"] / st["jacobi_tasks"] if st["jacobi_tasks"] else None,
        "sweeps_per_svd_fp64_finish": st["jacobi_sweeps"] / st["jacobi_tasks"] if st["jacobi_tasks"] else None,
        "amp_rel_err_vs_fp64": abs(amps[1] - amps[0]) / abs(amps[0]),
        "error_workload": f"{w0.name}: {w0.n} qubits, chi_max {w0.chi}",
    }
    fx = os.path.join(ROOT, "tests", "golden", "config1_exact.npz")
    if os.path.exists(fx) and w.n == 50:
        ref = np.load(fx)
        m1 = W.CudaMps(w.n, w.chi, ctx=ctx, precision=W.PRECISION_FP32)
        m1.set_split_rule(W.SPLIT_RULE_EXACT)
        m1.apply_gates(w.gates)
        rec = m1.split_records()
        norm2 = m1.expectation(["I" * w.n], [1.0]).real
        m1.close()
        rr = ref["records"]
        out["exact_rule_vs_oracle"] = {
            "chi_path_shape_bit_exact": bool(len(rr) == len(rec) and all(
                np.array_equal(rr[k], rec[k]) for k in ("left_site", "rows", "cols", "path", "chi"))),
            "max_weight_diff": float(np.max(np.abs(rr["discarded_weight"] - rec["discarded_weight"])))
            if len(rr) == len(rec) else None,
            "norm2_rel_err": abs(norm2 - float(ref["norm2"])) / float(ref["norm2"]),
            "note": "the 50-qubit state's norm^2 (1.2e-30 after 2804 truncating splits) against the FP64 oracle; "
                    "the oracle drifts against itself under a change of FP64 SVD by tests/golden/config1_drift.npz",
        }
    return out


def measured_tf32_peak(torch) -> float:
    """cuBLAS TF32 GEMM throughput (TFLOP/s, FP32 operands with TF32 tensor
    math), best of 5 on 8192^3: the roofline of the tensor-core GEMM."""
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    try:
        n = 8192
        a = torch.randn(n, n, dtype=torch.float32, device="cuda")
        b = torch.randn(n, n, dtype=torch.float32, device="cuda")
        torch.matmul(a, b)
        torch.cuda.synchronize()
        best = 0.0
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            e1.synchronize()
            best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
        del a, b
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old
    return best


def whole_circuit_profile(W, torch, ctx, w, rule, precision: int, flush, merge=None) -> tuple[float, int, dict]:
    """One untimed warm-up pass and one timed pass of the whole circuit from
    |0...0> with per-kernel events: (ms, splits, kernel milliseconds)."""
    m = W.CudaMps(w.n, w.chi, ctx=ctx, precision=precision)
    m.set_split_rule(rule)
    if merge is not None:
        m.set_merge(merge)
    stream = torch.cuda.ExternalStream(m.stream())
    ms = 0.0
    for k in range(2):
        m.reset()
        m.reset_stats()
        m.set_profiling(k == 1)
        flush.fill_(float(np.random.random()))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m.apply_gates(w.gates)
        m.amplitude_at_compact_zero()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
    m.set_profiling(False)
    st = m.kernel_stats()
    splits = m.split_count()
    m.close()
    return ms, splits, st["milliseconds"]


def tensor_core_leg(W, torch, ctx, w, rule, flush, gemm_only: bool = False) -> dict:
    """The tcgen05 complex GEMM (wqc_tc_zgemm: 3xTF32 split products, FP32
    accumulation in tensor memory, TMA-fed) on 4096^3 against cuBLAS TF32
    measured here, then the tensor-core form (WQC_PRECISION_TF32X3: every
    merge on that GEMM) on the whole headline circuit beside the plain form,
    and its error against FP64 on the 16-qubit chi 32 brickwork."""
    from wqc_cuda import tc as T

    peak = measured_tf32_peak(torch)
    rng = np.random.default_rng(2024)
    n = 4096
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    b = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    reps = 10
    c, ms = T.zgemm(a, b, reps=reps, ctx=ctx)
    rows = rng.choice(n, 64, replace=False)
    ref = a[rows] @ b
    err = float(np.linalg.norm(c[rows] - ref) / np.linalg.norm(ref))
    del a, b, c
    tensor = 24.0 * n ** 3 / (ms * 1e-3) / 1e12  # 3 products x 2 flops x m x 2n x 2k of the real embedding
    out = {
        "gemm": {
            "shape": f"complex {n} x {n} x {n}, operands resident, {reps} launches",
            "kernel_ms": ms,
            "complex_tflops": 8.0 * n ** 3 / (ms * 1e-3) / 1e12,
            "roofline": {"bound": "tensor", "achieved": tensor, "peak": peak, "unit": "TFLOP/s",
                         "frac": tensor / peak,
                         "peak_source": "cuBLAS TF32 GEMM (torch.matmul, FP32 8192^3, TF32 math) measured in this run",
                         "work": "24 m n k: three TF32 products (lo*hi, hi*lo, hi*hi) of the m x 2k by 2k x 2n "
                                 "real embedding"},
            "rel_err_vs_fp64": err,
            "error_sample": "64 random rows against numpy FP64",
        },
    }
    # the same product from int8 digit slices (45 slice products, exact int32
    # accumulation): FP64-level, on the integer tensor pipe
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    b = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    c, ms8 = T.zgemm(a, b, reps=5, ctx=ctx, form="int8")
    ref = a[rows] @ b
    err8 = float(np.linalg.norm(c[rows] - ref) / np.linalg.norm(ref))
    del a, b, c
    out["gemm_int8"] = {
        "shape": f"complex {n} x {n} x {n}, operands resident, 5 launches",
        "kernel_ms": ms8,
        "complex_tflops": 8.0 * n ** 3 / (ms8 * 1e-3) / 1e12,
        "int8_tops": 360.0 * n ** 3 / (ms8 * 1e-3) / 1e12,
        "work": "360 m n k int8 ops: 45 digit-slice products of the m x 2k by 2k x 2n real embedding",
        "rel_err_vs_fp64": err8,
        "error_sample": "64 random rows against numpy FP64",
    }
    if gemm_only:
        return out
    fp64_ms, fp64_splits, fp64_k = whole_circuit_profile(W, torch, ctx, w, rule, W.PRECISION_FP64, flush,
                                                         merge=W.MERGE_FFMA)
    i8_ms, i8_splits, i8_k = whole_circuit_profile(W, torch, ctx, w, rule, W.PRECISION_FP64, flush,
                                                   merge=W.MERGE_TC_INT8)
    out["int8_merge"] = {
        "form": "plain FP64 form with every merge from int8 digit slices on the tensor cores (WQC_MERGE_TC_INT8, "
                "the single-state default)",
        "value": i8_splits / (i8_ms * 1e-3),
        "ffma_value": fp64_splits / (fp64_ms * 1e-3),
        "unit": UNIT,
        "merge_ms": i8_k["merge_gate"],
        "ffma_merge_ms": fp64_k["merge_gate"],
    }
    tc_ms, tc_splits, tc_k = whole_circuit_profile(W, torch, ctx, w, rule, W.PRECISION_TF32X3, flush)
    w0 = C.config0()
    amps, recs = [], []
    for prec in (W.PRECISION_FP64, W.PRECISION_TF32X3):
        m0 = W.CudaMps(w0.n, w0.chi, ctx=ctx, precision=prec)
        m0.apply_gates(w0.gates)
        amps.append(m0.amplitude_at_compact_zero())
        recs.append(m0.split_records())
        m0.close()
    out["form"] = {
        "form": "WQC_PRECISION_TF32X3: every merge on the tcgen05 GEMM (theta in FP32-level precision, the 4x4 "
                "gate in FP64), the precision form's two-phase Jacobi, singular values below 1e-6 of the largest "
                "counted as zero",
        "workload": "whole circuit from |0...0>, one timed pass per form with per-kernel events",
        "value": tc_splits / (tc_ms * 1e-3),
        "fp64_value": fp64_splits / (fp64_ms * 1e-3),
        "unit": UNIT,
        "merge_ms": tc_k["merge_gate"],
        "fp64_merge_ms": fp64_k["merge_gate"],
        "fp64_merge": "FP64 FMA tiles",
        "splits": tc_splits,
        "fp64_splits": fp64_splits,
        "amp_rel_err_vs_fp64": abs(amps[1] - amps[0]) / abs(amps[0]),
        "kept_chi_differs": int(np.count_nonzero(recs[0]["chi"] != recs[1]["chi"])) if len(recs[0]) == len(recs[1])
        else None,
        "error_workload": f"{w0.name}: {w0.n} qubits, chi_max {w0.chi}, against the plain FP64 form",
    }
    return out


def oracle_gradient_sample(n, chi, lists, labels, coeffs, budget_s: float, threads: int):
    """CPU leg of the differentiation form: threads run whole shifted circuits
    (and the observable) on the oracle until `budget_s`; returns (circuits
    done, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    O.lib()
    done = [0] * threads
    secs = [0.0] * threads
    barrier = threading.Barrier(threads)

    def worker(t):
        barrier.wait()
        t0 = time.perf_counter()
        k = t
        while k < len(lists) and time.perf_counter() - t0 < budget_s:
            o = O.run(n, chi, lists[k])
            o.expectation(labels, coeffs)
            done[t] += 1
            k += threads
        secs[t] = time.perf_counter() - t0

    ths = [threading.Thread(target=worker, args=(t,)) for t in range(threads)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    return sum(done), max(secs)


def differentiation_leg(W, torch, ctx, flush, cpu_budget: float) -> dict:
    """Config 3's workload: the 32-qubit hardware-efficient ansatz (8 layers
    of RY, RZ on every qubit and a CZ ladder; 512 parameters), observable
    sum Z_i Z_i+1 + 0.5 sum X_i, chi_max 64.  One full gradient by the
    adjoint (forward with checkpoints every 2 layers, reverse sweep with SVD
    backward through the truncated splits), and one by the parameter-shift
    rule: 1025 circuits (unshifted + two per parameter) as slices of one
    batch, the observable evaluated on every slice.  Through truncating
    splits the two are different quantities (the adjoint is the derivative
    of the truncated map); their distance is reported."""
    from wqc_cuda import gradients as G

    n, chi = 32, 64
    gates, pidx, _ = C.hea_ansatz(n, 8)
    labels, coeffs = C.zz_x_observable(n)
    lists, _ = G.shifted_circuits(gates, pidx)
    b = W.CudaBatch([n] * len(lists), [chi] * len(lists), ctx=ctx)
    stream = torch.cuda.ExternalStream(b.stream())
    flush.fill_(float(np.random.random()))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    b.apply_slices(lists)
    vals = b.expectations(labels, coeffs).real
    e1.record(stream)
    e1.synchronize()
    wall = time.perf_counter() - t0
    dev_s = e0.elapsed_time(e1) * 1e-3
    splits = b.split_count()
    b.close()
    grad = 0.5 * (vals[1::2] - vals[2::2])
    # The adjoint: forward with checkpoints, then the reverse sweep (wall clock
    # of the two C ABI calls, which synchronise the state's stream).
    adj_runs = []
    for _ in range(2):  # the first is a warm-up
        m = W.CudaMps(n, chi, ctx=ctx)
        flush.fill_(float(np.random.random()))
        torch.cuda.synchronize()
        ta = time.perf_counter()
        adj = W.Adjoint(m, gates, C.hea_checkpoints(n, 8, 2))
        tb = time.perf_counter()
        fa, ga = adj.backward(labels, coeffs)
        tc = time.perf_counter()
        adj.close()
        m.close()
        adj_runs.append((tb - ta, tc - tb, fa, ga))
    fwd_s, bwd_s, fa, ga = adj_runs[-1]
    adj_grad = np.zeros(len(grad))
    for i, p in enumerate(pidx):
        if p >= 0:
            adj_grad[p] += ga[i]
    out = {
        "workload": "hea32_l8_chi64: 32 qubits, 8 layers RY/RZ + CZ ladder, 512 parameters, "
                    "sum Z_i Z_i+1 + 0.5 sum X_i (63 terms), chi_max 64, FP64",
        "method": "adjoint (checkpoints every 2 layers) and parameter shift on the batching form",
        "adjoint_seconds": fwd_s + bwd_s,
        "adjoint_forward_seconds": fwd_s,
        "adjoint_backward_seconds": bwd_s,
        "adjoint_value": fa,
        "adjoint_vs_shift_max_abs_diff": float(np.abs(adj_grad - grad).max()),
        "circuits": len(lists),
        "gradient_seconds": dev_s,
        "gradient_seconds_e2e": wall,
        "applies_per_s": splits / dev_s,
        "value": float(vals[0]),
        "grad_norm": float(np.linalg.norm(grad)),
    }
    if cpu_budget > 0:
        threads = os.cpu_count() or 1
        done, secs = oracle_gradient_sample(n, chi, lists, labels, coeffs, cpu_budget, threads)
        out["cpu_baseline"] = {
            "value": (done / secs) / len(lists) if done else None,
            "unit": "gradients/s",
            "cores": threads,
            "kind": "port",
            "sample": f"FP64 restatement, whole shifted circuits + observable, one per thread on {threads} threads: "
                      f"{done} of {len(lists)} circuits in {secs:.1f} s",
        }
    return out


def oracle_saturated_splits(budget_s: float):
    """CPU leg of the large-chi form: the oracle on isolated saturated splits
    of the chi 256 circuit (512 x 512 theta of random 256-bond sites, one CNOT,
    reference rule: the range finder at ell 272), one thread, until budget_s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import wqc_cuda as W

    rng = np.random.default_rng(7)
    done, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < budget_s:
        o = O.OracleMps(4, 256)
        for i, (l, r) in enumerate([(1, 256), (256, 256), (256, 256), (256, 1)]):
            t = rng.normal(size=(l, 2, r)) + 1j * rng.normal(size=(l, 2, r))
            o.set_site(i, t / np.linalg.norm(t))
        o.apply_2q_at(1, W.CNOT4, True)
        done += 1
    return done, time.perf_counter() - t0


def large_chi_leg(W, torch, ctx, flush, cpu_budget: float) -> dict:
    """Config 4's workload: 100 qubits, depth 100 blocks (RZ.RY.RZ on both
    qubits, CNOT, RY on both, CNOT, RZ.RY.RZ on both, alternating pairs; every
    10th layer a CCNOT on an adjacent triple and an H layer), chi_max 256, in
    the plain and the precision form, one pass each from |0> to <0|psi>."""
    w = C.config4()
    out = {"workload": f"{w.name}: {w.n} qubits, chi_max {w.chi}, {len(w.gates)} gates, split rule reference"}
    for name, prec in (("fp64", W.PRECISION_FP64), ("fp32", W.PRECISION_FP32)):
        m = W.CudaMps(w.n, w.chi, ctx=ctx, precision=prec)
        stream = torch.cuda.ExternalStream(m.stream())
        flush.fill_(float(np.random.random()))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m.apply_gates(w.gates)
        m.amplitude_at_compact_zero()
        e1.record(stream)
        e1.synchronize()
        sec = e0.elapsed_time(e1) * 1e-3
        rec = m.split_records()
        out[name] = {
            "applies_per_s": len(rec) / sec,
            "seconds": sec,
            "splits": int(len(rec)),
            "splits_512x512": int(np.sum((rec["rows"] == 512) & (rec["cols"] == 512))),
            "paths": [int(x) for x in np.bincount(rec["path"], minlength=3)],
            "peak_vram_bytes": m.peak_vram_bytes(),
        }
        m.close()
    out["fp32_speedup"] = out["fp32"]["applies_per_s"] / out["fp64"]["applies_per_s"]
    if cpu_budget > 0:
        done, secs = oracle_saturated_splits(cpu_budget)
        out["cpu_baseline"] = {
            "value": done / secs,
            "unit": UNIT,
            "cores": 1,
            "kind": "port",
            "sample": f"FP64 restatement, one thread: {done} isolated saturated 512x512 splits (random 256-bond sites, "
                      f"CNOT, range finder at ell 272) in {secs:.1f} s; the circuit's own first layers would take "
                      f"tens of minutes to reach saturation on one thread",
        }
    return out


def batch_leg(W, torch, ctx, count: int, flush, cpu_budget: float, precision: int = 0) -> dict:
    """The batching form: `count` independent slices (width U[20,60], depth
    U[10,50], chi_max from {16,32,64,128}) in one device state, one pass from
    |0...0> to every slice's <0...0|psi>.  Latency of a slice = device time
    from the start of the pass to the end of the wave holding its last split."""
    slices = C.config2_slices(count)
    b = W.CudaBatch([s.n for s in slices], [s.chi for s in slices], ctx=ctx, precision=precision)
    stream = torch.cuda.ExternalStream(b.stream())
    gate_lists = [s.gates for s in slices]
    b.set_profiling(True)
    flush.fill_(float(np.random.random()))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    b.apply_slices(gate_lists)
    amps = b.amplitudes()
    e1.record(stream)
    e1.synchronize()
    wall = time.perf_counter() - t0
    dev_s = e0.elapsed_time(e1) * 1e-3
    lat = np.sort(b.slice_times_ms())
    splits = int(b.split_count())
    stats = b.kernel_stats()
    out = {
        "workload": f"{count} slices: width U[20,60], depth U[10,50], chi_max U{{16,32,64,128}}, RY/RZ + CNOT "
                    f"brickwork, own seed each; {'precision form (complex64 Jacobi)' if precision else 'plain FP64'}"
                    f", split rule reference",
        "slices": count,
        "slices_per_s": count / dev_s,
        "e2e_slices_per_s": count / wall,
        "p50_ms": float(np.percentile(lat, 50)),
        "p99_ms": float(np.percentile(lat, 99)),
        "applies": splits,
        "applies_per_s": splits / dev_s,
        "gpu_launches": stats["total_launches"],
        "peak_vram_bytes": b.peak_vram_bytes(),
        "finite_amplitudes": bool(np.all(np.isfinite(amps))),
    }
    b.close()
    if cpu_budget > 0:
        threads = os.cpu_count() or 1
        done, secs = oracle_batch_sample(slices, cpu_budget, threads)
        per_slice = splits / count
        out["cpu_baseline"] = {
            "value": done / secs / per_slice,
            "unit": "slices/s",
            "cores": threads,
            "kind": "port",
            "sample": f"FP64 restatement, one slice per thread on {threads} threads (slices 0..{threads - 1} "
                      f"from their start, {cpu_budget:.0f} s): {done} splits in {secs:.1f} s, converted at the "
                      f"batch's mean of {per_slice:.0f} splits per slice",
        }
    return out


def aggregate_ranks(dist, device, dev_ms: float, wall_s: float):
    """Max over ranks of the timed steps' device and wall times.  Every rank
    runs its own replica (a circuit does not shard: weak scaling, no
    collective on the data path), so the whole job's throughput is the work of
    all ranks over the slowest rank's time; this reduction, at the end of the
    timed region, is the only collective."""
    if dist is None:
        return dev_ms, wall_s
    import torch

    t = torch.tensor([dev_ms, wall_s], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t[0]), float(t[1])


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = workload(args.workload, args.depth)
    g0, windows = timed_windows(w, SATURATED_LAYERS.get(args.workload, 0), args.steps)
    threads = os.cpu_count() or 1
    splits, secs, _ = oracle_windows(w, g0, windows, threads)
    value = splits / secs
    sample = (f"{threads} independent replicas (one thread each) of the FP64 restatement of the reference CPU path; "
              f"each runs gates 0..{g0} untimed, then the {len(windows)} timed windows of gates {g0}..{len(w.gates)} "
              f"(one per step, each closed by a <0...0|psi> read): {splits} splits over all replicas in "
              f"{secs:.1f} s (slowest replica)")
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": len(windows),
        "warmup": args.warmup,
        "ms_per_step": 1000.0 * secs / len(windows),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(w, "reference", g0, windows),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU leg
# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                if int(parts[0]) != self.gpu_index:
                    continue
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def measured_fp64_peak(torch) -> float:
    """cuBLAS DGEMM throughput (TFLOP/s), best of 5, the FP64 roofline."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


def record_flops(W, recs) -> float:
    """Algorithmic SVD flops of the splits in `recs` (the Jacobi's work)."""
    flops = 0.0
    for r in recs:
        if int(r["path"]) == 1:
            flops += W.svd_flops(int(r["ell"]), int(r["cols"]))
        elif int(r["path"]) == 2:
            flops += W.svd_flops(int(r["ell"]), int(r["cols"])) + W.svd_flops(int(r["rows"]), int(r["cols"]))
        else:
            flops += W.svd_flops(int(r["rows"]), int(r["cols"]))
    return flops


def measured_copy_peak(torch) -> float:
    """Device-to-device copy bandwidth (GB/s, read + write bytes), best of 5
    over 1 GiB: the HBM roofline of the streaming kernels."""
    x = torch.empty(1 << 27, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    x.fill_(1.0)
    y.copy_(x)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        y.copy_(x)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * x.numel() * 8 / (e0.elapsed_time(e1) * 1e-3) / 1e9)
    del x, y
    return best


def one_qubit_layer_leg(W, torch, ctx, peak_gbs: float) -> dict:
    """apply_1q_kernel on a wave that streams: a layer of RY on every site of
    a saturated chi 256, 100-site state (98 sites of 256 x 2 x 256 complex128,
    ~200 MB, read and written once by one launch), timed by the kernel's own
    CUDA events; algorithmic bytes 2 * sum_i l_i 2 r_i * 16."""
    n, chi = 100, 256
    m = W.CudaMps(n, chi, ctx=ctx)
    rng = np.random.default_rng(11)
    nbytes = 0
    for q in range(n):
        l = 1 if q == 0 else chi
        r = 1 if q == n - 1 else chi
        t = (rng.standard_normal((l, 2, r)) + 1j * rng.standard_normal((l, 2, r))) / np.sqrt(2 * r)
        m.set_site(q, t)
        nbytes += 2 * t.size * 16
    layer = C.gates_array([C.g1(C.RY, q, 0.1 + 0.01 * q) for q in range(n)])
    m.apply_gates(layer)  # warm-up
    m.synchronize()
    best_ms = None
    for _ in range(5):
        m.reset_stats()
        m.set_profiling(True)
        m.apply_gates(layer)
        m.synchronize()
        st = m.kernel_stats()
        m.set_profiling(False)
        ms = st["milliseconds"]["one_qubit"]
        best_ms = ms if best_ms is None else min(best_ms, ms)
    m.close()
    gbs = nbytes / (best_ms * 1e-3) / 1e9
    return {
        "kernel": "apply_1q_kernel",
        "bytes_per_launch": nbytes,
        "ms_per_launch": best_ms,
        "achieved_gbs": gbs,
        "peak_gbs": peak_gbs,
        "frac": gbs / peak_gbs if peak_gbs else None,
        "peak_source": "device-to-device copy of 1 GiB measured in this run (MEASURED_PEAKS.json absent)",
    }


def unfused_pass_bytes(tree) -> int:
    """Bytes a gate-at-a-time executor moves on this tree: every gate node
    reads and writes its whole state once (2 * 16 * 2^legs)."""
    legs = {}
    total = 0
    for i, nd in enumerate(tree["nodes"]):
        ops = [nd["left"], nd["right"]]
        if any("gate" in r for r in ops):
            st = next(r for r in ops if "gate" not in r)
            k = legs.pop(st["node"]) if "node" in st else 1
            total += 2 * (16 << k)
            legs[i] = k
        else:
            legs[i] = sum(legs.pop(r["node"]) if "node" in r else 1 for r in ops)
    return total


def oracle_exact_sample(n: int, gates, budget_s: float) -> tuple[float, int, float]:
    """The oracle's C loops (exact.rs's apply_in_place, one thread, as the
    reference runs it) applying the circuit's gates to a full n-qubit state
    until the budget is spent: (seconds per gate, gates applied, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import exact as OX

    rng = np.random.default_rng(5)
    data = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)) * (2.0 ** (-(n + 1) / 2))
    wires = list(range(n))
    t0 = time.perf_counter()
    done = 0
    while done < len(gates) and time.perf_counter() - t0 < budget_s:
        OX.apply_in_place(data, wires, gates[done])
        done += 1
    sec = time.perf_counter() - t0
    return sec / max(done, 1), done, sec


def exact_tree_leg(W, ctx, peak_gbs: float, cpu_budget: float) -> dict:
    """An exact contraction tree (src/tn/exact.rs) on the device: the greedy
    plan (src/tn/plan.rs) of a 25-qubit RY + CNOT brickwork of depth 20, the
    widest state the 1 GiB peak admits, contracted for the amplitude of
    |0...0>.  The state (512 MiB) is larger than L2, so no flush is needed
    between repetitions.  Device time from the executor's CUDA events; the
    passes' bytes are 2 * 16 * 2^legs per pass over the 25-leg state."""
    from wqc_cuda import exact as X
    from wqc_cuda import exact_plan as P

    n, depth = 25, 20
    gates = C.ry_cnot_brickwork(n, depth)
    tree = P.plan_greedy(n, gates)
    ex = X.ExactContractor(ctx)
    tiles = {}
    for tile in (12, 13):
        ex.set_tile_bits(tile)
        ex.contract(n, gates, tree, 0)  # warm-up: arena and tables
        runs = []
        for _ in range(5):
            t0 = time.perf_counter()
            amp = ex.contract(n, gates, tree, 0)
            wall = time.perf_counter() - t0
            runs.append((ex.stats(), wall, amp))
        tiles[tile] = runs
    ex.close()
    by_tile = {t: min(r[0]["device_ms"] for r in runs) for t, runs in tiles.items()}
    tile = min(by_tile, key=by_tile.get)
    st, wall, amp = min(tiles[tile], key=lambda r: r[0]["device_ms"])
    best_wall = min(r[1] for r in tiles[tile])
    amps_equal = all(r[2] == amp for runs in tiles.values() for r in runs)
    pass_gbs = st["pass_bytes"] / (st["pass_ms"] * 1e-3) / 1e9
    unfused = unfused_pass_bytes(tree)
    out = {
        "workload": f"brickwork{n}_d{depth}: {n} qubits, RY + CNOT brickwork of depth {depth} ({len(gates)} gates), "
                    f"greedy exact tree ({len(tree['nodes'])} nodes, declared peak {tree['peak_bytes']} B)",
        "gates_per_s": len(gates) / (st["device_ms"] * 1e-3),
        "e2e_gates_per_s": len(gates) / best_wall,
        "device_ms": st["device_ms"],
        "e2e_ms": best_wall * 1e3,
        "launches": st["launches"],
        "passes": st["passes"],
        "exchanges": st["exchanges"],
        "outer_products": st["outer_products"],
        "tile_bits": tile,
        "device_ms_by_tile_bits": by_tile,
        "amplitude": [amp.real, amp.imag],
        "amplitude_same_for_every_tile_and_run": amps_equal,
        "roofline": {
            "bound": "hbm", "kernel": "exact_pass_reg_kernel (passes over tensors of >= 2^20 amplitudes)",
            "achieved": pass_gbs, "peak": peak_gbs, "unit": "GB/s", "frac": pass_gbs / peak_gbs if peak_gbs else None,
            "pass_ms": st["pass_ms"], "pass_bytes": st["pass_bytes"],
            "peak_source": "device-to-device copy of 1 GiB measured in this run (MEASURED_PEAKS.json absent)",
        },
        "unfused_bytes": unfused,
        "unfused_ms_at_peak": unfused / (peak_gbs * 1e9) * 1e3 if peak_gbs else None,
        "note": "e2e: wall clock of wqc_exact_contract (host walk and plan, table upload, device work, amplitude "
                "to host); unfused_ms_at_peak: the HBM time a gate-at-a-time pass would need at the copy peak",
    }
    if cpu_budget > 0:
        per_gate, done, sec = oracle_exact_sample(n, gates, cpu_budget)
        out["cpu_baseline"] = {
            "value": 1.0 / per_gate, "unit": "gates/s", "cores": 1, "kind": "port",
            "sample": f"the oracle's C loops of exact.rs's apply_in_place (one thread, as the reference) on a "
                      f"{n}-qubit state: the circuit's first {done} gates in {sec:.1f} s",
        }
    return out


def network_tree_leg(W, ctx, fp64_peak: float, cpu_budget: float) -> dict:
    """A network contraction tree (src/tn/network.rs) on the device: the
    plain greedy tree (the orchestrator's first pass) of the 5 x 5 grid
    circuit of depth 12 -- 25 qubits, 769 contractions, 290 GFLOP of complex
    GEMM, declared peak 554 MB -- contracted for <0...0|U|0...0>.  Device
    time from the executor's CUDA events; the GEMMs' flops (8 m n k each)
    over their own event time, against the FP64 DGEMM measured in this run."""
    from wqc_cuda import network as N
    from wqc_cuda import network_plan as NP

    n, side, depth = 25, 5, 12
    gates = C.grid(side, depth)
    tree = NP.greedy_tree(n, gates)
    net = N.NetworkContractor(ctx)
    net.contract(n, gates, tree)  # warm-up: arena, cuBLAS
    runs = []
    for _ in range(5):
        t0 = time.perf_counter()
        amp = net.contract(n, gates, tree)
        runs.append((net.stats(), time.perf_counter() - t0, amp))
    net.close()
    st, _, amp = min(runs, key=lambda r: r[0]["device_ms"])
    best_wall = min(r[1] for r in runs)
    tflops = st["gemm_flops"] / (st["gemm_ms"] * 1e-3) / 1e12 if st["gemm_ms"] else None
    out = {
        "workload": f"grid{side}x{side}_d{depth}: {n} qubits, RY + RZ on every qubit and CNOTs along rows and "
                    f"columns, depth {depth} ({len(gates)} gates); greedy network tree ({len(tree['nodes'])} "
                    f"contractions, declared peak {tree['peak_bytes']} B)",
        "contractions_per_s": len(tree["nodes"]) / (st["device_ms"] * 1e-3),
        "device_ms": st["device_ms"],
        "e2e_ms": best_wall * 1e3,
        "gemm_ms": st["gemm_ms"],
        "permute_ms": st["permute_ms"],
        "gemms": st["gemms"],
        "small_contractions": st["small"],
        "launches": st["launches"],
        "permutes": st["permutes"],
        "gemm_gflop": st["gemm_flops"] / 1e9,
        "permute_bytes": st["permute_bytes"],
        "amplitude": [amp.real, amp.imag],
        "amplitude_same_every_run": all(r[2] == amp for r in runs),
        "roofline": {
            "bound": "fp64", "kernel": "cuBLAS ZGEMM of the large contractions (each timed with CUDA events; the "
                                       "level-batched small ones are in device_ms only)",
            "achieved": tflops, "peak": fp64_peak, "unit": "TFLOP/s",
            "frac": tflops / fp64_peak if tflops and fp64_peak else None,
            "peak_source": "FP64 cuBLAS DGEMM 8192^3 measured in this run",
        },
        "note": "e2e: wall clock of wqc_network_contract (host walk and plan, leaf upload, device work, amplitude "
                "to host)",
    }
    if cpu_budget > 0:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import network as ON

        kinds = {"ket0": ON.KET0, "gate": ON.GATE, "node": ON.NODE, "bra0": ON.BRA0, "control": ON.CONTROL,
                 "target": ON.TARGET}
        nodes = [tuple((kinds[k], v) for side_ in (nd["left"], nd["right"]) for k, v in side_.items())
                 for nd in tree["nodes"]]
        t0 = time.perf_counter()
        ON.contract(n, gates, nodes, tree["peak_bytes"])
        sec = time.perf_counter() - t0
        out["cpu_baseline"] = {
            "value": len(tree["nodes"]) / sec, "unit": "contractions/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"the oracle (numpy permutes, multithreaded BLAS ZGEMM on the host's {os.cpu_count()} "
                      f"threads) on the whole tree: {sec:.2f} s",
        }
    return out


def trace_loop_leg(W, ctx, w) -> dict:
    """The production call pattern of the reference's trace loop
    (src/tn/trace.rs:55-187) on the headline circuit: rotation runs folded,
    disjoint layers batched, and before every traced step one
    wqc_mps_site_amplitudes_many call (control probabilities and first-time
    target amplitudes), each a synchronising device read; wall clock of the
    whole loop through the C ABI."""
    from wqc_cuda import trace_replay as TR

    m = W.CudaMps(w.n, w.chi, ctx=ctx)
    TR.replay(m, w.n, w.gates[:200])  # warm-up
    m.reset()
    t0 = time.perf_counter()
    reads = TR.replay(m, w.n, w.gates)
    amp = m.amplitude_at_compact_zero()
    sec = time.perf_counter() - t0
    splits = m.split_count()
    m.close()
    return {
        "workload": f"{w.name}: the trace loop's steps and reads, split rule reference",
        "e2e_applies_per_s": splits / sec,
        "seconds": sec,
        "steps_with_reads": len(reads),
        "reads": int(sum(len(t) for t, _ in reads)),
        "unit": UNIT,
        "amplitude": [amp.real, amp.imag],
        "note": "wall clock of every C ABI call of the loop (gate plans in host memory, reads to host memory)",
    }


def exact_rule_leg(W, torch, ctx, flush) -> dict:
    """The headline circuit under the exact split rule (an exact SVD on every
    split, so the result does not depend on the range finder's rank-48 test
    matrix), one pass from |0...0>, checked against the oracle's fixture
    (tests/golden/config1_exact.npz): kept chi and split paths per split,
    discarded weights, the norm and the amplitude."""
    w = C.config1()
    m = W.CudaMps(w.n, w.chi, ctx=ctx)
    m.set_split_rule(W.SPLIT_RULE_EXACT)
    stream = torch.cuda.ExternalStream(m.stream())
    flush.fill_(float(np.random.random()))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    m.apply_gates(w.gates)
    amp = m.amplitude_at_compact_zero()
    e1.record(stream)
    e1.synchronize()
    sec = e0.elapsed_time(e1) * 1e-3
    rec = m.split_records()
    norm2 = m.expectation(["I" * w.n], [1.0]).real
    out = {
        "workload": f"{w.name}: {w.n} qubits, chi_max {w.chi}, plain FP64, split rule exact",
        "applies_per_s": len(rec) / sec,
        "seconds": sec,
        "amplitude": [amp.real, amp.imag],
        "norm2": norm2,
    }
    fx = os.path.join(ROOT, "tests", "golden", "config1_exact.npz")
    if os.path.exists(fx):
        ref = np.load(fx)
        rr = ref["records"]
        out["vs_oracle"] = {
            "splits_equal": bool(len(rr) == len(rec)),
            "chi_path_shape_bit_exact": bool(len(rr) == len(rec) and all(
                np.array_equal(rr[k], rec[k]) for k in ("left_site", "rows", "cols", "path", "chi"))),
            "max_weight_diff": float(np.max(np.abs(rr["discarded_weight"] - rec["discarded_weight"])))
            if len(rr) == len(rec) else None,
            "norm2_rel_err": abs(norm2 - float(ref["norm2"])) / float(ref["norm2"]) if "norm2" in ref else None,
            "amp_abs_err": abs(amp - complex(ref["amplitude"])),
            "oracle_amplitude": [complex(ref["amplitude"]).real, complex(ref["amplitude"]).imag],
        }
    m.close()
    return out


def run_cuda(args) -> None:
    import torch

    import wqc_cuda as W

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.tree_only:
        # The contraction-tree legs alone (profiling runs): one JSON line.
        ctx = W.Context(local)
        budget = 0.0 if args.no_cpu_baseline else args.cpu_budget
        legs = {}
        if args.tree_only in ("exact", "both"):
            legs["exact_tree"] = exact_tree_leg(W, ctx, measured_copy_peak(torch), budget)
        if args.tree_only in ("network", "both"):
            legs["network_tree"] = network_tree_leg(W, ctx, measured_fp64_peak(torch), budget)
        if rank == 0:
            print(json.dumps(legs), flush=True)
        return
    w = workload(args.workload, args.depth)
    g0, windows = timed_windows(w, SATURATED_LAYERS.get(args.workload, 0), args.steps)
    rule = W.SPLIT_RULE_EXACT if args.split_rule == "exact" else W.SPLIT_RULE_REFERENCE
    if args.tensor_core_only == "merge":
        ctx = W.Context(local)
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
        ms, splits, kms = whole_circuit_profile(W, torch, ctx, w, rule, W.PRECISION_FP64, flush,
                                                merge=W.MERGE_TC_INT8)
        if rank == 0:
            print(json.dumps({"int8_merge_pass": {"ms": ms, "splits": splits, "merge_ms": kms["merge_gate"]}}),
                  flush=True)
        return
    if args.tensor_core_only:
        ctx = W.Context(local)
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
        leg = tensor_core_leg(W, torch, ctx, w, rule, flush, gemm_only=args.tensor_core_only == "gemm")
        if rank == 0:
            print(json.dumps({"tensor_core": leg}), flush=True)
        return
    ctx = W.Context(local)
    # Jacobi cluster sizes measured on this device (or loaded from the
    # fingerprinted cache), before any timed work.
    t_tune = time.perf_counter()
    tuned = 0 if args.no_autotune else ctx.autotune(os.environ.get("WQC_TUNE_PATH"), 120.0)
    tune_s = time.perf_counter() - t_tune
    m = W.CudaMps(w.n, w.chi, ctx=ctx)
    m.set_split_rule(rule)
    stream = torch.cuda.ExternalStream(m.stream())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    peak = measured_fp64_peak(torch) if rank == 0 else None

    def whole_pass():
        m.reset()
        flush.fill_(float(np.random.random()))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m.apply_gates(w.gates)
        amp = m.amplitude_at_compact_zero()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), amp

    for _ in range(args.warmup):
        whole_pass()
    # Timed steps: each reruns the prefix untimed, then times the whole range.
    rng_gates = w.gates[g0:]
    steps = args.steps
    dev_ms, wall_s = [], []
    splits, flops = 0, 0.0
    timed_counts = dict.fromkeys(("h2d_bytes", "d2h_bytes", "total_launches", "jacobi_tasks", "jacobi_sweeps"), 0)
    jac_launches = 0
    m.reset_stats()
    clocks = ClockSampler(local)
    clocks.start()
    amp = 0j
    for _ in range(steps):
        m.set_profiling(False)
        m.reset()
        if g0:
            m.apply_gates(w.gates[:g0])
        m.amplitude_at_compact_zero()
        prefix_splits = m.split_count()
        st0 = m.kernel_stats()
        m.set_profiling(True)
        flush.fill_(float(np.random.random()))
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        m.apply_gates(rng_gates)
        amp = m.amplitude_at_compact_zero()
        e1.record(stream)
        e1.synchronize()
        wall_s.append(time.perf_counter() - t0)
        dev_ms.append(e0.elapsed_time(e1))
        st1 = m.kernel_stats()
        for k in ("h2d_bytes", "d2h_bytes", "total_launches", "jacobi_tasks", "jacobi_sweeps"):
            timed_counts[k] += st1[k] - st0[k]
        jac_launches += st1["launches"]["jacobi_svd"] - st0["launches"]["jacobi_svd"]
        recs = m.split_records()[prefix_splits:]
        splits += len(recs)
        flops += record_flops(W, recs)
    clk = clocks.stop()
    m.set_profiling(False)
    stats = m.kernel_stats()  # kernel milliseconds: events are recorded in the timed regions only
    stats.update(timed_counts)
    total_dev_ms, total_wall = aggregate_ranks(dist, "cuda", sum(dev_ms), sum(wall_s))
    value = world * splits / (total_dev_ms * 1e-3)
    e2e = world * splits / total_wall
    jac_ms = stats["milliseconds"]["jacobi_svd"]
    jac_n = jac_launches
    achieved = flops / (jac_ms * 1e-3) / 1e12 if jac_ms > 0 else None
    whole_ms, whole_amp = whole_pass()
    whole_splits = m.split_count()
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": steps,
            "warmup": args.warmup,
            "ms_per_step": total_dev_ms / steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded generator, same circuit every run)",
            "config": dict(workload_config(w, args.split_rule, g0, windows),
                           merge="int8 digit slices on the tcgen05 tensor cores, FP64-level (the state default)"),
            "e2e": {
                "value": e2e,
                "unit": UNIT,
                "h2d_bytes_per_step": stats["h2d_bytes"] // steps,
                "d2h_bytes_per_step": stats["d2h_bytes"] // steps,
                "note": "wall clock of wqc_mps_apply_gates(host gate list of the window) + wqc_mps_amplitude_zero "
                        "(host result) per step",
            },
            "roofline": {
                "bound": "fp64",
                "kernel": "jacobi_cluster_kernel (FP64 one-sided Jacobi SVD)",
                "achieved": achieved,
                "peak": peak,
                "unit": "TFLOP/s",
                "frac": (achieved / peak) if (achieved and peak) else None,
                "traffic": 767232,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one saturated launch "
                                  "(five exact 256 x 256 splits on 16-CTA clusters); W stays in shared memory",
                "peak_source": "FP64 cuBLAS DGEMM 8192^3 measured in this run (the FP64 pipe: no tensor-core "
                               "instruction is issued; MEASURED_PEAKS.json has no FP64 figure)",
                "flops_per_step": flops / steps,
                "kernel_ms_per_step": jac_ms / steps,
                "launches_per_step": jac_n / steps,
                "svds_per_step": stats["jacobi_tasks"] / steps,
                "sweeps_per_svd": (stats["jacobi_sweeps"] / stats["jacobi_tasks"]) if stats["jacobi_tasks"] else None,
                "flop_count": "4*(14*q*p^2 + 8*p^3) per decomposed p x q matrix (Golub-Van Loan), complex",
            },
            "kernel_ms_per_step": {k: v / steps for k, v in stats["milliseconds"].items()},
            "gpu_launches": stats["total_launches"],
            "clocks": clk,
            "autotune": {"tuned_shapes": tuned, "seconds": tune_s},
            "amplitude": [amp.real, amp.imag],
            "whole_circuit": {
                "applies_per_s": whole_splits / (whole_ms * 1e-3),
                "seconds": whole_ms * 1e-3,
                "splits": whole_splits,
                "amplitude": [whole_amp.real, whole_amp.imag],
                "note": "one pass of the whole circuit from |0...0>, CUDA events, L2 flushed before",
            },
        }
        if world == 1 and not args.no_cpu_baseline:
            s1, secs, nwin = oracle_windows(w, g0, windows, 1, budget_s=args.cpu_budget)
            line["cpu_baseline"] = {
                "value": s1 / secs,
                "unit": UNIT,
                "cores": 1,
                "kind": "port",
                "sample": f"FP64 restatement on 1 thread (the reference MPS path is single-threaded): gates 0..{g0} "
                          f"untimed, then the first {nwin} of the {steps} timed windows ({s1} splits) in {secs:.1f} s",
            }
        if world == 1 and args.workload == "config1" and args.exact_rule_leg:
            line["exact_rule"] = exact_rule_leg(W, torch, ctx, flush)
        if world == 1 and args.trace_leg:
            line["trace_loop"] = trace_loop_leg(W, ctx, w)
        copy_peak = measured_copy_peak(torch) if world == 1 and (args.hbm_leg or args.exact_tree_leg) else 0.0
        if world == 1 and args.hbm_leg:
            line["one_qubit_layer"] = one_qubit_layer_leg(W, torch, ctx, copy_peak)
        if world == 1 and args.exact_tree_leg:
            line["exact_tree"] = exact_tree_leg(W, ctx, copy_peak, 0.0 if args.no_cpu_baseline else args.cpu_budget)
        if world == 1 and args.network_tree_leg:
            line["network_tree"] = network_tree_leg(W, ctx, peak, 0.0 if args.no_cpu_baseline else args.cpu_budget)
        if world == 1 and args.batch_slices > 0:
            line["batch"] = batch_leg(W, torch, ctx, args.batch_slices, flush,
                                      0.0 if args.no_cpu_baseline else args.cpu_budget)
        if world == 1 and args.differentiation_leg:
            line["differentiation"] = differentiation_leg(W, torch, ctx, flush,
                                                          0.0 if args.no_cpu_baseline else args.cpu_budget)
        if world == 1 and args.large_chi_leg:
            line["large_chi"] = large_chi_leg(W, torch, ctx, flush, 0.0 if args.no_cpu_baseline else args.cpu_budget)
        if world == 1 and args.tensor_core_leg:
            line["tensor_core"] = tensor_core_leg(W, torch, ctx, w, rule, flush)
        if world == 1 and args.precision_leg:
            line["precision_form"] = precision_leg(W, torch, ctx, w, rule, 2, flush, whole_splits / (whole_ms * 1e-3))
            if args.batch_slices > 0:
                line["precision_form"]["batch"] = batch_leg(W, torch, ctx, args.batch_slices, flush, 0.0,
                                                            W.PRECISION_FP32)
        print(json.dumps(line), flush=True)
    m.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("cuda", "reference"), default="cuda")
    ap.add_argument("--workload", choices=("config1", "config0", "config4"), default="config1",
                    help="config1: 50 qubits, depth 40, chi 128 (the headline); config0: 16 qubits, chi 32; "
                         "config4: 100 qubits, chi 256 (--depth layers, default 100)")
    ap.add_argument("--depth", type=int, default=0,
                    help="layers of the config1 / config4 circuit (0: their full 40 / 100; a prefix for profiling)")
    ap.add_argument("--split-rule", choices=("reference", "exact"), default="reference")
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the cost model's Jacobi cluster sizes")
    ap.add_argument("--no-hbm-leg", dest="hbm_leg", action="store_false",
                    help="skip the one-qubit layer over a saturated chi 256 state (HBM bandwidth of apply_1q_kernel)")
    ap.add_argument("--no-exact-tree-leg", dest="exact_tree_leg", action="store_false",
                    help="skip the 25-qubit exact contraction tree (wqc_exact_contract)")
    ap.add_argument("--no-network-tree-leg", dest="network_tree_leg", action="store_false",
                    help="skip the 25-qubit grid network contraction tree (wqc_network_contract)")
    ap.add_argument("--tree-only", choices=("exact", "network", "both"), default=None,
                    help="run only the contraction-tree leg(s) and print them (for profiling)")
    ap.add_argument("--no-trace-leg", dest="trace_leg", action="store_false",
                    help="skip the trace loop's call pattern (per-step reads) on the headline circuit")
    ap.add_argument("--no-exact-rule-leg", dest="exact_rule_leg", action="store_false",
                    help="skip the headline circuit under the exact split rule, checked against the oracle fixture")
    ap.add_argument("--no-differentiation-leg", dest="differentiation_leg", action="store_false",
                    help="skip the parameter-shift gradient of the 32-qubit ansatz run after the timed steps")
    ap.add_argument("--no-large-chi-leg", dest="large_chi_leg", action="store_false",
                    help="skip the 100-qubit chi 256 circuit run after the timed steps")
    ap.add_argument("--no-precision-leg", dest="precision_leg", action="store_false",
                    help="skip the precision-form (complex64 Jacobi) leg run after the timed steps")
    ap.add_argument("--no-tensor-core-leg", dest="tensor_core_leg", action="store_false",
                    help="skip the tcgen05 GEMM and the tensor-core form (WQC_PRECISION_TF32X3)")
    ap.add_argument("--tensor-core-only", choices=("gemm", "form", "merge"), default=None,
                    help="run only the tensor-core leg (gemm: the 4096^3 GEMMs alone; merge: one pass of the "
                         "circuit with the int8-slice merges) and print it (for profiling)")
    ap.add_argument("--batch-slices", type=int, default=512,
                    help="slices of the batching-form leg run once after the timed steps (0 = skip)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_cuda(args)


if __name__ == "__main__":
    main()
