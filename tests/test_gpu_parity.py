"""Parity of the cuda backend with the FP64 oracle, through the C ABI.

Tolerances (plain FP64 form): amplitudes within 1e-10 relative, guarded by
1e-12 of the state norm for tiny amplitudes; per-split discarded weights
within 1e-12 absolute; kept bond (chi), split path and bond dimensions
bit-exact.  The reference's own dense-comparison tests use 1e-8 to 1e-12
(src/tn/mps.rs:1482-2113); those are checked against the dense oracle.
"""
import numpy as np
import pytest

import dense as D
import oracle as O
import wqc_cuda as W
from wqc_cuda import circuits as C

pytestmark = pytest.mark.gpu

AMP_RTOL = 1e-10
DISC_ATOL = 1e-12  # per split, times max(1, |weight|): the weights are not normalised (no canonical form)


def rel_err(a: complex, b: complex, norm: float = 1.0) -> float:
    return abs(a - b) / max(abs(b), 1e-12 * norm)


def amp_err(a: complex, b: complex, n: int) -> float:
    """Relative error of an amplitude, guarded by 2^(-n/2), the typical size of
    an amplitude of an n-qubit unit state: <0|psi> of a deep circuit is a
    cancelling sum of much larger terms, and rounding in those terms is what
    a tiny amplitude can be checked against."""
    return abs(a - b) / max(abs(b), 2.0 ** (-n / 2.0))


def oracle_drift(n, chi, gates, rule=0):
    """The oracle's own per-split weight drift between its two FP64 SVDs."""
    return O.self_drift(n, chi, gates, rule=rule)


def assert_records_match(got, ref, drift=None):
    """Shapes, paths and kept chi bit-exact; discarded weights within
    DISC_ATOL (times the weight's size), plus, for long truncating runs, ten
    times the oracle's own drift between two SVDs up to that split."""
    assert len(got) == len(ref), f"split count {len(got)} != {len(ref)}"
    for k in ("left_site", "rows", "cols", "ell", "path", "chi"):
        bad = np.nonzero(got[k] != ref[k])[0]
        assert bad.size == 0, f"{k} differs at splits {bad[:10]}: got {got[k][bad[:10]]} ref {ref[k][bad[:10]]}"
    d = np.abs(got["discarded_weight"] - ref["discarded_weight"])
    tol = DISC_ATOL * np.maximum(1.0, np.abs(ref["discarded_weight"]))
    if drift is not None:
        tol = tol + 10.0 * np.maximum.accumulate(drift)
    bad = np.nonzero(d > tol)[0]
    assert bad.size == 0, (f"discarded weight differs at splits {bad[:5]}: got {got['discarded_weight'][bad[:5]]} "
                           f"ref {ref['discarded_weight'][bad[:5]]}")


def run_both(n, chi, gates, ctx):
    m = W.CudaMps(n, chi, ctx=ctx)
    m.apply_gates(gates)
    o = O.run(n, chi, gates)
    return m, o


def test_backend_label_and_h_amplitude(cuda_ctx):
    m = W.CudaMps(1, 2, ctx=cuda_ctx)
    m.apply_gates(C.gates_array([C.g1(C.H, 0)]))
    a = m.amplitude_at_compact_zero()
    assert abs(a - 1 / np.sqrt(2)) < 1e-12
    assert m.backend_label() == "cuda"
    assert m.peak_vram_bytes() > 0


def random_circuit(rng, n, depth):
    gl = []
    for _ in range(depth):
        k = rng.random()
        q = int(rng.integers(0, n))
        others = [w for w in range(n) if w != q]
        if n >= 3 and k < 0.08:
            c2 = int(rng.choice(others))
            t = int(rng.choice([w for w in others if w != c2]))
            gl.append(C.g3(q, c2, t))
        elif n >= 2 and k < 0.35:
            t = int(rng.choice(others))
            gl.append(C.g2(C.CNOT if rng.random() < 0.5 else C.CZ, q, t))
        elif k < 0.65:
            gl.append(C.g1((C.RX, C.RY, C.RZ)[int(rng.integers(0, 3))], q, rng.uniform(-7, 7)))
        else:
            gl.append(C.g1((C.H, C.X, C.Y, C.Z, C.S, C.T)[int(rng.integers(0, 6))], q))
    return C.gates_array(gl)


def test_random_small_circuits_match_oracle_and_dense(cuda_ctx):
    """The reference's random_circuits_match_dense shape (mps.rs:1922-1972):
    1-6 qubits, every gate type, exact bond."""
    rng = np.random.default_rng(0x5EED20261128)
    for case in range(60):
        n = int(rng.integers(1, 7))
        g = random_circuit(rng, n, int(rng.integers(1, 25)))
        m, o = run_both(n, 128, g, cuda_ctx)
        d = D.Dense(n)
        d.apply_gates(g)
        got = m.to_dense_state()
        assert np.abs(got - d.state).max() < 1e-9, f"case {case}"
        assert_records_match(m.split_records(), o.records())
        assert np.array_equal(m.bond_dims(), o.bond_dims())


def test_ccnot_every_order_matches_dense(cuda_ctx):
    """mps.rs:1977-1994: CCNOT in every wire order on 3-5 qubits, 1e-10."""
    def spread(n, phase):
        out = []
        for q in range(n):
            out.append(C.g1(C.RY, q, 0.3 + 0.4 * q + phase))
            out.append(C.g1(C.RZ, q, 0.7 - 0.2 * q + phase))
        return out
    for n in (3, 4):
        for c1 in range(n):
            for c2 in range(n):
                for t in range(n):
                    if len({c1, c2, t}) < 3:
                        continue
                    g = C.gates_array(spread(n, 0.1) + [C.g3(c1, c2, t)] + spread(n, -0.25))
                    m = W.run(n, 128, g, ctx=cuda_ctx)
                    d = D.Dense(n)
                    d.apply_gates(g)
                    assert np.abs(m.to_dense_state() - d.state).max() < 1e-10


def test_nonadjacent_gates_match_dense(cuda_ctx):
    """mps.rs:1516-1540."""
    g = C.gates_array([C.g1(C.H, 0), C.g1(C.H, 1), C.g2(C.CNOT, 0, 2), C.g2(C.CZ, 3, 1), C.g2(C.CNOT, 2, 0)])
    m = W.run(4, 8, g, ctx=cuda_ctx)
    d = D.Dense(4)
    d.apply_gates(g)
    assert np.abs(m.to_dense_state() - d.state).max() < 1e-8


def test_exact_zero_through_rank_one_split(cuda_ctx):
    """mps.rs:2102-2113."""
    g = C.gates_array([C.g1(C.X, 0), C.g2(C.CZ, 1, 0), C.g1(C.RX, 1, -0.736), C.g2(C.CZ, 1, 0),
                       C.g2(C.CNOT, 0, 1), C.g2(C.CZ, 1, 0)])
    m = W.run(2, 128, g, ctx=cuda_ctx)
    d = D.Dense(2)
    d.apply_gates(g)
    assert np.abs(m.to_dense_state() - d.state).max() < 1e-12


def test_config0_brickwork16_chi32_parity(cuda_ctx):
    """16 qubits, depth 20 RY/RZ + CNOT brickwork at chi 32: heavy truncation."""
    w = C.config0()
    m, o = run_both(w.n, w.chi, w.gates, cuda_ctx)
    a, b = m.amplitude_at_compact_zero(), o.amplitude_zero()
    assert rel_err(a, b) < AMP_RTOL, (a, b)
    assert_records_match(m.split_records(), o.records())
    assert np.array_equal(m.bond_dims(), o.bond_dims())


def _random_sites(rng, dims, scale=1.0):
    out = []
    for l, r in dims:
        t = rng.normal(size=(l, 2, r)) + 1j * rng.normal(size=(l, 2, r))
        out.append(scale * t / np.linalg.norm(t))
    return out


def _theta(site_l, site_r):
    return np.einsum("asg,gtb->astb", site_l, site_r)


def test_range_finder_split_matches_oracle_on_rank_24_theta(cuda_ctx):
    """A 192x192 split at chi 96 takes the seeded range finder (mps.rs:929-981).
    The reference's Rademacher test matrix has rank 48, so the range finder is
    fully determined only when theta*Omega keeps theta's rank (here rank 24;
    at rank 40 it already drops to 36).  Then the GPU's Omega, products,
    Householder QR, projected SVD and Q-absorption must reproduce the
    oracle's kept product, rank and discarded weight."""
    rng = np.random.default_rng(40)
    sites = _random_sites(rng, [(1, 96), (96, 12), (12, 96), (96, 1)])
    m = W.CudaMps(4, 96, ctx=cuda_ctx)
    o = O.OracleMps(4, 96)
    for i, s in enumerate(sites):
        m.set_site(i, s)
        o.set_site(i, s)
    info = m.apply_two_qubit_at_positions(1, 2, W.CNOT4, True, want_info=True)
    o.apply_2q_at(1, W.CNOT4, True)
    ref = o.records()[0]
    assert int(ref["path"]) == 1 and int(info["path"]) == 1, (ref, info)
    assert int(info["chi"]) == int(ref["chi"]) == 24, (ref, info)
    got, want = _theta(m.site(1), m.site(2)), _theta(o.site(1), o.site(2))
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err <= 1e-12, err
    assert abs(float(info["discarded_weight"]) - float(ref["discarded_weight"])) <= DISC_ATOL


def test_range_finder_fallback_matches_oracle(cuda_ctx):
    """needs_f64_fallback (svd_guard.rs:58-76, mps.rs:1027-1032): a 192x192
    theta of rank 48 with singular values graded from 3 to 0.3.  The range
    finder's B keeps 64 rows of rounding noise, which the oracle puts inside
    the (1e-14, 1e-10] band for every scale of theta from 0.1 to 100 (3 is
    in the middle), so the ambiguity test sends the split to the exact SVD,
    whose own noise (~1e-15) stays far below the 1e-12 cut: path
    RSVD_FALLBACK and chi 48 on both sides, and the kept product is unique."""
    rng = np.random.default_rng(7)
    rank, bond = 48, 96
    ul, _ = np.linalg.qr(rng.normal(size=(2 * bond, rank)) + 1j * rng.normal(size=(2 * bond, rank)))
    vr, _ = np.linalg.qr(rng.normal(size=(2 * bond, rank)) + 1j * rng.normal(size=(2 * bond, rank)))
    sig = 3.0 * np.geomspace(1.0, 0.1, rank)
    outer = _random_sites(rng, [(1, bond), (bond, 1)])
    sites = [outer[0], (ul * sig).reshape(bond, 2, rank), vr.conj().T.reshape(rank, 2, bond), outer[1]]
    m = W.CudaMps(4, bond, ctx=cuda_ctx)
    o = O.OracleMps(4, bond)
    for i, s in enumerate(sites):
        m.set_site(i, s)
        o.set_site(i, s)
    eye = np.eye(4, dtype=np.complex128)
    info = m.apply_two_qubit_at_positions(1, 2, eye, True, want_info=True)
    o.apply_2q_at(1, eye, True)
    ref = o.records()[0]
    assert int(ref["path"]) == 2 and int(info["path"]) == 2, (ref, info)
    assert int(info["chi"]) == int(ref["chi"]) == rank, (ref, info)
    got, want = _theta(m.site(1), m.site(2)), _theta(o.site(1), o.site(2))
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err <= 1e-12, err
    assert abs(float(info["discarded_weight"]) - float(ref["discarded_weight"])) <= DISC_ATOL


def test_exact_and_range_finder_splits_in_one_wave(cuda_ctx):
    """One level holding a range-finder split (sites 1-2, the rank-24 theta)
    and an exact split (sites 4-5): the exact SVD runs on the state's second
    stream while the range finder runs on the first.  Both splits, the bonds
    and the amplitude must equal the oracle's."""
    rng = np.random.default_rng(41)
    sites = _random_sites(rng, [(1, 96), (96, 12), (12, 96), (96, 8), (8, 16), (16, 8), (8, 1)])
    gates = C.gates_array([C.g2(C.CNOT, 1, 2), C.g2(C.CZ, 4, 5)])
    _, level, nlev = W.schedule(7, gates)
    assert nlev == 1 and list(level) == [0, 0]
    m = W.CudaMps(7, 96, ctx=cuda_ctx)
    o = O.OracleMps(7, 96)
    for i, s in enumerate(sites):
        m.set_site(i, s)
        o.set_site(i, s)
    m.apply_gates(gates)
    o.apply_gates(gates)
    got, ref = m.split_records(), o.records()
    assert list(ref["path"]) == [1, 0]
    assert_records_match(got, ref)
    assert list(m.bond_dims()) == list(o.bond_dims())
    for p in (1, 4):
        a, b = _theta(m.site(p), m.site(p + 1)), _theta(o.site(p), o.site(p + 1))
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-12, p
    assert rel_err(m.amplitude_zero(), o.amplitude_zero()) < AMP_RTOL


PRECISION_FORM_AMP_RTOL = 1e-6  # the precision form's stated error bound against the FP64 oracle


def test_precision_form_tracks_the_fp64_oracle(cuda_ctx):
    """WQC_PRECISION_FP32: complex64 Jacobi sweeps (carrying X V and V) as
    the first phase of every SVD, then V made orthonormal in FP64, X V formed
    in FP64 and FP64 sweeps to finish.  On the 16-qubit chi 32 brickwork (150
    truncating splits) the amplitude stays within PRECISION_FORM_AMP_RTOL of
    the FP64 oracle, shapes, paths and kept chi are bit-exact, and the
    discarded weights agree as the plain form's long runs do (1e-12 plus the
    oracle's own drift between two FP64 SVDs)."""
    w = C.config0()
    m = W.CudaMps(w.n, w.chi, ctx=cuda_ctx, precision=W.PRECISION_FP32)
    m.apply_gates(w.gates)
    o = O.run(w.n, w.chi, w.gates)
    a, b = m.amplitude_zero(), o.amplitude_zero()
    assert rel_err(a, b) < PRECISION_FORM_AMP_RTOL, (a, b)
    assert_records_match(m.split_records(), o.records(), drift=oracle_drift(w.n, w.chi, w.gates))


def test_precision_form_batch_tracks_the_fp64_oracle(cuda_ctx):
    """The batching form in the precision form: every slice's amplitude
    within PRECISION_FORM_AMP_RTOL of its FP64 oracle run (guarded as the
    plain batch test), split shapes, paths and kept chi bit-exact."""
    slices = C.config2_slices(6, seed=98)
    for s in slices:
        s.chi = min(s.chi, 32)
    b = W.CudaBatch([s.n for s in slices], [s.chi for s in slices], ctx=cuda_ctx, precision=W.PRECISION_FP32)
    b.apply_slices([s.gates for s in slices])
    amps = b.amplitudes()
    recs = b.slice_records()
    for i, s in enumerate(slices):
        o = O.run(s.n, s.chi, s.gates)
        assert amp_err(amps[i], o.amplitude_zero(), s.n) < PRECISION_FORM_AMP_RTOL, (i, amps[i], o.amplitude_zero())
        ref = o.records()
        for k in ("left_site", "rows", "cols", "ell", "path", "chi"):
            assert np.array_equal(recs[i][k], ref[k]), (i, k)


@pytest.mark.parametrize("bond", [64, 128, 256])
def test_exact_split_of_full_rank_theta_matches_oracle(cuda_ctx, bond):
    """2*bond x 2*bond full-rank theta through the exact rule (cluster-resident
    Jacobi at its largest size for chi 128; the staged Jacobi, columns in the
    global workspace, for 512 x 512 at chi 256): kept product, rank, discarded
    weight."""
    rng = np.random.default_rng(bond)
    sites = _random_sites(rng, [(1, bond), (bond, bond), (bond, bond), (bond, 1)])
    m = W.CudaMps(4, bond, ctx=cuda_ctx)
    m.set_split_rule(W.SPLIT_RULE_EXACT)
    o = O.OracleMps(4, bond)
    o.set_split_rule(1)
    for i, s in enumerate(sites):
        m.set_site(i, s)
        o.set_site(i, s)
    info = m.apply_two_qubit_at_positions(1, 2, W.CZ4, False, want_info=True)
    o.apply_2q_at(1, W.CZ4, False)
    ref = o.records()[0]
    assert int(info["chi"]) == int(ref["chi"]) == bond, (ref, info)
    got, want = _theta(m.site(1), m.site(2)), _theta(o.site(1), o.site(2))
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err <= 1e-11, err
    assert abs(float(info["discarded_weight"]) - float(ref["discarded_weight"])) <= DISC_ATOL


def test_precision_form_staged_split_at_chi_256(cuda_ctx):
    """The precision form's staged Jacobi (complex64 columns and V in the
    global workspace, then the FP64 finish) on a full-rank 512 x 512 theta
    under the exact rule: kept product, rank and discarded weight as the
    plain form's."""
    rng = np.random.default_rng(512)
    sites = _random_sites(rng, [(1, 256), (256, 256), (256, 256), (256, 1)])
    m = W.CudaMps(4, 256, ctx=cuda_ctx, precision=W.PRECISION_FP32)
    m.set_split_rule(W.SPLIT_RULE_EXACT)
    o = O.OracleMps(4, 256)
    o.set_split_rule(1)
    for i, s in enumerate(sites):
        m.set_site(i, s)
        o.set_site(i, s)
    info = m.apply_two_qubit_at_positions(1, 2, W.CZ4, False, want_info=True)
    o.apply_2q_at(1, W.CZ4, False)
    ref = o.records()[0]
    assert int(info["chi"]) == int(ref["chi"]) == 256, (ref, info)
    got, want = _theta(m.site(1), m.site(2)), _theta(o.site(1), o.site(2))
    assert np.abs(got - want).max() / np.abs(want).max() <= 1e-11
    assert abs(float(info["discarded_weight"]) - float(ref["discarded_weight"])) <= DISC_ATOL


def test_range_finder_split_at_chi_256_matches_oracle(cuda_ctx):
    """A 512x512 split at chi 256 takes the range finder (ell 272); B^H
    (512 x 272) exceeds a cluster's shared memory and runs on the staged
    Jacobi.  At this shape the reference's Rademacher rows repeat every 64
    rows and theta's columns (t, b) split at 256, so Omega cannot tell the
    t = 0 and t = 1 halves apart and Y = A A^H A Omega has half of theta's
    rank: the range finder is rounding-determined for a generic theta.  With
    the t = 1 half empty (right site's t = 1 slice zero, diagonal CZ) theta
    keeps rank 12 in Y and the result is unique."""
    rng = np.random.default_rng(256)
    sites = _random_sites(rng, [(1, 256), (256, 12), (12, 256), (256, 1)])
    sites[2][:, 1, :] = 0
    m = W.CudaMps(4, 256, ctx=cuda_ctx)
    o = O.OracleMps(4, 256)
    for i, s in enumerate(sites):
        m.set_site(i, s)
        o.set_site(i, s)
    info = m.apply_two_qubit_at_positions(1, 2, W.CZ4, False, want_info=True)
    o.apply_2q_at(1, W.CZ4, False)
    ref = o.records()[0]
    assert int(ref["path"]) == 1 and int(info["path"]) == 1, (ref, info)
    assert int(info["ell"]) == 272 and int(info["chi"]) == int(ref["chi"]) == 12, (ref, info)
    got, want = _theta(m.site(1), m.site(2)), _theta(o.site(1), o.site(2))
    assert np.abs(got - want).max() / np.abs(want).max() <= 1e-12
    assert abs(float(info["discarded_weight"]) - float(ref["discarded_weight"])) <= DISC_ATOL


def test_exact_rule_circuit_parity_at_chi_96(cuda_ctx):
    """The workload that saturates at 192x192 splits, under the exact rule on
    both sides: amplitude, ranks and discarded weights."""
    g = C.gates_array(C.random_layers(18, 12, seed=7))
    m = W.run(18, 96, g, ctx=cuda_ctx, rule=W.SPLIT_RULE_EXACT)
    o = O.run(18, 96, g, rule=1)
    assert_records_match(m.split_records(), o.records(), drift=oracle_drift(18, 96, g, rule=1))
    a, b = m.amplitude_at_compact_zero(), o.amplitude_zero()
    assert rel_err(a, b) < AMP_RTOL, (a, b)


def test_reference_rule_takes_the_same_paths(cuda_ctx):
    """Under the reference rule the same workload takes the range finder on
    its saturated splits.  Omega has rank 48 there, so the kept subspace of a
    rank > 48 split is set by rounding in the reference itself; the decision
    sequence up to the first such split is compared, and both sides must
    take the range finder."""
    g = C.gates_array(C.random_layers(18, 12, seed=7))
    m = W.run(18, 96, g, ctx=cuda_ctx)
    got, ref = m.split_records(), O.run(18, 96, g).records()
    assert len(got) == len(ref)
    first = int(np.argmax(ref["path"] != 0))
    assert (ref["path"] != 0).any() and got["path"][first] != 0
    assert_records_match(got[:first], ref[:first])


def test_site_amplitudes_match_oracle(cuda_ctx):
    g = C.gates_array(C.ry_rz_brickwork(10, 6, seed=3))
    m, o = run_both(10, 16, g, cuda_ctx)
    for t in (0, 4, 9):
        ga, oa = m.site_amplitudes(t), o.site_amplitudes(t)
        for x, y in zip(ga, oa):
            assert rel_err(x, y) < 1e-10


def test_pauli_expectation_matches_dense(cuda_ctx):
    n = 8
    g = C.gates_array(C.ry_rz_brickwork(n, 5, seed=11))
    m = W.run(n, 64, g, ctx=cuda_ctx)
    d = D.Dense(n)
    d.apply_gates(g)
    labels, coeffs = C.zz_x_observable(n)
    labels = labels + ["Y" * n, "XYZI" * (n // 4)]
    coeffs = np.concatenate([coeffs, [0.25 + 0.5j, -1.0]])
    ref = sum(c * D.pauli_expectation(d.state, lab) for lab, c in zip(labels, coeffs))
    got = m.expectation(labels, coeffs)
    assert abs(got - ref) < 1e-10


def test_time_split_rejects_truncation(cuda_ctx):
    """reject_truncation errors instead of cutting (mps.rs:1137-1144, 1650-1661)."""
    def brick(n, depth):
        out = []
        for layer in range(depth):
            for q in range(n):
                out.append(C.g1(C.RY, q, 0.17 + 0.01 * (q + layer)))
            for q in range(layer % 2, n - 1, 2):
                out.append(C.g2(C.CNOT, q, q + 1))
        return out
    g = C.gates_array(brick(16, 8) + [C.g2(C.CNOT, 0, 15)])
    m = W.CudaMps(16, 16, reject_truncation=True, ctx=cuda_ctx)
    with pytest.raises(W.WqcCudaError) as e:
        m.apply_gates(g)
        m.synchronize()
    assert e.value.code == W.ERR_TRUNCATION_REJECTED


def test_batch_of_uneven_slices_matches_single_runs_and_oracle(cuda_ctx):
    """The batching form: slices of different width, depth and chi_max in one
    state.  Every slice must give bit for bit what a batch holding only that
    slice gives (batch invariance: SVD launch shapes depend on each split's
    shape, not on the other slices), agree with the single-state path (whose
    SVD clusters are sized for latency, so the rotation order and the last
    bits differ) in split shapes, paths and kept chi exactly and in the
    amplitude within AMP_RTOL, and match its own oracle run: amplitude
    within AMP_RTOL, split shapes, paths and kept chi bit-exact over the
    whole run, and discarded weights over every split within 1e-12 plus ten
    times the oracle's own drift between its two SVDs.  The deepest slices
    (about 1000 truncating splits at chi 32) carry rounding differences into
    later truncations: the oracle's Golub-Kahan and Jacobi runs of the same
    slice drift apart to ~5e-9 in the last weights, the size of the drift
    between device and oracle (test_oracle_drift_under_a_change_of_svd pins
    that on the CPU)."""
    slices = C.config2_slices(12, seed=99)
    for s in slices:  # keep the oracle side short
        s.chi = min(s.chi, 32)
    b = W.CudaBatch([s.n for s in slices], [s.chi for s in slices], ctx=cuda_ctx)
    b.set_profiling(True)
    b.apply_slices([s.gates for s in slices])
    amps = b.amplitudes()
    recs = b.slice_records()
    times = b.slice_times_ms()
    assert np.all(times > 0)
    for i, s in enumerate(slices):
        one = W.CudaBatch([s.n], [s.chi], ctx=cuda_ctx)
        one.apply_slices([s.gates])
        assert np.array_equal(recs[i], one.slice_records()[0]), i
        assert amps[i] == one.amplitudes()[0], i
        m = W.CudaMps(s.n, s.chi, ctx=cuda_ctx)
        m.apply_gates(s.gates)
        single = m.split_records()
        for k in ("left_site", "rows", "cols", "ell", "path", "chi"):
            assert np.array_equal(recs[i][k], single[k]), (i, k)
        assert amp_err(amps[i], m.amplitude_zero(), s.n) < AMP_RTOL, (i, amps[i], m.amplitude_zero())
        o = O.run(s.n, s.chi, s.gates)
        ref = o.records()
        assert amp_err(amps[i], o.amplitude_zero(), s.n) < AMP_RTOL, (i, amps[i], o.amplitude_zero())
        for k in ("left_site", "rows", "cols", "ell", "path", "chi"):
            assert np.array_equal(recs[i][k], ref[k]), (i, k)
        assert_records_match(recs[i], ref, drift=oracle_drift(s.n, s.chi, s.gates))
