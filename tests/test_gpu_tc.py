"""The tcgen05 tensor-core complex GEMM (wqc_tc_zgemm) against an FP64
GEMM (numpy).

Tolerance: 3xTF32 split products (hi = tf32(x), lo = tf32(x - hi); lo*hi +
hi*lo + hi*hi) are exact in FP32; the error comes from accumulating them in
FP32 in tensor memory.  Each of the two hi*hi accumulators takes k/8 updates
(2k real K values, 8 per MMA, alternate K blocks), and each update may lose
up to one FP32 unit roundoff (2^-24) of the accumulator: the bound is
2^-24 * max(16, k/4), every entry within it times |A_i| |B_j| (row and
column 2-norms) of the FP64 product and the whole within it relative in
the Frobenius norm (measured: 3.4e-7 at k = 128, 2.4e-6 at k = 1000, about
a fifth of the bound).  One TF32 product alone (10 mantissa bits) would be
off by ~5e-4.
"""
import numpy as np
import pytest

from wqc_cuda import ERR_INVALID, WqcCudaError
from wqc_cuda import tc as T

pytestmark = pytest.mark.gpu


def tol(k: int) -> float:
    return 2.0 ** -24 * max(16.0, k / 4.0)


def cplx(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def check(a, b, c):
    ref = a @ b
    scale = np.outer(np.linalg.norm(a, axis=1), np.linalg.norm(b, axis=0))
    entry = np.max(np.abs(c - ref) / np.maximum(scale, 1e-300))
    fro = np.linalg.norm(c - ref) / max(np.linalg.norm(ref), 1e-300)
    t = tol(a.shape[1])
    assert entry <= t, (entry, t)
    assert fro <= t, (fro, t)
    return entry, fro


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (5, 7, 3), (128, 64, 16), (129, 65, 17), (256, 256, 128),
                                   (200, 300, 1000), (1024, 512, 384)])
def test_matches_fp64_gemm(cuda_ctx, m, n, k):
    rng = np.random.default_rng(m * 7919 + n * 31 + k)
    a, b = cplx(rng, m, k), cplx(rng, k, n)
    c, ms = T.zgemm(a, b, ctx=cuda_ctx)
    check(a, b, c)
    assert ms > 0


def test_merge_shaped_operands_and_scales(cuda_ctx):
    """Site-like operands: a unit-norm left site times a right site with
    singular values spread over 12 decades (columns scaled), the shapes of
    a saturated chi 128 merge (256 x 128 times 128 x 256)."""
    rng = np.random.default_rng(5)
    q, _ = np.linalg.qr(cplx(rng, 256, 128))
    s = np.logspace(0, -12, 128)
    r = (s[:, None] * cplx(rng, 128, 256)) / np.sqrt(256)
    c, _ = T.zgemm(q, r, ctx=cuda_ctx)
    check(q, r, c)


def test_repeated_launches_give_the_same_product(cuda_ctx):
    rng = np.random.default_rng(11)
    a, b = cplx(rng, 300, 257), cplx(rng, 257, 190)
    c1, _ = T.zgemm(a, b, reps=1, ctx=cuda_ctx)
    c5, ms = T.zgemm(a, b, reps=5, ctx=cuda_ctx)
    assert np.array_equal(c1, c5) and ms > 0


def test_sizes_are_checked_before_device_work(cuda_ctx):
    with pytest.raises(WqcCudaError) as e:
        T.zgemm(np.zeros((0, 4)), np.zeros((4, 3)), ctx=cuda_ctx)
    assert e.value.code == ERR_INVALID
    with pytest.raises(ValueError):
        T.zgemm(np.zeros((3, 4)), np.zeros((5, 3)), ctx=cuda_ctx)


# ---------------------------------------------------------------------------
# The tensor-core form (WQC_PRECISION_TF32X3): every merge on the tensor cores.
# ---------------------------------------------------------------------------
import oracle as O  # noqa: E402
import wqc_cuda as W  # noqa: E402
from wqc_cuda import circuits as C  # noqa: E402


def _sites(rng, dims):
    out = []
    for l, r in dims:
        t = rng.normal(size=(l, 2, r)) + 1j * rng.normal(size=(l, 2, r))
        out.append(t / np.linalg.norm(t))
    return out


def _unitary4(rng):
    q, r = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))
    return q * (np.diag(r) / np.abs(np.diag(r)))


@pytest.mark.parametrize("bond", [32, 128])
def test_tensor_core_merge_of_one_full_rank_split(cuda_ctx, bond):
    """One exact-rule split of a full-rank theta under a random 4x4 unitary:
    the kept product against the oracle's FP64 theta' within the merge's
    FP32-level error, rank bit-exact."""
    rng = np.random.default_rng(bond + 1)
    sites = _sites(rng, [(1, bond), (bond, bond), (bond, bond), (bond, 1)])
    u = _unitary4(rng)
    m = W.CudaMps(4, bond, ctx=cuda_ctx, precision=W.PRECISION_TF32X3)
    m.set_split_rule(W.SPLIT_RULE_EXACT)
    o = O.OracleMps(4, bond)
    o.set_split_rule(1)
    for i, s in enumerate(sites):
        m.set_site(i, s)
        o.set_site(i, s)
    info = m.apply_two_qubit_at_positions(1, 2, u, False, want_info=True)
    o.apply_2q_at(1, u, False)
    ref = o.records()[0]
    assert int(info["chi"]) == int(ref["chi"]) == bond
    got = np.einsum("asg,gtb->astb", m.site(1), m.site(2))
    want = np.einsum("asg,gtb->astb", o.site(1), o.site(2))
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    print(f"tc merge split bond {bond}: theta rel err {err:.3e}")
    assert err <= 1e-5, err


def test_tensor_core_form_on_the_16_qubit_brickwork(cuda_ctx):
    """The 16-qubit chi 32 brickwork (150 truncating splits) in the
    tensor-core form against the FP64 oracle."""
    w = C.config0()
    m = W.CudaMps(w.n, w.chi, ctx=cuda_ctx, precision=W.PRECISION_TF32X3)
    m.apply_gates(w.gates)
    o = O.run(w.n, w.chi, w.gates)
    a, b = m.amplitude_zero(), o.amplitude_zero()
    err = abs(a - b) / max(abs(b), 2.0 ** (-w.n / 2.0))
    got, ref = m.split_records(), o.records()
    bad = {k: int(np.count_nonzero(got[k] != ref[k])) for k in ("rows", "cols", "path", "chi")}
    wd = float(np.max(np.abs(got["discarded_weight"] - ref["discarded_weight"])))
    print(f"tc form config0: amp {a} oracle {b} rel err {err:.3e}; record mismatches {bad}; weight diff {wd:.3e}")
    assert err <= 1e-3, err


# ---------------------------------------------------------------------------
# int8 digit slices on the tensor cores (wqc_tc_zgemm_int8, WQC_MERGE_TC_INT8).
# Each row of A and column of B2 is scaled by a power of two and cut into 9
# signed 7-bit digits; digit products are exact in int32.  Truncation leaves
# less than 2^-63 of each scaled value and the dropped slice products less
# than 2^-60 of the scales; what remains is the FP64 rounding of the final
# sum, so every entry lies within 2^-49 * 2k of the product of its row's and
# column's largest |re|, |im| -- FP64-level -- and the whole within 1e-14
# relative (measured values are printed).
# ---------------------------------------------------------------------------
from test_gpu_parity import assert_records_match, oracle_drift  # noqa: E402


def int8_bound(a, b):
    ra = np.maximum(np.abs(a.real), np.abs(a.imag)).max(axis=1)
    cb = np.maximum(np.abs(b.real), np.abs(b.imag)).max(axis=0)
    return 2.0 ** -49 * (2 * a.shape[1]) * np.outer(ra, cb)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (5, 7, 3), (128, 32, 32), (129, 65, 33), (256, 256, 128),
                                   (300, 200, 1000), (1024, 512, 384)])
def test_int8_slices_match_fp64(cuda_ctx, m, n, k):
    rng = np.random.default_rng(m * 131 + n * 17 + k)
    a, b = cplx(rng, m, k), cplx(rng, k, n)
    c, ms = T.zgemm(a, b, ctx=cuda_ctx, form="int8")
    ref = a @ b
    err = np.abs(c - ref)
    bound = int8_bound(a, b)
    fro = np.linalg.norm(c - ref) / np.linalg.norm(ref)
    print(f"int8 slices {m}x{n}x{k}: max err / bound {np.max(err / bound):.3e}, rel err {fro:.3e}, {ms:.4f} ms")
    assert np.all(err <= bound), np.max(err / bound)
    assert fro <= 1e-14, fro
    assert ms > 0


def test_int8_slices_follow_row_and_column_scales(cuda_ctx):
    """Rows and columns 10^-60..10^60 apart: the power-of-two scales keep
    every entry within its own bound."""
    rng = np.random.default_rng(3)
    a = cplx(rng, 200, 96) * 10.0 ** rng.uniform(-60, 60, size=(200, 1))
    b = cplx(rng, 96, 150) * 10.0 ** rng.uniform(-60, 60, size=(1, 150))
    c, _ = T.zgemm(a, b, ctx=cuda_ctx, form="int8")
    assert np.all(np.abs(c - a @ b) <= int8_bound(a, b))


@pytest.mark.parametrize("bond", [32, 128])
def test_int8_merge_of_one_full_rank_split(cuda_ctx, bond):
    """The plain FP64 form with int8-slice merges: one exact-rule split of a
    full-rank theta under a random 4x4 unitary, the kept product against the
    oracle within the plain form's 1e-11, rank bit-exact."""
    rng = np.random.default_rng(bond + 7)
    sites = _sites(rng, [(1, bond), (bond, bond), (bond, bond), (bond, 1)])
    u = _unitary4(rng)
    m = W.CudaMps(4, bond, ctx=cuda_ctx)
    m.set_split_rule(W.SPLIT_RULE_EXACT)
    m.set_merge(W.MERGE_TC_INT8)
    o = O.OracleMps(4, bond)
    o.set_split_rule(1)
    for i, s in enumerate(sites):
        m.set_site(i, s)
        o.set_site(i, s)
    info = m.apply_two_qubit_at_positions(1, 2, u, False, want_info=True)
    o.apply_2q_at(1, u, False)
    assert int(info["chi"]) == int(o.records()[0]["chi"]) == bond
    got = np.einsum("asg,gtb->astb", m.site(1), m.site(2))
    want = np.einsum("asg,gtb->astb", o.site(1), o.site(2))
    err = np.abs(got - want).max() / np.abs(want).max()
    print(f"int8 merge split bond {bond}: theta err {err:.3e}")
    assert err <= 1e-11, err


def test_int8_merges_keep_the_plain_form_parity(cuda_ctx):
    """The 16-qubit chi 32 brickwork (150 truncating splits) with every merge
    from int8 slices: the plain form's bar against the oracle (amplitude
    1e-10, records bit-exact, weights within 1e-12 plus the oracle's drift)."""
    w = C.config0()
    m = W.run(w.n, w.chi, w.gates, ctx=cuda_ctx, merge=W.MERGE_TC_INT8)
    o = O.run(w.n, w.chi, w.gates)
    a, b = m.amplitude_zero(), o.amplitude_zero()
    err = abs(a - b) / max(abs(b), 1e-12)
    print(f"int8 merges config0: amp rel err {err:.3e}")
    assert err < 1e-10, (a, b)
    assert_records_match(m.split_records(), o.records(), drift=oracle_drift(w.n, w.chi, w.gates))
    st = m.kernel_stats()
    assert st["launches"]["merge_gate"] > 0


def test_merge_selector_is_checked(cuda_ctx):
    m = W.CudaMps(4, 8, ctx=cuda_ctx)
    with pytest.raises(WqcCudaError) as e:
        m.set_merge(7)
    assert e.value.code == ERR_INVALID
    t = W.CudaMps(4, 8, ctx=cuda_ctx, precision=W.PRECISION_TF32X3)
    with pytest.raises(WqcCudaError):
        t.set_merge(W.MERGE_TC_INT8)
    m.set_merge(W.MERGE_TC_INT8)
    m.set_merge(W.MERGE_FFMA)
