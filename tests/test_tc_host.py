"""CPU models of the tensor-core merges' arithmetic (no device work).

The kernels in wqc-core_b200/csrc/tc_gemm.cu and tc_ozaki.cu rest on three
pieces of exact arithmetic; these tests restate each in numpy and check the
claims the kernels' bounds are built on:

* the real embedding: A's rows as they lie in memory (re, im interleaved)
  times B2 = [[Br, Bi], [-Bi, Br]] blocks gives C interleaved the same way,
  with the merge's B-row order (a tile of 128 real columns holds 32 values
  of b for both t) -- the order the merge epilogue reads back;
* the 3xTF32 split: hi = tf32(x), lo = tf32(x - hi) leaves less than
  2^-21 of |x|, and TF32 products are exact in FP32;
* the int8 digit slices: 9 signed 7-bit digits by truncation of x 2^-e
  reconstruct x to 2^-63 of 2^e, every digit lies in [-127, 127], the slice
  products with p + q < 9 (accumulated per diagonal as the tensor memory
  does) give C within the kernels' bound, the dropped ones stay below 2^-60
  of the scales, no accumulator can leave int32 for k <= 4096, and eight
  digits leave a dropped part 2^7 times larger.
"""
import numpy as np

MAX_INT32 = 2 ** 31 - 1


def cplx(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def embed_a(a):
    """m x k complex -> m x 2k real, K index 2g + c."""
    return np.stack([a.real, a.imag], axis=-1).reshape(a.shape[0], -1)


def b2_entry(v, p, c):
    return (v.real if c == 0 else -v.imag) if p == 0 else (v.imag if c == 0 else v.real)


def embed_b_plain(b):
    """k x n complex -> 2n x 2k real rows (row 2 col + p), K-major."""
    k, n = b.shape
    out = np.zeros((2 * n, 2 * k))
    for col in range(n):
        for p in range(2):
            for g in range(k):
                for c in range(2):
                    out[2 * col + p, 2 * g + c] = b2_entry(b[g, col], p, c)
    return out


def test_real_embedding_gives_the_complex_product():
    rng = np.random.default_rng(1)
    a, b = cplx(rng, 7, 5), cplx(rng, 5, 6)
    c = embed_a(a) @ embed_b_plain(b).T
    got = c[:, 0::2] + 1j * c[:, 1::2]
    assert np.allclose(got, a @ b, rtol=0, atol=1e-13)


def test_merge_row_order_and_epilogue_reproduce_theta_with_the_gate():
    """tc_prep_merge_kernel's B rows (R' = 128 nt + 2 q + p, q = 32 t + b - 32 nt)
    and the epilogue's partner-row 4x4 give theta' = U (L R) of mps.rs:812-866."""
    rng = np.random.default_rng(2)
    dl, k, dr = 5, 6, 37
    L, R = cplx(rng, dl, 2, k), cplx(rng, k, 2, dr)
    U = cplx(rng, 4, 4)
    rows, ntiles = 2 * dl, (dr + 31) // 32
    A = embed_a(L.reshape(rows, k))
    B = np.zeros((ntiles * 128, 2 * k))
    for rr in range(ntiles * 128):
        nt, w = divmod(rr, 128)
        q, p = divmod(w, 2)
        t, b = q // 32, nt * 32 + q % 32
        if b < dr:
            for g in range(k):
                for c in range(2):
                    B[rr, 2 * g + c] = b2_entry(R[g, t, b], p, c)
    D = A @ B.T
    theta = np.zeros((rows, 2 * dr), dtype=complex)
    for row in range(rows):
        s_own, partner = row & 1, row ^ 1
        for nt in range(ntiles):
            for i in range(32):
                b = nt * 32 + i
                if b >= dr:
                    continue
                o = [D[row, nt * 128 + 2 * (32 * t + i)] + 1j * D[row, nt * 128 + 2 * (32 * t + i) + 1] for t in (0, 1)]
                pr = [D[partner, nt * 128 + 2 * (32 * t + i)] + 1j * D[partner, nt * 128 + 2 * (32 * t + i) + 1]
                      for t in (0, 1)]
                th = {(s_own, 0): o[0], (s_own, 1): o[1], (1 - s_own, 0): pr[0], (1 - s_own, 1): pr[1]}
                for to in range(2):
                    u = U[s_own * 2 + to]
                    theta[row, to * dr + b] = sum(u[si * 2 + ti] * th[(si, ti)] for si in (0, 1) for ti in (0, 1))
    plain = np.einsum("asg,gtb->astb", L, R).reshape(dl, 2, 2, dr)
    want = np.einsum("xy,ayb->axb", U, plain.reshape(dl, 4, dr)).reshape(rows, 2 * dr)
    assert np.allclose(theta, want, rtol=0, atol=1e-12)


def tf32_rna(x):
    """cvt.rna.tf32.f32: keep 10 mantissa bits, round to nearest, ties away."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x1000) & 0xFFFFE000
    return u.astype(np.uint32).view(np.float32)


def test_three_tf32_split_and_exact_products():
    rng = np.random.default_rng(3)
    x = rng.standard_normal(20000) * 10.0 ** rng.uniform(-8, 8, 20000)
    hi = tf32_rna(x.astype(np.float32))
    lo = tf32_rna((x - hi.astype(np.float64)).astype(np.float32))
    rel = np.abs(x - hi.astype(np.float64) - lo.astype(np.float64)) / np.abs(x)
    assert rel.max() < 2.0 ** -21, rel.max()
    # an 11-bit by 11-bit significand product has 22 bits: exact in FP32
    y = tf32_rna(rng.standard_normal(20000).astype(np.float32))
    prod32 = (hi * y).astype(np.float64)
    assert np.array_equal(prod32, hi.astype(np.float64) * y.astype(np.float64))


SLICES = 9


def scale_exponent(mx):
    return 0 if mx == 0 else int(np.frexp(mx)[1])


def digits(x, e, slices=SLICES):
    v = np.ldexp(x, -e)
    out = []
    for _ in range(slices):
        v = v * 128.0
        t = np.trunc(v)
        out.append(t.astype(np.int64))
        v = v - t
    return np.stack(out), v  # digits (slice-major) and the remainder in units of 2^-7 slices


def int8_gemm_model(a, b, slices=SLICES):
    """The scheme of oz_zgemm_kernel on the real embedding: row / column
    scales, digit planes, int accumulators per diagonal p + q < slices, FP64
    combination by Horner.  Returns C and the largest |accumulator|."""
    A, B = embed_a(a), embed_b_plain(b)  # m x 2k, 2n x 2k (rows = output columns)
    ea = np.array([scale_exponent(np.abs(r).max()) for r in A])
    fb = np.array([scale_exponent(np.abs(r).max()) for r in B])
    da = np.stack([digits(A[i], ea[i], slices)[0] for i in range(A.shape[0])], axis=1)  # slice, row, K
    db = np.stack([digits(B[j], fb[j], slices)[0] for j in range(B.shape[0])], axis=1)
    assert np.abs(da).max() <= 127 and np.abs(db).max() <= 127
    acc = np.zeros((slices, A.shape[0], B.shape[0]), dtype=np.int64)
    for p in range(slices):
        for q in range(slices - p):
            acc[p + q] += da[p] @ db[q].T
    v = acc[slices - 1].astype(np.float64)
    for d in range(slices - 2, -1, -1):
        v = v / 128.0 + acc[d]
    C = np.ldexp(v, ea[:, None] + fb[None, :] - 14)
    return C[:, 0::2] + 1j * C[:, 1::2], int(np.abs(acc).max())


def test_digits_reconstruct_to_two_to_the_minus_63():
    rng = np.random.default_rng(4)
    x = rng.standard_normal(5000) * 10.0 ** rng.uniform(-30, 30, 5000)
    e = scale_exponent(np.abs(x).max())
    d, rem = digits(x, e)
    assert np.abs(d).max() <= 127
    assert np.all(np.sign(d[0][d[0] != 0]) == np.sign(x[d[0] != 0]))  # truncation keeps the sign
    assert np.abs(rem).max() < 1.0  # remainder below one unit of the last digit: below 2^-63 of 2^e


def dropped_part(a, b, slices):
    """Largest |sum of the slice products with p + q >= slices| over the
    entries, relative to the row and column scales, in exact integers."""
    A, B = embed_a(a), embed_b_plain(b)
    ea = np.array([scale_exponent(np.abs(r).max()) for r in A])
    fb = np.array([scale_exponent(np.abs(r).max()) for r in B])
    da = np.stack([digits(A[i], ea[i], slices)[0] for i in range(A.shape[0])], axis=1)
    db = np.stack([digits(B[j], fb[j], slices)[0] for j in range(B.shape[0])], axis=1)
    drop = np.zeros((A.shape[0], B.shape[0]))
    for p in range(slices):
        for q in range(slices):
            if p + q >= slices:
                drop += (da[p] @ db[q].T).astype(np.float64) * 2.0 ** (-7 * (p + q + 2))
    return np.abs(drop).max()  # in units of 2^(e_r + f_c) <= 4 x the scales


def test_int8_slices_meet_the_bound_and_nine_digits_drop_less():
    rng = np.random.default_rng(5)
    for m, n, k in ((9, 7, 5), (24, 16, 40), (12, 10, 129)):
        a = cplx(rng, m, k) * 10.0 ** rng.uniform(-20, 20, size=(m, 1))
        b = cplx(rng, k, n) * 10.0 ** rng.uniform(-20, 20, size=(1, n))
        ref = a @ b
        c9, _ = int8_gemm_model(a, b, 9)
        ra = np.maximum(np.abs(a.real), np.abs(a.imag)).max(axis=1)
        cb = np.maximum(np.abs(b.real), np.abs(b.imag)).max(axis=0)
        assert np.all(np.abs(c9 - ref) <= 2.0 ** -49 * (2 * k) * np.outer(ra, cb))
        # the dropped products: below 2^-60 of the scales per K term with nine
        # digits, 2^7 times more with eight
        d9, d8 = dropped_part(a, b, 9), dropped_part(a, b, 8)
        assert d9 <= 2.0 ** -60 * (2 * k), d9
        assert d8 > 16.0 * d9, (d8, d9)


def test_merge_operands_scale_together_along_k():
    """The bound is relative to each row's and column's largest values, not
    to the terms of each dot product: where large entries of a row meet small
    entries of a column the relative error grows.  The merge's operands do
    not do that -- L = U sqrt(S) and R = sqrt(S) V^H shrink together along
    the inner index -- and its theta stays at FP64-level relative error."""
    rng = np.random.default_rng(6)
    k = 24
    s = np.logspace(0, -12, k)
    U = np.linalg.qr(cplx(rng, 64, k))[0]
    V = np.linalg.qr(cplx(rng, 40, k))[0]
    L, R = U * np.sqrt(s), (np.sqrt(s)[:, None] * V.conj().T)
    c, _ = int8_gemm_model(L, R)
    ref = L @ R
    assert np.linalg.norm(c - ref) / np.linalg.norm(ref) < 1e-14


def test_int32_accumulators_cannot_overflow_up_to_k_4096():
    # at most 9 products on a diagonal, 2k real terms each of |d e| <= 127^2
    assert 9 * 2 * 4096 * 127 * 127 <= MAX_INT32
    # the largest accumulator of an all-max operand pair stays inside the same bound
    a = np.full((2, 64), 0.999 + 0.999j)
    b = np.full((64, 3), 0.999 - 0.999j)
    _, amax = int8_gemm_model(a, b)
    assert amax <= 9 * 2 * 64 * 127 * 127


def test_anti_correlated_scales_keep_the_maxima_bound_only():
    """The caveat the header states: where a row's large entries meet a
    column's small ones along K, the error is small against the maxima but
    not against the result itself (FP64 FMA would keep ~1e-16 relative)."""
    rng = np.random.default_rng(7)
    k = 32
    w = np.logspace(0, -12, k)
    a = cplx(rng, 6, k) * w              # row entries shrink along K
    b = cplx(rng, k, 5) / w[:, None] * 1e-12  # column entries grow along K
    c, _ = int8_gemm_model(a, b)
    ref = a @ b
    ra = np.maximum(np.abs(a.real), np.abs(a.imag)).max(axis=1)
    cb = np.maximum(np.abs(b.real), np.abs(b.imag)).max(axis=0)
    assert np.all(np.abs(c - ref) <= 2.0 ** -49 * (2 * k) * np.outer(ra, cb))
    assert np.max(np.abs(c - ref) / np.abs(ref)) > 1e-10

