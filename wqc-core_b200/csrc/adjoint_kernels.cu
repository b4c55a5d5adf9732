// Device kernels of the adjoint (reverse-mode) pass of the differentiation
// form: the cotangents of the site tensors for a Pauli-sum observable, the
// reverse of a one-qubit gate, and the reverse of a two-site apply (merge,
// 4x4 gate, truncated SVD split with sqrt(S) absorbed on both sides).
//
// What is differentiated is the reference's forward path: apply_one_qubit
// (src/tn/mps.rs:333-351), apply_two_qubit_at_positions (mps.rs:377-429:
// merge 484-514, 4x4 on theta 833-866) and truncated_svd_split
// (mps.rs:1124-1171: L = U_k sqrt(S_k), R = sqrt(S_k) V_k^H, kept chi by
// retained_chi, svd_guard.rs:25-35), then f = sum_t Re(c_t) <psi|P_t|psi>
// (src/expectation.rs:98-200).  The reference has no reverse mode.
//
// The split's reverse is the complex SVD's reverse mode over the thin SVD
// theta = U S V^H (all p = min(m, n) columns), the cotangents of the dropped
// columns set to zero -- which keeps the truncation term, the coupling of
// every kept column to every dropped one through 1/(s_j^2 - s_i^2):
//   theta_bar = U Z V^H + U Q2^H + Q1 V^H, with
//   Q1 = U_bar S^-1, Q2 = V_bar S^-1, M = U^H U_bar, N = V^H V_bar,
//   Z = F o ((M - M^H) S + S (N - N^H)) + diag(s_bar + i Im(M_ii - N_ii) / 2 s_i)
//       - M S^-1 - (N S^-1)^H,
//   F_ij = (s_j^2 - s_i^2) / ((s_j^2 - s_i^2)^2 + eps), eps = 1e-24 s_max^4
// (Lorentzian broadening of 1/(s_j^2 - s_i^2) for near-degenerate values).
// The last two terms of Z fold the projections (I - U U^H) and (I - V V^H)
// of the non-square parts in.  Columns whose singular value is below 1e-14
// of the largest are null directions: they are left out of U and V and
// enter through those projections.  The device Jacobi keeps W = X V (one
// side); the other side is recovered as theta^H U S^-1 or theta V S^-1.
#include "common.cuh"
#include "split_kernels.cuh"

namespace wqc {

constexpr double kAdjNullRel = 1e-14;
constexpr double kAdjLorentz = 1e-24;

__device__ __forceinline__ double2 pauli_conj_row(char ch, const double2* a, int s, size_t stride) {
    // sum_{s'} P[s'][s] conj(A[s'])  with A[s'] = a[s' * stride]
    const double2 a0 = cconj(a[0]), a1 = cconj(a[stride]);
    switch (ch) {
        case 'X': return s == 0 ? a1 : a0;
        case 'Y': return s == 0 ? cmake(-a1.y, a1.x) : cmake(a0.y, -a0.x);  // P[1][0] = i, P[0][1] = -i
        case 'Z': return s == 0 ? a0 : cmake(-a1.x, -a1.y);
        default: return s == 0 ? a0 : a1;
    }
}

// Left and right environments of every site for each Pauli term (one CTA
// per term).  EL_q[a][a'] (ket a, bra a') contracts sites 0..q-1 of
// <psi| P |psi>; ER_q[b][b'] contracts sites q+1..n-1.  With
// At[a', s, b'] = sum_{s'} P[s'][s] conj(A[a', s', b']):
//   EL_{q+1}[b][b'] = sum_{a, a', s} EL_q[a][a'] A[a, s, b] At[a', s, b'],
//   ER_{q-1}[a][a'] = sum_{b, b', s} A[a, s, b] ER_q[b][b'] At[a', s, b'].
// envs: (n + 1) cap^2 entries per term for EL, then n cap^2 for ER;
// tmp: cap * 2 * cap per term.  vals[t] = <psi|P_t|psi> = EL_n[0][0].
__global__ void __launch_bounds__(256) adj_pauli_envs_kernel(DeviceMps mps, const char* labels, int nterms, int cap,
                                                             double2* envs, double2* tmp_all, double2* vals) {
    const int t = blockIdx.x;
    if (t >= nterms) return;
    const int n = mps.n;
    const size_t E = size_t(cap) * cap;
    double2* EL = envs + size_t(t) * (2 * n + 1) * E;
    double2* ER = EL + size_t(n + 1) * E;
    double2* tmp = tmp_all + size_t(t) * 2 * E;
    const char* lab = labels + size_t(t) * n;
    if (threadIdx.x == 0) {
        EL[0] = cmake(1.0, 0.0);
        ER[size_t(n - 1) * E] = cmake(1.0, 0.0);
    }
    __syncthreads();
    for (int q = 0; q < n; ++q) {
        const int l = mps.dl[q], r = mps.dr[q];
        const double2* A = mps.site[q];
        const double2* cur = EL + size_t(q) * E;  // l x l
        double2* nxt = EL + size_t(q + 1) * E;    // r x r
        const char ch = lab[n - 1 - q];
        // tmp[a'][s][b] = sum_a cur[a][a'] A[a, s, b]
        for (long e = threadIdx.x; e < long(l) * 2 * r; e += blockDim.x) {
            const int ap = int(e / (2 * r)), rem = int(e % (2 * r));
            double2 acc = cmake(0, 0);
            for (int a = 0; a < l; ++a) cfma(acc, cur[size_t(a) * l + ap], A[size_t(a) * 2 * r + rem]);
            tmp[e] = acc;
        }
        __syncthreads();
        for (long e = threadIdx.x; e < long(r) * r; e += blockDim.x) {
            const int b = int(e / r), bp = int(e % r);
            double2 acc = cmake(0, 0);
            for (int ap = 0; ap < l; ++ap)
                for (int s = 0; s < 2; ++s)
                    cfma(acc, tmp[(size_t(ap) * 2 + s) * r + b],
                         pauli_conj_row(ch, A + size_t(ap) * 2 * r + bp, s, size_t(r)));
            nxt[e] = acc;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) vals[t] = EL[size_t(n) * E];
    for (int q = n - 1; q > 0; --q) {
        const int l = mps.dl[q], r = mps.dr[q];
        const double2* A = mps.site[q];
        const double2* cur = ER + size_t(q) * E;  // r x r
        double2* nxt = ER + size_t(q - 1) * E;    // l x l
        const char ch = lab[n - 1 - q];
        // tmp[a][s][b'] = sum_b A[a, s, b] cur[b][b']
        for (long e = threadIdx.x; e < long(l) * 2 * r; e += blockDim.x) {
            const int as = int(e / r), bp = int(e % r);
            double2 acc = cmake(0, 0);
            for (int b = 0; b < r; ++b) cfma(acc, A[size_t(as) * r + b], cur[size_t(b) * r + bp]);
            tmp[e] = acc;
        }
        __syncthreads();
        for (long e = threadIdx.x; e < long(l) * l; e += blockDim.x) {
            const int a = int(e / l), ap = int(e % l);
            double2 acc = cmake(0, 0);
            for (int s = 0; s < 2; ++s)
                for (int bp = 0; bp < r; ++bp)
                    cfma(acc, tmp[(size_t(a) * 2 + s) * r + bp],
                         pauli_conj_row(ch, A + size_t(ap) * 2 * r + bp, s, size_t(r)));
            nxt[e] = acc;
        }
        __syncthreads();
    }
}

// Holes of site q for the terms of one chunk (grid: sites x terms):
// H[a, s, b] = sum_{a', b'} EL_q[a][a'] At[a', s, b'] ER_q[b][b'], written to
// holes[(t * n + q) * cap * 2 * cap]; half-products in tmp (same layout).
__global__ void __launch_bounds__(256) adj_pauli_holes_kernel(DeviceMps mps, const char* labels, int t0, int cap,
                                                              const double2* envs, double2* tmp_all,
                                                              double2* holes) {
    const int q = blockIdx.x, tl = blockIdx.y, t = t0 + tl;
    const int n = mps.n;
    const size_t E = size_t(cap) * cap, S = size_t(cap) * 2 * cap;
    const double2* EL = envs + size_t(t) * (2 * n + 1) * E + size_t(q) * E;
    const double2* ER = envs + size_t(t) * (2 * n + 1) * E + size_t(n + 1 + q) * E;
    double2* tmp = tmp_all + (size_t(tl) * n + q) * S;
    double2* H = holes + (size_t(tl) * n + q) * S;
    const int l = mps.dl[q], r = mps.dr[q];
    const double2* A = mps.site[q];
    const char ch = labels[size_t(t) * n + (n - 1 - q)];
    for (long e = threadIdx.x; e < long(l) * 2 * r; e += blockDim.x) {
        const int a = int(e / (2 * r)), s = int((e / r) % 2), bp = int(e % r);
        double2 acc = cmake(0, 0);
        for (int ap = 0; ap < l; ++ap)
            cfma(acc, EL[size_t(a) * l + ap], pauli_conj_row(ch, A + size_t(ap) * 2 * r + bp, s, size_t(r)));
        tmp[e] = acc;
    }
    __syncthreads();
    for (long e = threadIdx.x; e < long(l) * 2 * r; e += blockDim.x) {
        const long as = e / r;
        const int b = int(e % r);
        double2 acc = cmake(0, 0);
        for (int bp = 0; bp < r; ++bp) cfma(acc, tmp[as * r + bp], ER[size_t(b) * r + bp]);
        H[e] = acc;
    }
}

// bar[q][e] (+)= sum over the chunk's terms, in term order, 2 Re(c_t) conj(H).
__global__ void __launch_bounds__(256) adj_pauli_accumulate_kernel(DeviceMps mps, double2* const* bars,
                                                                   const double2* holes, const double* coef_re,
                                                                   int t0, int count, int cap, int first) {
    const int q = blockIdx.y;
    const int n = mps.n;
    const size_t S = size_t(cap) * 2 * cap;
    const long len = long(mps.dl[q]) * 2 * mps.dr[q];
    for (long e = long(blockIdx.x) * blockDim.x + threadIdx.x; e < len; e += long(gridDim.x) * blockDim.x) {
        double2 acc = first ? cmake(0, 0) : bars[q][e];
        for (int tl = 0; tl < count; ++tl) {
            const double2 h = holes[(size_t(tl) * n + q) * S + e];
            const double c2 = 2.0 * coef_re[t0 + tl];
            acc.x += c2 * h.x;
            acc.y -= c2 * h.y;
        }
        bars[q][e] = acc;
    }
}

// Reverse of a one-qubit gate A' = u A at a site of shape dims[0] x 2 x
// dims[1] (one CTA): grad[slot] = Re <bar, du A_before> when du is given
// (a rotation angle), then bar <- u^H bar.
__global__ void __launch_bounds__(256) adj_one_qubit_kernel(double2* bar, const double2* before, const int* dims,
                                                            Adj1q g, double* grad) {
    const int l = dims[0], r = dims[1];
    __shared__ double red[8];
    double part = 0;
    for (long e = threadIdx.x; e < long(l) * r; e += blockDim.x) {
        const long a = e / r, b = e % r;
        double2* p0 = bar + (a * 2) * r + b;
        double2* p1 = p0 + r;
        const double2 y0 = *p0, y1 = *p1;
        if (g.has_du) {
            const double2 x0 = before[(a * 2) * r + b], x1 = before[(a * 2 + 1) * r + b];
            const double2 d0 = cadd(cmul(g.du[0], x0), cmul(g.du[1], x1));
            const double2 d1 = cadd(cmul(g.du[2], x0), cmul(g.du[3], x1));
            part += y0.x * d0.x + y0.y * d0.y + y1.x * d1.x + y1.y * d1.y;  // Re(conj(y) d)
        }
        // u^H y: (u^H)[s][x] = conj(u[x][s])
        *p0 = cadd(cconjmul(g.u[0], y0), cconjmul(g.u[2], y1));
        *p1 = cadd(cconjmul(g.u[1], y0), cconjmul(g.u[3], y1));
    }
    if (!g.has_du) return;
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) s += red[w];
        grad[g.slot] = s;
    }
}

// ----- reverse of a split -------------------------------------------------
// Workspace matrices are column-major with leading dimension R (= 2 chi_max).
__device__ __forceinline__ int adj_active(const AdjSplit& A, int i, double smax) {
    return A.sigma[A.perm[i]] > kAdjNullRel * smax;
}

// Stage 1 (grid-stride over R x R): the side of the SVD that W holds (U for
// theta, V for theta^H), scaled to unit columns and sorted by descending
// singular value; s^-1 and sqrt(s); U_bar = L_bar sqrt(s) and V_bar =
// R_bar^H sqrt(s) over the kept columns (zero elsewhere).
__global__ void __launch_bounds__(256) adj_split_prep_kernel(AdjSplit A) {
    const SplitState S = *A.st;
    const int m = S.rows, n = S.cols, N = min(m, n), M = max(m, n), k = S.chi, R = A.R;
    const double smax = N > 0 ? A.sigma[A.perm[0]] : 0.0;
    double2* Wside = S.w_rows_of_src ? A.V : A.U;
    const long stride = long(gridDim.x) * blockDim.x;
    for (long e = long(blockIdx.x) * blockDim.x + threadIdx.x; e < long(R) * R; e += stride) {
        const int i = int(e / R), j = int(e % R);  // column i, row j
        const bool col = i < N && adj_active(A, i, smax);
        const double s = i < N ? A.sigma[A.perm[i]] : 0.0;
        const double inv = col ? 1.0 / s : 0.0;
        if (j == 0 && i < R) {
            A.inv[i] = inv;
            A.sq[i] = (i < N && s > 0.0) ? sqrt(s) : 0.0;
        }
        Wside[e] = (col && j < M) ? cscale(A.w[size_t(A.perm[i]) * M + j], inv) : cmake(0, 0);
        const double sq = (i < N && s > 0.0) ? sqrt(s) : 0.0;
        // L_bar: m x k row-major (site p's cotangent [dl][2][k]); R_bar: k x n row-major.
        A.Ub[e] = (i < k && j < m) ? cscale(A.bar_l[size_t(j) * k + i], sq) : cmake(0, 0);
        A.Vb[e] = (i < k && j < n) ? cscale(cconj(A.bar_r[size_t(i) * n + j]), sq) : cmake(0, 0);
        if (i >= N || !col) {  // keep the other side's columns zero where there is no vector
            double2* other = S.w_rows_of_src ? A.U : A.V;
            other[e] = cmake(0, 0);
        }
    }
}

// The split's GEMMs as 32 x 32 FP64 tiles over strided, optionally
// conjugated views, with the dimensions read from the tape's SplitState.
// Stages (kAdjStage*): Other, the side W does not hold (V = theta^H U s^-1,
// or U = theta V s^-1); M = U^H U_bar; N = V^H V_bar; T1 += U Z;
// theta_bar = T1 V^H; theta_bar += U Q2^H; the cotangent of site p,
// theta_bar0 A_{p+1}^H; the cotangent of site p+1, A_p^H theta_bar0.

struct ZView {
    const double2* p;
    long rs, cs;
    int conj;
};

__device__ __forceinline__ double2 zat(const ZView& v, int i, int k) {
    const double2 x = v.p[i * v.rs + k * v.cs];
    return v.conj ? cconj(x) : x;
}

constexpr int kAdjT = 32, kAdjK = 16;

__global__ void __launch_bounds__(256) adj_split_gemm_kernel(AdjSplit A, int stage) {
    const SplitState S = *A.st;
    const int m = S.rows, n = S.cols, N = min(m, n), R = A.R, kin = S.k;
    ZView a, b;
    double2* c;
    long crs, ccs;
    int M_, N_, K_;
    bool acc = false;
    const double* cscale_by = nullptr;
    switch (stage) {
        case kAdjStageOther:
            if (!S.w_rows_of_src) {  // V (n x N) = theta^H (n x m) U (m x N), columns / s
                a = {A.theta, 1, n, 1};
                b = {A.U, 1, R, 0};
                c = A.V; M_ = n; N_ = N; K_ = m;
            } else {  // U (m x N) = theta (m x n) V (n x N), columns / s
                a = {A.theta, n, 1, 0};
                b = {A.V, 1, R, 0};
                c = A.U; M_ = m; N_ = N; K_ = n;
            }
            crs = 1; ccs = R; cscale_by = A.inv;
            break;
        case kAdjStageM:
            a = {A.U, R, 1, 1}; b = {A.Ub, 1, R, 0}; c = A.M; crs = 1; ccs = R; M_ = N; N_ = N; K_ = m;
            break;
        case kAdjStageN:
            a = {A.V, R, 1, 1}; b = {A.Vb, 1, R, 0}; c = A.Nm; crs = 1; ccs = R; M_ = N; N_ = N; K_ = n;
            break;
        case kAdjStageT1:
            a = {A.U, 1, R, 0}; b = {A.Z, 1, R, 0}; c = A.T1; crs = 1; ccs = R; M_ = m; N_ = N; K_ = N; acc = true;
            break;
        case kAdjStageTb:
            a = {A.T1, 1, R, 0}; b = {A.V, R, 1, 1}; c = A.tb; crs = 1; ccs = R; M_ = m; N_ = n; K_ = N;
            break;
        case kAdjStageTb2:
            a = {A.U, 1, R, 0}; b = {A.Vb, R, 1, 1}; c = A.tb; crs = 1; ccs = R; M_ = m; N_ = n; K_ = N; acc = true;
            break;
        case kAdjStageBarL:  // (m x kin) row-major = tb0 (m x n) * A_{p+1}^H (n x kin)
            a = {A.tb0, 1, R, 0}; b = {A.site_r, 1, n, 1}; c = A.bar_l; crs = kin; ccs = 1; M_ = m; N_ = kin; K_ = n;
            break;
        default:  // kAdjStageBarR: (kin x n) row-major = A_p^H (kin x m) * tb0 (m x n)
            a = {A.site_l, 1, kin, 1}; b = {A.tb0, 1, R, 0}; c = A.bar_r; crs = n; ccs = 1; M_ = kin; N_ = n; K_ = m;
            break;
    }
    const int i0 = blockIdx.y * kAdjT, j0 = blockIdx.x * kAdjT;
    if (i0 >= M_ || j0 >= N_) return;
    __shared__ double2 As[kAdjT][kAdjK + 1];
    __shared__ double2 Bs[kAdjK][kAdjT + 1];
    const int tid = threadIdx.x, tr = tid / 16, tc = tid % 16;
    double2 accv[2][2] = {{cmake(0, 0), cmake(0, 0)}, {cmake(0, 0), cmake(0, 0)}};
    for (int k0 = 0; k0 < K_; k0 += kAdjK) {
        for (int e = tid; e < kAdjT * kAdjK; e += 256) {
            const int r = e / kAdjK, cc = e % kAdjK;
            As[r][cc] = (i0 + r < M_ && k0 + cc < K_) ? zat(a, i0 + r, k0 + cc) : cmake(0, 0);
        }
        for (int e = tid; e < kAdjK * kAdjT; e += 256) {
            const int r = e / kAdjT, cc = e % kAdjT;
            Bs[r][cc] = (k0 + r < K_ && j0 + cc < N_) ? zat(b, k0 + r, j0 + cc) : cmake(0, 0);
        }
        __syncthreads();
#pragma unroll 4
        for (int cc = 0; cc < kAdjK; ++cc) {
            const double2 a0 = As[tr][cc], a1 = As[tr + 16][cc];
            const double2 b0 = Bs[cc][tc], b1 = Bs[cc][tc + 16];
            cfma(accv[0][0], a0, b0);
            cfma(accv[0][1], a0, b1);
            cfma(accv[1][0], a1, b0);
            cfma(accv[1][1], a1, b1);
        }
        __syncthreads();
    }
    for (int x = 0; x < 2; ++x)
        for (int y = 0; y < 2; ++y) {
            const int i = i0 + tr + 16 * x, j = j0 + tc + 16 * y;
            if (i >= M_ || j >= N_) continue;
            double2 v = accv[x][y];
            if (cscale_by) v = cscale(v, cscale_by[j]);
            double2* dst = c + i * crs + j * ccs;
            *dst = acc ? cadd(*dst, v) : v;
        }
}

// Stage 3 (grid-stride over R x R): s_bar, then Z, T1 = U_bar s^-1 (= Q1)
// and V_bar <- V_bar s^-1 (= Q2).  s_bar_i = (Re(U_i^H L_bar_i) +
// Re(R_bar_i V_i)) / (2 sqrt(s_i)) = Re(M_ii + N_ii) / (2 s_i) since
// U_bar_i = L_bar_i sqrt(s_i) and V_bar_i = R_bar_i^H sqrt(s_i).
__global__ void __launch_bounds__(256) adj_split_assemble_kernel(AdjSplit A) {
    const SplitState S = *A.st;
    const int m = S.rows, n = S.cols, N = min(m, n), k = S.chi, R = A.R;
    const double smax = N > 0 ? A.sigma[A.perm[0]] : 0.0;
    const double eps = kAdjLorentz * smax * smax * smax * smax;
    const long stride = long(gridDim.x) * blockDim.x;
    for (long e = long(blockIdx.x) * blockDim.x + threadIdx.x; e < long(R) * R; e += stride) {
        const int j = int(e / R), i = int(e % R);  // column j, row i
        if (i < N && j < N) {
            const double si = A.sigma[A.perm[i]], sj = A.sigma[A.perm[j]];
            const double inv_i = A.inv[i], inv_j = A.inv[j];
            const double2 Mij = A.M[size_t(j) * R + i], Mji = A.M[size_t(i) * R + j];
            const double2 Nij = A.Nm[size_t(j) * R + i], Nji = A.Nm[size_t(i) * R + j];
            double2 z;
            if (i == j) {
                const double sbar = (i < k && inv_i > 0.0) ? 0.5 * (Mij.x + Nij.x) * inv_i : 0.0;
                z = cmake(sbar, 0.5 * (Mij.y - Nij.y) * inv_i);
            } else if (inv_i > 0.0 && inv_j > 0.0) {
                const double d2 = sj * sj - si * si;
                const double F = d2 / (d2 * d2 + eps);
                const double2 mm = csub(Mij, cconj(Mji)), nn = csub(Nij, cconj(Nji));
                z = cscale(cadd(cscale(mm, sj), cscale(nn, si)), F);
            } else {
                z = cmake(0, 0);
            }
            // - M_ij / s_j (j kept) - conj(N_ji) / s_i (i kept)
            if (j < k) z = csub(z, cscale(Mij, inv_j));
            if (i < k) z = csub(z, cscale(cconj(Nji), inv_i));
            A.Z[e] = z;
        } else if (j < R && i < R) {
            A.Z[e] = cmake(0, 0);
        }
        // Q1 into T1 (m rows), Q2 in place of V_bar (n rows)
        if (j < N) {
            if (i < m) A.T1[e] = cscale(A.Ub[e], A.inv[j]);
            if (i < n) A.Vb[e] = cscale(A.Vb[e], A.inv[j]);
        }
    }
}

// Stage 5: the gate's reverse, theta_bar0[(a, si, ti, b)] = sum_{so, to}
// conj(u[(so, to), (si, ti)]) theta_bar[(a, so, to, b)].
__global__ void __launch_bounds__(256) adj_split_gate_kernel(AdjSplit A) {
    const SplitState S = *A.st;
    const int dl = S.dl, dr = S.dr, R = A.R;
    const long stride = long(gridDim.x) * blockDim.x;
    for (long e = long(blockIdx.x) * blockDim.x + threadIdx.x; e < long(dl) * dr; e += stride) {
        const int a = int(e / dr), b = int(e % dr);
        double2 y[4];
        for (int so = 0; so < 2; ++so)
            for (int to = 0; to < 2; ++to) y[so * 2 + to] = A.tb[size_t(to * dr + b) * R + (a * 2 + so)];
        for (int si = 0; si < 2; ++si)
            for (int ti = 0; ti < 2; ++ti) {
                double2 acc = cmake(0, 0);
                for (int x = 0; x < 4; ++x) cfma_conj(acc, A.u[x * 4 + si * 2 + ti], y[x]);
                A.tb0[size_t(ti * dr + b) * R + (a * 2 + si)] = acc;
            }
    }
}

}  // namespace wqc
