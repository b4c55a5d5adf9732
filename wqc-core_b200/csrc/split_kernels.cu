// Two-site split pipeline: merge + 4x4 gate, range finder (reference rule),
// one-sided Jacobi SVD in a thread-block cluster, cut, and sqrt(S) absorption.
//
// Reference path: src/tn/mps.rs:377-429 (two-site apply), 484-514 (merge),
// 833-866 (4x4 on theta), 937-981 (split dispatch), 983-1053 (range finder),
// 1124-1171 (truncated split), src/tn/svd_guard.rs:25-76 (truncation rule,
// ambiguity test), 91-139 (dust zeroing before the SVD).
//
// Every kernel takes the wave's job array and reads the job's bond dimensions
// from device memory, so a whole circuit can be enqueued without the host
// waiting on the device.
#include <cooperative_groups.h>

#include "common.cuh"
#include "split_kernels.cuh"

namespace cg = cooperative_groups;

namespace wqc {

// ---------------------------------------------------------------------------
// prepare: bond dims and the exact / range-finder decision (mps.rs:937-954).
// ---------------------------------------------------------------------------
__global__ void prepare_kernel(const SplitJob* jobs, SplitState* st, int njobs, DeviceMps mps) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    const SplitJob& J = jobs[j];
    SplitState s{};
    if (*mps.cancel) {  // cancelled: every later kernel of this wave skips the job
        s.skip = 1;
        st[j] = s;
        if (j == 0) atomicOr(mps.status, kStatusCancelled);
        return;
    }
    s.dl = mps.dl[J.p];
    s.dr = mps.dr[J.p + 1];
    s.k = min(mps.dr[J.p], mps.dl[J.p + 1]);
    s.rows = 2 * s.dl;
    s.cols = 2 * s.dr;
    s.ell = min(min(J.chi_max + kRsvdOversample, s.rows), s.cols);
    const unsigned long long f = (unsigned long long)s.rows * s.cols * s.ell;
    const unsigned long long side = kRsvdMinSide;
    const bool worth = f >= side * side * side;
    s.use_rsvd = (!J.reject && !J.exact_only && s.ell > 0 && s.ell < min(s.rows, s.cols) && worth) ? 1 : 0;
    s.need_exact = s.use_rsvd ? 0 : 1;
    s.path = s.use_rsvd ? WQC_SPLIT_RSVD : WQC_SPLIT_EXACT;
    s.w_rows_of_src = s.rows < s.cols ? 1 : 0;
    st[j] = s;
}

// ---------------------------------------------------------------------------
// merge + gate: theta'[(a,s'),(t',b)] = sum_{s,t} U[s't',st] sum_g L[a,s,g] R[g,t,b]
// One thread owns one (a, b) pair and its 2x2 physical block.  L and R tiles
// are staged in shared memory.
// ---------------------------------------------------------------------------
constexpr int kMergeTA = 16, kMergeTB = 16, kMergeTK = 16;

__global__ void __launch_bounds__(256) merge_gate_kernel(const SplitJob* jobs, const SplitState* st,
                                                         const SlotBuffers* slots, DeviceMps mps) {
    const int j = blockIdx.z;
    const SplitJob& J = jobs[j];
    const SplitState S = st[j];
    const int a0 = blockIdx.y * kMergeTA, b0 = blockIdx.x * kMergeTB;
    if (S.skip || a0 >= S.dl || b0 >= S.dr) return;
    const double2* L = mps.site[J.p];      // [dl][2][k']  with k' = dr of site p
    const double2* R = mps.site[J.p + 1];  // [k''][2][dr] with k'' = dl of site p+1
    const int ldl = mps.dr[J.p];           // row stride of L's (a,s) rows
    const int k = S.k;
    const int dr = S.dr;
    __shared__ double2 Ls[2 * kMergeTA][kMergeTK + 1];
    __shared__ double2 Rs[kMergeTK][2 * kMergeTB + 1];
    __shared__ double2 U[16];
    const int tid = threadIdx.x;
    if (tid < 16) U[tid] = J.u[tid];
    const int ta = tid / kMergeTB, tb = tid % kMergeTB;
    const int a = a0 + ta, b = b0 + tb;
    double2 acc[4] = {cmake(0, 0), cmake(0, 0), cmake(0, 0), cmake(0, 0)};  // [s][t]
    for (int g0 = 0; g0 < k; g0 += kMergeTK) {
        // L tile: rows (a0..a0+TA) x s, cols g
        for (int e = tid; e < 2 * kMergeTA * kMergeTK; e += 256) {
            const int r = e / kMergeTK, c = e % kMergeTK;
            const int aa = a0 + r / 2, ss = r % 2, gg = g0 + c;
            Ls[r][c] = (aa < S.dl && gg < k) ? L[(size_t(aa) * 2 + ss) * ldl + gg] : cmake(0, 0);
        }
        for (int e = tid; e < kMergeTK * 2 * kMergeTB; e += 256) {
            const int r = e / (2 * kMergeTB), c = e % (2 * kMergeTB);
            const int gg = g0 + r, tt = c / kMergeTB, bb = b0 + c % kMergeTB;
            Rs[r][c] = (gg < k && bb < dr) ? R[(size_t(gg) * 2 + tt) * dr + bb] : cmake(0, 0);
        }
        __syncthreads();
#pragma unroll 4
        for (int c = 0; c < kMergeTK; ++c) {
            const double2 l0 = Ls[2 * ta][c], l1 = Ls[2 * ta + 1][c];
            const double2 r0 = Rs[c][tb], r1 = Rs[c][kMergeTB + tb];
            cfma(acc[0], l0, r0);
            cfma(acc[1], l0, r1);
            cfma(acc[2], l1, r0);
            cfma(acc[3], l1, r1);
        }
        __syncthreads();
    }
    if (a >= S.dl || b >= dr) return;
    double2* th = slots[J.slot].theta;
    const int cols = S.cols;
    for (int so = 0; so < 2; ++so)
        for (int to = 0; to < 2; ++to) {
            double2 v = cmake(0, 0);
            for (int q = 0; q < 4; ++q) cfma(v, U[(so * 2 + to) * 4 + q], acc[q]);
            th[size_t(a * 2 + so) * cols + to * dr + b] = v;
        }
}

// ---------------------------------------------------------------------------
// Rademacher test matrix (mps.rs:1103-1122), generated in parallel: element i
// is the LCG state after i+1 steps from (salt | 1), reached by composing the
// affine map x -> a x + c with itself (exact 64-bit wrapping arithmetic).
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long lcg_jump(unsigned long long x, unsigned long long n) {
    unsigned long long A = 1ull, Cc = 0ull;            // accumulated map
    unsigned long long a = 6364136223846793005ull, c = 1ull;  // current power
    while (n) {
        if (n & 1ull) {
            A = A * a;
            Cc = Cc * a + c;
        }
        c = c * (a + 1ull);
        a = a * a;
        n >>= 1;
    }
    return A * x + Cc;
}

__global__ void omega_kernel(const SplitJob* jobs, const SplitState* st, const SlotBuffers* slots) {
    const int j = blockIdx.y;
    const SplitState S = st[j];
    if (!S.use_rsvd) return;
    const long total = long(S.cols) * S.ell;
    const unsigned long long salt =
        ((unsigned long long)S.rows * 0x9E37ull + (unsigned long long)S.cols) * 0x9E37ull + (unsigned long long)S.ell;
    const double scale = 1.0 / sqrt(double(S.cols));
    double2* om = slots[jobs[j].slot].omega;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const unsigned long long s = lcg_jump(salt | 1ull, (unsigned long long)i + 1ull);
        om[i] = cmake((s & 0x100ull) == 0 ? scale : -scale, (s & 0x200ull) == 0 ? scale : -scale);
    }
}

// ---------------------------------------------------------------------------
// Batched complex FP64 GEMM for the range finder.  C(m x n) = A(m x k) B(k x n)
// with strided / conjugated operand views derived per job from its state.
// ---------------------------------------------------------------------------
struct MatView {
    const double2* p;
    long rs, cs;
    int conj;
};

__device__ __forceinline__ double2 view_at(const MatView& v, int i, int kk) {
    const double2 x = v.p[i * v.rs + kk * v.cs];
    return v.conj ? cconj(x) : x;
}

constexpr int kGemmT = 32, kGemmK = 16;

__global__ void __launch_bounds__(256) rsvd_gemm_kernel(const SplitJob* jobs, const SplitState* st,
                                                        const SlotBuffers* slots, int stage) {
    const int j = blockIdx.z;
    const SplitState S = st[j];
    if (!S.use_rsvd) return;
    const SlotBuffers B = slots[jobs[j].slot];
    const int rows = S.rows, cols = S.cols, ell = S.ell;
    MatView A, Bv;
    double2* Cp;
    long c_rs, c_cs;
    int m, n, k;
    switch (stage) {
        case kStageY0:  // Y0 = theta * Omega   (rows x ell)
            A = {B.theta, cols, 1, 0};
            Bv = {B.omega, ell, 1, 0};
            Cp = B.y0; c_rs = ell; c_cs = 1; m = rows; n = ell; k = cols;
            break;
        case kStageZ:  // Z = theta^H * Y0    (cols x ell)
            A = {B.theta, 1, cols, 1};
            Bv = {B.y0, ell, 1, 0};
            Cp = B.zr; c_rs = ell; c_cs = 1; m = cols; n = ell; k = rows;
            break;
        case kStageY:  // Y = theta * Z, stored column-major for the QR
            A = {B.theta, cols, 1, 0};
            Bv = {B.zr, ell, 1, 0};
            Cp = B.y; c_rs = 1; c_cs = rows; m = rows; n = ell; k = cols;
            break;
        default:  // kStageB: B = Q^H * theta  (ell x cols), Q column-major rows x ell
            A = {B.q, rows, 1, 1};
            Bv = {B.theta, cols, 1, 0};
            Cp = B.b; c_rs = cols; c_cs = 1; m = ell; n = cols; k = rows;
            break;
    }
    const int i0 = blockIdx.y * kGemmT, n0 = blockIdx.x * kGemmT;
    if (i0 >= m || n0 >= n) return;
    __shared__ double2 As[kGemmT][kGemmK + 1];
    __shared__ double2 Bs[kGemmK][kGemmT + 1];
    const int tid = threadIdx.x;
    const int tr = tid / 16, tc = tid % 16;  // 2x2 outputs per thread
    double2 acc[2][2] = {{cmake(0, 0), cmake(0, 0)}, {cmake(0, 0), cmake(0, 0)}};
    for (int k0 = 0; k0 < k; k0 += kGemmK) {
        for (int e = tid; e < kGemmT * kGemmK; e += 256) {
            const int r = e / kGemmK, c = e % kGemmK;
            As[r][c] = (i0 + r < m && k0 + c < k) ? view_at(A, i0 + r, k0 + c) : cmake(0, 0);
        }
        for (int e = tid; e < kGemmK * kGemmT; e += 256) {
            const int r = e / kGemmT, c = e % kGemmT;
            Bs[r][c] = (k0 + r < k && n0 + c < n) ? view_at(Bv, k0 + r, n0 + c) : cmake(0, 0);
        }
        __syncthreads();
#pragma unroll 4
        for (int c = 0; c < kGemmK; ++c) {
            const double2 a0 = As[tr][c], a1 = As[tr + 16][c];
            const double2 b0 = Bs[c][tc], b1 = Bs[c][tc + 16];
            cfma(acc[0][0], a0, b0);
            cfma(acc[0][1], a0, b1);
            cfma(acc[1][0], a1, b0);
            cfma(acc[1][1], a1, b1);
        }
        __syncthreads();
    }
    for (int x = 0; x < 2; ++x)
        for (int y = 0; y < 2; ++y) {
            const int i = i0 + tr + 16 * x, jj = n0 + tc + 16 * y;
            if (i < m && jj < n) Cp[i * c_rs + jj * c_cs] = acc[x][y];
        }
}

// ---------------------------------------------------------------------------
// Householder QR of Y (rows x ell, column-major) and the thin Q, one CTA per
// job (LAPACK zgeqr2 + zung2r conventions; thin Q is unique up to column
// phases, which the range finder's results do not depend on).
// ---------------------------------------------------------------------------
constexpr int kQrThreads = 512;

__device__ double block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double t = 0;
    const int nw = blockDim.x >> 5;
    for (int w = 0; w < nw; ++w) t += red[w];  // every thread sums in the same order
    __syncthreads();
    return t;
}

__global__ void __launch_bounds__(kQrThreads) householder_qr_kernel(const SplitJob* jobs, const SplitState* st,
                                                                    const SlotBuffers* slots) {
    const int j = blockIdx.x;
    const SplitState S = st[j];
    if (!S.use_rsvd) return;
    const SlotBuffers B = slots[jobs[j].slot];
    const int m = S.rows, n = S.ell;
    double2* y = B.y;
    double2* q = B.q;
    double2* tau = B.tau;
    __shared__ double red[kQrThreads / 32];
    __shared__ double2 v[512];
    __shared__ double2 s_tau;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = kQrThreads / 32;
    for (int c = 0; c < n; ++c) {
        double2* col = y + size_t(c) * m;
        double part = 0;
        for (int i = c + 1 + tid; i < m; i += kQrThreads) part += cnorm2(col[i]);
        const double xnorm2 = block_sum(part, red);
        const double2 alpha = col[c];
        double2 t = cmake(0, 0);
        double2 sc = cmake(0, 0);
        double beta = alpha.x;
        const bool trivial = (xnorm2 == 0.0 && alpha.y == 0.0);
        if (!trivial) {
            beta = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2);
            if (alpha.x >= 0) beta = -beta;
            t = cmake((beta - alpha.x) / beta, -alpha.y / beta);
            // sc = 1 / (alpha - beta)
            const double2 d = cmake(alpha.x - beta, alpha.y);
            const double dn = d.x * d.x + d.y * d.y;
            sc = cmake(d.x / dn, -d.y / dn);
        }
        __syncthreads();  // everyone has read col[c]
        for (int i = c + 1 + tid; i < m; i += kQrThreads) {
            const double2 x = trivial ? col[i] : cmul(col[i], sc);
            col[i] = x;
            v[i] = x;
        }
        if (tid == 0) {
            col[c] = cmake(beta, 0.0);
            v[c] = cmake(1.0, 0.0);
            tau[c] = t;
            s_tau = t;
        }
        __syncthreads();
        if (!trivial) {
            const double2 tc = cconj(s_tau);  // apply H^H
            for (int kk = c + 1 + wid; kk < n; kk += nw) {
                double2* ck = y + size_t(kk) * m;
                double2 w = cmake(0, 0);
                for (int i = c + lane; i < m; i += 32) cfma_conj(w, v[i], ck[i]);
                for (int o = 16; o > 0; o >>= 1) {
                    w.x += __shfl_xor_sync(0xffffffffu, w.x, o);
                    w.y += __shfl_xor_sync(0xffffffffu, w.y, o);
                }
                w = cmul(tc, w);
                for (int i = c + lane; i < m; i += 32) ck[i] = csub(ck[i], cmul(v[i], w));
            }
        }
        __syncthreads();
    }
    // Thin Q = H_0 ... H_{n-1} [I; 0], accumulated backward.
    for (int e = tid; e < m * n; e += kQrThreads) {
        const int r = e % m, c = e / m;
        q[e] = cmake(r == c ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    for (int c = n - 1; c >= 0; --c) {
        const double2* col = y + size_t(c) * m;
        for (int i = c + 1 + tid; i < m; i += kQrThreads) v[i] = col[i];
        if (tid == 0) {
            v[c] = cmake(1.0, 0.0);
            s_tau = tau[c];
        }
        __syncthreads();
        const double2 tc = s_tau;
        if (tc.x != 0.0 || tc.y != 0.0) {
            for (int kk = c + wid; kk < n; kk += nw) {
                double2* ck = q + size_t(kk) * m;
                double2 w = cmake(0, 0);
                for (int i = c + lane; i < m; i += 32) cfma_conj(w, v[i], ck[i]);
                for (int o = 16; o > 0; o >>= 1) {
                    w.x += __shfl_xor_sync(0xffffffffu, w.x, o);
                    w.y += __shfl_xor_sync(0xffffffffu, w.y, o);
                }
                w = cmul(tc, w);
                for (int i = c + lane; i < m; i += 32) ck[i] = csub(ck[i], cmul(v[i], w));
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// The same Householder QR and thin Q on a thread-block cluster: CTA r holds
// columns [r*cpc, (r+1)*cpc) of Y and of Q in shared memory.  At step c the
// owner of column c forms the reflector, publishes v_c and tau_c in a
// double-buffered slot of its shared memory and updates its own trailing
// columns; after one cluster barrier the CTAs to its right copy v_c through
// distributed shared memory and update theirs.  Q is then accumulated
// backward with every reflector read from its owner.  Same arithmetic as the
// single-CTA kernel above.  With kGlobalCols the columns stay in the slot's
// Y and Q buffers (L2-resident) instead of shared memory, for shapes whose
// columns do not fit (Y of 512 x 272 at chi 256); only the reflector
// broadcast and the local reflector copy live in shared memory.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void reflect_columns(double2* cols, int ldc, int count, const double2* v, double2 t,
                                                int c, int m, int lane, int wid, int nw) {
    for (int kk = wid; kk < count; kk += nw) {
        double2* ck = cols + size_t(kk) * ldc;
        double2 w = cmake(0, 0);
        for (int i = c + lane; i < m; i += 32) cfma_conj(w, v[i], ck[i]);
        for (int o = 16; o > 0; o >>= 1) {
            w.x += __shfl_xor_sync(0xffffffffu, w.x, o);
            w.y += __shfl_xor_sync(0xffffffffu, w.y, o);
        }
        w = cmul(t, w);
        for (int i = c + lane; i < m; i += 32) ck[i] = csub(ck[i], cmul(v[i], w));
    }
}

// Split cluster barrier: arrive (releasing this thread's writes) and wait
// (acquiring the others') as two steps, so a CTA can work between them.
__device__ __forceinline__ void cluster_arrive_release() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait_acquire() {
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

template <bool kGlobalCols>
__global__ void __launch_bounds__(kQrClusterThreads, 1) qr_cluster_kernel(const SplitJob* jobs, const SplitState* st,
                                                                           const SlotBuffers* slots) {
    cg::cluster_group cluster = cg::this_cluster();
    const int C = int(cluster.num_blocks());
    const int rank = int(cluster.block_rank());
    const int j = blockIdx.x / C;
    const SplitState S = st[j];
    if (!S.use_rsvd) return;  // uniform over the cluster
    const SlotBuffers B = slots[jobs[j].slot];
    const int m = S.rows, n = S.ell;
    const int cpc = (n + C - 1) / C;
    const int c0 = min(n, rank * cpc), c1 = min(n, c0 + cpc), nloc = c1 - c0;
    extern __shared__ __align__(16) double2 qsm[];
    double2* Ys = kGlobalCols ? B.y + size_t(c0) * m : qsm;                      // cpc columns of m
    double2* Qs = kGlobalCols ? B.q + size_t(c0) * m : qsm + size_t(cpc) * m;    // cpc columns of m
    double2* bcast = kGlobalCols ? qsm : qsm + size_t(2) * cpc * m;              // 2 slots of m
    double2* vloc = bcast + size_t(2) * m;                                        // m
    double2* taus = vloc + m;                                                     // cpc local tau values
    __shared__ double red[kQrClusterThreads / 32];
    __shared__ double2 s_tau[2];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = kQrClusterThreads / 32;
    if (!kGlobalCols)
        for (int e = tid; e < nloc * m; e += kQrClusterThreads) Ys[e] = B.y[size_t(c0) * m + e];
    __syncthreads();
    for (int c = 0; c < n; ++c) {
        const int owner = c / cpc;
        const int slot = c & 1;
        if (rank == owner) {
            double2* col = Ys + size_t(c - c0) * m;
            double part = 0;
            for (int i = c + 1 + tid; i < m; i += kQrClusterThreads) part += cnorm2(col[i]);
            const double xnorm2 = block_sum(part, red);
            const double2 alpha = col[c];
            double2 t = cmake(0, 0), sc = cmake(0, 0);
            double beta = alpha.x;
            const bool trivial = (xnorm2 == 0.0 && alpha.y == 0.0);
            if (!trivial) {
                beta = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2);
                if (alpha.x >= 0) beta = -beta;
                t = cmake((beta - alpha.x) / beta, -alpha.y / beta);
                const double2 d = cmake(alpha.x - beta, alpha.y);
                const double dn = d.x * d.x + d.y * d.y;
                sc = cmake(d.x / dn, -d.y / dn);
            }
            __syncthreads();
            double2* bv = bcast + size_t(slot) * m;
            for (int i = c + 1 + tid; i < m; i += kQrClusterThreads) {
                const double2 x = trivial ? col[i] : cmul(col[i], sc);
                col[i] = x;
                bv[i] = x;
            }
            if (tid == 0) {
                col[c] = cmake(beta, 0.0);
                bv[c] = cmake(1.0, 0.0);
                taus[c - c0] = t;
                s_tau[slot] = t;
            }
            __syncthreads();
            // v_c and tau_c are published: release them to the cluster, then
            // update this CTA's trailing columns while the others copy v_c.
            cluster_arrive_release();
            if (!trivial)
                reflect_columns(Ys + size_t(c - c0 + 1) * m, m, c1 - c - 1, bv, cconj(t), c, m, lane, wid, nw);
            // The wait below orders nothing written after the arrive: the
            // next column's norm must not start before every warp's update.
            __syncthreads();
            cluster_wait_acquire();
        } else {
            cluster_arrive_release();
            cluster_wait_acquire();
            if (rank > owner && nloc > 0) {
                const double2* rv = cluster.map_shared_rank(bcast, owner) + size_t(slot) * m;
                for (int i = c + tid; i < m; i += kQrClusterThreads) vloc[i] = rv[i];
                const double2 t = *cluster.map_shared_rank(&s_tau[slot], owner);
                __syncthreads();
                if (t.x != 0.0 || t.y != 0.0) reflect_columns(Ys, m, nloc, vloc, cconj(t), c, m, lane, wid, nw);
                __syncthreads();
            }
        }
    }
    if (kGlobalCols) __threadfence();
    cluster.sync();  // every reflector is final
    for (int e = tid; e < nloc * m; e += kQrClusterThreads) {
        const int r = e % m, cc = c0 + e / m;
        Qs[e] = cmake(r == cc ? 1.0 : 0.0, 0.0);
    }
    // Backward accumulation, Q = H_0 ... H_{n-1} E.  Reflector c-1 is read
    // from its owner into registers before reflector c is applied, and
    // stored into the other half of a double buffer (vloc / bcast) after,
    // so the distributed-shared-memory latency overlaps the update.
    double2 pv[kQrRowsPerThread];
    double2 ptau = cmake(0, 0);
    auto pull = [&](int c) {
        const int owner = c / cpc;
        const double2* rcol = kGlobalCols ? B.y + size_t(c) * m
                                          : cluster.map_shared_rank(Ys, owner) + size_t(c - owner * cpc) * m;
#pragma unroll
        for (int k = 0; k < kQrRowsPerThread; ++k) {
            const int i = c + 1 + tid + k * kQrClusterThreads;
            if (i < m) pv[k] = kGlobalCols ? __ldcg(rcol + i) : rcol[i];
        }
        if (tid == 0) ptau = *(cluster.map_shared_rank(taus, owner) + (c - owner * cpc));
    };
    auto place = [&](int c, double2* dst, int sl) {
#pragma unroll
        for (int k = 0; k < kQrRowsPerThread; ++k) {
            const int i = c + 1 + tid + k * kQrClusterThreads;
            if (i < m) dst[i] = pv[k];
        }
        if (tid == 0) {
            dst[c] = cmake(1.0, 0.0);
            s_tau[sl] = ptau;
        }
    };
    int cur = 0;
    if (nloc > 0) {
        pull(c1 - 1);
        place(c1 - 1, vloc, 0);
    }
    __syncthreads();
    for (int c = nloc > 0 ? c1 - 1 : -1; c >= 0; --c) {
        if (c > 0) pull(c - 1);
        const double2 t = s_tau[cur];
        const int first = max(c, c0);
        if ((t.x != 0.0 || t.y != 0.0) && first < c1)
            reflect_columns(Qs + size_t(first - c0) * m, m, c1 - first, cur ? bcast : vloc, t, c, m, lane, wid,
                            nw);
        if (c > 0) place(c - 1, cur ? vloc : bcast, cur ^ 1);
        __syncthreads();
        cur ^= 1;
    }
    if (!kGlobalCols) {
        for (int e = tid; e < nloc * m; e += kQrClusterThreads) B.q[size_t(c0) * m + e] = Qs[e];
        for (int e = tid; e < nloc * m; e += kQrClusterThreads) B.y[size_t(c0) * m + e] = Ys[e];
    }
    if (tid < nloc) B.tau[c0 + tid] = taus[tid];
    cluster.sync();  // no CTA leaves while another may still read its shared memory
}

// ---------------------------------------------------------------------------
// One-sided Hestenes Jacobi SVD on a thread-block cluster.
//
// The tall working matrix W (M x N, padded to N' = 2*C*b columns) is held
// column by column in the shared memory of the C CTAs of one cluster: CTA r
// holds block r ("top") and block 2C-1-r ("bottom"), b columns each.  The
// right rotations are not accumulated: at convergence W = X V = U Sigma, and
// the cut recovers the other side from W and X (absorb_kernel), which keeps
// the step's shared-memory traffic (its bound) to W's M rows.  A sweep orthogonalises the pairs inside each block, then
// runs 2C-1 block steps of the b*b cross pairs, rotating the blocks between
// CTAs by the circle method through distributed shared memory.  Each pair
// rotation is the reference's rephase-then-real-rotation (svd_guard.rs:
// 174-199), with column dot products reduced by warp shuffles.
// ---------------------------------------------------------------------------
struct JacobiCtl {
    int rot;
    unsigned long long relmax_bits;  // largest |gamma|/sqrt(alpha beta) seen this sweep (non-negative double bits)
    double fro_part;
    double chk_in, chk_out;  // this CTA's share of ||X||_F^2 (after dust zeroing) and of sum sigma^2
};

// The Frobenius part of the reference's factorisation check (svd_reproduces,
// svd_guard.rs:234-255): sum sigma^2 must equal ||X||_F^2 of the dust-zeroed
// matrix to SVD_CHECK_TOL = 1e-9 relative (plus 1e-28).  The precision form's
// complex64 columns carry ~1e-6 of rounding, so it is held to 1e-4.  The
// probe-vector part needs V, which this Jacobi does not accumulate.
constexpr double kSvdCheckTol = 1e-9;
constexpr double kSvdCheckTolFp32 = 1e-4;

__device__ __forceinline__ double block_total(double v, double* red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double t = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t += red[w];
    return t;
}

__device__ __forceinline__ int circle_at(int pos, int step, int b) {
    if (pos == 0) return 0;
    const int m = b - 1;
    int v = (pos - 1 - step) % m;
    if (v < 0) v += m;
    return v + 1;
}

// Rotates columns xp, xq (each W then Z, `len` entries, W part `M`).  All
// lanes compute bitwise-identical reductions (xor butterfly), so the branch is
// warp-uniform.  Returns 1 when a rotation was applied.
//
// Two guards keep every applied rotation unitary and the sweep finite:
// |gamma| is taken with hypot when |gamma|^2 nears the subnormal range, so
// the phase stays of unit modulus; and a pair whose smaller column has
// alpha <= floor = (1e-15 ||W||_F)^2 (FP32 columns: (1e-6 ||W||_F)^2) is left
// alone.  Such a column is at the storage's rounding level: its direction is
// noise, rotating it against another column changes nothing above
// floor * ||W||_F^2, and rotating it anyway lets exactly parallel columns (a
// rank-deficient theta) be re-rotated every sweep until their products go
// subnormal, and pairs of noise columns keep |gamma|/sqrt(alpha beta) near
// 1e-8 forever (seen on a 256 x 144 range-finder matrix of the 50-qubit
// circuit, which then never met the stop test).
//
// The columns are complex128 (double2) in the plain form and complex64
// (float2) in the precision form.  The precision form accumulates the dot
// products and applies the rotation in FP32; the rotation parameters, the
// tests against tol and the noise floor, and the convergence measure are
// FP64 in both.
template <typename T>
struct JacobiReal;
template <>
struct JacobiReal<double2> {
    using R = double;
};
template <>
struct JacobiReal<float2> {
    using R = float;
};

// Warp sums of four values, every lane receiving the same four totals (so
// branches on them stay warp-uniform).  Instead of four butterflies (20
// shuffles) the first two levels split the values between the lane halves
// (lanes with bit 4 clear keep a, b and pass g, h; then bit 3 picks one of
// the two), three more levels finish one value per quarter of the warp, and
// four broadcasts from lanes 0, 8, 16, 24 hand out the totals: 10 shuffles,
// on the dependent chain of every rotation round.
template <typename R>
__device__ __forceinline__ void warp_sum4(R& a, R& b, R& g, R& h, int lane) {
    const bool hi = lane & 16;
    R k0 = hi ? g : a, k1 = hi ? h : b;
    k0 += __shfl_xor_sync(0xffffffffu, hi ? a : g, 16);
    k1 += __shfl_xor_sync(0xffffffffu, hi ? b : h, 16);
    const bool b3 = lane & 8;
    R v = b3 ? k1 : k0;
    v += __shfl_xor_sync(0xffffffffu, b3 ? k0 : k1, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    a = __shfl_sync(0xffffffffu, v, 0);
    b = __shfl_sync(0xffffffffu, v, 8);
    g = __shfl_sync(0xffffffffu, v, 16);
    h = __shfl_sync(0xffffffffu, v, 24);
}

// Rotation parameters from alpha = |p|^2, beta = |q|^2, gamma = <p, q>:
// returns false when the pair is left alone (noise-level column, or already
// orthogonal to tol), else c and w = s * phase.
__device__ __forceinline__ bool jacobi_params(double a, double bb, double gr, double gi, double tol, double noise_floor,
                                              double& relmax, double& c, double& wr, double& wi) {
    // Squared forms keep the dependent chain short: |gamma|^2 against
    // tol^2 alpha beta, one reciprocal square root for the phase.
    const double g2 = fma(gr, gr, gi * gi);
    const double ab = a * bb;
    if (fmin(a, bb) <= noise_floor) return false;  // the smaller column is at the storage's rounding level
    relmax = fmax(relmax, g2 / ab);  // squared ratio; the caller compares with squared bounds
    if (g2 == 0.0 || g2 <= tol * tol * ab) return false;
    double pr, pi, zeta;
    if (g2 > 1e-290) {
        const double inv_g = rsqrt(g2);
        pr = gr * inv_g;
        pi = gi * inv_g;
        zeta = 0.5 * (bb - a) * inv_g;
    } else {  // |gamma|^2 near the subnormal range: hypot keeps the phase of unit modulus
        const double g = hypot(gr, gi);
        pr = gr / g;
        pi = gi / g;
        zeta = (bb - a) / (2.0 * g);
    }
    // tan = sign(zeta) / (|zeta| + u) with u = sqrt(1 + zeta^2) gives
    // c^2 = (u + |zeta|) / (2u) and s^2 = 1 / (2u (u + |zeta|)): after one
    // reciprocal square root, c and s are two independent ones, no division.
    const double az = fabs(zeta);
    const double q = fma(zeta, zeta, 1.0);
    const double ru = rsqrt(q);
    const double u = q * ru;
    const double c2 = fma(0.5 * az, ru, 0.5);
    c = c2 * rsqrt(c2);
    const double s = copysign(rsqrt(2.0 * u * (u + az)), zeta);
    // With w = s * phase the rephased rotation (svd_guard.rs:189-197) is
    // xp' = c xp - conj(w) xq,  xq' = w xp + c xq   (|phase| = 1).
    wr = s * pr;
    wi = s * pi;
    return true;
}

template <typename T>
__device__ __forceinline__ int jacobi_rotate(T* __restrict__ xp, T* __restrict__ xq, int M, int len, double tol,
                                             double noise_floor, int lane, double& relmax) {
    using R = typename JacobiReal<T>::R;
    // Two rows per lane per iteration into two accumulator sets: the loads
    // of the second row overlap the first's FMAs and the dependent chains
    // are half as long (the columns are distinct, hence __restrict__).
    R a_ = 0, b_ = 0, gr_ = 0, gi_ = 0, a1 = 0, b1 = 0, gr1 = 0, gi1 = 0;
    int r0 = lane;
    for (; r0 + 32 < M; r0 += 64) {
        const T u = xp[r0], v = xq[r0], u1 = xp[r0 + 32], v1 = xq[r0 + 32];
        a_ = fma(u.x, u.x, fma(u.y, u.y, a_));
        b_ = fma(v.x, v.x, fma(v.y, v.y, b_));
        gr_ = fma(u.x, v.x, fma(u.y, v.y, gr_));
        gi_ = fma(u.x, v.y, fma(-u.y, v.x, gi_));
        a1 = fma(u1.x, u1.x, fma(u1.y, u1.y, a1));
        b1 = fma(v1.x, v1.x, fma(v1.y, v1.y, b1));
        gr1 = fma(u1.x, v1.x, fma(u1.y, v1.y, gr1));
        gi1 = fma(u1.x, v1.y, fma(-u1.y, v1.x, gi1));
    }
    if (r0 < M) {
        const T u = xp[r0], v = xq[r0];
        a_ = fma(u.x, u.x, fma(u.y, u.y, a_));
        b_ = fma(v.x, v.x, fma(v.y, v.y, b_));
        gr_ = fma(u.x, v.x, fma(u.y, v.y, gr_));
        gi_ = fma(u.x, v.y, fma(-u.y, v.x, gi_));
    }
    a_ += a1;
    b_ += b1;
    gr_ += gr1;
    gi_ += gi1;
    warp_sum4(a_, b_, gr_, gi_, lane);
    double c64, wr64, wi64;
    if (!jacobi_params(a_, b_, gr_, gi_, tol, noise_floor, relmax, c64, wr64, wi64)) return 0;
    const R wr = R(wr64), wi = R(wi64), cr = R(c64);
    auto rot = [&](const T u, const T v, T& p, T& q) {
        p.x = fma(cr, u.x, -fma(wr, v.x, wi * v.y));
        p.y = fma(cr, u.y, -fma(wr, v.y, -wi * v.x));
        q.x = fma(wr, u.x, fma(-wi, u.y, cr * v.x));
        q.y = fma(wr, u.y, fma(wi, u.x, cr * v.y));
    };
    // Four rows per lane per iteration: all loads issue before the stores.
    int r = lane;
    for (; r + 96 < len; r += 128) {
        T u[4], v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            u[k] = xp[r + 32 * k];
            v[k] = xq[r + 32 * k];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            T p, q;
            rot(u[k], v[k], p, q);
            xp[r + 32 * k] = p;
            xq[r + 32 * k] = q;
        }
    }
    for (; r < len; r += 32) {
        T p, q;
        rot(xp[r], xq[r], p, q);
        xp[r] = p;
        xq[r] = q;
    }
    return 1;
}

// The same rotation with p held in registers (rows lane + 32 k, M <= 32 *
// kJacobiRegRows): in a block step warp i keeps its top column for all b
// rounds, so only the partner q moves through shared memory (the step is
// bound by shared-memory bandwidth).
constexpr int kJacobiRegRows = 8;

template <typename T>
__device__ __forceinline__ int jacobi_rotate_reg(T (&u)[kJacobiRegRows], T* __restrict__ xq, int M, int len,
                                                 T* __restrict__ xp_tail, double tol, double noise_floor, int lane,
                                                 double& relmax) {
    using R = typename JacobiReal<T>::R;
    T v[kJacobiRegRows];
#pragma unroll
    for (int k = 0; k < kJacobiRegRows; ++k) {
        const int r = lane + 32 * k;
        if (r < M) {
            v[k] = xq[r];
        } else {
            v[k].x = v[k].y = R(0);
        }
    }
    R a_ = 0, b_ = 0, gr_ = 0, gi_ = 0, a1 = 0, b1 = 0, gr1 = 0, gi1 = 0;
#pragma unroll
    for (int k = 0; k < kJacobiRegRows; k += 2) {
        a_ = fma(u[k].x, u[k].x, fma(u[k].y, u[k].y, a_));
        b_ = fma(v[k].x, v[k].x, fma(v[k].y, v[k].y, b_));
        gr_ = fma(u[k].x, v[k].x, fma(u[k].y, v[k].y, gr_));
        gi_ = fma(u[k].x, v[k].y, fma(-u[k].y, v[k].x, gi_));
        a1 = fma(u[k + 1].x, u[k + 1].x, fma(u[k + 1].y, u[k + 1].y, a1));
        b1 = fma(v[k + 1].x, v[k + 1].x, fma(v[k + 1].y, v[k + 1].y, b1));
        gr1 = fma(u[k + 1].x, v[k + 1].x, fma(u[k + 1].y, v[k + 1].y, gr1));
        gi1 = fma(u[k + 1].x, v[k + 1].y, fma(-u[k + 1].y, v[k + 1].x, gi1));
    }
    a_ += a1;
    b_ += b1;
    gr_ += gr1;
    gi_ += gi1;
    warp_sum4(a_, b_, gr_, gi_, lane);
    double c64, wr64, wi64;
    if (!jacobi_params(a_, b_, gr_, gi_, tol, noise_floor, relmax, c64, wr64, wi64)) return 0;
    const R wr = R(wr64), wi = R(wi64), cr = R(c64);
#pragma unroll
    for (int k = 0; k < kJacobiRegRows; ++k) {
        const int r = lane + 32 * k;
        if (r < M) {
            T p, q;
            p.x = fma(cr, u[k].x, -fma(wr, v[k].x, wi * v[k].y));
            p.y = fma(cr, u[k].y, -fma(wr, v[k].y, -wi * v[k].x));
            q.x = fma(wr, u[k].x, fma(-wi, u[k].y, cr * v[k].x));
            q.y = fma(wr, u[k].y, fma(wi, u[k].x, cr * v[k].y));
            u[k] = p;
            xq[r] = q;
        }
    }
    // Rows M .. len-1 (the right rotations accumulated in the precision
    // form's first phase) stay in shared memory for both columns.
    for (int r = M + lane; r < len; r += 32) {
        const T x = xp_tail[r], y = xq[r];
        T p, q;
        p.x = fma(cr, x.x, -fma(wr, y.x, wi * y.y));
        p.y = fma(cr, x.y, -fma(wr, y.y, -wi * y.x));
        q.x = fma(wr, x.x, fma(-wi, x.y, cr * y.x));
        q.y = fma(wr, x.y, fma(wi, x.x, cr * y.y));
        xp_tail[r] = p;
        xq[r] = q;
    }
    return 1;
}

// Block copy into another CTA's shared memory: eight local loads, then eight
// remote stores (which do not stall the thread).
template <typename T>
__device__ __forceinline__ void dsmem_push(T* __restrict__ dst, const T* __restrict__ src, size_t n, int tid,
                                           int nthreads) {
    size_t e = tid;
    const size_t st = nthreads;
    for (; e + 7 * st < n; e += 8 * st) {
        T v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = src[e + u * st];
#pragma unroll
        for (int u = 0; u < 8; ++u) dst[e + u * st] = v[u];
    }
    for (; e < n; e += st) dst[e] = src[e];
}

__device__ __forceinline__ void jacobi_task(const SplitJob& J, const SplitState& S, const SlotBuffers& B, int mode,
                                            const double2*& src, int& sr, int& sc, int& ld, int& rows_of_src) {
    if (mode == kJacobiRsvd) {  // W = B^H, B is ell x cols row-major
        src = B.b;
        sr = S.ell;
        sc = S.cols;
        ld = S.cols;
        rows_of_src = 1;
    } else {  // exact: W = theta (rows >= cols) or theta^H
        src = B.theta;
        sr = S.rows;
        sc = S.cols;
        ld = S.cols;
        rows_of_src = S.w_rows_of_src;
    }
}

__device__ __forceinline__ bool jacobi_active(const SplitState& S, int mode) {
    if (mode == kJacobiRsvd) return S.use_rsvd != 0;
    // The exact path's two modes never overlap: prepare sets path EXACT, and a
    // fallback changes a range-finder split's path to RSVD_FALLBACK only.
    if (mode == kJacobiExact) return S.need_exact != 0 && S.path == WQC_SPLIT_EXACT;
    return S.need_exact != 0 && S.path == WQC_SPLIT_RSVD_FALLBACK;
}

template <typename T>
__device__ __forceinline__ T to_store(double2 x);
template <>
__device__ __forceinline__ double2 to_store<double2>(double2 x) {
    return x;
}
template <>
__device__ __forceinline__ float2 to_store<float2>(double2 x) {
    return make_float2(float(x.x), float(x.y));
}
__device__ __forceinline__ double2 to_f64(double2 x) { return x; }
__device__ __forceinline__ double2 to_f64(float2 x) { return make_double2(x.x, x.y); }

template <typename T, bool kReg>
__global__ void __launch_bounds__(kReg ? kJacobiRegThreads : kJacobiThreads) jacobi_cluster_kernel(
    const SplitJob* jobs, SplitState* st, const SlotBuffers* slots, const int* idx, int mode, int phase,
    int max_sweeps, int* status, unsigned long long* counters) {
    constexpr bool kF64 = sizeof(T) == sizeof(double2);
    cg::cluster_group cluster = cg::this_cluster();
    const int C = int(cluster.num_blocks());
    const int rank = int(cluster.block_rank());
    const int j = idx[blockIdx.x / C];
    const SplitState S = st[j];
    if (!jacobi_active(S, mode)) return;  // uniform over the cluster
    const SplitJob& J = jobs[j];
    const SlotBuffers Bf = slots[J.slot];
    const double2* src;
    int sr, sc, ld, rows_of_src;
    jacobi_task(J, S, Bf, mode, src, sr, sc, ld, rows_of_src);
    const int M = rows_of_src ? sc : sr;
    const int N = rows_of_src ? sr : sc;
    const int quantum = 4 * C;
    const int Np = ((N + quantum - 1) / quantum) * quantum;
    const int b = Np / (2 * C);
    // W only, the other side's vectors are recovered from W after the SVD;
    // the precision form's first phase also carries V (N rows under W).
    const int vrows = phase == kPhaseFp32V ? N : 0;
    const int len = M + vrows;
    const bool colmajor = rows_of_src || phase == kPhaseFinish;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    __shared__ JacobiCtl ctl;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int nthreads = blockDim.x;  // a multiple of 32, at most kJacobiThreads
    const int nwarps = nthreads / 32;
    auto buf = [&](int k) { return smem + size_t(k) * b * len; };
    __shared__ double red[kJacobiThreads / 32];

    if (tid == 0) ctl.rot = 0;
    // Buffer roles and block ids after xk block exchanges, the same on every
    // CTA without reading a neighbour's state: CTA 0 keeps its top block
    // (position 0) in buffer 0 and receives into buffer 1; every other CTA
    // turns its (top, bottom, spare) buffers one place per exchange; the
    // blocks at positions 1 .. 2C-1 move one position on per exchange, so
    // position p holds block circle_at(p, xk, 2C).
    int xk = 0;
    auto top_buf_of = [&](int r, int k) { return r == 0 ? 0 : (3 - k % 3) % 3; };
    auto bot_buf_of = [&](int r, int k) { return r == 0 ? 1 : (4 - k % 3) % 3; };
    auto spare_buf_of = [&](int k) { return (5 - k % 3) % 3; };
    // Frobenius norm over the columns this CTA loads, then over the cluster.
    // The precision form's finishing phase starts from X V (column-major in
    // the slot's W buffer), formed from the dust-zeroed X.
    const double2* wsrc = Bf.w;
    auto src_at = [&](int i, int col) -> double2 {
        if (phase == kPhaseFinish) return wsrc[size_t(col) * M + i];
        return rows_of_src ? cconj(src[size_t(col) * ld + i]) : src[size_t(i) * ld + col];
    };
    double part = 0;
    for (int half = 0; half < 2; ++half) {
        const int id = half == 0 ? rank : 2 * C - 1 - rank;
        for (int e = tid; e < b * M; e += nthreads) {
            int c, i;
            if (colmajor) { c = e / M; i = e % M; } else { i = e / b; c = e % b; }
            const int col = id * b + c;
            if (col < N) part += cnorm2(src_at(i, col));
        }
    }
    {
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == 0) red[wid] = part;
        __syncthreads();
        if (tid == 0) {
            double t = 0;
            for (int w = 0; w < nwarps; ++w) t += red[w];
            ctl.fro_part = t;
        }
    }
    cluster.sync();
    double fro2 = 0;
    for (int r = 0; r < C; ++r) fro2 += cluster.map_shared_rank(&ctl, r)->fro_part;
    const double dust = sqrt(fro2) * kDustRel;
    const double dust2 = dust * dust;
    double chk_in = 0, chk_out = 0;
    // Load W (dust-zeroed; padding columns zero).
    for (int half = 0; half < 2; ++half) {
        const int id = half == 0 ? rank : 2 * C - 1 - rank;
        T* base = buf(half);
        for (int e = tid; e < b * M; e += nthreads) {
            int c, i;
            if (colmajor) { c = e / M; i = e % M; } else { i = e / b; c = e % b; }
            const int col = id * b + c;
            double2 x = col < N ? src_at(i, col) : cmake(0, 0);
            if (phase != kPhaseFinish && cnorm2(x) < dust2) x = cmake(0, 0);
            chk_in += cnorm2(x);
            base[size_t(c) * len + i] = to_store<T>(x);
        }
        for (int e = tid; e < b * vrows; e += nthreads) {  // V = I (padding columns: zero)
            const int c = e / vrows, i = e % vrows;
            base[size_t(c) * len + M + i] = to_store<T>(cmake(id * b + c == i ? 1.0 : 0.0, 0.0));
        }
    }
    __syncthreads();
    // Pairs count as orthogonal at |gamma| <= tol sqrt(alpha beta), just
    // above the rounding of an M <= 512 dot product (sqrt(M) eps: 5e-15 in
    // FP64, 3e-6 in FP32), so the sweeps stop and the singular values are
    // exact to second order.  A sweep that every pair entered orthogonal to
    // stop_rel ends the iteration: one-sided Jacobi converges quadratically,
    // so that sweep leaves them at about stop_rel^2 <= tol.  Columns at the
    // storage's rounding level against ||W||_F are left alone (noise floor).
    const double tol = kF64 ? 1e-14 : 4e-6;
    const double stop_rel2 = kF64 ? 1e-16 : 4e-6;  // squared: 1e-8 and 2e-3
    const double noise_floor = (kF64 ? 1e-30 : 1e-12) * fro2;  // squared column norm: 1e-15 (1e-6) of ||W||_F
    int sweep = 0;
    bool converged = false;
    int ctl_rot_last = 0;
    unsigned long long ctl_relmax_bits_last = 0ull;
    for (; sweep < max_sweeps; ++sweep) {
        if (tid == 0) {
            ctl.rot = 0;
            ctl.relmax_bits = 0ull;
        }
        __syncthreads();
        int my_rot = 0;
        double my_rel = 0.0;
        // Pairs inside each block (circle method on b columns).
        for (int step = 0; step < b - 1; ++step) {
            for (int pq = wid; pq < b; pq += nwarps) {
                const bool top = pq < b / 2;
                const int i = top ? pq : pq - b / 2;
                T* base = buf(top ? top_buf_of(rank, xk) : bot_buf_of(rank, xk));
                const int e1 = circle_at(i, step, b), e2 = circle_at(b - 1 - i, step, b);
                my_rot += jacobi_rotate(base + size_t(e1) * len, base + size_t(e2) * len, M, len, tol, noise_floor, lane, my_rel);
            }
            __syncthreads();
        }
        // Cross pairs between the two blocks, 2C-1 block steps.  Warp i pairs
        // its top column i with bottom column (i + k) % b in round k; when
        // every warp owns one top column and it fits, the column stays in
        // registers for the b rounds.
        const bool reg_path = kReg && M <= 32 * kJacobiRegRows && nwarps >= b;
        for (int bs = 0; bs < 2 * C - 1; ++bs) {
            T* tb = buf(top_buf_of(rank, xk));
            T* bb = buf(bot_buf_of(rank, xk));
            if (reg_path) {
                T u[kJacobiRegRows];
                T* col = tb + size_t(wid) * len;
                if (wid < b) {
#pragma unroll
                    for (int kk = 0; kk < kJacobiRegRows; ++kk) {
                        const int r = lane + 32 * kk;
                        if (r < M) {
                            u[kk] = col[r];
                        } else {
                            u[kk].x = u[kk].y = 0;
                        }
                    }
                }
                for (int k = 0; k < b; ++k) {
                    if (wid < b)
                        my_rot += jacobi_rotate_reg(u, bb + size_t((wid + k) % b) * len, M, len, col, tol,
                                                    noise_floor, lane, my_rel);
                    __syncthreads();
                }
                if (wid < b) {
#pragma unroll
                    for (int kk = 0; kk < kJacobiRegRows; ++kk) {
                        const int r = lane + 32 * kk;
                        if (r < M) col[r] = u[kk];
                    }
                }
                __syncthreads();
            } else {
                for (int k = 0; k < b; ++k) {
                    for (int i = wid; i < b; i += nwarps) {
                        const int e2 = (i + k) % b;
                        my_rot += jacobi_rotate(tb + size_t(i) * len, bb + size_t(e2) * len, M, len, tol, noise_floor,
                                                lane, my_rel);
                    }
                    __syncthreads();
                }
            }
            if (C == 1) continue;
            // Circle rotation of blocks between CTAs (push protocol, one spare
            // buffer, two cluster barriers).  Phase 1: as soon as its own
            // rotations are done, CTA r <= C-2 stores the block that moves to
            // CTA r+1's top position (CTA 0: its bottom block, the others:
            // their top) into CTA r+1's spare buffer, which CTA r+1 does not
            // touch while it rotates.  After the barrier, when every CTA has
            // finished rotating and sending, phase 2: CTA r >= 1 stores its
            // bottom block over CTA r-1's old top (CTA 0: its old bottom),
            // both already sent.  The second barrier makes the received
            // blocks visible.  Remote stores do not wait for DSMEM latency
            // as remote loads do (measured: ~2700 cycles per pulled block of
            // 66 KB).  Roles and block ids follow from the exchange count.
            const size_t blk = size_t(b) * len;
            if (rank <= C - 2) {
                const int src = rank == 0 ? bot_buf_of(0, xk) : top_buf_of(rank, xk);
                dsmem_push(cluster.map_shared_rank(smem, rank + 1) + size_t(spare_buf_of(xk)) * blk, buf(src), blk,
                           tid, nthreads);
            }
            cluster.sync();
            if (rank >= 1) {
                const int dst = rank - 1;
                const int dbuf = dst == 0 ? bot_buf_of(0, xk) : top_buf_of(dst, xk);
                dsmem_push(cluster.map_shared_rank(smem, dst) + size_t(dbuf) * blk, buf(bot_buf_of(rank, xk)), blk,
                           tid, nthreads);
            }
            ++xk;
            cluster.sync();
        }
        // Cluster-wide rotation count decides convergence.
        if (lane == 0 && my_rot) atomicAdd(&ctl.rot, my_rot);
        if (lane == 0 && my_rel > 0.0) atomicMax(&ctl.relmax_bits, (unsigned long long)__double_as_longlong(my_rel));
        __syncthreads();
        int total = 0;
        double relmax = 0.0;
        if (C == 1) {
            total = ctl.rot;
            relmax = __longlong_as_double((long long)ctl.relmax_bits);
            __syncthreads();
        } else {
            cluster.sync();
            for (int r = 0; r < C; ++r) {
                const JacobiCtl* rc = cluster.map_shared_rank(&ctl, r);
                total += rc->rot;
                relmax = fmax(relmax, __longlong_as_double((long long)rc->relmax_bits));
            }
            cluster.sync();
        }
        // Converged when nothing rotated, or when every pair entered this
        // sweep orthogonal to stop_rel (FP64: 1e-8, leaving them at about
        // 1e-16, below the rotation tolerance, so a verification sweep would
        // rotate nothing).
        ctl_rot_last = total;
        ctl_relmax_bits_last = (unsigned long long)__double_as_longlong(relmax);
        if (total == 0 || relmax < stop_rel2) {  // relmax holds squared ratios
            converged = true;
            break;
        }
    }
    if (tid == 0 && rank == 0) {
        if (!converged) {
            atomicOr(status, kStatusJacobiNoConvergence);
            // The first such split, its last sweep's rotation count and largest
            // squared |gamma| / sqrt(alpha beta), for the error message.
            if (atomicCAS(status + 1, 0, J.seq + 1) == 0) {
                const unsigned long long bits = ctl_relmax_bits_last;
                status[2] = ctl_rot_last;
                status[3] = int(bits >> 32);
                status[4] = int(bits & 0xffffffffull);
            }
        }
        if (phase != kPhaseFp32V) atomicAdd(counters + 0, 1ull);
        atomicAdd(counters + (phase == kPhaseFp32V ? 2 : 1), (unsigned long long)(converged ? sweep + 1 : sweep));
    }
    if (phase == kPhaseFp32V) {
        // The accumulated V (FP64) for the finishing phase, and ||X||_F^2
        // for its dust zeroing of X.
        for (int half = 0; half < 2; ++half) {
            const int id = circle_at(half == 0 ? rank : 2 * C - 1 - rank, xk, 2 * C);
            const T* base = buf(half == 0 ? top_buf_of(rank, xk) : bot_buf_of(rank, xk));
            for (int c = wid; c < b; c += nwarps) {
                const int col = id * b + c;
                if (col >= N) continue;
                for (int r = lane; r < N; r += 32) Bf.z[size_t(col) * N + r] = to_f64(base[size_t(c) * len + M + r]);
            }
        }
        if (rank == 0 && tid == 0) st[j].fro2 = fro2;
        cluster.sync();  // no CTA leaves while another may still read its shared memory
        return;
    }
    // Write back: W columns and column norms.
    for (int half = 0; half < 2; ++half) {
        const int id = circle_at(half == 0 ? rank : 2 * C - 1 - rank, xk, 2 * C);
        const T* base = buf(half == 0 ? top_buf_of(rank, xk) : bot_buf_of(rank, xk));
        for (int c = wid; c < b; c += nwarps) {
            const int col = id * b + c;
            if (col >= N) continue;
            const T* x = base + size_t(c) * len;
            double s2 = 0;  // column norms in FP64 in both forms
            for (int r = lane; r < M; r += 32) {
                const double2 v = to_f64(x[r]);
                s2 = fma(v.x, v.x, fma(v.y, v.y, s2));
                Bf.w[size_t(col) * M + r] = v;
            }
            for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
            if (lane == 0) {
                Bf.sigma[col] = sqrt(s2);
                chk_out += s2;
            }
        }
    }
    // Factorisation check over the cluster (every CTA reaches it: the loop
    // above ends on a cluster-uniform decision).
    {
        const double in_cta = block_total(chk_in, red);
        const double out_cta = block_total(chk_out, red);
        if (tid == 0) {
            ctl.chk_in = in_cta;
            ctl.chk_out = out_cta;
        }
        cluster.sync();
        if (rank == 0 && tid == 0) {
            double tin = 0, tout = 0;
            for (int r = 0; r < C; ++r) {
                const JacobiCtl* rc = cluster.map_shared_rank(&ctl, r);
                tin += rc->chk_in;
                tout += rc->chk_out;
            }
            const double tol = kF64 ? kSvdCheckTol : kSvdCheckTolFp32;
            if (fabs(tout - tin) > tol * tin + 1e-28) atomicOr(status, kStatusSvdCheck);
        }
        cluster.sync();  // no CTA leaves while rank 0 reads its shared memory
    }
}

// ---------------------------------------------------------------------------
// The same Jacobi SVD for working matrices too large for a cluster's shared
// memory (theta up to 512 x 512 at chi 256: W takes 4 MB in FP64, a 16-CTA
// cluster holds 3.6 MB with two working blocks per CTA).  The padded W
// columns live in the slot's global workspace `gs`, which stays in L2.
// The N' = 2Kb columns form 2K blocks of b; a sweep runs 2K-1 steps of the
// circle method over the blocks (position 0 fixed, block at position p at
// step s: circle_at(p, s, 2K)), and at each step CTA r takes the block pairs
// r, r+C, ... < K: it loads both blocks into shared memory, rotates the b*b
// cross pairs (and, at a sweep's first step, the pairs inside each block),
// and stores them back.  One cluster barrier separates the steps: every
// block is held by one pair per step, so a block's store and its next load
// are ordered by that barrier.  Rotation rule, tolerances, stop test and
// outputs are those of jacobi_cluster_kernel.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kJacobiStagedThreads) jacobi_staged_kernel(const SplitJob* jobs, SplitState* st,
                                                                         const SlotBuffers* slots, const int* idx,
                                                                         int mode, int phase, int max_sweeps, int b,
                                                                         int* status, unsigned long long* counters) {
    constexpr bool kF64 = sizeof(T) == sizeof(double2);
    cg::cluster_group cluster = cg::this_cluster();
    const int C = int(cluster.num_blocks());
    const int rank = int(cluster.block_rank());
    const int j = idx[blockIdx.x / C];
    const SplitState S = st[j];
    if (!jacobi_active(S, mode)) return;  // uniform over the cluster
    const SplitJob& J = jobs[j];
    const SlotBuffers Bf = slots[J.slot];
    const double2* src;
    int sr, sc, ld, rows_of_src;
    jacobi_task(J, S, Bf, mode, src, sr, sc, ld, rows_of_src);
    const int M = rows_of_src ? sc : sr;
    const int N = rows_of_src ? sr : sc;
    const int K = (N + 2 * b - 1) / (2 * b);
    const int nblk = 2 * K;
    const int Np = nblk * b;
    const int vrows = phase == kPhaseFp32V ? N : 0;  // as in jacobi_cluster_kernel
    const int len = M + vrows;
    const size_t blk = size_t(b) * len;
    T* G = reinterpret_cast<T*>(Bf.gs);
    if (G == nullptr) {  // a state sized without the workspace (uniform over the cluster)
        if (threadIdx.x == 0 && rank == 0) atomicOr(status, kStatusBadShape);
        return;
    }

    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sA = reinterpret_cast<T*>(smem_raw);
    T* sB = sA + blk;
    __shared__ JacobiCtl ctl;
    __shared__ double red[kJacobiStagedThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int nthreads = blockDim.x;
    const int nwarps = nthreads / 32;
    const double2* wsrc = Bf.w;
    auto src_at = [&](int i, int col) -> double2 {
        if (phase == kPhaseFinish) return wsrc[size_t(col) * M + i];
        return rows_of_src ? cconj(src[size_t(col) * ld + i]) : src[size_t(i) * ld + col];
    };
    if (tid == 0) ctl.rot = 0;
    // Frobenius norm: CTA r reads columns r, r+C, ...
    double part = 0;
    for (int col = rank; col < N; col += C)
        for (int i = tid; i < M; i += nthreads) part += cnorm2(src_at(i, col));
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if (lane == 0) red[wid] = part;
    __syncthreads();
    if (tid == 0) {
        double t = 0;
        for (int w = 0; w < nwarps; ++w) t += red[w];
        ctl.fro_part = t;
    }
    cluster.sync();
    double fro2 = 0;
    for (int r = 0; r < C; ++r) fro2 += cluster.map_shared_rank(&ctl, r)->fro_part;
    const double dust = sqrt(fro2) * kDustRel;
    const double dust2 = dust * dust;
    // W (dust-zeroed, zero padding columns) into the workspace.
    double chk_in = 0, chk_out = 0;
    for (int col = rank; col < Np; col += C) {
        T* x = G + size_t(col) * len;
        for (int i = tid; i < M; i += nthreads) {
            double2 v = col < N ? src_at(i, col) : cmake(0, 0);
            if (phase != kPhaseFinish && cnorm2(v) < dust2) v = cmake(0, 0);
            chk_in += cnorm2(v);
            x[i] = to_store<T>(v);
        }
        for (int i = tid; i < vrows; i += nthreads) x[M + i] = to_store<T>(cmake(col == i ? 1.0 : 0.0, 0.0));
    }
    __threadfence();
    cluster.sync();
    const double tol = kF64 ? 1e-14 : 4e-6;
    const double stop_rel2 = kF64 ? 1e-16 : 4e-6;
    const double noise_floor = (kF64 ? 1e-30 : 1e-12) * fro2;  // squared column norm: 1e-15 (1e-6) of ||W||_F
    int sweep = 0;
    bool converged = false;
    int ctl_rot_last = 0;
    unsigned long long ctl_relmax_bits_last = 0ull;
    for (; sweep < max_sweeps; ++sweep) {
        if (tid == 0) {
            ctl.rot = 0;
            ctl.relmax_bits = 0ull;
        }
        __syncthreads();
        int my_rot = 0;
        double my_rel = 0.0;
        for (int step = 0; step < nblk - 1; ++step) {
            for (int ps = rank; ps < K; ps += C) {
                const int ida = circle_at(ps, step, nblk), idb = circle_at(nblk - 1 - ps, step, nblk);
                const T* ga = G + size_t(ida) * blk;
                const T* gb = G + size_t(idb) * blk;
                for (size_t e = tid; e < blk; e += nthreads) {
                    sA[e] = __ldcg(ga + e);
                    sB[e] = __ldcg(gb + e);
                }
                __syncthreads();
                if (step == 0) {  // pairs inside each block, once per sweep
                    // Circle method on bb = b rounded up to even positions; for
                    // an odd b the extra position is a dummy and its pair is
                    // skipped (uniformly per warp).
                    const int bb = b + (b & 1);
                    for (int s2 = 0; s2 < bb - 1; ++s2) {
                        for (int pq = wid; pq < bb; pq += nwarps) {
                            const bool top = pq < bb / 2;
                            const int i = top ? pq : pq - bb / 2;
                            T* base = top ? sA : sB;
                            const int e1 = circle_at(i, s2, bb), e2 = circle_at(bb - 1 - i, s2, bb);
                            if (e1 < b && e2 < b)
                                my_rot += jacobi_rotate(base + size_t(e1) * len, base + size_t(e2) * len, M, len,
                                                        tol, noise_floor, lane, my_rel);
                        }
                        __syncthreads();
                    }
                }
                for (int k = 0; k < b; ++k) {
                    for (int i = wid; i < b; i += nwarps) {
                        const int e2 = (i + k) % b;
                        my_rot += jacobi_rotate(sA + size_t(i) * len, sB + size_t(e2) * len, M, len, tol,
                                                noise_floor, lane, my_rel);
                    }
                    __syncthreads();
                }
                T* wa = G + size_t(ida) * blk;
                T* wb = G + size_t(idb) * blk;
                for (size_t e = tid; e < blk; e += nthreads) {
                    wa[e] = sA[e];
                    wb[e] = sB[e];
                }
                __syncthreads();  // the next pair's loads overwrite sA, sB
            }
            __threadfence();
            cluster.sync();
        }
        if (lane == 0 && my_rot) atomicAdd(&ctl.rot, my_rot);
        if (lane == 0 && my_rel > 0.0) atomicMax(&ctl.relmax_bits, (unsigned long long)__double_as_longlong(my_rel));
        __syncthreads();
        int total = 0;
        double relmax = 0.0;
        cluster.sync();
        for (int r = 0; r < C; ++r) {
            const JacobiCtl* rc = cluster.map_shared_rank(&ctl, r);
            total += rc->rot;
            relmax = fmax(relmax, __longlong_as_double((long long)rc->relmax_bits));
        }
        cluster.sync();
        ctl_rot_last = total;
        ctl_relmax_bits_last = (unsigned long long)__double_as_longlong(relmax);
        if (total == 0 || relmax < stop_rel2) {
            converged = true;
            break;
        }
    }
    if (tid == 0 && rank == 0) {
        if (!converged) {
            atomicOr(status, kStatusJacobiNoConvergence);
            // The first such split, its last sweep's rotation count and largest
            // squared |gamma| / sqrt(alpha beta), for the error message.
            if (atomicCAS(status + 1, 0, J.seq + 1) == 0) {
                const unsigned long long bits = ctl_relmax_bits_last;
                status[2] = ctl_rot_last;
                status[3] = int(bits >> 32);
                status[4] = int(bits & 0xffffffffull);
            }
        }
        if (phase != kPhaseFp32V) atomicAdd(counters + 0, 1ull);
        atomicAdd(counters + (phase == kPhaseFp32V ? 2 : 1), (unsigned long long)(converged ? sweep + 1 : sweep));
    }
    if (phase == kPhaseFp32V) {  // V (FP64) and ||X||_F^2 for the finishing phase
        for (int col = rank + C * wid; col < N; col += C * nwarps)
            for (int r = lane; r < N; r += 32) Bf.z[size_t(col) * N + r] = to_f64(__ldcg(G + size_t(col) * len + M + r));
        if (rank == 0 && tid == 0) st[j].fro2 = fro2;
        cluster.sync();
        return;
    }
    // Write back W and the column norms; CTA r takes columns r, r+C, ...,
    // one warp per column.
    for (int col = rank + C * wid; col < N; col += C * nwarps) {
        const T* x = G + size_t(col) * len;
        double s2 = 0;
        for (int r = lane; r < M; r += 32) {
            const double2 v = to_f64(__ldcg(x + r));
            s2 = fma(v.x, v.x, fma(v.y, v.y, s2));
            Bf.w[size_t(col) * M + r] = v;
        }
        for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        if (lane == 0) {
            Bf.sigma[col] = sqrt(s2);
            chk_out += s2;
        }
    }
    // Factorisation check over the cluster, as in jacobi_cluster_kernel.
    {
        const double in_cta = block_total(chk_in, red);
        const double out_cta = block_total(chk_out, red);
        if (tid == 0) {
            ctl.chk_in = in_cta;
            ctl.chk_out = out_cta;
        }
        cluster.sync();
        if (rank == 0 && tid == 0) {
            double tin = 0, tout = 0;
            for (int r = 0; r < C; ++r) {
                const JacobiCtl* rc = cluster.map_shared_rank(&ctl, r);
                tin += rc->chk_in;
                tout += rc->chk_out;
            }
            const double tol = kF64 ? kSvdCheckTol : kSvdCheckTolFp32;
            if (fabs(tout - tin) > tol * tin + 1e-28) atomicOr(status, kStatusSvdCheck);
        }
        cluster.sync();  // no CTA leaves while rank 0 reads its shared memory
    }
}

// ---------------------------------------------------------------------------
// The probe-vector half of the reference's factorisation check
// (svd_reproduces, svd_guard.rs:256-283): U Sigma V^H x must reproduce X x
// for the two fixed probes x_j = (sin t, cos t), t = (j + 1) (0.754877666 +
// p 0.56984029), to 1e-9 ||X||_F ||x|| + 1e-14.  The Jacobi keeps W = X V =
// U Sigma and no V, and U Sigma V^H x = U U^H X x over the columns with
// sigma > 0, so with y = X x the rebuilt vector is W diag(1/sigma^2) W^H y:
// it equals y only when W's columns are orthogonal and span X's range.
// Columns at the storage's rounding level (the Jacobi's noise floor) are
// left out: their direction is noise and they carry less than the tolerance.
// One CTA per (job, probe); a failure sets the same status as the Frobenius
// check ("failed its check").
// ---------------------------------------------------------------------------
constexpr int kProbeMax = 512;

__global__ void __launch_bounds__(256) svd_probe_kernel(const SplitJob* jobs, const SplitState* st,
                                                        const SlotBuffers* slots, int mode, int fp32, int* status) {
    const int j = blockIdx.x;
    const int probe = blockIdx.y;
    const SplitState S = st[j];
    if (!jacobi_active(S, mode)) return;
    const SplitJob& J = jobs[j];
    const SlotBuffers Bf = slots[J.slot];
    const double2* src;
    int sr, sc, ld, rows_of_src;
    jacobi_task(J, S, Bf, mode, src, sr, sc, ld, rows_of_src);
    const int M = rows_of_src ? sc : sr;
    const int N = rows_of_src ? sr : sc;
    if (M > kProbeMax || N > kProbeMax) {
        if (threadIdx.x == 0) atomicOr(status, kStatusBadShape);
        return;
    }
    __shared__ double2 xs[kProbeMax], ys[kProbeMax], zs[kProbeMax];
    __shared__ double red[8];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    const double step = 0.754877666 + double(probe) * 0.56984029;
    double fro2_part = 0;
    for (int c = tid; c < N; c += blockDim.x) {
        double sn, cs;
        sincos(double(c + 1) * step, &sn, &cs);
        xs[c] = cmake(sn, cs);
        const double sg = Bf.sigma[c];
        fro2_part += sg * sg;
    }
    for (int o = 16; o > 0; o >>= 1) fro2_part += __shfl_xor_sync(0xffffffffu, fro2_part, o);
    if (lane == 0) red[wid] = fro2_part;
    __syncthreads();
    double fro2 = 0;
    for (int w = 0; w < nw; ++w) fro2 += red[w];
    const double floor2 = (fp32 ? 1e-12 : 1e-30) * fro2;
    // y = X x, one warp per row.
    for (int i = wid; i < M; i += nw) {
        double2 acc = cmake(0, 0);
        for (int c = lane; c < N; c += 32) {
            const double2 a = rows_of_src ? cconj(src[size_t(c) * ld + i]) : src[size_t(i) * ld + c];
            cfma(acc, a, xs[c]);
        }
        for (int o = 16; o > 0; o >>= 1) {
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
        }
        if (lane == 0) ys[i] = acc;
    }
    __syncthreads();
    // z = diag(1/sigma^2) W^H y, one warp per column.
    for (int c = wid; c < N; c += nw) {
        const double sg = Bf.sigma[c];
        double2 acc = cmake(0, 0);
        if (sg * sg > floor2) {
            const double2* wc = Bf.w + size_t(c) * M;
            for (int i = lane; i < M; i += 32) cfma_conj(acc, wc[i], ys[i]);
            for (int o = 16; o > 0; o >>= 1) {
                acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
                acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
            }
            acc = cscale(acc, 1.0 / (sg * sg));
        }
        if (lane == 0) zs[c] = acc;
    }
    __syncthreads();
    // |y - W z|^2, one thread per row.
    double err2 = 0;
    for (int i = tid; i < M; i += blockDim.x) {
        double2 r = cmake(0, 0);
        for (int c = 0; c < N; ++c) cfma(r, Bf.w[size_t(c) * M + i], zs[c]);
        err2 += cnorm2(csub(ys[i], r));
    }
    for (int o = 16; o > 0; o >>= 1) err2 += __shfl_xor_sync(0xffffffffu, err2, o);
    __syncthreads();
    if (lane == 0) red[wid] = err2;
    __syncthreads();
    if (tid == 0) {
        double e2 = 0;
        for (int w = 0; w < nw; ++w) e2 += red[w];
        const double tol = fp32 ? 1e-4 : 1e-9;  // the Frobenius check's tolerance of each form
        if (!(sqrt(e2) <= tol * sqrt(fro2) * sqrt(double(N)) + 1e-14)) atomicOr(status, kStatusSvdCheck);
    }
}

// ---------------------------------------------------------------------------
// The precision form's FP64 products between its Jacobi phases (see
// split_kernels.cuh): 32 x 32 tiles, batched over the wave's jobs.  G lives
// in the slot's omega and y0 buffers and V' in zr and y (each pair holds
// 2 R ell >= R^2 entries); none of them is in use while an SVD of the job
// runs.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) precond_gemm_kernel(const SplitJob* jobs, const SplitState* st,
                                                           const SlotBuffers* slots, int mode, int stage) {
    const int j = blockIdx.z;
    const SplitState S = st[j];
    if (!jacobi_active(S, mode)) return;
    const SplitJob& J = jobs[j];
    const SlotBuffers B = slots[J.slot];
    const double2* src;
    int sr, sc, ld, rows_of_src;
    jacobi_task(J, S, B, mode, src, sr, sc, ld, rows_of_src);
    const int M = rows_of_src ? sc : sr, N = rows_of_src ? sr : sc;
    const bool last = stage == kPrecondXV;
    const int m = last ? M : N, n = N, k = N;
    const int i0 = blockIdx.y * kGemmT, n0 = blockIdx.x * kGemmT;
    if (i0 >= m || n0 >= n) return;
    // Two Newton-Schulz steps: V (z) -> zr -> z; then X V from z.
    const bool second = stage >= kPrecondGram2;
    const double2* V = last ? B.z : (second ? B.zr : B.z);
    double2* G = B.omega;
    double2* Vout = second ? B.z : B.zr;
    const bool gram = stage == kPrecondGram1 || stage == kPrecondGram2;
    const double dust2 = kDustRel * kDustRel * S.fro2;
    auto a_at = [&](int i, int kk) -> double2 {
        if (gram) return cconj(V[size_t(i) * N + kk]);  // V^H
        if (!last) return V[size_t(kk) * N + i];
        const double2 x = rows_of_src ? cconj(src[size_t(kk) * ld + i]) : src[size_t(i) * ld + kk];
        return cnorm2(x) < dust2 ? cmake(0, 0) : x;  // X, dust-zeroed as the first phase loaded it
    };
    auto b_at = [&](int kk, int jj) -> double2 {
        if (gram) return V[size_t(jj) * N + kk];
        if (!last) {
            const double2 g = G[size_t(jj) * N + kk];
            return cmake((kk == jj ? 1.5 : 0.0) - 0.5 * g.x, -0.5 * g.y);
        }
        return V[size_t(jj) * N + kk];
    };
    __shared__ double2 As[kGemmT][kGemmK + 1];
    __shared__ double2 Bs[kGemmK][kGemmT + 1];
    const int tid = threadIdx.x, tr = tid / 16, tc = tid % 16;
    double2 acc[2][2] = {{cmake(0, 0), cmake(0, 0)}, {cmake(0, 0), cmake(0, 0)}};
    for (int k0 = 0; k0 < k; k0 += kGemmK) {
        for (int e = tid; e < kGemmT * kGemmK; e += 256) {
            const int r = e / kGemmK, c = e % kGemmK;
            As[r][c] = (i0 + r < m && k0 + c < k) ? a_at(i0 + r, k0 + c) : cmake(0, 0);
        }
        for (int e = tid; e < kGemmK * kGemmT; e += 256) {
            const int r = e / kGemmT, c = e % kGemmT;
            Bs[r][c] = (k0 + r < k && n0 + c < n) ? b_at(k0 + r, n0 + c) : cmake(0, 0);
        }
        __syncthreads();
#pragma unroll 4
        for (int c = 0; c < kGemmK; ++c) {
            const double2 a0 = As[tr][c], a1 = As[tr + 16][c];
            const double2 b0 = Bs[c][tc], b1 = Bs[c][tc + 16];
            cfma(acc[0][0], a0, b0);
            cfma(acc[0][1], a0, b1);
            cfma(acc[1][0], a1, b0);
            cfma(acc[1][1], a1, b1);
        }
        __syncthreads();
    }
    double2* C = gram ? G : last ? B.w : Vout;
    const int ldc = last ? M : N;
    for (int x = 0; x < 2; ++x)
        for (int y = 0; y < 2; ++y) {
            const int i = i0 + tr + 16 * x, jj = n0 + tc + 16 * y;
            if (i < m && jj < n) C[size_t(jj) * ldc + i] = acc[x][y];
        }
}

// ---------------------------------------------------------------------------
// finalize: stable descending sort, truncation rule, ambiguity test,
// discarded weight and the split record.
// ---------------------------------------------------------------------------
__global__ void finalize_kernel(const SplitJob* jobs, SplitState* st, const SlotBuffers* slots, int mode,
                                int chi_max, double noise_rel, wqc_split_info* records, int* status) {
    const int j = blockIdx.x;
    SplitState& S = st[j];
    if (!jacobi_active(S, mode)) return;
    const SplitJob& J = jobs[j];
    const SlotBuffers B = slots[J.slot];
    const int N = mode == kJacobiRsvd ? S.ell : min(S.rows, S.cols);
    __shared__ double vals[1024];
    const int tid = threadIdx.x;
    // rank_j = #{i : s_i > s_j or (s_i == s_j and i < j)}
    for (int c = tid; c < N; c += blockDim.x) {
        const double sj = B.sigma[c];
        int r = 0;
        for (int i = 0; i < N; ++i) {
            const double si = B.sigma[i];
            r += (si > sj || (si == sj && i < c)) ? 1 : 0;
        }
        B.perm[r] = c;
    }
    __syncthreads();
    const double floor_abs = N > 0 ? noise_rel * B.sigma[B.perm[0]] : 0.0;
    for (int c = tid; c < N; c += blockDim.x) {
        double v = B.sigma[B.perm[c]];
        if (mode == kJacobiRsvd && v < kRsvdZero) v = 0.0;
        if (v < floor_abs) v = 0.0;
        vals[c] = v;
    }
    __syncthreads();
    if (tid != 0) return;
    // retained_chi (svd_guard.rs:25-35)
    int rank = 0;
    bool bad = false;
    for (int i = 0; i < N; ++i) {
        if (vals[i] > kSingularCutoff) ++rank;
        if (!isfinite(vals[i]) || vals[i] < 0.0) bad = true;
    }
    int chi = N == 0 ? 0 : min(min(max(rank, 1), J.chi_max > 0 ? J.chi_max : chi_max), min(S.rows, S.cols));
    if (mode == kJacobiRsvd) {
        // needs_f64_fallback (svd_guard.rs:58-76)
        bool fb = bad || chi == 0;
        for (int i = 0; i < N && !fb; ++i)
            if (vals[i] > 0.0 && fabs(vals[i] - kSingularCutoff) <= kCutoffAbsBand) fb = true;
        if (!fb && chi > 0 && chi < N) {
            const double kept = vals[chi - 1], dropped = vals[chi];
            const double scale = fmax(fmax(kept, dropped), 1e-30);
            if (fabs(kept - dropped) / scale < kChiRelGap) fb = true;
        }
        if (fb) {
            S.need_exact = 1;
            S.path = WQC_SPLIT_RSVD_FALLBACK;
            return;
        }
        S.final_kind = 1;
    } else {
        S.final_kind = 0;
        if (J.reject) {
            for (int i = chi; i < N; ++i)
                if (vals[i] > kSingularCutoff) {
                    atomicOr(status, kStatusTruncationRejected);
                    break;
                }
        }
        if (bad) atomicOr(status, kStatusNonFinite);
    }
    double disc = 0;
    for (int i = chi; i < N; ++i) disc += vals[i] * vals[i];
    S.chi = chi;
    S.discarded = disc;
    wqc_split_info info;
    info.left_site = J.p;
    info.rows = S.rows;
    info.cols = S.cols;
    info.ell = S.ell;
    info.path = S.path;
    info.chi = chi;
    info.discarded_weight = disc;
    records[J.seq] = info;
}

// ---------------------------------------------------------------------------
// Recovery of the side the Jacobi does not accumulate, as tiled batched
// GEMMs over the kept columns (m < chi, W column pc = perm[m]), with the
// s^-3/2 scale in the epilogue.  W = X V = U_X Sigma for X = theta, theta^H
// or B^H, so (kept columns, sigma > 0):
//   kRecoverBW:   T = B W_k                  (ell x chi, into the slot's z, column pc)
//   kRecoverQT:   L = Q T s^-3/2             (range finder, rows x chi, into site p)
//   kRecoverExact: R = s^-3/2 W_k^H theta    (theta, rows >= cols, into site p+1)
//                  L = theta W_k s^-3/2      (theta^H, rows < cols, into site p)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) recover_gemm_kernel(const SplitJob* jobs, const SplitState* st,
                                                           const SlotBuffers* slots, DeviceMps mps, int stage) {
    const int j = blockIdx.z;
    const SplitJob& J = jobs[j];
    const SplitState S = st[j];
    if (S.skip) return;
    const bool rf = S.final_kind == 1;
    if ((stage == kRecoverExact) == rf) return;
    const SlotBuffers B = slots[J.slot];
    const int rows = S.rows, cols = S.cols, ell = S.ell, chi = S.chi;
    // C[i][n] = sum_k A(i, k) Bm(k, n); which operand is gathered by perm
    // depends on the stage.
    int m, n, k, kind;
    if (stage == kRecoverBW) {
        m = ell; n = chi; k = cols; kind = 0;
    } else if (stage == kRecoverQT) {
        m = rows; n = chi; k = ell; kind = 1;
    } else if (!S.w_rows_of_src) {
        m = chi; n = cols; k = rows; kind = 2;
    } else {
        m = rows; n = chi; k = cols; kind = 3;
    }
    const int i0 = blockIdx.y * kGemmT, n0 = blockIdx.x * kGemmT;
    if (i0 >= m || n0 >= n) return;
    auto a_at = [&](int i, int kk) -> double2 {
        switch (kind) {
            case 0: return B.b[size_t(i) * cols + kk];                          // B[j][c]
            case 1: return B.q[size_t(kk) * rows + i];                          // Q[r][t]
            case 2: return cconj(B.w[size_t(B.perm[i]) * rows + kk]);          // conj W[r][pc(m)]
            default: return B.theta[size_t(i) * cols + kk];                     // theta[r][c]
        }
    };
    auto b_at = [&](int kk, int nn) -> double2 {
        switch (kind) {
            case 0: return B.w[size_t(B.perm[nn]) * cols + kk];                 // W[c][pc(m)]
            case 1: return B.z[size_t(B.perm[nn]) * ell + kk];                  // T[t][pc(m)]
            case 2: return B.theta[size_t(kk) * cols + nn];                     // theta[r][c]
            default: return B.w[size_t(B.perm[nn]) * cols + kk];                // W[c][pc(m)]
        }
    };
    __shared__ double2 As[kGemmT][kGemmK + 1];
    __shared__ double2 Bs[kGemmK][kGemmT + 1];
    const int tid = threadIdx.x;
    const int tr = tid / 16, tc = tid % 16;
    double2 acc[2][2] = {{cmake(0, 0), cmake(0, 0)}, {cmake(0, 0), cmake(0, 0)}};
    for (int k0 = 0; k0 < k; k0 += kGemmK) {
        for (int e = tid; e < kGemmT * kGemmK; e += 256) {
            const int r = e / kGemmK, c = e % kGemmK;
            As[r][c] = (i0 + r < m && k0 + c < k) ? a_at(i0 + r, k0 + c) : cmake(0, 0);
        }
        for (int e = tid; e < kGemmK * kGemmT; e += 256) {
            const int r = e / kGemmT, c = e % kGemmT;
            Bs[r][c] = (k0 + r < k && n0 + c < n) ? b_at(k0 + r, n0 + c) : cmake(0, 0);
        }
        __syncthreads();
#pragma unroll 4
        for (int c = 0; c < kGemmK; ++c) {
            const double2 a0 = As[tr][c], a1 = As[tr + 16][c];
            const double2 b0 = Bs[c][tc], b1 = Bs[c][tc + 16];
            cfma(acc[0][0], a0, b0);
            cfma(acc[0][1], a0, b1);
            cfma(acc[1][0], a1, b0);
            cfma(acc[1][1], a1, b1);
        }
        __syncthreads();
    }
    auto inv_s32 = [&](int mm) {
        const double sg = B.sigma[B.perm[mm]];
        return sg > 0.0 ? 1.0 / (sg * sqrt(sg)) : 0.0;
    };
    for (int x = 0; x < 2; ++x)
        for (int y = 0; y < 2; ++y) {
            const int i = i0 + tr + 16 * x, nn = n0 + tc + 16 * y;
            if (i >= m || nn >= n) continue;
            const double2 v = acc[x][y];
            switch (kind) {
                case 0: B.z[size_t(B.perm[nn]) * ell + i] = v; break;
                case 1: mps.site[J.p][size_t(i) * chi + nn] = cscale(v, inv_s32(nn)); break;
                case 2: mps.site[J.p + 1][size_t(i) * cols + nn] = cscale(v, inv_s32(i)); break;
                default: mps.site[J.p][size_t(i) * chi + nn] = cscale(v, inv_s32(nn)); break;
            }
        }
}

// ---------------------------------------------------------------------------
// absorb: the sides that are plain copies of W (L = W / sqrt(s) for theta,
// R = W^H / sqrt(s) for theta^H and B^H), and the new bond dims
// (mps.rs:1156-1168, 1039-1051).  The other side comes from
// recover_gemm_kernel.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) absorb_kernel(const SplitJob* jobs, const SplitState* st,
                                                     const SlotBuffers* slots, DeviceMps mps) {
    const int j = blockIdx.y;
    const SplitJob& J = jobs[j];
    const SplitState S = st[j];
    if (S.skip) return;
    const SlotBuffers B = slots[J.slot];
    const int chi = S.chi, rows = S.rows, cols = S.cols;
    const long stride = long(gridDim.x) * blockDim.x;
    const long t0 = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (S.final_kind == 0 && !S.w_rows_of_src) {
        // L = W / sqrt(s), W rows x cols; R comes from recover_gemm_kernel.
        double2* Ls = mps.site[J.p];
        for (long e = t0; e < long(rows) * chi; e += stride) {
            const int r = int(e / chi), m = int(e % chi);
            const int pc = B.perm[m];
            const double sg = B.sigma[pc];
            const double2 w = B.w[size_t(pc) * rows + r];
            Ls[e] = sg > 0.0 ? cscale(w, 1.0 / sqrt(sg)) : cmake(0, 0);  // L[(r/2)][r%2][m] at r*chi + m
        }
    } else {
        // R = W^H / sqrt(s), W cols x (ell or rows); L comes from recover_gemm_kernel.
        double2* Rs = mps.site[J.p + 1];
        for (long e = t0; e < long(chi) * cols; e += stride) {
            const int m = int(e / cols), c = int(e % cols);
            const int pc = B.perm[m];
            const double sg = B.sigma[pc];
            const double2 w = B.w[size_t(pc) * cols + c];
            Rs[e] = sg > 0.0 ? cscale(cconj(w), 1.0 / sqrt(sg)) : cmake(0, 0);  // R[m][c/dr][c%dr]
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        mps.dr[J.p] = chi;
        mps.dl[J.p + 1] = chi;
    }
}

}  // namespace wqc

namespace wqc {
const void* jacobi_kernel(bool fp32, bool reg) {
    if (reg)
        return fp32 ? reinterpret_cast<const void*>(jacobi_cluster_kernel<float2, true>)
                    : reinterpret_cast<const void*>(jacobi_cluster_kernel<double2, true>);
    return fp32 ? reinterpret_cast<const void*>(jacobi_cluster_kernel<float2, false>)
                : reinterpret_cast<const void*>(jacobi_cluster_kernel<double2, false>);
}

const void* qr_cluster(bool global_cols) {
    return global_cols ? reinterpret_cast<const void*>(qr_cluster_kernel<true>)
                       : reinterpret_cast<const void*>(qr_cluster_kernel<false>);
}

cudaError_t launch_qr_cluster(bool global_cols, const cudaLaunchConfig_t& cfg, const SplitJob* jobs,
                              const SplitState* st, const SlotBuffers* slots) {
    if (global_cols) return cudaLaunchKernelEx(&cfg, qr_cluster_kernel<true>, jobs, st, slots);
    return cudaLaunchKernelEx(&cfg, qr_cluster_kernel<false>, jobs, st, slots);
}

const void* jacobi_staged(bool fp32) {
    return fp32 ? reinterpret_cast<const void*>(jacobi_staged_kernel<float2>)
                : reinterpret_cast<const void*>(jacobi_staged_kernel<double2>);
}

cudaError_t launch_jacobi_staged(bool fp32, const cudaLaunchConfig_t& cfg, const SplitJob* jobs, SplitState* st,
                                 const SlotBuffers* slots, const int* idx, int mode, int phase, int max_sweeps, int b,
                                 int* status, unsigned long long* counters) {
    if (fp32)
        return cudaLaunchKernelEx(&cfg, jacobi_staged_kernel<float2>, jobs, st, slots, idx, mode, phase, max_sweeps, b,
                                  status, counters);
    return cudaLaunchKernelEx(&cfg, jacobi_staged_kernel<double2>, jobs, st, slots, idx, mode, phase, max_sweeps, b,
                              status, counters);
}

cudaError_t launch_jacobi(bool fp32, bool reg, const cudaLaunchConfig_t& cfg, const SplitJob* jobs, SplitState* st,
                          const SlotBuffers* slots, const int* idx, int mode, int phase, int max_sweeps, int* status,
                          unsigned long long* counters) {
    if (fp32 && reg)
        return cudaLaunchKernelEx(&cfg, jacobi_cluster_kernel<float2, true>, jobs, st, slots, idx, mode, phase,
                                  max_sweeps, status, counters);
    if (fp32)
        return cudaLaunchKernelEx(&cfg, jacobi_cluster_kernel<float2, false>, jobs, st, slots, idx, mode, phase,
                                  max_sweeps, status, counters);
    if (reg)
        return cudaLaunchKernelEx(&cfg, jacobi_cluster_kernel<double2, true>, jobs, st, slots, idx, mode, phase,
                                  max_sweeps, status, counters);
    return cudaLaunchKernelEx(&cfg, jacobi_cluster_kernel<double2, false>, jobs, st, slots, idx, mode, phase,
                              max_sweeps, status, counters);
}
}  // namespace wqc
