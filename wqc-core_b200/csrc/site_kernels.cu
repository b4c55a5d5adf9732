// Site-local kernels: 1-qubit gates, the <0...0|psi> chain, the trace
// feeders' environments, and Pauli-string expectations.
#include "common.cuh"
#include "split_kernels.cuh"

namespace wqc {

// One-qubit gates (mps.rs:333-351): site[a, s', b] = sum_s u[s'][s] site[a, s, b].
// Every gate queued for a site in this wave is applied in order while the
// pair (v0, v1) stays in registers: one read and one write of the site.
__global__ void __launch_bounds__(256) apply_1q_kernel(const OneQubitOp* ops, const double2* mats, DeviceMps mps) {
    const OneQubitOp op = ops[blockIdx.y];
    const int l = mps.dl[op.site], r = mps.dr[op.site];
    double2* s = mps.site[op.site];
    const long total = long(l) * r;
    for (long e = long(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += long(gridDim.x) * blockDim.x) {
        const long a = e / r, b = e % r;
        double2* p0 = s + (a * 2) * r + b;
        double2* p1 = p0 + r;
        double2 v0 = *p0, v1 = *p1;
        for (int g = 0; g < op.count; ++g) {
            const double2* u = mats + size_t(op.first + g) * 4;
            const double2 n0 = cadd(cmul(u[0], v0), cmul(u[1], v1));
            const double2 n1 = cadd(cmul(u[2], v0), cmul(u[3], v1));
            v0 = n0;
            v1 = n1;
        }
        *p0 = v0;
        *p1 = v1;
    }
}

// Every site back to |0> (mps.rs:101-109): [1, 0] with bonds 1.
__global__ void reset_sites_kernel(DeviceMps mps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        mps.status[0] = 0;
        mps.status[1] = 0;
    }
    if (i >= mps.n) return;
    mps.site[i][0] = cmake(1.0, 0.0);
    mps.site[i][1] = cmake(0.0, 0.0);
    mps.dl[i] = 1;
    mps.dr[i] = 1;
}

// <0...0|psi> (mps.rs:262-276): v <- v . site[:, 0, :] along the chain.  One
// CTA per state: block b runs sites seg[2b] .. seg[2b] + seg[2b+1] - 1 (the
// slices of a batch, or the single state).
__global__ void __launch_bounds__(512) amplitude_zero_kernel(DeviceMps mps, const int* seg, double2* out) {
    extern __shared__ double2 vbuf[];  // 2 * chi_max
    double2* v = vbuf;
    double2* nx = vbuf + mps.chi_max;
    const int first = seg[2 * blockIdx.x], count = seg[2 * blockIdx.x + 1];
    int len = 1;
    if (threadIdx.x == 0) v[0] = cmake(1.0, 0.0);
    __syncthreads();
    for (int i = first; i < first + count; ++i) {
        const int l = mps.dl[i], r = mps.dr[i];
        const double2* s = mps.site[i];
        const int la = min(l, len);
        for (int b = threadIdx.x; b < r; b += blockDim.x) {
            double2 acc = cmake(0, 0);
            for (int a = 0; a < la; ++a) cfma(acc, v[a], s[size_t(a) * 2 * r + b]);
            nx[b] = acc;
        }
        __syncthreads();
        double2* t = v;
        v = nx;
        nx = t;
        len = r;
    }
    if (threadIdx.x == 0) out[blockIdx.x] = len > 0 ? v[0] : cmake(0, 0);
}

// Trace feeders (mps.rs:679-740), incremental and batched.  The left
// environment of site i, L_i (length dl[i]), and the right environment,
// R_i (length dr[i]), contract every site left (right) of i with the
// all-ones physical vector; they stay cached in envL / envR (chi_max
// entries per site) between calls.  The host knows which sites its
// operations touched since the last call, so it passes the ranges still to
// compute: L_{lfrom+1} .. L_{lto} from L_{lfrom} (L_0 = [1] is written when
// lfrom == 0) and R_{rfrom-1} .. R_{rto} from R_{rfrom} (R_{n-1} = [1] when
// rfrom == n-1).  Then, for every target t, a_s = sum_{a,b} L_t[a]
// site_t[a, s, b] R_t[b] (out[2k], out[2k+1] for targets[k]).  One CTA: each
// environment step needs the previous one.
__global__ void __launch_bounds__(512) site_envs_kernel(DeviceMps mps, double2* envL, double2* envR, int lfrom,
                                                        int lto, int rfrom, int rto, const int* targets, int count,
                                                        double2* out) {
    const int cap = mps.chi_max;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    __shared__ double2 red[2][512 / 32];
    if (lfrom == 0 && tid == 0) envL[0] = cmake(1.0, 0.0);
    if (rfrom == mps.n - 1 && tid == 0) envR[size_t(mps.n - 1) * cap] = cmake(1.0, 0.0);
    __syncthreads();
    for (int i = lfrom; i < lto; ++i) {
        const int l = mps.dl[i], r = mps.dr[i];
        const int len = i == 0 ? 1 : mps.dr[i - 1];
        const double2* site = mps.site[i];
        const double2* cur = envL + size_t(i) * cap;
        double2* nxt = envL + size_t(i + 1) * cap;
        const int la = min(l, len);
        for (int b = tid; b < r; b += blockDim.x) {
            double2 acc = cmake(0, 0);
            for (int a = 0; a < la; ++a)
                for (int p = 0; p < 2; ++p) cfma(acc, cur[a], site[(size_t(a) * 2 + p) * r + b]);
            nxt[b] = acc;
        }
        __syncthreads();
    }
    for (int i = rfrom; i > rto; --i) {
        const int l = mps.dl[i], r = mps.dr[i];
        const int len = i == mps.n - 1 ? 1 : mps.dl[i + 1];
        const double2* site = mps.site[i];
        const double2* cur = envR + size_t(i) * cap;
        double2* nxt = envR + size_t(i - 1) * cap;
        const int rb = min(r, len);
        for (int a = tid; a < l; a += blockDim.x) {
            double2 acc = cmake(0, 0);
            for (int b = 0; b < rb; ++b)
                for (int p = 0; p < 2; ++p) cfma(acc, cur[b], site[(size_t(a) * 2 + p) * r + b]);
            nxt[a] = acc;
        }
        __syncthreads();
    }
    for (int k = 0; k < count; ++k) {
        const int t = targets[k];
        const int l = mps.dl[t], r = mps.dr[t];
        const int llen = t == 0 ? 1 : mps.dr[t - 1];
        const int rlen = t == mps.n - 1 ? 1 : mps.dl[t + 1];
        const double2* site = mps.site[t];
        const double2* le = envL + size_t(t) * cap;
        const double2* re = envR + size_t(t) * cap;
        double2 a0 = cmake(0, 0), a1 = cmake(0, 0);
        for (long e = tid; e < long(llen) * r; e += blockDim.x) {
            const int a = int(e / r), b = int(e % r);
            if (a >= l) continue;
            const double2 rv = b < rlen ? re[b] : cmake(1.0, 0.0);
            cfma(a0, le[a], cmul(site[(size_t(a) * 2) * r + b], rv));
            cfma(a1, le[a], cmul(site[(size_t(a) * 2 + 1) * r + b], rv));
        }
        for (int o = 16; o > 0; o >>= 1) {
            a0.x += __shfl_xor_sync(0xffffffffu, a0.x, o);
            a0.y += __shfl_xor_sync(0xffffffffu, a0.y, o);
            a1.x += __shfl_xor_sync(0xffffffffu, a1.x, o);
            a1.y += __shfl_xor_sync(0xffffffffu, a1.y, o);
        }
        if (lane == 0) {
            red[0][wid] = a0;
            red[1][wid] = a1;
        }
        __syncthreads();
        if (tid == 0) {
            double2 s0 = cmake(0, 0), s1 = cmake(0, 0);
            for (int w = 0; w < nw; ++w) {
                s0 = cadd(s0, red[0][w]);
                s1 = cadd(s1, red[1][w]);
            }
            out[2 * k] = s0;
            out[2 * k + 1] = s1;
        }
        __syncthreads();
    }
}

// The dense state (mps.rs:742-780 to_dense_state, 215-260
// contract_to_statevector), one site per launch: cur holds the contraction of
// sites 0..q-1 as [prefix][a] (prefix < 2^q, a < l); nxt gets
// [s 2^q + prefix][b] = sum_a cur[prefix][a] site[a, s, b].  Basis bit q is
// qubit q.  With prune, site entries with |x|^2 < 1e-30 count as zero, as
// to_dense_state's recursion skips them.
__global__ void __launch_bounds__(256) dense_step_kernel(const double2* cur, const double2* site, int l, int r,
                                                         long prefix, int prune, double2* nxt) {
    const long total = 2 * prefix * r;
    for (long e = long(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += long(gridDim.x) * blockDim.x) {
        const long basis = e / r;
        const int b = int(e % r);
        const int s = int(basis / prefix);
        const long pre = basis % prefix;
        double2 acc = cmake(0, 0);
        for (int a = 0; a < l; ++a) {
            const double2 x = site[(size_t(a) * 2 + s) * r + b];
            if (prune && cnorm2(x) < 1e-30) continue;
            cfma(acc, cur[pre * l + a], x);
        }
        nxt[e] = acc;
    }
}

// <psi|P|psi> for Pauli strings by transfer matrices, one CTA per term.
// env[l_ket][l_bra] lives in global scratch (two env_cap x env_cap buffers
// per term plus one for the half-contracted tensor).  Label character n-1-q
// acts on qubit q (src/expectation.rs:98-132).
__global__ void __launch_bounds__(256) pauli_expectation_kernel(DeviceMps mps, const char* labels, int nterms,
                                                                double2* scratch, int env_cap, double2* out) {
    const int t = blockIdx.x;
    if (t >= nterms) return;
    const size_t E = size_t(env_cap) * env_cap;
    double2* env = scratch + size_t(t) * 4 * E;
    double2* nxt = env + E;
    double2* tmp = env + 2 * E;  // [l_bra][s][r], up to env_cap * 2 * env_cap
    const char* lab = labels + size_t(t) * mps.n;
    if (threadIdx.x == 0) env[0] = cmake(1.0, 0.0);
    __syncthreads();
    int lk = 1;
    for (int q = 0; q < mps.n; ++q) {
        const int l = mps.dl[q], r = mps.dr[q];
        const double2* s = mps.site[q];
        const char ch = lab[mps.n - 1 - q];
        // tmp[lp][p][b] = sum_l env[l][lp] * s[l][p][b]
        for (long e = threadIdx.x; e < long(lk) * 2 * r; e += blockDim.x) {
            const int lp = int(e / (2 * r)), rem = int(e % (2 * r));
            double2 acc = cmake(0, 0);
            for (int a = 0; a < min(lk, l); ++a) cfma(acc, env[size_t(a) * lk + lp], s[size_t(a) * 2 * r + rem]);
            tmp[e] = acc;
        }
        __syncthreads();
        // next[b][bp] = sum_{lp, so, si} conj(s[lp][so][bp]) P[so][si] tmp[lp][si][b]
        for (long e = threadIdx.x; e < long(r) * r; e += blockDim.x) {
            const int b = int(e / r), bp = int(e % r);
            double2 acc = cmake(0, 0);
            for (int lp = 0; lp < min(lk, l); ++lp) {
                const double2 t0 = tmp[(size_t(lp) * 2 + 0) * r + b];
                const double2 t1 = tmp[(size_t(lp) * 2 + 1) * r + b];
                const double2 k0 = s[(size_t(lp) * 2 + 0) * r + bp];
                const double2 k1 = s[(size_t(lp) * 2 + 1) * r + bp];
                double2 y0, y1;  // (P t)[so]
                if (ch == 'X') { y0 = t1; y1 = t0; }
                else if (ch == 'Y') { y0 = cmake(t1.y, -t1.x); y1 = cmake(-t0.y, t0.x); }
                else if (ch == 'Z') { y0 = t0; y1 = cmake(-t1.x, -t1.y); }
                else { y0 = t0; y1 = t1; }
                cfma_conj(acc, k0, y0);
                cfma_conj(acc, k1, y1);
            }
            nxt[e] = acc;
        }
        __syncthreads();
        double2* sw = env;
        env = nxt;
        nxt = sw;
        lk = r;
    }
    if (threadIdx.x == 0) out[t] = env[0];
}

// <bra|ket> of two states by a left environment env[a][b] (ket bond a, bra
// bond b), as the time split's overlap (mps.rs:1423-1474), two launches per
// site so every step spreads over the GPU.  The reference caps the
// environment at 256 entries (its CPU cost); here it is bounded only by the
// scratch, chi_ket x chi_bra.
// tmp[b][s][a'] = sum_a env[a][b] K[a][s][a']   (bl x 2 x kr)
__global__ void __launch_bounds__(256) overlap_half_kernel(const double2* env, int kl, int bl, const double2* ket,
                                                           int kr, double2* tmp) {
    const long total = 2L * bl * kr;
    for (long e = long(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += long(gridDim.x) * blockDim.x) {
        const int ar = int(e % kr);
        const int s = int((e / kr) & 1);
        const int b = int(e / (2L * kr));
        double2 acc = cmake(0, 0);
        for (int a = 0; a < kl; ++a) cfma(acc, env[size_t(a) * bl + b], ket[(size_t(a) * 2 + s) * kr + ar]);
        tmp[e] = acc;
    }
}

// next[a'][b'] = sum_{b, s} tmp[b][s][a'] conj(B[b][s][b'])   (kr x br)
__global__ void __launch_bounds__(256) overlap_next_kernel(const double2* tmp, int bl, int kr, const double2* bra,
                                                           int br, double2* next) {
    const long total = long(kr) * br;
    for (long e = long(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += long(gridDim.x) * blockDim.x) {
        const int bp = int(e % br), ar = int(e / br);
        double2 acc = cmake(0, 0);
        for (int bs = 0; bs < 2 * bl; ++bs) cfma_conj(acc, bra[size_t(bs) * br + bp], tmp[size_t(bs) * kr + ar]);
        next[e] = acc;
    }
}

// ---------------------------------------------------------------------------
// Shot sampling from the MPS.  The reference samples terminal measurements
// from the dense statevector (src/sample.rs:85-131, 192-211), so only up to
// 20 qubits; on the MPS the same distribution |<b|psi>|^2 / <psi|psi> is
// drawn site by site (qubit q is site q).  With right environments
// E_q = sum_s A_q[s] E_{q+1} A_q[s]^H (E_n = 1), a shot carries a row vector
// v (v = 1 before site 0), draws s at site q with probability
// p_s / (p_0 + p_1), p_s = w_s E_{q+1} w_s^H, w_s = v A_q[s], and goes on
// with v = w_s / sqrt(p_s).  Every site is drawn, so the measured qubits get
// their marginal distribution.
// ---------------------------------------------------------------------------

// tmp[a][s][c'] = sum_c A[a][s][c] E[c][c'] for one site (l x 2 x r).
__global__ void __launch_bounds__(256) sample_env_half_kernel(const double2* site, int l, int r,
                                                              const double2* env_next, double2* tmp) {
    const long total = 2L * l * r;
    for (long e = long(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += long(gridDim.x) * blockDim.x) {
        const int cp = int(e % r);
        const double2* arow = site + (e / r) * r;
        double2 acc = cmake(0, 0);
        for (int c = 0; c < r; ++c) cfma(acc, arow[c], env_next[size_t(c) * r + cp]);
        tmp[e] = acc;
    }
}

// env[a][a'] = sum_{s, c'} tmp[a][s][c'] conj(A[a'][s][c'])  (l x l).
__global__ void __launch_bounds__(256) sample_env_kernel(const double2* site, int l, int r, const double2* tmp,
                                                         double2* env) {
    const long total = long(l) * l;
    for (long e = long(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += long(gridDim.x) * blockDim.x) {
        const double2* t = tmp + (e / l) * 2 * r;
        const double2* k = site + (e % l) * 2 * r;
        double2 acc = cmake(0, 0);
        for (int x = 0; x < 2 * r; ++x) cfma_conj(acc, k[x], t[x]);
        env[e] = acc;
    }
}

// SplitMix64 (Steele, Lea and Flood, OOPSLA 2014): the uniform draw of shot
// `shot` at site q is the top 53 bits of mix(mix(seed ^ mix(shot)) + q).
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double sample_uniform(unsigned long long seed, unsigned long long shot, int q) {
    const unsigned long long key = splitmix64(seed ^ splitmix64(shot));
    return double(splitmix64(key + (unsigned long long)q) >> 11) * 0x1.0p-53;
}

// One CTA per shot (grid-stride over shots).  envs + env_off[q] holds E_q
// (dl[q] x dl[q]; E_n is 1 x 1); bitpos[q] is the output bit of qubit q, or
// -1 when q is not measured.  Dynamic shared memory: 3 * chi_max complex.
__global__ void __launch_bounds__(256) sample_shots_kernel(DeviceMps mps, const double2* envs,
                                                           const unsigned long long* env_off, const int* bitpos,
                                                           unsigned long long seed, int shots,
                                                           unsigned long long* out) {
    extern __shared__ __align__(16) double2 sv[];
    double2* v = sv;
    double2* w0 = sv + mps.chi_max;
    double2* w1 = w0 + mps.chi_max;
    __shared__ double red[2][256 / 32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    for (int shot = blockIdx.x; shot < shots; shot += gridDim.x) {
        if (tid == 0) v[0] = cmake(1.0, 0.0);
        __syncthreads();
        unsigned long long bits = 0;
        for (int q = 0; q < mps.n; ++q) {
            const int l = mps.dl[q], r = mps.dr[q];
            const double2* A = mps.site[q];
            const double2* E = envs + env_off[q + 1];  // r x r
            for (int c = tid; c < r; c += blockDim.x) {
                double2 a0 = cmake(0, 0), a1 = cmake(0, 0);
                for (int a = 0; a < l; ++a) {
                    cfma(a0, v[a], A[(size_t(a) * 2 + 0) * r + c]);
                    cfma(a1, v[a], A[(size_t(a) * 2 + 1) * r + c]);
                }
                w0[c] = a0;
                w1[c] = a1;
            }
            __syncthreads();
            double part0 = 0, part1 = 0;
            for (int cp = tid; cp < r; cp += blockDim.x) {
                double2 x0 = cmake(0, 0), x1 = cmake(0, 0);
                for (int c = 0; c < r; ++c) {
                    const double2 e = E[size_t(c) * r + cp];
                    cfma(x0, w0[c], e);
                    cfma(x1, w1[c], e);
                }
                part0 += x0.x * w0[cp].x + x0.y * w0[cp].y;  // Re(x conj(w))
                part1 += x1.x * w1[cp].x + x1.y * w1[cp].y;
            }
            for (int o = 16; o > 0; o >>= 1) {
                part0 += __shfl_xor_sync(0xffffffffu, part0, o);
                part1 += __shfl_xor_sync(0xffffffffu, part1, o);
            }
            if (lane == 0) {
                red[0][wid] = part0;
                red[1][wid] = part1;
            }
            __syncthreads();
            double p0 = 0, p1 = 0;
            for (int w = 0; w < nw; ++w) {  // every thread sums in the same order
                p0 += red[0][w];
                p1 += red[1][w];
            }
            p0 = fmax(p0, 0.0);
            p1 = fmax(p1, 0.0);
            const double u = sample_uniform(seed, (unsigned long long)shot, q);
            const int s = (p0 + p1 > 0.0 && u * (p0 + p1) >= p0) ? 1 : 0;
            const double ps = s ? p1 : p0;
            const double scale = ps > 0.0 ? rsqrt(ps) : 1.0;
            const double2* ws = s ? w1 : w0;
            for (int c = tid; c < r; c += blockDim.x) v[c] = cscale(ws[c], scale);
            if (s && bitpos[q] >= 0) bits |= 1ull << bitpos[q];
            __syncthreads();
        }
        if (tid == 0) out[shot] = bits;
    }
}

}  // namespace wqc
