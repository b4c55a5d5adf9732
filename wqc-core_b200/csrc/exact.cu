// Exact contraction trees on the device: the walk of src/tn/exact.rs:136-241
// with every state tensor in HBM.
//
// The host walks the tree once, as the reference's `walk` does (tree shape,
// circuit order, shared wires, legs, live bytes and the peak), and plans the
// device work while it walks.  Each state tensor gets a place in one device
// arena; a gate node queues its gate on the state it applies to; an outer
// product first flushes the queues of its two inputs.  Nothing reaches the
// device until the whole walk has passed, so every failure the reference
// reports comes back before any launch.
//
// A flushed queue becomes passes.  A pass is a set of at most 12 positions of
// the tensor, positions 0-3 always among them (so a block reads runs of 256
// contiguous bytes), and the gates, in circuit order, whose wires all lie in
// it.  One block loads the 4096 amplitudes of one assignment of the other
// positions into shared memory, applies the pass's gates one after another,
// and writes them back: a 25-leg state crosses HBM once per pass instead of
// once per gate.  Gates stay in circuit order and every amplitude is
// computed with the reference's arithmetic (exact.rs:482-560: complex
// products as re*re - im*im, re*im + im*re, then sums, no fused multiply-add),
// so each amplitude is the value the reference computes.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/wqc_cuda.h"
#include "tree_common.h"

using namespace wqc;
using namespace wqc::tree;

namespace {

constexpr int kLowBits = 4;                      // positions every pass holds: 16 amplitudes, 256 bytes
constexpr int kMaxPassBits = 12;                 // 4096 amplitudes, 64 KB of shared memory per block
constexpr int kPassThreads = 256;
constexpr int kOuterThreads = 256;
constexpr int kTimedPassLegs = 20;               // passes timed one by one for the stats

enum PassKind : int32_t { kOne = 0, kCnot = 1, kCz = 2, kCcnot = 3 };

struct PassGate {
    int32_t kind;     // PassKind
    int32_t a, b, c;  // local bit positions: one-qubit a; CNOT/CZ control a, target b; CCNOT controls a, b, target c
    double2 u[4];     // one-qubit matrix, row-major (row = output amplitude)
};

struct PassHdr {
    uint32_t mask;   // tensor positions the pass holds (bit p: position p)
    int32_t legs;    // tensor legs
    int32_t local;   // popcount(mask)
    int32_t ngates;
};

// ---------------------------------------------------------------------------
// Device side.
// ---------------------------------------------------------------------------

// The reference's complex product and sum (num_complex, no contraction).
__device__ __forceinline__ double2 xmul(double2 a, double2 b) {
    return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                        __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 xadd(double2 a, double2 b) {
    return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}

// Bits of x placed, lowest first, at the set bits of mask.
__device__ __forceinline__ uint32_t deposit(uint32_t x, uint32_t mask) {
    uint32_t r = 0;
    for (uint32_t m = mask; m; m &= m - 1) {
        if (x & 1u) r |= m & (0u - m);
        x >>= 1;
    }
    return r;
}
// The bits of x at the set bits of mask, packed from bit 0.
__device__ __forceinline__ uint32_t extract(uint32_t x, uint32_t mask) {
    uint32_t r = 0, k = 1;
    for (uint32_t m = mask; m; m &= m - 1, k <<= 1)
        if (x & m & (0u - m)) r |= k;
    return r;
}
// p with a zero bit inserted at position b.
__device__ __forceinline__ uint32_t insert0(uint32_t p, int b) {
    const uint32_t lo = p & ((1u << b) - 1u);
    return ((p >> b) << (b + 1)) | lo;
}

// One pass: block `blockIdx.x` holds the amplitudes whose positions outside
// h.mask spell blockIdx.x; its 2^h.local amplitudes go through shared memory
// and the pass's gates.  Index bounds: blockIdx.x < 2^(legs - local), so base
// < 2^legs with the mask's bits clear; local indices < 2^local deposit into
// the mask's bits; every address is below 2^legs, the tensor's length.
__global__ void __launch_bounds__(kPassThreads) exact_pass_kernel(double2* __restrict__ state, PassHdr h,
                                                                   const PassGate* __restrict__ gates) {
    extern __shared__ double2 amp[];
    __shared__ uint32_t hi_off[1 << (kMaxPassBits - kLowBits)];
    const uint32_t all = h.legs >= 32 ? ~0u : ((1u << h.legs) - 1u);
    const uint32_t base = deposit(blockIdx.x, all & ~h.mask);
    const int low = h.local < kLowBits ? h.local : kLowBits;  // positions 0..low-1 are in the mask
    const uint32_t hi_mask = h.mask & ~((1u << low) - 1u);
    const uint32_t n_hi = 1u << (h.local - low);
    const uint32_t n = 1u << h.local;
    for (uint32_t t = threadIdx.x; t < n_hi; t += blockDim.x) hi_off[t] = deposit(t, hi_mask);
    __syncthreads();
    const uint32_t low_mask = (1u << low) - 1u;
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) amp[j] = state[base + hi_off[j >> low] + (j & low_mask)];
    __syncthreads();
    for (int g = 0; g < h.ngates; ++g) {
        const PassGate G = gates[g];
        if (G.kind == kOne) {
            const uint32_t bit = 1u << G.a;
            for (uint32_t p = threadIdx.x; p < (n >> 1); p += blockDim.x) {
                const uint32_t i0 = insert0(p, G.a), i1 = i0 | bit;
                const double2 v0 = amp[i0], v1 = amp[i1];
                amp[i0] = xadd(xmul(G.u[0], v0), xmul(G.u[1], v1));
                amp[i1] = xadd(xmul(G.u[2], v0), xmul(G.u[3], v1));
            }
        } else if (G.kind == kCnot || G.kind == kCz) {
            const int lo = G.a < G.b ? G.a : G.b, hi = G.a < G.b ? G.b : G.a;
            const uint32_t c = 1u << G.a, t = 1u << G.b;
            for (uint32_t p = threadIdx.x; p < (n >> 2); p += blockDim.x) {
                const uint32_t i = insert0(insert0(p, lo), hi);
                if (G.kind == kCnot) {
                    const double2 v10 = amp[i | c], v11 = amp[i | c | t];
                    amp[i | c] = v11;
                    amp[i | c | t] = v10;
                } else {
                    const double2 v11 = amp[i | c | t];
                    amp[i | c | t] = make_double2(-v11.x, -v11.y);
                }
            }
        } else {  // CCNOT
            int s0 = G.a, s1 = G.b, s2 = G.c;  // ascending for the zero insertions
            if (s0 > s1) { const int x = s0; s0 = s1; s1 = x; }
            if (s1 > s2) { const int x = s1; s1 = s2; s2 = x; }
            if (s0 > s1) { const int x = s0; s0 = s1; s1 = x; }
            const uint32_t both = (1u << G.a) | (1u << G.b), t = 1u << G.c;
            for (uint32_t p = threadIdx.x; p < (n >> 3); p += blockDim.x) {
                const uint32_t i = insert0(insert0(insert0(p, s0), s1), s2) | both;
                const double2 v = amp[i];
                amp[i] = amp[i | t];
                amp[i | t] = v;
            }
        }
        __syncthreads();
    }
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) state[base + hi_off[j >> low] + (j & low_mask)] = amp[j];
}

// ---------------------------------------------------------------------------
// Register-tiled passes over tensors of at least 5 + WB + RB legs.
//
// A block holds a tile of 2^(5 + WB + RB) amplitudes: its local bits 0-4 are
// the tensor's positions 0-4 (the lanes of a warp, so every warp-wide load or
// store is 512 contiguous bytes), the other WB + RB local bits are the tile's
// high positions, of which RB are register bits (each thread holds 2^RB
// amplitudes) and WB are warp bits.  A gate whose target is a register bit
// runs inside the thread; a target on a lane bit takes its partner by a warp
// shuffle; a target on a warp bit first needs an exchange, which rewrites the
// tile through shared memory with another choice of register bits.  Controls,
// diagonal gates and CZ act where their bits are, in the tile or outside it
// (bits of the block's base index).  The host plans the ops and the exchanges.
// ---------------------------------------------------------------------------
enum RegOpKind : int32_t { kXchg = 0, kDense = 1, kPerm = 2, kNeg = 3, kDiag = 4 };
enum RegForm : int32_t { kGeneral = 0, kReal = 1 };
constexpr int kLaneTarget = 16;  // RegOp::tgt >= kLaneTarget: lane bit tgt - kLaneTarget

// One op of a register-tiled pass, read by every thread with one 16-byte load
// plus the matrix it needs.  code: kind (bits 0-3) | form << 4 | tgt << 8 |
// c_lane << 16 | c_warp << 21 | c_reg << 26, where the c_ masks are the bits
// that must be set -- controls (kPerm), the sign bits (kNeg), the one bit that
// picks u[3] over u[0] (kDiag) -- among the lane, warp and register bits;
// c_out the same among the tensor positions outside the tile.  tgt is a
// register bit 0..3, or kLaneTarget + a lane bit.
struct RegOp {
    uint32_t code;
    uint32_t c_out;
    uint32_t x_reg, x_warp;  // kXchg: register / warp bits among the tile's high local bits
    double2 u[4];  // kDense, form kReal: u[0] = (u00, u01), u[1] = (u10, u11) real parts; otherwise the matrix
};

struct RegPassHdr {
    uint32_t mask;  // tensor positions of the tile (0-4 and the high ones)
    int32_t legs;
    int32_t nops;
    uint32_t reg0, warp0;  // register / warp bits among the high local bits at the start
};

// The reference's output amplitude A v0 + B v1 of a one-qubit gate row
// (u00 v0 + u01 v1, u10 v0 + u11 v1).  The real form drops the products of
// zero imaginary parts, signed zeros that leave every sum's value unchanged.
__device__ __forceinline__ double2 row_real(double a, double b, double2 v0, double2 v1) {
    return make_double2(__dadd_rn(__dmul_rn(a, v0.x), __dmul_rn(b, v1.x)),
                        __dadd_rn(__dmul_rn(a, v0.y), __dmul_rn(b, v1.y)));
}
__device__ __forceinline__ double2 row_general(double2 a, double2 b, double2 v0, double2 v1) {
    return xadd(xmul(a, v0), xmul(b, v1));
}

__device__ __forceinline__ double2 shfl_xor2(double2 v, int m) {
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// The four register bits' places among the high local bits, and the high
// local index of register r: the OR of the places of r's set bits, folded at
// compile time for each unrolled r.
template <int RB>
struct RegBits {
    uint32_t b[RB];
    __device__ __forceinline__ void set(uint32_t regm) {
#pragma unroll
        for (int i = 0; i < RB; ++i) {
            b[i] = regm & (0u - regm);
            regm &= regm - 1;
        }
    }
    __device__ __forceinline__ uint32_t at(int r) const {
        uint32_t x = 0;
#pragma unroll
        for (int i = 0; i < RB; ++i) x |= ((r >> i) & 1) ? b[i] : 0u;
        return x;
    }
};

__device__ __forceinline__ double2 sel(bool c, double2 a, double2 b) {
    return make_double2(c ? a.x : b.x, c ? a.y : b.y);
}

// One-qubit gates with two nonzero entries per row (H, Y, RX, RY; no
// controls).  On a register bit: pairs (r, r | 1 << TR) inside the thread.
template <int NR, int TR>
__device__ __forceinline__ void dense_reg_real(double2 (&v)[NR], double a, double b, double c, double d) {
    if constexpr ((1 << TR) < NR) {
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        if (r & (1 << TR)) continue;
        const int r1 = r | (1 << TR);
        const double2 v0 = v[r], v1 = v[r1];
        v[r] = row_real(a, b, v0, v1);
        v[r1] = row_real(c, d, v0, v1);
    }
    }
}
template <int NR, int TR>
__device__ __forceinline__ void dense_reg_general(double2 (&v)[NR], const double2 (&u)[4]) {
    if constexpr ((1 << TR) < NR) {
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        if (r & (1 << TR)) continue;
        const int r1 = r | (1 << TR);
        const double2 v0 = v[r], v1 = v[r1];
        v[r] = row_general(u[0], u[1], v0, v1);
        v[r1] = row_general(u[2], u[3], v0, v1);
    }
    }
}

// On a lane bit: the partner's amplitude by a warp shuffle.  The lane with
// the bit clear computes u00 v + u01 p, the lane with it set u11 v + u10 p
// -- the reference's u10 v0 + u11 v1 with the two terms of the sum swapped,
// which IEEE addition leaves bit-identical.
template <int NR>
__device__ __forceinline__ void dense_lane_real(double2 (&v)[NR], double a, double b, double c, double d, int tl,
                                                uint32_t lane) {
    const bool hi = (lane >> tl) & 1u;
    const double own = hi ? d : a, other = hi ? c : b;
#pragma unroll
    for (int r = 0; r < NR; ++r) v[r] = row_real(own, other, v[r], shfl_xor2(v[r], 1 << tl));
}
template <int NR>
__device__ __forceinline__ void dense_lane_general(double2 (&v)[NR], const double2 (&u)[4], int tl, uint32_t lane) {
    const bool hi = (lane >> tl) & 1u;
    const double2 own = hi ? u[3] : u[0], other = hi ? u[2] : u[1];
#pragma unroll
    for (int r = 0; r < NR; ++r) v[r] = row_general(own, other, v[r], shfl_xor2(v[r], 1 << tl));
}

// Swaps of the target pairs where the controls are set: thread-level
// controls select whole pairs; register-bit controls select pair by pair.
template <int NR, int TR>
__device__ __forceinline__ void perm_reg(double2 (&v)[NR], bool thread_ok, uint32_t c_reg) {
    if constexpr ((1 << TR) < NR) {
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        if (r & (1 << TR)) continue;
        const int r1 = r | (1 << TR);
        const bool ok = thread_ok && (uint32_t(r) & c_reg) == c_reg;
        const double2 v0 = v[r], v1 = v[r1];
        v[r] = sel(ok, v1, v0);
        v[r1] = sel(ok, v0, v1);
    }
    }
}

template <int WB, int RB>
__global__ void __launch_bounds__(32 << WB, (WB == 3 ? 2 : 1))
    exact_pass_reg_kernel(double2* __restrict__ state, RegPassHdr h, const RegOp* __restrict__ ops) {
    constexpr int HB = WB + RB;  // high local bits
    constexpr int NR = 1 << RB;  // amplitudes per thread
    extern __shared__ double2 xbuf[];  // 2^(9 + WB) amplitudes, used by exchanges
    __shared__ uint32_t hi_off[1 << HB];
    const uint32_t all = h.legs >= 32 ? ~0u : ((1u << h.legs) - 1u);
    const uint32_t base = deposit(blockIdx.x, all & ~h.mask);
    for (uint32_t t = threadIdx.x; t < (1u << HB); t += blockDim.x) hi_off[t] = deposit(t, h.mask & ~31u);
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    constexpr uint32_t kHiAll = (1u << HB) - 1u;  // keeps every tile index below 2^(9 + WB)
    RegBits<RB> rb;
    rb.set(h.reg0 & kHiAll);
    uint32_t wdep = deposit(w, h.warp0 & kHiAll);
    double2 v[NR];
    const double2* src = state + base + lane;
#pragma unroll
    for (int r = 0; r < NR; ++r) v[r] = src[hi_off[wdep | rb.at(r)]];
    for (int o = 0; o < h.nops; ++o) {
        const uint4 hd = __ldg(reinterpret_cast<const uint4*>(ops + o));
        const uint32_t code = hd.x;
        const int kind = int(code & 15u);
        const int tgt = int((code >> 8) & 255u);
        if (kind == kXchg) {
            __syncthreads();  // the previous exchange's reads are done
#pragma unroll
            for (int r = 0; r < NR; ++r) xbuf[lane | ((wdep | rb.at(r)) << 5)] = v[r];
            __syncthreads();
            rb.set(hd.z & kHiAll);
            wdep = deposit(w, hd.w & kHiAll);
#pragma unroll
            for (int r = 0; r < NR; ++r) v[r] = xbuf[lane | ((wdep | rb.at(r)) << 5)];
            continue;
        }
        const double2* u = ops[o].u;
        if (kind == kDense) {
            if (((code >> 4) & 15u) == kReal) {
                const double2 ab = __ldg(u), cd = __ldg(u + 1);
                switch (tgt) {
                    case 0: dense_reg_real<NR, 0>(v, ab.x, ab.y, cd.x, cd.y); break;
                    case 1: dense_reg_real<NR, 1>(v, ab.x, ab.y, cd.x, cd.y); break;
                    case 2: dense_reg_real<NR, 2>(v, ab.x, ab.y, cd.x, cd.y); break;
                    case 3: dense_reg_real<NR, 3>(v, ab.x, ab.y, cd.x, cd.y); break;
                    default: dense_lane_real<NR>(v, ab.x, ab.y, cd.x, cd.y, tgt - kLaneTarget, lane); break;
                }
            } else {
                const double2 m[4] = {__ldg(u), __ldg(u + 1), __ldg(u + 2), __ldg(u + 3)};
                switch (tgt) {
                    case 0: dense_reg_general<NR, 0>(v, m); break;
                    case 1: dense_reg_general<NR, 1>(v, m); break;
                    case 2: dense_reg_general<NR, 2>(v, m); break;
                    case 3: dense_reg_general<NR, 3>(v, m); break;
                    default: dense_lane_general<NR>(v, m, tgt - kLaneTarget, lane); break;
                }
            }
            continue;
        }
        const uint32_t c_lane = (code >> 16) & 31u, c_warp = (code >> 21) & 15u, c_reg = (code >> 26) & 15u;
        const uint32_t c_out = hd.y;
        if (kind == kDiag) {  // exactly one of the masks holds the gate's bit
            const bool thread_bit = (lane & c_lane) | (w & c_warp) | (base & c_out);
            const double2 u0 = __ldg(u), u3 = __ldg(u + 3);
#pragma unroll
            for (int r = 0; r < NR; ++r) v[r] = xmul(sel(thread_bit || (uint32_t(r) & c_reg), u3, u0), v[r]);
            continue;
        }
        const bool thread_ok = (lane & c_lane) == c_lane && (w & c_warp) == c_warp && (base & c_out) == c_out;
        if (kind == kPerm) {
            switch (tgt) {
                case 0: perm_reg<NR, 0>(v, thread_ok, c_reg); break;
                case 1: perm_reg<NR, 1>(v, thread_ok, c_reg); break;
                case 2: perm_reg<NR, 2>(v, thread_ok, c_reg); break;
                case 3: perm_reg<NR, 3>(v, thread_ok, c_reg); break;
                default: {
                    const int m = 1 << (tgt - kLaneTarget);
#pragma unroll
                    for (int r = 0; r < NR; ++r) {
                        const double2 p = shfl_xor2(v[r], m);
                        v[r] = sel(thread_ok && (uint32_t(r) & c_reg) == c_reg, p, v[r]);
                    }
                }
            }
        } else {  // kNeg
#pragma unroll
            for (int r = 0; r < NR; ++r)
                v[r] = sel(thread_ok && (uint32_t(r) & c_reg) == c_reg, make_double2(-v[r].x, -v[r].y), v[r]);
        }
    }
    double2* dst = state + base + lane;
#pragma unroll
    for (int r = 0; r < NR; ++r) dst[hi_off[wdep | rb.at(r)]] = v[r];
}

// out[i] = left[extract(i, lmask)] * right[extract(i, rmask)] over the sorted
// union of the two tensors' wires (exact.rs:444-480).  The extractions come
// from four 7-bit tables per operand (28 bits >= 26 legs).  Bounds: i <
// 2^legs; lmask and rmask partition the legs, so the extracted indices are
// below 2^popcount(lmask) and 2^popcount(rmask), the operands' lengths.
__global__ void __launch_bounds__(kOuterThreads) exact_outer_kernel(double2* __restrict__ out,
                                                                     const double2* __restrict__ left,
                                                                     const double2* __restrict__ right,
                                                                     uint32_t lmask, uint32_t rmask, int legs) {
    __shared__ uint32_t tl[4][128], tr[4][128];
    for (int e = threadIdx.x; e < 512; e += blockDim.x) {
        const uint32_t v = uint32_t(e & 127) << (7 * (e >> 7));
        tl[e >> 7][e & 127] = extract(v, lmask);
        tr[e >> 7][e & 127] = extract(v, rmask);
    }
    __syncthreads();
    const uint32_t total = 1u << legs;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const uint32_t c0 = i & 127, c1 = (i >> 7) & 127, c2 = (i >> 14) & 127, c3 = (i >> 21) & 127;
        const uint32_t li = tl[0][c0] | tl[1][c1] | tl[2][c2] | tl[3][c3];
        const uint32_t ri = tr[0][c0] | tr[1][c1] | tr[2][c2] | tr[3][c3];
        out[i] = xmul(left[li], right[ri]);
    }
}

// |0> into every ket slot: slot k is arena[2k], arena[2k+1].
__global__ void exact_kets_kernel(double2* __restrict__ kets, uint32_t count) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        kets[2 * size_t(k)] = make_double2(1.0, 0.0);
        kets[2 * size_t(k) + 1] = make_double2(0.0, 0.0);
    }
}

// out[k] = arena[where[k]]: the components the amplitudes multiply.
__global__ void exact_gather_kernel(const double2* __restrict__ arena, const uint64_t* __restrict__ where,
                                    uint32_t count, double2* __restrict__ out) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x)
        out[k] = arena[where[k]];
}

// ---------------------------------------------------------------------------
// Host side: the walk.
// ---------------------------------------------------------------------------

// declared_peak (exact.rs:87-97).
wqc_status declared_peak(const wqc_tree* tree, uint64_t* out) {
    if (!tree->has_peak) return failx("exact contraction tree requires a peak");
    if (tree->peak_bytes > kMaxPeakBytes) return failx("contraction tree peak exceeds 1 GiB");
    *out = tree->peak_bytes;
    return WQC_OK;
}

// Device work the walk plans.
struct PendingGate {
    uint32_t gate;
};
struct Buffer {
    uint64_t off = 0;  // element offset in the arena
    int legs = 0;
    bool ket = false;  // in the ket region (never freed)
    std::vector<uint32_t> pending;  // gates queued on this state, circuit order
};
struct Item {
    int kind;  // 0 shared-memory pass, 1 outer product, 2 register-tiled pass
    PassHdr hdr;
    RegPassHdr rhdr;
    int buf;             // pass: the state; outer: the result
    int lbuf, rbuf;      // outer: the operands
    uint32_t gate_off;   // pass: first gate (kind 0) or op (kind 2) in its table
    bool xchg;           // kind 2: the pass exchanges (needs the shared-memory tile)
    uint32_t lmask, rmask;
    int legs;
};

// How a gate runs in a register-tiled pass, and whether it may move past
// gates on other positions.  Gates whose arithmetic rounds (H, T, RX, RY, RZ)
// keep their circuit order among themselves; the others (X, Y, Z, S, CNOT,
// CZ, CCNOT) only permute amplitudes and multiply them by +-1 or +-i, which
// commutes exactly with any gate on other positions.
struct Sched {
    int kind = kDense;  // RegOpKind
    int form = kGeneral;
    bool exact = false;
    int tgt = -1;        // tensor position of the target (kDense, kPerm)
    uint32_t bits = 0;   // controls (kPerm), sign bits (kNeg), the bit (kDiag)
    uint32_t all = 0;    // every position the gate touches
    double2 u[4] = {};
};

struct Plan {
    bool on = false;
    int pass_bits = kMaxPassBits;
    int tile_wb = 3;  // warp bits of a register tile
    int tile_rb = 4;  // register bits: tiles of 2^(5 + tile_wb + tile_rb) amplitudes
    const wqc_gate* gates = nullptr;
    std::vector<Buffer> bufs;
    std::vector<Item> items;
    std::vector<PassGate> pass_gates;
    std::vector<RegOp> reg_ops;
    uint32_t exchanges = 0;
    Placer placer;
    uint32_t kets = 0;  // ket slots (32 bytes each) at the arena's start
    uint64_t bytes_moved = 0;
    uint32_t gate_total = 0;

    int new_ket() {
        Buffer b;
        b.ket = true;
        b.legs = 1;
        b.off = 2 * uint64_t(kets++);  // element offset inside the ket region
        bufs.push_back(std::move(b));
        return int(bufs.size()) - 1;
    }
    int new_state(int legs) {
        Buffer b;
        b.legs = legs;
        b.off = placer.alloc(16ull << legs) / 16;  // element offset inside the tensor region
        bufs.push_back(std::move(b));
        return int(bufs.size()) - 1;
    }
    void drop(int id) {
        Buffer& b = bufs[size_t(id)];
        if (!b.ket) placer.release(b.off * 16, 16ull << b.legs);
    }

    Sched classify(const wqc_gate& g, const std::vector<uint32_t>& wires) const {
        auto pos = [&](int q) { return int(std::lower_bound(wires.begin(), wires.end(), uint32_t(q)) - wires.begin()); };
        Sched s;
        switch (g.kind) {
            case WQC_GATE_CNOT:
                s.kind = kPerm, s.exact = true, s.tgt = pos(g.q1), s.bits = 1u << pos(g.q0);
                break;
            case WQC_GATE_CCNOT:
                s.kind = kPerm, s.exact = true, s.tgt = pos(g.q2), s.bits = (1u << pos(g.q0)) | (1u << pos(g.q1));
                break;
            case WQC_GATE_CZ:
                s.kind = kNeg, s.exact = true, s.bits = (1u << pos(g.q0)) | (1u << pos(g.q1));
                break;
            case WQC_GATE_X:
                s.kind = kPerm, s.exact = true, s.tgt = pos(g.q0);
                break;
            case WQC_GATE_Z:
                s.kind = kNeg, s.exact = true, s.bits = 1u << pos(g.q0);
                break;
            case WQC_GATE_S: case WQC_GATE_T: case WQC_GATE_RZ:
                s.kind = kDiag, s.exact = g.kind == WQC_GATE_S, s.bits = 1u << pos(g.q0);
                gate_matrix_2x2(g.kind, g.angle, s.u);
                break;
            default:  // H, Y, RX, RY
                s.kind = kDense, s.exact = g.kind == WQC_GATE_Y, s.tgt = pos(g.q0);
                gate_matrix_2x2(g.kind, g.angle, s.u);
                s.form = (s.u[0].y == 0.0 && s.u[1].y == 0.0 && s.u[2].y == 0.0 && s.u[3].y == 0.0) ? kReal : kGeneral;
                break;
        }
        s.all = s.bits | (s.tgt >= 0 ? 1u << s.tgt : 0u);
        return s;
    }

    // One register-tiled pass: the gates `g` (execution order) on a state of
    // `legs` legs whose targets outside positions 0-4 are `targets`.
    void emit_reg_pass(int id, int legs, const std::vector<Sched>& g, uint32_t targets) {
        const int HB = tile_wb + tile_rb;
        std::vector<int> hi;  // tensor positions of the high local bits, ascending
        for (int p = 5; p < legs; ++p)
            if (targets & (1u << p)) hi.push_back(p);
        for (int p = 5; p < legs && int(hi.size()) < HB; ++p)
            if (!(targets & (1u << p))) hi.push_back(p);
        std::sort(hi.begin(), hi.end());
        uint32_t mask = 0x1fu;
        for (int p : hi) mask |= 1u << p;
        auto hb_of = [&](int p) { return int(std::lower_bound(hi.begin(), hi.end(), p) - hi.begin()); };
        auto rank = [](uint32_t m, int b) { return __builtin_popcount(m & ((1u << b) - 1u)); };
        const uint32_t hi_all = (1u << HB) - 1u;
        // The high bit each op needs in registers, or -1.
        std::vector<int> use(g.size(), -1);
        for (size_t i = 0; i < g.size(); ++i)
            if ((g[i].kind == kDense || g[i].kind == kPerm) && g[i].tgt >= 5) use[i] = hb_of(g[i].tgt);
        uint32_t regm = 0;
        for (size_t i = 0; i < g.size() && __builtin_popcount(regm) < tile_rb; ++i)
            if (use[i] >= 0) regm |= 1u << use[i];
        for (int b = 0; b < HB && __builtin_popcount(regm) < tile_rb; ++b) regm |= 1u << b;
        Item it{};
        it.kind = 2;
        it.buf = id;
        it.legs = legs;
        it.gate_off = uint32_t(reg_ops.size());
        it.rhdr.mask = mask;
        it.rhdr.legs = legs;
        it.rhdr.reg0 = regm;
        it.rhdr.warp0 = hi_all & ~regm;
        for (size_t i = 0; i < g.size(); ++i) {
            if (use[i] >= 0 && !(regm & (1u << use[i]))) {
                // Keep in registers the four high bits needed soonest (Belady).
                std::vector<std::pair<size_t, int>> next;  // (next use, bit)
                for (int b = 0; b < HB; ++b) {
                    size_t nu = g.size() + 1;
                    for (size_t j = i; j < g.size(); ++j)
                        if (use[j] == b) {
                            nu = j;
                            break;
                        }
                    // prefer bits already in registers on ties
                    next.emplace_back(nu * 2 + ((regm >> b) & 1u ? 0 : 1), b);
                }
                std::sort(next.begin(), next.end());
                uint32_t nm = 0;
                for (int k = 0; k < tile_rb; ++k) nm |= 1u << next[size_t(k)].second;
                RegOp x{};
                x.code = uint32_t(kXchg);
                x.x_reg = nm;
                x.x_warp = hi_all & ~nm;
                reg_ops.push_back(x);
                regm = nm;
                it.xchg = true;
                ++exchanges;
            }
            const uint32_t warpm = hi_all & ~regm;
            RegOp op{};
            uint32_t tgt = 0, c_lane = 0, c_warp = 0, c_reg = 0;
            if (g[i].kind == kDense && g[i].form == kReal) {
                op.u[0] = make_double2(g[i].u[0].x, g[i].u[1].x);
                op.u[1] = make_double2(g[i].u[2].x, g[i].u[3].x);
            } else {
                for (int k = 0; k < 4; ++k) op.u[k] = g[i].u[k];
            }
            if (g[i].tgt >= 0)
                tgt = g[i].tgt < 5 ? uint32_t(kLaneTarget + g[i].tgt) : uint32_t(rank(regm, hb_of(g[i].tgt)));
            for (uint32_t m = g[i].bits; m; m &= m - 1) {
                const int p = __builtin_ctz(m);
                if (p < 5) {
                    c_lane |= 1u << p;
                } else if (mask & (1u << p)) {
                    const int b = hb_of(p);
                    if (regm & (1u << b)) c_reg |= 1u << rank(regm, b);
                    else c_warp |= 1u << rank(warpm, b);
                } else {
                    op.c_out |= 1u << p;
                }
            }
            op.code = uint32_t(g[i].kind) | uint32_t(g[i].form) << 4 | tgt << 8 | c_lane << 16 | c_warp << 21 |
                      c_reg << 26;
            reg_ops.push_back(op);
        }
        it.rhdr.nops = int(reg_ops.size() - it.gate_off);
        items.push_back(it);
        bytes_moved += 2 * (16ull << legs);
    }

    // The queued gates of a state of at least 9 + tile_wb legs as register-
    // tiled passes.  A pass takes, in circuit order, every gate whose target
    // fits its 4 + tile_wb high positions; a gate that does not fit waits for
    // the next pass, and so does every later gate that shares a position with
    // a waiting gate, or that rounds while a rounding gate waits.  The waiting
    // gates keep their order.
    void flush_reg(Buffer& b, const std::vector<uint32_t>& wires, int id) {
        const int cap = tile_wb + tile_rb;
        std::vector<Sched> pending;
        for (uint32_t gi : b.pending) pending.push_back(classify(gates[gi], wires));
        while (!pending.empty()) {
            std::vector<Sched> placed, waiting;
            uint32_t targets = 0, blocked = 0;
            bool chain_blocked = false;
            for (const Sched& s : pending) {
                bool take = !(s.all & blocked) && (s.exact || !chain_blocked);
                if (take && s.tgt >= 5 && !(targets & (1u << s.tgt))) {
                    if (__builtin_popcount(targets) < cap) targets |= 1u << s.tgt;
                    else take = false;
                }
                if (take) {
                    placed.push_back(s);
                } else {
                    waiting.push_back(s);
                    blocked |= s.all;
                    if (!s.exact) chain_blocked = true;
                }
            }
            emit_reg_pass(id, b.legs, placed, targets);
            pending.swap(waiting);
        }
    }

    // Turn the queued gates of a state into passes (wires are the state's
    // sorted open wires; position p holds wires[p]).
    void flush(int id, const std::vector<uint32_t>& wires) {
        Buffer& b = bufs[size_t(id)];
        if (b.pending.empty()) return;
        const int legs = b.legs;
        if (legs >= 5 + tile_wb + tile_rb) {
            flush_reg(b, wires, id);
            gate_total += uint32_t(b.pending.size());
            b.pending.clear();
            return;
        }
        auto pos_of = [&](uint32_t wire) {
            return int(std::lower_bound(wires.begin(), wires.end(), wire) - wires.begin());
        };
        const int pass_bits = std::min(legs, this->pass_bits);
        const uint32_t low = (1u << std::min(legs, kLowBits)) - 1u;
        uint32_t mask = low;
        std::vector<uint32_t> group;
        auto emit = [&]() {
            if (group.empty()) return;
            // Fill the pass up to pass_bits positions with the lowest free ones.
            uint32_t m = mask;
            for (int p = 0; p < legs && __builtin_popcount(m) < pass_bits; ++p) m |= 1u << p;
            Item it{};
            it.kind = 0;
            it.hdr.mask = m;
            it.hdr.legs = legs;
            it.hdr.local = __builtin_popcount(m);
            it.hdr.ngates = int(group.size());
            it.buf = id;
            it.gate_off = uint32_t(pass_gates.size());
            it.legs = legs;
            auto local = [&](int p) { return __builtin_popcount(m & ((1u << p) - 1u)); };
            for (uint32_t gi : group) {
                const wqc_gate& g = gates[gi];
                PassGate pg{};
                if (g.kind == WQC_GATE_CNOT || g.kind == WQC_GATE_CZ) {
                    pg.kind = g.kind == WQC_GATE_CNOT ? kCnot : kCz;
                    pg.a = local(pos_of(uint32_t(g.q0)));
                    pg.b = local(pos_of(uint32_t(g.q1)));
                } else if (g.kind == WQC_GATE_CCNOT) {
                    pg.kind = kCcnot;
                    pg.a = local(pos_of(uint32_t(g.q0)));
                    pg.b = local(pos_of(uint32_t(g.q1)));
                    pg.c = local(pos_of(uint32_t(g.q2)));
                } else {
                    pg.kind = kOne;
                    pg.a = local(pos_of(uint32_t(g.q0)));
                    gate_matrix_2x2(g.kind, g.angle, pg.u);
                }
                pass_gates.push_back(pg);
            }
            items.push_back(it);
            bytes_moved += 2 * (16ull << legs);
            group.clear();
            mask = low;
        };
        for (uint32_t gi : b.pending) {
            uint32_t gm = 0;
            for (uint32_t w : wires_of(gates[gi])) gm |= 1u << pos_of(w);
            if (__builtin_popcount(mask | gm) > pass_bits) emit();
            mask |= gm;
            group.push_back(gi);
        }
        emit();
        gate_total += uint32_t(b.pending.size());
        b.pending.clear();
    }
};

struct Live {
    bool gate = false;
    uint32_t gate_index = 0;
    std::vector<uint32_t> wires;
    int buf = -1;
};

using Key = std::pair<int, uint32_t>;  // RefId order: Ket < Gate < Node, then index

struct Walker {
    uint32_t n;
    const wqc_gate* gates;
    uint32_t gate_count;
    uint32_t node_count;
    Plan* plan;
    std::map<Key, Live> live;
    std::vector<char> consumed_nodes, consumed_gate, consumed_ket;
    uint32_t next_gate = 0;

    Walker(uint32_t n_, const wqc_gate* g, uint32_t gc, uint32_t nc, Plan* p)
        : n(n_), gates(g), gate_count(gc), node_count(nc), plan(p), consumed_nodes(nc, 0), consumed_gate(gc, 0),
          consumed_ket(n_, 0) {}

    static uint64_t occupied(const Live& t) { return t.gate ? 0 : (16ull << t.wires.size()); }
    uint64_t live_bytes() const {
        uint64_t s = 0;
        for (const auto& kv : live) s += occupied(kv.second);
        return s;
    }

    wqc_status next_unitary(uint32_t* out) const {
        for (uint32_t i = next_gate; i < gate_count; ++i)
            if (is_unitary(gates[i].kind)) {
                *out = i;
                return WQC_OK;
            }
        return failx("gates are out of circuit order");
    }

    // Walk::materialize (exact.rs:286-358).
    wqc_status materialize(Key id) {
        if (live.count(id)) return WQC_OK;
        if (id.first == WQC_TREE_KET0) {
            const uint32_t wire = id.second;
            if (wire >= n) return fail_index(wire, n);
            if (consumed_ket[wire]) return failx("contraction tree reuses a tensor");
            consumed_ket[wire] = 1;
            Live t;
            t.wires = {wire};
            if (plan->on) t.buf = plan->new_ket();
            live.emplace(id, std::move(t));
        } else if (id.first == WQC_TREE_GATE) {
            const uint32_t gi = id.second;
            if (gi >= gate_count) return failx("contraction tree gate is missing");
            if (!is_unitary(gates[gi].kind)) return failx("gate " + std::to_string(gi) + " is not a contraction leaf");
            uint32_t expected = 0;
            if (wqc_status s = next_unitary(&expected)) return s;
            if (gi != expected) return failx("gates are out of circuit order");
            next_gate = gi + 1;
            if (consumed_gate[gi]) return failx("contraction tree reuses a tensor");
            consumed_gate[gi] = 1;
            Live t;
            t.gate = true;
            t.gate_index = gi;
            live.emplace(id, std::move(t));
        } else {
            if (id.second < node_count && consumed_nodes[id.second]) return failx("contraction tree reuses a tensor");
            return failx("contraction tree tensor is not ready");
        }
        return WQC_OK;
    }

    // Walk::take (exact.rs:360-376).
    wqc_status take(Key id, Live* out) {
        auto it = live.find(id);
        if (it == live.end()) return failx("contraction tree tensor is not ready");
        *out = std::move(it->second);
        live.erase(it);
        if (id.first == WQC_TREE_NODE) {
            if (id.second >= node_count) return failx("contraction tree tensor is not ready");
            if (consumed_nodes[id.second]) return failx("contraction tree reuses a tensor");
            consumed_nodes[id.second] = 1;
        }
        return WQC_OK;
    }

    static wqc_status ref_id(const wqc_tree_ref& r, Key* out) {
        switch (r.kind) {
            case WQC_TREE_KET0: case WQC_TREE_GATE: case WQC_TREE_NODE:
                *out = Key(r.kind, r.index);
                return WQC_OK;
            case WQC_TREE_LEFT: case WQC_TREE_RIGHT: return failx("exact contraction has no split");
            case WQC_TREE_BRA0: return failx("exact contraction has no bra0");
            case WQC_TREE_CONTROL: case WQC_TREE_TARGET: return failx("exact contraction has no gate halves");
            default: return failx("unknown tensor reference kind " + std::to_string(r.kind));
        }
    }

    // walk (exact.rs:136-196) up to the sample.
    wqc_status run(const wqc_tree_node* nodes, uint64_t* peak_out) {
        uint64_t peak = 0;
        for (uint32_t index = 0; index < node_count; ++index) {
            const wqc_tree_node& node = nodes[index];
            if (node.op != 0) return failx("contraction tree mixes sweep steps and exact contractions");
            Key lid, rid;
            if (wqc_status s = ref_id(node.left, &lid)) return s;
            if (wqc_status s = ref_id(node.right, &rid)) return s;
            if (wqc_status s = materialize(lid)) return s;
            if (wqc_status s = materialize(rid)) return s;
            Live lt, rt;
            if (wqc_status s = take(lid, &lt)) return s;
            if (wqc_status s = take(rid, &rt)) return s;
            const bool allocating = !lt.gate && !rt.gate;
            const uint64_t inputs = occupied(lt) + occupied(rt);
            Live result;
            if (lt.gate || rt.gate) {
                // combine: (Gate, state) | (state, Gate) (exact.rs:390-411).
                Live& g = lt.gate ? lt : rt;
                Live& st = lt.gate ? rt : lt;
                if (st.gate) return failx("exact contraction does not contract two gates");
                for (uint32_t w : wires_of(gates[g.gate_index]))
                    if (!std::binary_search(st.wires.begin(), st.wires.end(), w))
                        return failx("gate wires are not open");
                result.wires = st.wires;
                result.buf = st.buf;
                if (plan->on) plan->bufs[size_t(st.buf)].pending.push_back(g.gate_index);
            } else {
                // outer (exact.rs:444-480).
                for (uint32_t w : lt.wires)
                    if (std::binary_search(rt.wires.begin(), rt.wires.end(), w)) return failx("tensors share a wire");
                result.wires = lt.wires;
                result.wires.insert(result.wires.end(), rt.wires.begin(), rt.wires.end());
                std::sort(result.wires.begin(), result.wires.end());
                if (result.wires.size() > size_t(kMaxOpenLegs)) return failx("contraction tree tensor exceeds 26 legs");
                if (plan->on) {
                    plan->flush(lt.buf, lt.wires);
                    plan->flush(rt.buf, rt.wires);
                    const int legs = int(result.wires.size());
                    result.buf = plan->new_state(legs);
                    Item it{};
                    it.kind = 1;
                    it.legs = legs;
                    it.buf = result.buf;
                    it.lbuf = lt.buf;
                    it.rbuf = rt.buf;
                    for (size_t p = 0; p < result.wires.size(); ++p) {
                        if (std::binary_search(lt.wires.begin(), lt.wires.end(), result.wires[p])) it.lmask |= 1u << p;
                        else it.rmask |= 1u << p;
                    }
                    plan->items.push_back(it);
                    plan->bytes_moved += (16ull << legs) + (16ull << lt.wires.size()) + (16ull << rt.wires.size());
                    plan->drop(lt.buf);
                    plan->drop(rt.buf);
                }
            }
            uint64_t during = live_bytes() + inputs;
            if (allocating) during += occupied(result);
            if (during > kMaxPeakBytes) return failx("contraction tree peak exceeds 1 GiB");
            peak = std::max(peak, during);
            live.emplace(Key(WQC_TREE_NODE, index), std::move(result));
        }
        for (uint32_t i = 0; i < gate_count; ++i)
            if (is_unitary(gates[i].kind) && !consumed_gate[i]) return failx("gate was not contracted");
        for (const auto& kv : live)
            if (kv.second.gate) return failx("gate was not contracted");
        *peak_out = peak;
        return WQC_OK;
    }
};


}  // namespace

// ---------------------------------------------------------------------------
// The executor.
// ---------------------------------------------------------------------------
struct wqc_exact {
    wqc_cuda_ctx* ctx = nullptr;
    int device = 0;
    int sm_count = 148;
    int pass_bits = kMaxPassBits;
    int tile_wb = 3, tile_rb = 4;  // register tiles: 2^tile_wb warps, 2^tile_rb amplitudes a thread
    cudaStream_t stream = nullptr;
    double2* arena = nullptr;
    uint64_t arena_bytes = 0;
    unsigned char* table = nullptr;  // device: pass gates, gather offsets, gathered components
    uint64_t table_bytes = 0;
    unsigned char* staging = nullptr;  // pinned host mirror of `table`
    uint64_t staging_bytes = 0;
    std::vector<cudaEvent_t> events;
    std::atomic<int> cancel{0};
    wqc_exact_stats stats{};
};

namespace {

wqc_status cuda_fail(const char* what, cudaError_t e) {
    return record_error(WQC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

wqc_status ensure_device(wqc_exact* ex, void** p, uint64_t* have, uint64_t need) {
    if (*have >= need) return WQC_OK;
    if (*p) {
        cudaFree(*p);
        *p = nullptr;
        *have = 0;
    }
    if (cudaMalloc(p, need) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        return record_oom(need, fr);
    }
    *have = need;
    (void)ex;
    return WQC_OK;
}

wqc_status ensure_staging(wqc_exact* ex, uint64_t need) {
    if (ex->staging_bytes >= need) return WQC_OK;
    if (ex->staging) cudaFreeHost(ex->staging);
    ex->staging = nullptr;
    ex->staging_bytes = 0;
    if (cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&ex->staging), need)) {
        cudaGetLastError();
        return cuda_fail("cudaMallocHost(exact staging)", e);
    }
    ex->staging_bytes = need;
    return WQC_OK;
}

cudaEvent_t event_at(wqc_exact* ex, size_t i) {
    while (ex->events.size() <= i) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        ex->events.push_back(e);
    }
    return ex->events[i];
}

// The reference's complex product on the host (num_complex Mul).
inline void host_mul(double& re, double& im, double br, double bi) {
    const double r = re * br - im * bi;
    const double i = re * bi + im * br;
    re = r;
    im = i;
}

}  // namespace

extern "C" {

wqc_status wqc_exact_create(wqc_cuda_ctx* ctx, wqc_exact** out) {
    if (!ctx || !out) return failx("null argument");
    auto* ex = new wqc_exact();
    ex->ctx = ctx;
    ex->device = context_device(ctx);
    ex->sm_count = context_sm_count(ctx);
    cudaError_t e = cudaSetDevice(ex->device);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(exact_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(sizeof(double2)) << kMaxPassBits);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(exact_pass_reg_kernel<3, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(sizeof(double2)) << 12);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(exact_pass_reg_kernel<4, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(sizeof(double2)) << 13);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ex->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete ex;
        return cuda_fail("exact executor setup", e);
    }
    *out = ex;
    return WQC_OK;
}

void wqc_exact_destroy(wqc_exact* ex) {
    if (!ex) return;
    cudaSetDevice(ex->device);
    if (ex->stream) cudaStreamSynchronize(ex->stream);
    for (cudaEvent_t e : ex->events) cudaEventDestroy(e);
    if (ex->arena) cudaFree(ex->arena);
    if (ex->table) cudaFree(ex->table);
    if (ex->staging) cudaFreeHost(ex->staging);
    if (ex->stream) cudaStreamDestroy(ex->stream);
    delete ex;
}

wqc_status wqc_exact_set_tile_bits(wqc_exact* ex, int32_t bits) {
    if (!ex) return failx("null executor");
    if (bits != 12 && bits != 13) return failx("tile bits must be 12 or 13");
    ex->tile_wb = bits == 13 ? 4 : 3;
    ex->tile_rb = 4;
    return WQC_OK;
}

void wqc_exact_cancel(wqc_exact* ex) {
    if (ex) ex->cancel.store(1);
}

wqc_status wqc_exact_last_stats(wqc_exact* ex, wqc_exact_stats* out) {
    if (!ex || !out) return failx("null argument");
    *out = ex->stats;
    return WQC_OK;
}

wqc_status wqc_exact_validate(uint32_t n, const wqc_gate* gates, uint32_t gate_count, const wqc_tree* tree,
                              const uint64_t* mps_order, uint32_t mps_len) {
    if (wqc_status s = check_tree(tree)) return s;
    uint64_t declared = 0;
    if (wqc_status s = declared_peak(tree, &declared)) return s;
    return check_shape(n, gates, gate_count, tree, mps_order, mps_len);
}

wqc_status wqc_exact_measured_peak(uint32_t n, const wqc_gate* gates, uint32_t gate_count, const wqc_tree* tree,
                                   uint64_t* peak) {
    if (wqc_status s = check_tree(tree)) return s;
    if (!peak) return failx("null argument");
    if (wqc_status s = check_shape(n, gates, gate_count, tree, nullptr, 0)) return s;
    Plan plan;  // off: validation and bytes only
    Walker w(n, gates, gate_count, tree->node_count, &plan);
    return w.run(tree->nodes, peak);
}

wqc_status wqc_exact_contract(wqc_exact* ex, uint32_t n, const wqc_gate* gates, uint32_t gate_count,
                              const wqc_tree* tree, const uint64_t* mps_order, uint32_t mps_len, const uint64_t* bits,
                              uint32_t count, double* out) {
    if (!ex) return failx("null executor");
    if (wqc_status s = check_tree(tree)) return s;
    if (count && (!bits || !out)) return failx("null argument");
    ex->stats = wqc_exact_stats{};
    // contract_exact_at: declared peak, then the walk, then the comparison.
    uint64_t declared = 0;
    if (wqc_status s = declared_peak(tree, &declared)) return s;
    if (wqc_status s = check_shape(n, gates, gate_count, tree, mps_order, mps_len)) return s;
    Plan plan;
    plan.on = true;
    plan.pass_bits = ex->pass_bits;
    plan.tile_wb = ex->tile_wb;
    plan.tile_rb = ex->tile_rb;
    plan.gates = gates;
    Walker w(n, gates, gate_count, tree->node_count, &plan);
    uint64_t peak = 0;
    if (wqc_status s = w.run(tree->nodes, &peak)) return s;
    // Flush what is still queued; then the components of each amplitude, the
    // live tensors in RefId order (exact.rs:198-231).
    std::vector<const Live*> order;
    std::vector<char> covered(n, 0);
    for (const auto& kv : w.live) {
        plan.flush(kv.second.buf, kv.second.wires);
        order.push_back(&kv.second);
        for (uint32_t wire : kv.second.wires) covered[wire] = 1;
    }
    if (declared != peak) return failx("contraction tree peak does not match");

    // Layout: ket slots, then the tensor region; table: pass gates, gather
    // offsets, gathered components.
    const uint64_t ket_elems = 2 * uint64_t(plan.kets);
    const uint64_t ket_bytes = (ket_elems * 16 + kAlign - 1) / kAlign * kAlign;
    const uint64_t arena_need = std::max<uint64_t>(ket_bytes + plan.placer.top, kAlign);
    const size_t T = order.size();
    const uint64_t gather_n = uint64_t(count) * T;
    if (gather_n > (1ull << 28)) return failx("too many amplitudes for one contraction");
    const uint64_t pg_bytes = (plan.pass_gates.size() * sizeof(PassGate) + kAlign - 1) / kAlign * kAlign;
    const uint64_t ops_bytes = (plan.reg_ops.size() * sizeof(RegOp) + kAlign - 1) / kAlign * kAlign;
    const uint64_t gates_bytes = pg_bytes + ops_bytes;
    const uint64_t where_bytes = (gather_n * sizeof(uint64_t) + kAlign - 1) / kAlign * kAlign;
    const uint64_t comp_bytes = std::max<uint64_t>(gather_n * sizeof(double2), 16);
    const uint64_t table_need = gates_bytes + where_bytes + comp_bytes;

    if (cudaError_t e = cudaSetDevice(ex->device)) return cuda_fail("cudaSetDevice", e);
    if (wqc_status s = ensure_device(ex, reinterpret_cast<void**>(&ex->arena), &ex->arena_bytes, arena_need)) return s;
    if (wqc_status s = ensure_device(ex, reinterpret_cast<void**>(&ex->table), &ex->table_bytes, table_need)) return s;
    if (wqc_status s = ensure_staging(ex, table_need)) return s;

    // Stage the pass gates and the gather offsets.
    if (!plan.pass_gates.empty())
        std::memcpy(ex->staging, plan.pass_gates.data(), plan.pass_gates.size() * sizeof(PassGate));
    if (!plan.reg_ops.empty())
        std::memcpy(ex->staging + pg_bytes, plan.reg_ops.data(), plan.reg_ops.size() * sizeof(RegOp));
    uint64_t* where = reinterpret_cast<uint64_t*>(ex->staging + gates_bytes);
    const uint64_t tensor_base = ket_bytes / 16;  // element offset of the tensor region
    for (uint32_t k = 0; k < count; ++k) {
        for (size_t t = 0; t < T; ++t) {
            const Live& L = *order[t];
            const Buffer& B = plan.bufs[size_t(L.buf)];
            uint64_t index = 0;
            for (size_t p = 0; p < L.wires.size(); ++p)
                if (L.wires[p] < 64 && ((bits[k] >> L.wires[p]) & 1ull)) index |= 1ull << p;
            where[uint64_t(k) * T + t] = (B.ket ? 0 : tensor_base) + B.off + index;
        }
    }
    cudaStream_t st = ex->stream;
    const uint64_t upload = gates_bytes + gather_n * sizeof(uint64_t);
    if (upload)
        if (cudaError_t e = cudaMemcpyAsync(ex->table, ex->staging, upload, cudaMemcpyHostToDevice, st))
            return cuda_fail("cudaMemcpyAsync(exact tables)", e);
    const PassGate* d_gates = reinterpret_cast<const PassGate*>(ex->table);
    const RegOp* d_ops = reinterpret_cast<const RegOp*>(ex->table + pg_bytes);
    const uint64_t* d_where = reinterpret_cast<const uint64_t*>(ex->table + gates_bytes);
    double2* d_comp = reinterpret_cast<double2*>(ex->table + gates_bytes + where_bytes);
    double2* kets = ex->arena;
    double2* tensors = ex->arena + tensor_base;
    auto at = [&](int id) {
        const Buffer& B = plan.bufs[size_t(id)];
        return (B.ket ? kets : tensors) + B.off;
    };

    size_t ev = 0;
    cudaEvent_t e0 = event_at(ex, ev++), e1 = event_at(ex, ev++);
    if (!e0 || !e1) return record_error(WQC_ERR_CUDA, "cudaEventCreate failed");
    cudaEventRecord(e0, st);
    uint32_t launches = 0, passes = 0, outers = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> timed;
    auto bail = [&](wqc_status s) {
        cudaStreamSynchronize(st);
        return s;
    };
    if (plan.kets) {
        exact_kets_kernel<<<std::min<uint32_t>((plan.kets + 255) / 256, 1024), 256, 0, st>>>(kets, plan.kets);
        ++launches;
    }
    for (const Item& it : plan.items) {
        if (ex->cancel.exchange(0)) return bail(record_error(WQC_ERR_CANCELLED, "computation cancelled: the client has gone"));
        if (it.kind == 0 || it.kind == 2) {
            const bool time_it = it.legs >= kTimedPassLegs;
            cudaEvent_t a = nullptr, b = nullptr;
            if (time_it) {
                a = event_at(ex, ev++);
                b = event_at(ex, ev++);
                if (!a || !b) return bail(record_error(WQC_ERR_CUDA, "cudaEventCreate failed"));
                cudaEventRecord(a, st);
            }
            if (it.kind == 0) {
                const uint32_t grid = 1u << (it.legs - it.hdr.local);
                exact_pass_kernel<<<grid, kPassThreads, size_t(16) << it.hdr.local, st>>>(at(it.buf), it.hdr,
                                                                                           d_gates + it.gate_off);
            } else {
                const int tile = 5 + plan.tile_wb + plan.tile_rb;  // grid: one block per tile, 2^(legs - tile) tiles
                const uint32_t grid = 1u << (it.legs - tile);
                const size_t smem = it.xchg ? size_t(16) << tile : 0;
                if (plan.tile_wb == 3)
                    exact_pass_reg_kernel<3, 4><<<grid, 256, smem, st>>>(at(it.buf), it.rhdr, d_ops + it.gate_off);
                else
                    exact_pass_reg_kernel<4, 4><<<grid, 512, smem, st>>>(at(it.buf), it.rhdr, d_ops + it.gate_off);
            }
            if (time_it) {
                cudaEventRecord(b, st);
                timed.emplace_back(a, b);
                ex->stats.pass_bytes += 2 * (16ull << it.legs);
            }
            ++passes;
        } else {
            const uint64_t total = 1ull << it.legs;
            const uint32_t grid = uint32_t(std::min<uint64_t>((total + kOuterThreads - 1) / kOuterThreads,
                                                              uint64_t(ex->sm_count) * 8));
            exact_outer_kernel<<<grid, kOuterThreads, 0, st>>>(at(it.buf), at(it.lbuf), at(it.rbuf), it.lmask, it.rmask,
                                                               it.legs);
            ++outers;
        }
        ++launches;
        if (cudaError_t e = cudaGetLastError()) return bail(cuda_fail("exact contraction launch", e));
    }
    if (gather_n) {
        exact_gather_kernel<<<uint32_t(std::min<uint64_t>((gather_n + 255) / 256, 1024)), 256, 0, st>>>(
            ex->arena, d_where, uint32_t(gather_n), d_comp);
        ++launches;
        if (cudaError_t e = cudaGetLastError()) return bail(cuda_fail("exact gather launch", e));
        if (cudaError_t e = cudaMemcpyAsync(ex->staging, d_comp, gather_n * sizeof(double2), cudaMemcpyDeviceToHost, st))
            return bail(cuda_fail("cudaMemcpyAsync(exact components)", e));
    }
    cudaEventRecord(e1, st);
    if (cudaError_t e = cudaStreamSynchronize(st)) return cuda_fail("exact contraction", e);

    // sample (exact.rs:198-231): the product in RefId order; a set bit on a
    // wire no live tensor holds makes the amplitude zero.
    const double2* comp = reinterpret_cast<const double2*>(ex->staging);
    for (uint32_t k = 0; k < count; ++k) {
        double re = 1.0, im = 0.0;
        for (size_t t = 0; t < T; ++t) host_mul(re, im, comp[uint64_t(k) * T + t].x, comp[uint64_t(k) * T + t].y);
        for (uint32_t wire = 0; wire < n && wire < 64; ++wire)
            if (!covered[wire] && ((bits[k] >> wire) & 1ull)) {
                re = 0.0;
                im = 0.0;
                break;
            }
        out[2 * size_t(k)] = re;
        out[2 * size_t(k) + 1] = im;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    ex->stats.device_ms = ms;
    for (auto& ab : timed) {
        float t = 0.f;
        cudaEventElapsedTime(&t, ab.first, ab.second);
        ex->stats.pass_ms += t;
    }
    ex->stats.launches = launches;
    ex->stats.exchanges = plan.exchanges;
    ex->stats.passes = passes;
    ex->stats.outer_products = outers;
    ex->stats.gates = plan.gate_total;
    ex->stats.bytes_moved = plan.bytes_moved;
    ex->stats.arena_bytes = ex->arena_bytes;
    return WQC_OK;
}

}  // extern "C"
