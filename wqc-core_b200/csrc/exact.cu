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

namespace wqc {
wqc_status record_error(wqc_status code, const std::string& msg);  // executor.cu
wqc_status record_oom(uint64_t required, uint64_t available);
wqc_status check_circuit_gate(int n, const wqc_gate& g);
void gate_matrix_2x2(int kind, double theta, double2 out[4]);
int context_device(const wqc_cuda_ctx* ctx);
int context_sm_count(const wqc_cuda_ctx* ctx);
}  // namespace wqc

using namespace wqc;

namespace {

constexpr int kMaxOpenLegs = 26;                 // exact.rs:25
constexpr uint64_t kMaxPeakBytes = 1ull << 30;   // exact.rs:27
constexpr int kLowBits = 4;                      // positions every pass holds: 16 amplitudes, 256 bytes
constexpr int kMaxPassBits = 12;                 // 4096 amplitudes, 64 KB of shared memory per block
constexpr int kPassThreads = 256;
constexpr int kOuterThreads = 256;
constexpr uint64_t kAlign = 256;                 // arena placement granularity (bytes)
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

wqc_status failx(const std::string& msg) { return record_error(WQC_ERR_INVALID, msg); }
wqc_status fail_index(uint64_t index, uint64_t limit) {
    return record_error(WQC_ERR_QUBIT_OUT_OF_RANGE, "Qubit index " + std::to_string(index) +
                                                        " out of bounds (limit: " + std::to_string(limit) + ")");
}

bool is_unitary(int kind) { return kind >= WQC_GATE_H && kind <= WQC_GATE_CCNOT; }

std::vector<uint32_t> wires_of(const wqc_gate& g) {
    switch (g.kind) {
        case WQC_GATE_CNOT: case WQC_GATE_CZ: return {uint32_t(g.q0), uint32_t(g.q1)};
        case WQC_GATE_CCNOT: return {uint32_t(g.q0), uint32_t(g.q1), uint32_t(g.q2)};
        default: return {uint32_t(g.q0)};
    }
}

// canonicalize_site_order (src/tn/tree.rs:442-457) with validate_site_order
// (src/tn/site_order.rs:7-31): an empty or identity order is "no order".
wqc_status canonical_empty(uint32_t n, const uint64_t* order, uint32_t len, bool* empty) {
    *empty = true;
    if (len == 0) return WQC_OK;
    if (len != n)
        return failx("mps_site_order length " + std::to_string(len) + " != qubit_count " + std::to_string(n));
    std::vector<char> seen(n, 0);
    for (uint32_t i = 0; i < len; ++i) {
        if (order[i] >= n) return fail_index(order[i], n);
        if (seen[order[i]])
            return failx("mps_site_order is not a permutation (duplicate logical " + std::to_string(order[i]) + ")");
        seen[order[i]] = 1;
    }
    for (uint32_t i = 0; i < len; ++i)
        if (order[i] != i) *empty = false;
    return WQC_OK;
}

// check_shape (exact.rs:99-134).
wqc_status check_shape(uint32_t n, const wqc_gate* gates, uint32_t gate_count, const wqc_tree* tree,
                       const uint64_t* mps_order, uint32_t mps_len) {
    if (n == 0) return record_error(WQC_ERR_INVALID_QUBIT_COUNT, "Invalid qubit count: 0. Max limit is 40.");
    if (gate_count && !gates) return failx("null gate list");
    for (uint32_t i = 0; i < gate_count; ++i)
        if (wqc_status s = check_circuit_gate(int(std::min<uint32_t>(n, 0x7fffffff)), gates[i])) return s;
    if (tree->site_order_len && !tree->site_order) return failx("null site order");
    std::vector<uint64_t> so(tree->site_order, tree->site_order + tree->site_order_len);
    bool empty = true;
    if (wqc_status s = canonical_empty(n, so.data(), uint32_t(so.size()), &empty)) return s;
    if (!empty) return failx("contraction tree keeps parent wire numbers");
    if (mps_order) {
        for (uint32_t i = 0; i < mps_len; ++i)
            if (mps_order[i] > 0xffffffffull) return failx("qubit index exceeds u32");
        if (wqc_status s = canonical_empty(n, mps_order, mps_len, &empty)) return s;
        if (!empty) return failx("mps_site_order does not match the contraction tree");
    }
    return WQC_OK;
}

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
    int kind;  // 0 pass, 1 outer
    PassHdr hdr;
    int buf;             // pass: the state; outer: the result
    int lbuf, rbuf;      // outer: the operands
    uint32_t gate_off;   // pass: first gate in the pass-gate table
    uint32_t lmask, rmask;
    int legs;
};

// First-fit placement of tensors in the arena, done while planning; the
// device work runs in plan order on one stream, so a freed range is reused
// only by work that comes after its last reader.
struct Placer {
    std::map<uint64_t, uint64_t> free_;  // byte offset -> bytes
    uint64_t top = 0;
    uint64_t alloc(uint64_t bytes) {
        bytes = (bytes + kAlign - 1) / kAlign * kAlign;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                const uint64_t off = it->first, rest = it->second - bytes;
                free_.erase(it);
                if (rest) free_[off + bytes] = rest;
                return off;
            }
        }
        // Grow from the top, merging a free range that ends there.
        if (!free_.empty()) {
            auto last = std::prev(free_.end());
            if (last->first + last->second == top) {
                const uint64_t off = last->first;
                free_.erase(last);
                top = off + bytes;
                return off;
            }
        }
        const uint64_t off = top;
        top += bytes;
        return off;
    }
    void release(uint64_t off, uint64_t bytes) {
        bytes = (bytes + kAlign - 1) / kAlign * kAlign;
        auto it = free_.emplace(off, bytes).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }
};

struct Plan {
    bool on = false;
    int pass_bits = kMaxPassBits;
    const wqc_gate* gates = nullptr;
    std::vector<Buffer> bufs;
    std::vector<Item> items;
    std::vector<PassGate> pass_gates;
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

    // Turn the queued gates of a state into passes (wires are the state's
    // sorted open wires; position p holds wires[p]).
    void flush(int id, const std::vector<uint32_t>& wires) {
        Buffer& b = bufs[size_t(id)];
        if (b.pending.empty()) return;
        const int legs = b.legs;
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

wqc_status check_tree(const wqc_tree* tree) {
    if (!tree) return failx("null contraction tree");
    if (tree->node_count && !tree->nodes) return failx("null contraction tree nodes");
    return WQC_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// The executor.
// ---------------------------------------------------------------------------
struct wqc_exact {
    wqc_cuda_ctx* ctx = nullptr;
    int device = 0;
    int sm_count = 148;
    int pass_bits = kMaxPassBits;
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
    if (const char* env = std::getenv("WQC_EXACT_PASS_BITS")) {
        const int b = std::atoi(env);
        if (b >= kLowBits + 3 && b <= kMaxPassBits) ex->pass_bits = b;
    }
    cudaError_t e = cudaSetDevice(ex->device);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(exact_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(sizeof(double2)) << kMaxPassBits);
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
    const uint64_t gates_bytes = (plan.pass_gates.size() * sizeof(PassGate) + kAlign - 1) / kAlign * kAlign;
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
        if (it.kind == 0) {
            const bool time_it = it.legs >= kTimedPassLegs;
            cudaEvent_t a = nullptr, b = nullptr;
            if (time_it) {
                a = event_at(ex, ev++);
                b = event_at(ex, ev++);
                if (!a || !b) return bail(record_error(WQC_ERR_CUDA, "cudaEventCreate failed"));
                cudaEventRecord(a, st);
            }
            const uint32_t grid = 1u << (it.legs - it.hdr.local);
            exact_pass_kernel<<<grid, kPassThreads, size_t(16) << it.hdr.local, st>>>(at(it.buf), it.hdr,
                                                                                       d_gates + it.gate_off);
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
    ex->stats.passes = passes;
    ex->stats.outer_products = outers;
    ex->stats.gates = plan.gate_total;
    ex->stats.bytes_moved = plan.bytes_moved;
    ex->stats.arena_bytes = ex->arena_bytes;
    return WQC_OK;
}

}  // extern "C"
