// Network contraction trees on the device: the walk of src/tn/network.rs
// (<0...0|U|0...0> of a circuit as one tensor network) with its tensors in
// HBM.
//
// The host walks the tree once, as the reference's `walk` does (leaves,
// shared legs, reordered copies, live bytes and the peak), and plans the
// device work while it walks.  Leaves (|0> and <0| vectors, gate tensors,
// gate halves) are built on the host -- at most 64 amplitudes each -- and
// uploaded together into a region of the arena that is never reused; every
// other tensor gets a place in the arena's reusable region.  A large node
// reorders each operand that is not already in [shared legs, free legs]
// order (network_permute_kernel, a gather through four 7-bit index tables)
// and multiplies the two with a complex GEMM (cuBLAS ZGEMM): the result's
// legs are the right operand's free legs (low bits), then the left's
// (network.rs:591-664).  Small nodes -- most of a circuit's tree -- read
// their operands in place through index tables, one block each, and every
// run of them between two large nodes is launched level by level (a node's
// level: one more than its deepest input made in the same run), so a tree of
// hundreds of small joins costs a few launches.  Nothing reaches the device until the whole walk has
// passed, so every failure the reference reports comes back before any
// launch.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/wqc_cuda.h"
#include "tree_common.h"

using namespace wqc;
using namespace wqc::tree;

namespace {

constexpr int kPermuteThreads = 256;

// ---------------------------------------------------------------------------
// Device side.
// ---------------------------------------------------------------------------

// Source position of each destination bit: destination bit b reads bit src[b].
struct PermuteMap {
    uint8_t src[32];
};

// dst[i] = src[gather(i)]: destination bit b of i is source bit map.src[b]
// (network.rs:756-777).  The gather index comes from four 7-bit tables (28
// bits >= 26 legs).  Bounds: i < 2^legs; the map is a permutation of 0..legs-1,
// so gather(i) < 2^legs, the source's length.
__global__ void __launch_bounds__(kPermuteThreads) network_permute_kernel(double2* __restrict__ dst,
                                                                          const double2* __restrict__ src,
                                                                          PermuteMap map, int legs) {
    __shared__ uint32_t tab[4][128];
    for (int e = threadIdx.x; e < 512; e += blockDim.x) {
        const int c = e >> 7, v = e & 127;
        uint32_t out = 0;
        for (int j = 0; j < 7; ++j) {
            const int b = 7 * c + j;
            if (b < legs && ((v >> j) & 1)) out |= 1u << map.src[b];
        }
        tab[c][v] = out;
    }
    __syncthreads();
    const uint32_t total = 1u << legs;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x)
        dst[i] = src[tab[0][i & 127] | tab[1][(i >> 7) & 127] | tab[2][(i >> 14) & 127] | tab[3][(i >> 21) & 127]];
}

// One small contraction per block: C[i][j] = sum_x L[lf[i] + ls[x]] R[rf[j] + rs[x]]
// with the operands read in place through offset tables (no reordered
// copies).  The result is row-major m x n: index j | i << log2 n,
// the right operand's free legs low (network.rs:591-664).
struct SmallJob {
    uint64_t l, r, c;      // element offsets in the arena
    uint32_t m, n, k;
    uint32_t lf, ls, rf, rs;  // offsets of the four index tables in the table array
};

constexpr int kSmallThreads = 128;

// When a join has fewer outputs than threads (down to a single scalar), the
// threads of one output split its sum over x and add their parts through
// shared memory; the parts are added in thread order.
__global__ void __launch_bounds__(kSmallThreads) network_small_kernel(double2* __restrict__ arena,
                                                                      const SmallJob* __restrict__ jobs,
                                                                      const uint32_t* __restrict__ tab) {
    __shared__ double2 part[kSmallThreads];
    const SmallJob J = jobs[blockIdx.x];
    const double2* L = arena + J.l;
    const double2* R = arena + J.r;
    double2* out = arena + J.c;
    const uint32_t* lf = tab + J.lf;
    const uint32_t* ls = tab + J.ls;
    const uint32_t* rf = tab + J.rf;
    const uint32_t* rs = tab + J.rs;
    const uint32_t outs = J.m * J.n;  // a power of two
    const uint32_t tpo = outs >= kSmallThreads ? 1u : kSmallThreads / outs;  // threads per output
    const uint32_t slot = threadIdx.x / tpo, piece = threadIdx.x % tpo;
    for (uint32_t first = 0; first < outs; first += kSmallThreads / tpo) {
        const uint32_t o = first + slot;
        double re = 0.0, im = 0.0;
        if (o < outs) {
            const uint32_t i = o / J.n, j = o - i * J.n;
            const uint32_t li = lf[i], rj = rf[j];
            for (uint32_t x = piece; x < J.k; x += tpo) {
                const double2 a = L[li + ls[x]], b = R[rj + rs[x]];
                re = fma(a.x, b.x, fma(-a.y, b.y, re));
                im = fma(a.x, b.y, fma(a.y, b.x, im));
            }
        }
        if (tpo == 1) {
            if (o < outs) out[o] = make_double2(re, im);
            continue;
        }
        part[threadIdx.x] = make_double2(re, im);
        __syncthreads();
        if (piece == 0 && o < outs) {
            double2 acc = part[threadIdx.x];
            for (uint32_t q = 1; q < tpo; ++q) {
                acc.x += part[threadIdx.x + q].x;
                acc.y += part[threadIdx.x + q].y;
            }
            out[o] = acc;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------

// Network::build (network.rs:62-96): edge w leaves ket0(w); each gate numbers
// its outputs next, in wire order; bonds come after every wire edge, by gate
// index.
struct Network {
    std::vector<uint32_t> bra;                 // edge of bra0(w)
    std::vector<std::vector<uint32_t>> gate;   // inputs, then outputs, in the gate's wire order; empty: not unitary
    uint32_t wire_edges = 0;

    wqc_status build(uint32_t n, const wqc_gate* gates, uint32_t count) {
        std::vector<uint32_t> current(n);
        for (uint32_t w = 0; w < n; ++w) current[w] = w;
        uint64_t next = n;
        gate.assign(count, {});
        for (uint32_t i = 0; i < count; ++i) {
            if (!is_unitary(gates[i].kind)) continue;
            std::vector<uint32_t> wires = wires_of(gates[i]);
            std::vector<uint32_t> legs;
            for (uint32_t w : wires) legs.push_back(current[w]);
            for (uint32_t w : wires) {
                current[w] = uint32_t(next);
                legs.push_back(uint32_t(next));
                if (++next > 0xffffffffull) return failx("contraction tree has too many edges");
            }
            gate[i] = legs;
        }
        if (next + count > 0xffffffffull) return failx("contraction tree has too many edges");
        bra = current;
        wire_edges = uint32_t(next);
        return WQC_OK;
    }
};

// apply_in_place (exact.rs:482-560) on a vector over a gate's own wires (in
// the gate's order: wire k is bit k), with the reference's arithmetic: the
// columns of a gate tensor (network.rs:431-445).
void host_apply(std::vector<double2>& d, const wqc_gate& g) {
    auto mul = [](double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); };
    auto add = [](double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); };
    const size_t len = d.size();
    if (g.kind == WQC_GATE_CNOT || g.kind == WQC_GATE_CZ) {
        // the 4x4 product with CNOT's or CZ's entries (gates.rs), summed left to right
        double2 m[16] = {};  // [co][to][ci][ti]
        auto at = [&](int co, int to, int ci, int ti) -> double2& { return m[((co * 2 + to) * 2 + ci) * 2 + ti]; };
        at(0, 0, 0, 0) = make_double2(1, 0);
        at(0, 1, 0, 1) = make_double2(1, 0);
        if (g.kind == WQC_GATE_CNOT) {
            at(1, 0, 1, 1) = make_double2(1, 0);
            at(1, 1, 1, 0) = make_double2(1, 0);
        } else {
            at(1, 0, 1, 0) = make_double2(1, 0);
            at(1, 1, 1, 1) = make_double2(-1, 0);
        }
        const size_t ctrl = 1, tgt = 2;
        for (size_t i = 0; i < len; ++i) {
            if ((i & ctrl) || (i & tgt)) continue;
            const double2 v00 = d[i], v10 = d[i | ctrl], v01 = d[i | tgt], v11 = d[i | ctrl | tgt];
            auto amp = [&](int co, int to) {
                return add(add(add(mul(at(co, to, 0, 0), v00), mul(at(co, to, 1, 0), v10)), mul(at(co, to, 0, 1), v01)),
                           mul(at(co, to, 1, 1), v11));
            };
            const double2 a00 = amp(0, 0), a10 = amp(1, 0), a01 = amp(0, 1), a11 = amp(1, 1);
            d[i] = a00;
            d[i | ctrl] = a10;
            d[i | tgt] = a01;
            d[i | ctrl | tgt] = a11;
        }
    } else if (g.kind == WQC_GATE_CCNOT) {
        for (size_t i = 0; i < len; ++i)
            if ((i & 1) && (i & 2) && !(i & 4)) std::swap(d[i], d[i | 4]);
    } else {
        double2 u[4];
        gate_matrix_2x2(g.kind, g.angle, u);
        for (size_t i = 0; i < len; i += 2) {
            const double2 v0 = d[i], v1 = d[i + 1];
            d[i] = add(mul(u[0], v0), mul(u[1], v1));
            d[i + 1] = add(mul(u[2], v0), mul(u[3], v1));
        }
    }
}

// gate_tensor (network.rs:431-445): entry input | output << m is
// <output|U|input>.
std::vector<double2> gate_tensor(const wqc_gate& g) {
    const size_t m = wires_of(g).size(), dim = size_t(1) << m;
    std::vector<double2> data(dim * dim, make_double2(0, 0));
    for (size_t in = 0; in < dim; ++in) {
        std::vector<double2> col(dim, make_double2(0, 0));
        col[in] = make_double2(1, 0);
        host_apply(col, g);
        for (size_t out = 0; out < dim; ++out) data[in | (out << m)] = col[out];
    }
    return data;
}

// half_tensor (network.rs:371-392): entry input | output << 1 | bond << 2.
std::vector<double2> half_tensor(int half, bool target_is_z) {
    std::vector<double2> out(8);
    for (int index = 0; index < 8; ++index) {
        const int input = index & 1, output = (index >> 1) & 1, bond = index >> 2;
        double value;
        if (half == 0) value = (input == output && output == bond) ? 1.0 : 0.0;
        else if (bond == 0) value = input == output ? 1.0 : 0.0;
        else if (target_is_z) value = input != output ? 0.0 : (input == 1 ? -1.0 : 1.0);
        else value = input != output ? 1.0 : 0.0;
        out[size_t(index)] = make_double2(value, 0.0);
    }
    return out;
}

constexpr uint8_t kWhole = 1, kControl = 2, kTarget = 4, kHalves = kControl | kTarget;

struct Tensor {
    std::vector<uint32_t> legs;
    int buf = -1;
    uint64_t bytes() const { return 16ull << legs.size(); }
};

struct Buffer {
    uint64_t off = 0;  // element offset in its region
    int legs = 0;
    bool leaf = false;  // in the leaf region (never reused)
};

struct Op {
    int kind;  // 0 permute, 1 gemm, 2 small contraction (batched by level)
    int src, dst;          // permute
    PermuteMap map;
    int legs;
    int a, b, c;           // gemm / small: C (m x n) = A (m x k) B (n x k)^T, row-major
    uint64_t m, k, n;
    int level;             // small: 1 + the deepest small input of its segment
    uint32_t lf, ls, rf, rs;  // small: index tables
};

// A contraction this small (result, work and operands) runs in one block of
// a batched launch; the rest reorder and go through cuBLAS.
constexpr uint64_t kSmallResult = 1ull << 14, kSmallWork = 1ull << 16;
constexpr size_t kSmallLegs = 14;

struct NetPlan {
    bool on = false;
    std::vector<Buffer> bufs;
    std::vector<Op> ops;
    std::vector<double2> leaf_data;  // the leaf region's contents
    Placer placer;
    uint64_t permute_bytes = 0;
    double gemm_flops = 0;
    std::vector<uint32_t> tables;       // small contractions' index tables
    std::map<int, int> seg_level;       // buffers made in the open segment of small contractions -> level
    std::vector<int> seg_frees;         // buffers the open segment consumed, released when it closes

    // Small contractions between two large ones form a segment; its
    // launches run level by level, so a range it frees is reused only after
    // the segment.
    void close_segment() {
        for (int id : seg_frees) drop(id);
        seg_frees.clear();
        seg_level.clear();
    }

    int new_leaf(const std::vector<double2>& data, int legs) {
        Buffer b;
        b.leaf = true;
        b.legs = legs;
        b.off = leaf_data.size();
        leaf_data.insert(leaf_data.end(), data.begin(), data.end());
        // keep every leaf 256-byte aligned
        while (leaf_data.size() % (kAlign / 16)) leaf_data.push_back(make_double2(0, 0));
        bufs.push_back(b);
        return int(bufs.size()) - 1;
    }
    int new_tensor(int legs) {
        Buffer b;
        b.legs = legs;
        b.off = placer.alloc(16ull << legs) / 16;
        bufs.push_back(b);
        return int(bufs.size()) - 1;
    }
    void drop(int id) {
        const Buffer& b = bufs[size_t(id)];
        if (!b.leaf) placer.release(b.off * 16, 16ull << b.legs);
    }
};

struct Leaves {
    const Network* net;
    const wqc_gate* gates;
    uint32_t gate_count;
    uint32_t n;
    NetPlan* plan;
    std::vector<char> ket, bra;
    std::vector<uint8_t> gate;

    wqc_status mark(std::vector<char>& used, uint32_t wire) {
        if (wire >= n) return fail_index(wire, n);
        if (used[wire]) return failx("contraction tree reuses a tensor");
        used[wire] = 1;
        return WQC_OK;
    }
    Tensor basis_zero(uint32_t edge) {
        Tensor t;
        t.legs = {edge};
        if (plan->on) t.buf = plan->new_leaf({make_double2(1, 0), make_double2(0, 0)}, 1);
        return t;
    }
    wqc_status take_gate(uint32_t index, uint8_t part) {
        const uint8_t used = gate[index];
        if (used & part) return failx("contraction tree reuses a tensor");
        if (used != 0 && ((used | part) & kWhole)) return failx("contraction tree mixes a gate and its halves");
        gate[index] = uint8_t(used | part);
        return WQC_OK;
    }
    wqc_status whole(uint32_t index, Tensor* out) {
        if (index >= gate_count) return failx("contraction tree gate is missing");
        if (net->gate[index].empty()) return failx("gate " + std::to_string(index) + " is not a contraction leaf");
        if (wqc_status s = take_gate(index, kWhole)) return s;
        out->legs = net->gate[index];
        if (plan->on) out->buf = plan->new_leaf(gate_tensor(gates[index]), int(out->legs.size()));
        return WQC_OK;
    }
    wqc_status half(uint32_t index, int which, Tensor* out) {
        if (index >= gate_count) return failx("contraction tree gate is missing");
        const int kind = gates[index].kind;
        if (kind != WQC_GATE_CNOT && kind != WQC_GATE_CZ) return failx("gate " + std::to_string(index) + " has no halves");
        const std::vector<uint32_t>& legs = net->gate[index];
        if (legs.size() != 4) return failx("gate " + std::to_string(index) + " is not a contraction leaf");
        if (wqc_status s = take_gate(index, which == 0 ? kControl : kTarget)) return s;
        out->legs = {legs[size_t(which)], legs[size_t(2 + which)], net->wire_edges + index};
        if (plan->on) out->buf = plan->new_leaf(half_tensor(which, kind == WQC_GATE_CZ), 3);
        return WQC_OK;
    }
};

struct NetWalker {
    uint32_t n;
    const wqc_gate* gates;
    uint32_t gate_count;
    NetPlan* plan;
    Network net;
    std::map<uint32_t, Tensor> live;
    uint64_t live_bytes = 0;

    // take (network.rs:250-282).
    wqc_status take(const wqc_tree_ref& r, uint32_t index, Leaves& leaves, Tensor* out) {
        switch (r.kind) {
            case WQC_TREE_NODE: {
                if (r.index >= index) return failx("contraction tree tensor is not ready");
                auto it = live.find(r.index);
                if (it == live.end()) return failx("contraction tree reuses a tensor");
                *out = std::move(it->second);
                live.erase(it);
                live_bytes -= out->bytes();
                return WQC_OK;
            }
            case WQC_TREE_KET0:
                if (wqc_status s = leaves.mark(leaves.ket, r.index)) return s;
                *out = leaves.basis_zero(r.index);
                return WQC_OK;
            case WQC_TREE_BRA0:
                if (wqc_status s = leaves.mark(leaves.bra, r.index)) return s;
                *out = leaves.basis_zero(net.bra[r.index]);
                return WQC_OK;
            case WQC_TREE_GATE: return leaves.whole(r.index, out);
            case WQC_TREE_CONTROL: return leaves.half(r.index, 0, out);
            case WQC_TREE_TARGET: return leaves.half(r.index, 1, out);
            case WQC_TREE_LEFT: case WQC_TREE_RIGHT: return failx("contraction tree network has no split");
            default: return failx("unknown tensor reference kind " + std::to_string(r.kind));
        }
    }

    // contract_pair (network.rs:591-664): legs, working bytes, and the device
    // work of the join.
    wqc_status contract_pair(const Tensor& left, const Tensor& right, Tensor* result, uint64_t* working) {
        std::vector<uint32_t> shared, left_free, right_free;
        for (uint32_t l : left.legs)
            if (std::find(right.legs.begin(), right.legs.end(), l) != right.legs.end()) shared.push_back(l);
        auto is_shared = [&](uint32_t l) { return std::find(shared.begin(), shared.end(), l) != shared.end(); };
        for (uint32_t l : left.legs)
            if (!is_shared(l)) left_free.push_back(l);
        for (uint32_t l : right.legs)
            if (!is_shared(l)) right_free.push_back(l);
        std::vector<uint32_t> legs = right_free;
        legs.insert(legs.end(), left_free.begin(), left_free.end());
        if (legs.size() > size_t(kMaxOpenLegs)) return failx("contraction tree tensor exceeds 26 legs");
        std::vector<uint32_t> left_order = shared, right_order = shared;
        left_order.insert(left_order.end(), left_free.begin(), left_free.end());
        right_order.insert(right_order.end(), right_free.begin(), right_free.end());
        uint64_t work = 16ull << legs.size();
        const bool left_moves = left.legs != left_order, right_moves = right.legs != right_order;
        if (left_moves) work = std::max(work, left.bytes());
        if (right_moves) work = std::max(work, right.bytes());
        *working = work;
        result->legs = legs;
        if (!plan->on) return WQC_OK;
        const uint64_t m = 1ull << left_free.size(), k = 1ull << shared.size(), n_ = 1ull << right_free.size();
        if (m * n_ <= kSmallResult && m * n_ * k <= kSmallWork && left.legs.size() <= kSmallLegs &&
            right.legs.size() <= kSmallLegs) {
            // One block of a batched launch reads both operands in place.
            auto table = [&](const std::vector<uint32_t>& of, const std::vector<uint32_t>& legs_) {
                const uint32_t at = uint32_t(plan->tables.size());
                for (uint64_t x = 0; x < (1ull << legs_.size()); ++x) {
                    uint32_t off = 0;
                    for (size_t b = 0; b < legs_.size(); ++b)
                        if ((x >> b) & 1)
                            off |= 1u << (std::find(of.begin(), of.end(), legs_[b]) - of.begin());
                    plan->tables.push_back(off);
                }
                return at;
            };
            Op op{};
            op.kind = 2;
            op.a = left.buf;
            op.b = right.buf;
            result->buf = plan->new_tensor(int(legs.size()));
            op.c = result->buf;
            op.m = m;
            op.k = k;
            op.n = n_;
            op.legs = int(legs.size());
            op.lf = table(left.legs, left_free);
            op.ls = table(left.legs, shared);
            op.rf = table(right.legs, right_free);
            op.rs = table(right.legs, shared);
            int lv = 0;
            for (int in : {left.buf, right.buf}) {
                auto it = plan->seg_level.find(in);
                if (it != plan->seg_level.end()) lv = std::max(lv, it->second);
            }
            op.level = lv + 1;
            plan->seg_level[result->buf] = op.level;
            plan->ops.push_back(op);
            plan->gemm_flops += 8.0 * double(m) * double(n_) * double(k);
            plan->seg_frees.push_back(left.buf);
            plan->seg_frees.push_back(right.buf);
            return WQC_OK;
        }
        plan->close_segment();
        // Device work: reorder what is out of order, then C = A B^T.
        auto reorder = [&](const Tensor& t, const std::vector<uint32_t>& to) {
            const int L = int(t.legs.size());
            const int dst = plan->new_tensor(L);
            Op op{};
            op.kind = 0;
            op.src = t.buf;
            op.dst = dst;
            op.legs = L;
            for (int b = 0; b < L; ++b)
                op.map.src[b] = uint8_t(std::find(t.legs.begin(), t.legs.end(), to[size_t(b)]) - t.legs.begin());
            plan->ops.push_back(op);
            plan->permute_bytes += 2 * (16ull << L);
            return dst;
        };
        const int a = left_moves ? reorder(left, left_order) : left.buf;
        const int b = right_moves ? reorder(right, right_order) : right.buf;
        result->buf = plan->new_tensor(int(legs.size()));
        Op op{};
        op.kind = 1;
        op.a = a;
        op.b = b;
        op.c = result->buf;
        op.m = 1ull << left_free.size();
        op.k = 1ull << shared.size();
        op.n = 1ull << right_free.size();
        op.legs = int(legs.size());
        plan->ops.push_back(op);
        plan->gemm_flops += 8.0 * double(op.m) * double(op.n) * double(op.k);
        if (left_moves) plan->drop(a);
        if (right_moves) plan->drop(b);
        plan->drop(left.buf);
        plan->drop(right.buf);
        return WQC_OK;
    }

    // walk (network.rs:183-248).
    wqc_status run(const wqc_tree* tree, const std::atomic<int>* cancel, uint64_t* peak_out, int* root_buf) {
        if (tree->kind != 1) return failx("contraction tree is not a network");
        if (wqc_status s = net.build(n, gates, gate_count)) return s;
        Leaves leaves{&net, gates, gate_count, n, plan, std::vector<char>(n, 0), std::vector<char>(n, 0),
                      std::vector<uint8_t>(gate_count, 0)};
        uint64_t peak = 0;
        for (uint32_t index = 0; index < tree->node_count; ++index) {
            if (cancel && cancel->load()) return record_error(WQC_ERR_CANCELLED, "computation cancelled: the client has gone");
            const wqc_tree_node& node = tree->nodes[index];
            if (node.op != 0) return failx("contraction tree mixes sweep steps and network contractions");
            Tensor left, right;
            if (wqc_status s = take(node.left, index, leaves, &left)) return s;
            if (wqc_status s = take(node.right, index, leaves, &right)) return s;
            const uint64_t inputs = left.bytes() + right.bytes();
            Tensor result;
            uint64_t working = 0;
            if (wqc_status s = contract_pair(left, right, &result, &working)) return s;
            const uint64_t during = live_bytes + inputs + working;
            if (during > kMaxPeakBytes) return failx("contraction tree peak exceeds 1 GiB");
            peak = std::max(peak, during);
            live_bytes += result.bytes();
            live.emplace(index, std::move(result));
        }
        bool out = false;
        for (uint32_t w = 0; w < n; ++w) out |= !leaves.ket[w] || !leaves.bra[w];
        for (uint32_t i = 0; i < gate_count; ++i)
            if (!net.gate[i].empty() && leaves.gate[i] != kWhole && leaves.gate[i] != kHalves) out = true;
        if (out) return failx("contraction tree leaves a leaf out");
        if (live.size() != 1 || !live.begin()->second.legs.empty())
            return failx("contraction tree does not end in one scalar");
        *peak_out = peak;
        if (root_buf) *root_buf = live.begin()->second.buf;
        return WQC_OK;
    }
};

// declared_peak (network.rs:171-181).
wqc_status net_declared_peak(const wqc_tree* tree, uint64_t* out) {
    if (!tree->has_peak) return failx("contraction tree requires a peak");
    if (tree->peak_bytes > kMaxPeakBytes) return failx("contraction tree peak exceeds 1 GiB");
    *out = tree->peak_bytes;
    return WQC_OK;
}

}  // namespace

struct wqc_network {
    wqc_cuda_ctx* ctx = nullptr;
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    cublasHandle_t blas = nullptr;
    double2* arena = nullptr;
    uint64_t arena_bytes = 0;
    unsigned char* table = nullptr;  // small contractions' index tables and jobs
    uint64_t table_bytes = 0;
    double2* host_root = nullptr;  // pinned
    unsigned char* staging = nullptr;  // pinned leaf upload
    uint64_t staging_bytes = 0;
    std::vector<cudaEvent_t> events;
    std::atomic<int> cancel{0};
    wqc_network_stats stats{};
};

namespace {

wqc_status ncuda(const char* what, cudaError_t e) {
    return record_error(WQC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

cudaEvent_t net_event(wqc_network* net, size_t i) {
    while (net->events.size() <= i) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        net->events.push_back(e);
    }
    return net->events[i];
}

}  // namespace

extern "C" {

wqc_status wqc_network_create(wqc_cuda_ctx* ctx, wqc_network** out) {
    if (!ctx || !out) return failx("null argument");
    auto* net = new wqc_network();
    net->ctx = ctx;
    net->device = context_device(ctx);
    net->sm_count = context_sm_count(ctx);
    cudaError_t e = cudaSetDevice(net->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&net->host_root), sizeof(double2));
    if (e != cudaSuccess) {
        wqc_network_destroy(net);
        return ncuda("network executor setup", e);
    }
    if (cublasCreate(&net->blas) != CUBLAS_STATUS_SUCCESS || cublasSetStream(net->blas, net->stream) != CUBLAS_STATUS_SUCCESS) {
        wqc_network_destroy(net);
        return record_error(WQC_ERR_CUDA, "cublasCreate failed");
    }
    *out = net;
    return WQC_OK;
}

void wqc_network_destroy(wqc_network* net) {
    if (!net) return;
    cudaSetDevice(net->device);
    if (net->stream) cudaStreamSynchronize(net->stream);
    if (net->blas) cublasDestroy(net->blas);
    for (cudaEvent_t e : net->events) cudaEventDestroy(e);
    if (net->arena) cudaFree(net->arena);
    if (net->table) cudaFree(net->table);
    if (net->host_root) cudaFreeHost(net->host_root);
    if (net->staging) cudaFreeHost(net->staging);
    if (net->stream) cudaStreamDestroy(net->stream);
    delete net;
}

void wqc_network_cancel(wqc_network* net) {
    if (net) net->cancel.store(1);
}

wqc_status wqc_network_last_stats(wqc_network* net, wqc_network_stats* out) {
    if (!net || !out) return failx("null argument");
    *out = net->stats;
    return WQC_OK;
}

wqc_status wqc_network_measured_peak(uint32_t n, const wqc_gate* gates, uint32_t gate_count, const wqc_tree* tree,
                                     uint64_t* peak) {
    if (wqc_status s = check_tree(tree)) return s;
    if (!peak) return failx("null argument");
    if (tree->kind != 1) return failx("contraction tree is not a network");
    if (wqc_status s = check_shape(n, gates, gate_count, tree, nullptr, 0)) return s;
    NetPlan plan;
    NetWalker w{n, gates, gate_count, &plan, {}, {}, 0};
    return w.run(tree, nullptr, peak, nullptr);
}

wqc_status wqc_network_validate(uint32_t n, const wqc_gate* gates, uint32_t gate_count, const wqc_tree* tree,
                                const uint64_t* mps_order, uint32_t mps_len) {
    if (wqc_status s = check_tree(tree)) return s;
    uint64_t declared = 0, peak = 0;
    if (wqc_status s = net_declared_peak(tree, &declared)) return s;
    if (tree->kind != 1) return failx("contraction tree is not a network");
    if (wqc_status s = check_shape(n, gates, gate_count, tree, mps_order, mps_len)) return s;
    NetPlan plan;
    NetWalker w{n, gates, gate_count, &plan, {}, {}, 0};
    if (wqc_status s = w.run(tree, nullptr, &peak, nullptr)) return s;
    if (declared != peak) return failx("contraction tree peak does not match");
    return WQC_OK;
}

wqc_status wqc_network_contract(wqc_network* net, uint32_t n, const wqc_gate* gates, uint32_t gate_count,
                                const wqc_tree* tree, const uint64_t* mps_order, uint32_t mps_len, double out[2]) {
    if (!net) return failx("null executor");
    if (wqc_status s = check_tree(tree)) return s;
    if (!out) return failx("null argument");
    net->stats = wqc_network_stats{};
    uint64_t declared = 0, peak = 0;
    if (wqc_status s = net_declared_peak(tree, &declared)) return s;
    if (tree->kind != 1) return failx("contraction tree is not a network");
    if (wqc_status s = check_shape(n, gates, gate_count, tree, mps_order, mps_len)) return s;
    NetPlan plan;
    plan.on = true;
    NetWalker w{n, gates, gate_count, &plan, {}, {}, 0};
    int root = -1;
    if (net->cancel.exchange(0)) return record_error(WQC_ERR_CANCELLED, "computation cancelled: the client has gone");
    if (wqc_status s = w.run(tree, &net->cancel, &peak, &root)) {
        net->cancel.store(0);
        return s;
    }
    if (declared != peak) return failx("contraction tree peak does not match");

    const uint64_t leaf_bytes = (plan.leaf_data.size() * 16 + kAlign - 1) / kAlign * kAlign;
    const uint64_t need = std::max<uint64_t>(leaf_bytes + plan.placer.top, kAlign);
    auto offset_of = [&](int id) {
        const Buffer& B = plan.bufs[size_t(id)];
        return (B.leaf ? 0 : leaf_bytes / 16) + B.off;
    };
    // The small contractions' launches: each run of them between two large
    // contractions, level by level (`batches`: first job, job count, and the
    // op index the run ends before).
    std::vector<SmallJob> jobs;
    struct Batch {
        uint32_t first, count;
        size_t before;
    };
    std::vector<Batch> batches;
    for (size_t i = 0; i < plan.ops.size();) {
        if (plan.ops[i].kind != 2) {
            ++i;
            continue;
        }
        size_t j = i;
        int top = 0;
        while (j < plan.ops.size() && plan.ops[j].kind == 2) top = std::max(top, plan.ops[j++].level);
        for (int lv = 1; lv <= top; ++lv) {
            Batch b{uint32_t(jobs.size()), 0, j};
            for (size_t q = i; q < j; ++q) {
                const Op& op = plan.ops[q];
                if (op.level != lv) continue;
                jobs.push_back(SmallJob{offset_of(op.a), offset_of(op.b), offset_of(op.c), uint32_t(op.m),
                                        uint32_t(op.n), uint32_t(op.k), op.lf, op.ls, op.rf, op.rs});
                ++b.count;
            }
            if (b.count) batches.push_back(b);
        }
        i = j;
    }
    const uint64_t tab_bytes = (plan.tables.size() * 4 + kAlign - 1) / kAlign * kAlign;
    const uint64_t jobs_bytes = (jobs.size() * sizeof(SmallJob) + kAlign - 1) / kAlign * kAlign;
    const uint64_t stage_bytes = std::max<uint64_t>(leaf_bytes + tab_bytes + jobs_bytes, kAlign);
    if (cudaError_t e = cudaSetDevice(net->device)) return ncuda("cudaSetDevice", e);
    if (net->arena_bytes < need) {
        if (net->arena) cudaFree(net->arena);
        net->arena = nullptr;
        net->arena_bytes = 0;
        if (cudaMalloc(reinterpret_cast<void**>(&net->arena), need) != cudaSuccess) {
            cudaGetLastError();
            size_t fr = 0, tot = 0;
            cudaMemGetInfo(&fr, &tot);
            return record_oom(need, fr);
        }
        net->arena_bytes = need;
    }
    if (net->table_bytes < tab_bytes + jobs_bytes) {
        if (net->table) cudaFree(net->table);
        net->table = nullptr;
        net->table_bytes = 0;
        if (cudaMalloc(reinterpret_cast<void**>(&net->table), tab_bytes + jobs_bytes) != cudaSuccess) {
            cudaGetLastError();
            size_t fr = 0, tot = 0;
            cudaMemGetInfo(&fr, &tot);
            return record_oom(tab_bytes + jobs_bytes, fr);
        }
        net->table_bytes = tab_bytes + jobs_bytes;
    }
    if (net->staging_bytes < stage_bytes) {
        if (net->staging) cudaFreeHost(net->staging);
        net->staging = nullptr;
        net->staging_bytes = 0;
        if (cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&net->staging), stage_bytes)) {
            cudaGetLastError();
            return ncuda("cudaMallocHost(network leaves)", e);
        }
        net->staging_bytes = stage_bytes;
    }
    cudaStream_t st = net->stream;
    double2* leaves = net->arena;
    double2* tensors = net->arena + leaf_bytes / 16;
    auto at = [&](int id) {
        const Buffer& B = plan.bufs[size_t(id)];
        return (B.leaf ? leaves : tensors) + B.off;
    };
    auto bail = [&](wqc_status s) {
        cudaStreamSynchronize(st);
        return s;
    };
    size_t ev = 0;
    cudaEvent_t e0 = net_event(net, ev++), e1 = net_event(net, ev++);
    if (!e0 || !e1) return record_error(WQC_ERR_CUDA, "cudaEventCreate failed");
    cudaEventRecord(e0, st);
    if (!plan.leaf_data.empty()) {
        std::memcpy(net->staging, plan.leaf_data.data(), plan.leaf_data.size() * 16);
        if (cudaError_t e = cudaMemcpyAsync(leaves, net->staging, plan.leaf_data.size() * 16, cudaMemcpyHostToDevice, st))
            return bail(ncuda("cudaMemcpyAsync(network leaves)", e));
    }
    const uint32_t* d_tab = reinterpret_cast<const uint32_t*>(net->table);
    const SmallJob* d_jobs = reinterpret_cast<const SmallJob*>(net->table + tab_bytes);
    if (!jobs.empty()) {
        unsigned char* h = net->staging + leaf_bytes;
        std::memcpy(h, plan.tables.data(), plan.tables.size() * 4);
        std::memcpy(h + tab_bytes, jobs.data(), jobs.size() * sizeof(SmallJob));
        if (cudaError_t e = cudaMemcpyAsync(net->table, h, tab_bytes + jobs.size() * sizeof(SmallJob),
                                            cudaMemcpyHostToDevice, st))
            return bail(ncuda("cudaMemcpyAsync(network jobs)", e));
    }
    size_t next_batch = 0;
    uint32_t small_launches = 0;
    auto run_batches = [&](size_t before) -> wqc_status {
        while (next_batch < batches.size() && batches[next_batch].before <= before) {
            const Batch& b = batches[next_batch++];
            network_small_kernel<<<b.count, kSmallThreads, 0, st>>>(net->arena, d_jobs + b.first, d_tab);
            if (cudaError_t e = cudaGetLastError()) return ncuda("network small-contraction launch", e);
            ++small_launches;
        }
        return WQC_OK;
    };
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> timed;
    uint32_t permutes = 0, gemms = 0;
    const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
    for (size_t oi = 0; oi < plan.ops.size(); ++oi) {
        const Op& op = plan.ops[oi];
        if (op.kind == 2) continue;  // launched in batches
        if (wqc_status s = run_batches(oi)) return bail(s);
        if (net->cancel.exchange(0)) return bail(record_error(WQC_ERR_CANCELLED, "computation cancelled: the client has gone"));
        const bool time_it = true;  // the large contractions are few: each is timed
        cudaEvent_t a = nullptr, b = nullptr;
        if (time_it) {
            a = net_event(net, ev++);
            b = net_event(net, ev++);
            if (!a || !b) return bail(record_error(WQC_ERR_CUDA, "cudaEventCreate failed"));
            cudaEventRecord(a, st);
        }
        if (op.kind == 0) {
            const uint64_t total = 1ull << op.legs;
            const uint32_t grid = uint32_t(std::min<uint64_t>((total + kPermuteThreads - 1) / kPermuteThreads,
                                                              uint64_t(net->sm_count) * 8));
            network_permute_kernel<<<grid, kPermuteThreads, 0, st>>>(at(op.dst), at(op.src), op.map, op.legs);
            if (cudaError_t e = cudaGetLastError()) return bail(ncuda("network permute launch", e));
            ++permutes;
        } else {
            // Row-major C (m x n) = A (m x k) B^T: column-major C^T = B^T' A with
            // B read transposed (cublas: op T on a k x n matrix) and A as k x m.
            const cublasStatus_t s = cublasZgemm(
                net->blas, CUBLAS_OP_T, CUBLAS_OP_N, int(op.n), int(op.m), int(op.k), &one,
                reinterpret_cast<const cuDoubleComplex*>(at(op.b)), int(op.k),
                reinterpret_cast<const cuDoubleComplex*>(at(op.a)), int(op.k), &zero,
                reinterpret_cast<cuDoubleComplex*>(at(op.c)), int(op.n));
            if (s != CUBLAS_STATUS_SUCCESS) return bail(record_error(WQC_ERR_CUDA, "cublasZgemm failed: status " + std::to_string(int(s))));
            ++gemms;
        }
        if (time_it) {
            cudaEventRecord(b, st);
            timed.push_back({op.kind, {a, b}});
        }
    }
    if (wqc_status s = run_batches(plan.ops.size())) return bail(s);
    if (cudaError_t e = cudaMemcpyAsync(net->host_root, at(root), sizeof(double2), cudaMemcpyDeviceToHost, st))
        return bail(ncuda("cudaMemcpyAsync(network root)", e));
    cudaEventRecord(e1, st);
    if (cudaError_t e = cudaStreamSynchronize(st)) return ncuda("network contraction", e);
    out[0] = net->host_root->x;
    out[1] = net->host_root->y;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    net->stats.device_ms = ms;
    for (auto& t : timed) {
        float x = 0.f;
        cudaEventElapsedTime(&x, t.second.first, t.second.second);
        (t.first == 0 ? net->stats.permute_ms : net->stats.gemm_ms) += x;
    }
    net->stats.nodes = tree->node_count;
    net->stats.permutes = permutes;
    net->stats.gemms = gemms;
    net->stats.launches = permutes + gemms + small_launches;
    net->stats.small = uint32_t(jobs.size());
    net->stats.permute_bytes = plan.permute_bytes;
    net->stats.gemm_flops = plan.gemm_flops;
    net->stats.arena_bytes = net->arena_bytes;
    return WQC_OK;
}

}  // extern "C"
