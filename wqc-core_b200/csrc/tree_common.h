// Host-side pieces shared by the two tree executors (exact.cu, network.cu):
// the reference's shape checks of a ContractionTree and the arena placement
// of its tensors.  Host code only.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <iterator>
#include <map>
#include <string>
#include <vector>

#include "../../include/wqc_cuda.h"

namespace wqc {
wqc_status record_error(wqc_status code, const std::string& msg);  // executor.cu
wqc_status record_oom(uint64_t required, uint64_t available);
wqc_status check_circuit_gate(int n, const wqc_gate& g);
void gate_matrix_2x2(int kind, double theta, double2 out[4]);
int context_device(const wqc_cuda_ctx* ctx);
int context_sm_count(const wqc_cuda_ctx* ctx);

namespace tree {

constexpr int kMaxOpenLegs = 26;                // exact.rs:25
constexpr uint64_t kMaxPeakBytes = 1ull << 30;  // exact.rs:27
constexpr uint64_t kAlign = 256;                // arena placement granularity (bytes)

inline wqc_status failx(const std::string& msg) { return record_error(WQC_ERR_INVALID, msg); }
inline wqc_status fail_index(uint64_t index, uint64_t limit) {
    return record_error(WQC_ERR_QUBIT_OUT_OF_RANGE, "Qubit index " + std::to_string(index) +
                                                        " out of bounds (limit: " + std::to_string(limit) + ")");
}

inline bool is_unitary(int kind) { return kind >= WQC_GATE_H && kind <= WQC_GATE_CCNOT; }

inline std::vector<uint32_t> wires_of(const wqc_gate& g) {
    switch (g.kind) {
        case WQC_GATE_CNOT: case WQC_GATE_CZ: return {uint32_t(g.q0), uint32_t(g.q1)};
        case WQC_GATE_CCNOT: return {uint32_t(g.q0), uint32_t(g.q1), uint32_t(g.q2)};
        default: return {uint32_t(g.q0)};
    }
}

// canonicalize_site_order (src/tn/tree.rs:442-457) with validate_site_order
// (src/tn/site_order.rs:7-31): an empty or identity order is "no order".
inline wqc_status canonical_empty(uint32_t n, const uint64_t* order, uint32_t len, bool* empty) {
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
inline wqc_status check_shape(uint32_t n, const wqc_gate* gates, uint32_t gate_count, const wqc_tree* tree,
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

inline wqc_status check_tree(const wqc_tree* tree) {
    if (!tree) return failx("null contraction tree");
    if (tree->node_count && !tree->nodes) return failx("null contraction tree nodes");
    return WQC_OK;
}

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

}  // namespace tree
}  // namespace wqc
