/* Plain-data types shared by the cuda MPS backend's C ABI (wqc_cuda.h) and the
 * FP64 CPU oracle used by the tests.  No CUDA or torch types appear here.
 *
 * Gate encoding mirrors the reference's `Gate` enum (src/engine.rs, serde tag
 * "type"): one record per gate, qubit operands in declaration order.
 */
#ifndef WQC_TYPES_H
#define WQC_TYPES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Gate kinds, in the order of the reference enum (src/engine.rs). */
enum wqc_gate_kind {
    WQC_GATE_H = 0,
    WQC_GATE_X = 1,
    WQC_GATE_Y = 2,
    WQC_GATE_Z = 3,
    WQC_GATE_S = 4,
    WQC_GATE_T = 5,
    WQC_GATE_RX = 6,
    WQC_GATE_RY = 7,
    WQC_GATE_RZ = 8,
    WQC_GATE_CNOT = 9,     /* q0 = control, q1 = target */
    WQC_GATE_CZ = 10,      /* q0 = control, q1 = target */
    WQC_GATE_CCNOT = 11,   /* q0 = control 1, q1 = control 2, q2 = target */
    WQC_GATE_MEASURE = 12, /* no-op for the MPS executor (mps.rs:294) */
    WQC_GATE_RESET = 13,   /* no-op for the MPS executor */
    WQC_GATE_IF = 14       /* no-op for the MPS executor */
};

typedef struct wqc_gate {
    int32_t kind;
    int32_t q0, q1, q2;
    double angle; /* RX/RY/RZ only */
} wqc_gate;

/* How a two-site split was cut.  The reference chooses between an exact SVD
 * and a seeded randomized SVD (src/tn/mps.rs:937-981). */
enum wqc_split_path {
    WQC_SPLIT_EXACT = 0,         /* exact SVD, range finder not attempted */
    WQC_SPLIT_RSVD = 1,          /* range finder accepted */
    WQC_SPLIT_RSVD_FALLBACK = 2  /* range finder rejected, exact SVD used */
};

/* One record per two-site split (merge + 4x4 gate + SVD + truncation), in the
 * order the reference would perform them.  The discarded weight is the sum of
 * squared singular values past the kept bond: over the exact SVD's values, or
 * over the projected matrix's values when the range finder is accepted.  The
 * reference computes no discarded weight; this field is an addition. */
typedef struct wqc_split_info {
    int32_t left_site;
    int32_t rows;   /* 2 * left bond */
    int32_t cols;   /* 2 * right bond */
    int32_t ell;    /* range-finder width min(chi_max + 16, rows, cols) */
    int32_t path;   /* enum wqc_split_path */
    int32_t chi;    /* kept bond after the split */
    double discarded_weight;
} wqc_split_info;

#ifdef __cplusplus
}
#endif

#endif /* WQC_TYPES_H */
