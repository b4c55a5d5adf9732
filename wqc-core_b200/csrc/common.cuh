// Shared device types and helpers for the cuda MPS backend (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/wqc_types.h"

namespace wqc {

// ---------------------------------------------------------------------------
// Complex FP64 as double2 (x = re, y = im).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ double2 cmake(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__host__ __device__ __forceinline__ double2 cconjmul(double2 a, double2 b) {
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double cnorm2(double2 a) { return a.x * a.x + a.y * a.y; }
// acc += a * b
__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}
// acc += conj(a) * b
__device__ __forceinline__ void cfma_conj(double2& acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(-a.y, b.x, acc.y);
}

// ---------------------------------------------------------------------------
// Constants of the reference truncation rule (src/tn/svd_guard.rs, mps.rs).
// ---------------------------------------------------------------------------
constexpr double kSingularCutoff = 1e-12;  // svd_guard.rs:12
constexpr double kChiRelGap = 1e-3;        // svd_guard.rs:15
constexpr double kCutoffAbsBand = 1e-10;   // svd_guard.rs:18
constexpr double kDustRel = 1e-14;         // svd_guard.rs:92-97
constexpr double kRsvdZero = 1e-14;        // mps.rs:1022-1026 (cutoff * 1e-2)
constexpr int kRsvdMinSide = 160;          // mps.rs:794
constexpr int kRsvdOversample = 16;        // mps.rs:795

// Device status bits (sticky, read by the host after a synchronisation).
enum : int {
    kStatusOk = 0,
    kStatusTruncationRejected = 1 << 0,  // mps.rs:1137-1144
    kStatusJacobiNoConvergence = 1 << 1,
    kStatusBadShape = 1 << 2,
    kStatusNonFinite = 1 << 3,
    kStatusCancelled = 1 << 4,
    kStatusSvdCheck = 1 << 5,  // sum sigma^2 != ||X||_F^2 (svd_guard.rs:234-255)
    kStatusDeviceTimeout = 1 << 6,  // a bounded wait on an mbarrier gave up
};

// ---------------------------------------------------------------------------
// Split pipeline descriptors.  One SplitJob per two-site split in a wave; the
// host writes the static part, kernels write SplitState.
// ---------------------------------------------------------------------------
struct SplitJob {
    int p;            // left site, right site is p + 1
    int seq;          // index of this split in program order (record slot)
    int slot;         // workspace slot
    int reject;       // reject_truncation (time-split halves)
    int exact_only;   // split rule: exact SVD on every split, no range finder
    int chi_max;      // max bond dimension of the state (or batch slice) the split belongs to
    double2 u[16];    // effective 4x4 on theta: u[(so*2+to)*4 + si*2+ti]
};

struct SplitState {
    int dl, dr, k;       // left bond of p, right bond of p+1, inner bond
    int rows, cols, ell; // theta is rows x cols, range-finder width ell
    int use_rsvd;        // range finder attempted
    int need_exact;      // exact SVD of theta required
    int path;            // enum wqc_split_path
    int chi;             // kept bond
    int final_kind;      // 0: exact on theta, 1: rsvd accepted
    int w_rows_of_src;   // exact Jacobi: 1 when W = theta^H (rows < cols)
    int skip;            // cancelled before this wave: nothing is computed or written
    double discarded;
    double fro2;         // ||X||_F^2 seen by the precision form's first Jacobi phase
};

// Per-slot workspace pointers (device memory carved from one arena).
struct SlotBuffers {
    double2* theta;  // rows x cols, row-major
    double2* omega;  // cols x ell, row-major
    double2* y0;     // rows x ell, row-major
    double2* zr;     // cols x ell, row-major
    double2* y;      // rows x ell, column-major (QR works in place)
    double2* q;      // rows x ell, column-major
    double2* b;      // ell x cols, row-major
    double2* w;      // Jacobi output W, M x N column-major
    double2* z;      // Jacobi output Z, N x N column-major
    double* sigma;   // N
    int* perm;       // N: sorted position -> column
    double2* tau;    // ell Householder scalars
    void* gs;        // staged Jacobi workspace (padded W and Z columns), chi_max > 128 only
};

// One Jacobi SVD task: decompose X where column j of the tall working matrix
// W (M x N, M >= N) is column j of src (rows_of_src = 0, M = src rows) or the
// conjugate of row j of src (rows_of_src = 1, M = src cols).  src is
// row-major with leading dimension ld.
struct SvdTask {
    const double2* src;
    int src_rows, src_cols, ld;
    int rows_of_src;
    int active;
    double2* w_out;  // M x N column-major
    double2* z_out;  // N x N column-major
    double* sigma;   // N
};

struct DeviceMps {
    double2** site;  // n pointers, each of capacity chi_cap * 2 * chi_cap
    int* dl;         // left bond of each site
    int* dr;         // right bond of each site
    int n;
    int chi_max;
    int* status;          // sticky status bits
    const int* cancel;    // host-mapped cancel word (src/cancel.rs analogue)
};

}  // namespace wqc
