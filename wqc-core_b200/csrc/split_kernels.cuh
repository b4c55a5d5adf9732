// Kernel entry points of the two-site split pipeline and the site kernels.
#pragma once

#include "common.cuh"

namespace wqc {

enum { kStageY0 = 0, kStageZ = 1, kStageY = 2, kStageB = 3 };
// Jacobi / finalize modes: the range finder's B^H; theta of a split that takes
// the exact path from the start; theta of a range-finder split that fell back.
enum { kJacobiRsvd = 0, kJacobiExact = 1, kJacobiFallback = 2 };
// Threads of the cluster Jacobi: one warp per column pair of a block per step.
// The variant for columns of at most kJacobiRegMaxRows rows keeps each
// warp's top column in registers through a block step and is limited to 12
// warps (170 registers per thread); the other variant, like the staged
// Jacobi, takes up to 16 warps.
constexpr int kJacobiThreads = 512;
constexpr int kJacobiRegThreads = 384;
constexpr int kJacobiRegMaxRows = 256;
constexpr int kJacobiStagedThreads = 512;
inline int jacobi_max_warps(int M) { return (M <= kJacobiRegMaxRows ? kJacobiRegThreads : kJacobiThreads) / 32; }

__global__ void prepare_kernel(const SplitJob* jobs, SplitState* st, int njobs, DeviceMps mps);
__global__ void merge_gate_kernel(const SplitJob* jobs, const SplitState* st, const SlotBuffers* slots,
                                  DeviceMps mps);
__global__ void omega_kernel(const SplitJob* jobs, const SplitState* st, const SlotBuffers* slots);
__global__ void rsvd_gemm_kernel(const SplitJob* jobs, const SplitState* st, const SlotBuffers* slots, int stage);
__global__ void householder_qr_kernel(const SplitJob* jobs, const SplitState* st, const SlotBuffers* slots);
constexpr int kQrClusterThreads = 256;
constexpr int kQrRowsPerThread = 8;  // rows of one reflector each thread holds: Y of at most 2048 rows
// The cluster Householder QR (columns in shared memory, or with global_cols
// in the slot's Y and Q buffers), reached through these host functions.
const void* qr_cluster(bool global_cols);
cudaError_t launch_qr_cluster(bool global_cols, const cudaLaunchConfig_t& cfg, const SplitJob* jobs,
                              const SplitState* st, const SlotBuffers* slots);
// Shared memory of the cluster QR for an m x n Y on a cluster of C CTAs.
inline size_t qr_cluster_smem_bytes(int m, int n, int C, bool global_cols = false) {
    const int cpc = (n + C - 1) / C;
    return ((global_cols ? size_t(0) : size_t(2) * cpc * m) + size_t(3) * m + cpc) * sizeof(double2);
}
// The cluster Jacobi SVD kernel (a template over the column type: complex128
// in the plain form, complex64 in the precision form), reached from other
// files through these host functions.
const void* jacobi_kernel(bool fp32, bool reg);
// Phases of a Jacobi SVD: the plain one; the precision form's first phase
// (complex64 columns carrying W = X V and the accumulated V, written out as
// FP64 for the finish); and its finishing phase (FP64 sweeps that start from
// X V, formed in FP64 by precond_gemm_kernel).
enum { kPhasePlain = 0, kPhaseFp32V = 1, kPhaseFinish = 2 };
cudaError_t launch_jacobi(bool fp32, bool reg, const cudaLaunchConfig_t& cfg, const SplitJob* jobs, SplitState* st,
                          const SlotBuffers* slots, const int* idx, int mode, int phase, int max_sweeps, int* status,
                          unsigned long long* counters);
// The staged variant for working matrices beyond a cluster's shared memory:
// columns in the slot's `gs` workspace, blocks of b columns (b even).
const void* jacobi_staged(bool fp32);
cudaError_t launch_jacobi_staged(bool fp32, const cudaLaunchConfig_t& cfg, const SplitJob* jobs, SplitState* st,
                                 const SlotBuffers* slots, const int* idx, int mode, int phase, int max_sweeps, int b,
                                 int* status, unsigned long long* counters);
// The precision form's FP64 products between its two Jacobi phases, for the
// jobs active in `mode`, in stage order: G = V^H V and V <- V (3 I - G) / 2
// twice (Newton-Schulz: V^H V - I goes from ~1e-6 after the complex64
// rotations to ~1e-12, then to FP64 rounding), then X V into the slot's W
// buffer, X dust-zeroed as the first phase loaded it.
enum { kPrecondGram1 = 0, kPrecondStep1, kPrecondGram2, kPrecondStep2, kPrecondXV, kPrecondStages };
__global__ void precond_gemm_kernel(const SplitJob* jobs, const SplitState* st, const SlotBuffers* slots, int mode,
                                    int stage);
// Shape of the staged Jacobi for an M x N working matrix on a cluster of C
// CTAs: the block width b <= 16 whose two blocks fit `smem_limit` and whose
// sweep is shortest, counted in dependent rotation rounds: (2K-1) steps of
// ceil(K / C) block pairs per CTA, b rounds each, K = ceil(N / 2b) pairs.
// 0 if none fits.  Also returns the shared memory of that choice.
inline int jacobi_staged_b(int M, int N, size_t elem, size_t smem_limit, size_t* smem, int C = 16) {
    int best = 0;
    long best_rounds = 0;
    size_t best_bytes = 0;
    for (int b = 2; b <= 16; ++b) {
        const int K = (N + 2 * b - 1) / (2 * b);
        const size_t len = size_t(M);
        const size_t bytes = size_t(2) * b * len * elem;
        if (bytes > smem_limit) continue;
        const long rounds = long(2 * K - 1) * ((K + C - 1) / C) * b;
        if (!best || rounds < best_rounds) {
            best = b;
            best_rounds = rounds;
            best_bytes = bytes;
        }
    }
    if (best && smem) *smem = best_bytes;
    return best;
}
// Elements (double2) of the `gs` workspace for two-site matrices up to R x R.
inline size_t jacobi_staged_elems(int R) { return size_t(R + 32) * size_t(R); }
// Probe-vector factorisation check of every active Jacobi task (grid: jobs x 2).
__global__ void svd_probe_kernel(const SplitJob* jobs, const SplitState* st, const SlotBuffers* slots, int mode,
                                 int fp32, int* status);
// noise_rel: singular values below noise_rel * (largest) count as zero (0 in
// the plain form; the precision form's FP32 rounding level).
__global__ void finalize_kernel(const SplitJob* jobs, SplitState* st, const SlotBuffers* slots, int mode,
                                int chi_max, double noise_rel, wqc_split_info* records, int* status);
enum { kRecoverBW = 0, kRecoverQT = 1, kRecoverExact = 2 };
__global__ void recover_gemm_kernel(const SplitJob* jobs, const SplitState* st, const SlotBuffers* slots,
                                    DeviceMps mps, int stage);
__global__ void absorb_kernel(const SplitJob* jobs, const SplitState* st, const SlotBuffers* slots,
                              DeviceMps mps);

// Site kernels (site_kernels.cu).
struct OneQubitOp {
    int site;
    int first;  // first gate in the 2x2 array
    int count;  // gates applied in order
};
__global__ void apply_1q_kernel(const OneQubitOp* ops, const double2* mats, DeviceMps mps);
__global__ void amplitude_zero_kernel(DeviceMps mps, const int* seg, double2* out);
__global__ void reset_sites_kernel(DeviceMps mps);
__global__ void site_envs_kernel(DeviceMps mps, double2* envL, double2* envR, int lfrom, int lto, int rfrom, int rto,
                                 const int* targets, int count, double2* out);
__global__ void dense_step_kernel(const double2* cur, const double2* site, int l, int r, long prefix, int prune,
                                  double2* nxt);
__global__ void pauli_expectation_kernel(DeviceMps mps, const char* labels, int nterms, double2* scratch,
                                         int env_cap, double2* out);
__global__ void overlap_half_kernel(const double2* env, int kl, int bl, const double2* ket, int kr, double2* tmp);
__global__ void overlap_next_kernel(const double2* tmp, int bl, int kr, const double2* bra, int br, double2* next);
__global__ void sample_env_half_kernel(const double2* site, int l, int r, const double2* env_next, double2* tmp);
__global__ void sample_env_kernel(const double2* site, int l, int r, const double2* tmp, double2* env);
__global__ void sample_shots_kernel(DeviceMps mps, const double2* envs, const unsigned long long* env_off,
                                    const int* bitpos, unsigned long long seed, int shots, unsigned long long* out);

// Adjoint kernels (adjoint_kernels.cu).
struct Adj1q {
    double2 u[4];   // the gate, row-major
    double2 du[4];  // d u / d angle (rotations)
    int has_du;
    int slot;       // gradient slot of this gate instance
};
// One split of the reverse sweep: the tape's copies of its forward inputs
// and outputs, the cotangent sites it updates, and the workspace matrices
// (column-major, leading dimension R = 2 chi_max).
struct AdjSplit {
    const SplitState* st;
    const double2* theta;   // rows x cols, row-major
    const double2* w;       // Jacobi W, M x N column-major
    const double* sigma;    // N
    const int* perm;        // N: sorted position -> column
    const double2* site_l;  // site p before the split: [dl][2][k]
    const double2* site_r;  // site p+1 before the split: [k][2][dr]
    double2* bar_l;         // cotangent of site p
    double2* bar_r;         // cotangent of site p+1
    double2 u[16];          // effective 4x4 of the gate on theta
    double2 *U, *V, *Ub, *Vb, *M, *Nm, *Z, *T1, *tb, *tb0;
    double *inv, *sq;
    int R;
};
enum { kAdjStageOther = 0, kAdjStageM, kAdjStageN, kAdjStageT1, kAdjStageTb, kAdjStageTb2, kAdjStageBarL,
       kAdjStageBarR };
__global__ void adj_pauli_envs_kernel(DeviceMps mps, const char* labels, int nterms, int cap, double2* envs,
                                      double2* tmp_all, double2* vals);
__global__ void adj_pauli_holes_kernel(DeviceMps mps, const char* labels, int t0, int cap, const double2* envs,
                                       double2* tmp_all, double2* holes);
__global__ void adj_pauli_accumulate_kernel(DeviceMps mps, double2* const* bars, const double2* holes,
                                            const double* coef_re, int t0, int count, int cap, int first);
__global__ void adj_one_qubit_kernel(double2* bar, const double2* before, const int* dims, Adj1q g, double* grad);
__global__ void adj_split_prep_kernel(AdjSplit A);
__global__ void adj_split_gemm_kernel(AdjSplit A, int stage);
__global__ void adj_split_assemble_kernel(AdjSplit A);
__global__ void adj_split_gate_kernel(AdjSplit A);

// Jacobi shared-memory footprint for a working matrix of M rows and N columns
// on a cluster of C CTAs, `elem` bytes per complex entry.
inline size_t jacobi_smem_bytes(int M, int N, int C, size_t elem = sizeof(double2)) {
    const int quantum = 4 * C;
    const int Np = ((N + quantum - 1) / quantum) * quantum;
    const int b = Np / (2 * C);
    const int nbuf = C == 1 ? 2 : 3;
    return size_t(nbuf) * b * M * elem;  // W columns only (plus padding columns)
}

}  // namespace wqc
