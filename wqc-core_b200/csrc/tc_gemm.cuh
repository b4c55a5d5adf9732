// Complex GEMM on the tcgen05 tensor cores with 3xTF32 split products.
//
// A complex product C = A B (A m x k, B k x n) runs as one real GEMM on the
// real embedding: A's rows as they lie in memory (re, im interleaved along k:
// an m x 2k real matrix) times B2 (2k x 2n real) whose 2 x 2 blocks are
// [[Br, Bi], [-Bi, Br]], so that C's rows come out interleaved the same way.
// Each FP64 operand x is split into two TF32 values hi = tf32(x) and
// lo = tf32(x - hi); the product sums A_lo B_hi + A_hi B_lo + A_hi B_hi in FP32
// in tensor memory (the lo * lo term is below FP32 rounding).
//
// Operands are staged by a prep kernel as TF32 planes in global memory, K
// innermost, zero beyond the problem: A planes [job][hi|lo][Rpad][Kpad] and B
// planes [job][hi|lo][Npad][Kpad] (one row per real output column).  TMA
// loads 128-row x 32-column boxes of them with the 128-byte swizzle into
// shared memory; one thread issues the MMAs (M = N = 128, K = 8 per
// instruction) into a 128 x 128 FP32 accumulator in tensor memory; four warps
// read it back with tcgen05.ld for the epilogue.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace wqc {

constexpr int kTcTileM = 128;     // rows of a CTA tile (one TMEM lane each)
constexpr int kTcTileN = 128;     // real columns of a CTA tile (64 complex)
constexpr int kTcKBlock = 32;     // real K values per stage (128 bytes of FP32)
constexpr int kTcStages = 3;
constexpr int kTcThreads = 128;
constexpr int kTcBoxBytes = kTcTileM * kTcKBlock * 4;  // one plane's box: 16 KB
constexpr int kTcStageBytes = 4 * kTcBoxBytes;         // A hi, A lo, B hi, B lo
constexpr int kTcSmemBytes = kTcStages * kTcStageBytes + 1024;  // + alignment of the swizzled tiles

// Padded staging extents for complex problems up to m x k times k x n.
__host__ __device__ inline int tc_kpad(int k) { return ((2 * k + kTcKBlock - 1) / kTcKBlock) * kTcKBlock; }
__host__ __device__ inline int tc_rpad(int m) { return ((m + kTcTileM - 1) / kTcTileM) * kTcTileM; }
__host__ __device__ inline int tc_npad(int n) { return ((2 * n + kTcTileN - 1) / kTcTileN) * kTcTileN; }

// Tensor map over `planes` planes of rows x kpad FP32 values (K innermost),
// boxes of 32 x 128 with the 128-byte swizzle.  False if the driver refuses.
bool tc_encode_planes(CUtensorMap* map, void* base, int kpad, int rows, int planes);

// Epilogue of the two-site merge (mps.rs:812-866): theta'[(a,s'),(t',b)] =
// sum_{s,t} U[s't',st] theta[(a,s),(t,b)], written as FP64 into the slot's
// theta.  B's rows are ordered so that a tile holds 32 values of b for both t.
struct TcMergeArgs {
    const SplitJob* jobs;
    const SplitState* st;
    const SlotBuffers* slots;
};
// Plain epilogue: C (m x n complex FP64, row-major, leading dimension ldc).
struct TcPlainArgs {
    int m, n, k;
    double2* C;
    int ldc;
};

// Stage the merge operands of every job of a wave (L and R sites, shapes from
// the SplitState written by prepare_kernel) in one launch: grid (a_blocks +
// N tiles x kpad / 32, jobs).
__global__ void tc_prep_merge_kernel(const SplitJob* jobs, const SplitState* st, DeviceMps mps, float* a_planes,
                                     float* b_planes, int rpad, int npad, int kpad, int a_blocks);
// Stage a plain problem (A m x k, B k x n, row-major complex FP64).
__global__ void tc_prep_plain_kernel(const double2* A, const double2* B, int m, int n, int k, float* a_planes,
                                     float* b_planes, int rpad, int npad, int kpad);

cudaError_t launch_tc_merge(const CUtensorMap& ma, const CUtensorMap& mb, dim3 grid, cudaStream_t s,
                            const TcMergeArgs& args, int* status);
cudaError_t launch_tc_plain(const CUtensorMap& ma, const CUtensorMap& mb, dim3 grid, cudaStream_t s,
                            const TcPlainArgs& args, int* status);

// ---------------------------------------------------------------------------
// FP64-accurate complex GEMM from int8 slices (the Ozaki scheme) on the
// tcgen05 tensor cores, kind::i8 (tc_ozaki.cu).  Each row r of A (the real
// embedding, as above) is scaled by 2^-e_r so that its largest entry lies in
// [1/2, 1), each real column c of B2 by 2^-f_c, and every scaled value x is
// cut into kOzSlices = 9 signed 7-bit digits, x = sum_p d_p 2^-7(p+1) + eps
// with |eps| < 2^-63 (digits by truncation: |d_p| <= 127, the sign of x).
// The slice products A_p B_q are exact in int32; those with p + q = d share
// accumulator d (at most 9 products of K <= 8192 terms of |d_p e_q| <= 127^2:
// below 2^31), and the products with p + q >= kOzSlices are dropped (all
// together below 2^-60 of the two scales).  The epilogue sums the
// accumulators in FP64, C[r][c] = 2^(e_r + f_c - 14) sum_d acc_d 2^-7d, so
// the FP64 rounding of that sum is the error that remains.
//
// Staging: digit planes [job][slice][Rpad][Kpad] (A) and [job][slice][Npad]
// [Kpad] (B, one row per real output column), int8, K innermost, zero beyond
// the problem; exponents e [job][Rpad] and f [job][Npad / 2] (one per complex
// output column: both real columns of a complex column have the same B2
// column maximum).  TMA loads 64-byte x 128-row (A) and 64-byte x 64-row (B)
// boxes with the 64-byte swizzle; one thread issues the 45 MMAs (M = 128,
// N = 32, K = 32 bytes) of each 32-byte K step into 9 int32 accumulators in
// tensor memory (9 x 32 of its 512 columns: nine accumulators of 64 columns
// would not fit, hence the narrow tile).
// ---------------------------------------------------------------------------
constexpr int kOzSlices = 9;                                      // digits per operand: 63 bits
constexpr int kOzTileM = 128;                                     // rows of a CTA tile
constexpr int kOzTileN = 32;                                      // real columns of a CTA tile (16 complex)
constexpr int kOzTileC = kOzTileN / 2;                            // complex columns of a CTA tile
constexpr int kOzKBlock = 64;                                     // int8 K values per stage (64-byte rows)
constexpr int kOzStages = 2;
constexpr int kOzThreads = 128;
constexpr int kOzABox = kOzTileM * kOzKBlock;                     // one A slice's box: 8 KB
constexpr int kOzBBox = kOzTileN * kOzKBlock;                     // one B slice's box: 2 KB
constexpr int kOzStageBytes = kOzSlices * (kOzABox + kOzBBox);    // 90 KB
constexpr int kOzSmemBytes = kOzStages * kOzStageBytes + 1024;    // + alignment of the swizzled tiles

__host__ __device__ inline int oz_kpad(int k) { return ((2 * k + kOzKBlock - 1) / kOzKBlock) * kOzKBlock; }
__host__ __device__ inline int oz_rpad(int m) { return ((m + kOzTileM - 1) / kOzTileM) * kOzTileM; }
__host__ __device__ inline int oz_npad(int n) { return ((2 * n + kOzTileN - 1) / kOzTileN) * kOzTileN; }

// Staging of one set of jobs: digit planes, exponents and their tensor maps.
struct OzPlanes {
    int8_t* a = nullptr;   // [jobs][kOzSlices][rpad][kpad]
    int8_t* b = nullptr;   // [jobs][kOzSlices][npad][kpad]
    int* ea = nullptr;     // [jobs][rpad]
    int* eb = nullptr;     // [jobs][npad / 2]
    int rpad = 0, npad = 0, kpad = 0, jobs = 0;
    CUtensorMap map_a{}, map_b{};
};
// Bytes of the staging for `jobs` problems up to rpad x kpad times kpad x npad.
size_t oz_planes_bytes(int jobs, int rpad, int npad, int kpad);
// Carve the staging out of `base` (oz_planes_bytes long, 256-byte aligned)
// and encode its tensor maps; false if the driver refuses a map.
bool oz_planes_init(OzPlanes* P, void* base, int jobs, int rpad, int npad, int kpad);

// Stage the merge operands of every job of a wave (grid: a_blocks + N tiles
// of 8 values of b x kpad / 64 K chunks, jobs); a_blocks blocks take 8 rows
// of A each in turn.
__global__ void oz_prep_merge_kernel(const SplitJob* jobs, const SplitState* st, DeviceMps mps, OzPlanes P,
                                     int a_blocks);
cudaError_t launch_oz_merge(const OzPlanes& P, dim3 grid, cudaStream_t s, const TcMergeArgs& args, int* status);
// Plain problems (wqc_tc_zgemm_int8).
__global__ void oz_prep_plain_kernel(const double2* A, const double2* B, int m, int n, int k, OzPlanes P,
                                     int a_blocks);
cudaError_t launch_oz_plain(const OzPlanes& P, dim3 grid, cudaStream_t s, const TcPlainArgs& args, int* status);

}  // namespace wqc
