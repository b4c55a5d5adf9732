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

}  // namespace wqc
