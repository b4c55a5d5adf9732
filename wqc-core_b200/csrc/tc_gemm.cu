// Complex GEMM on the tcgen05 tensor cores (kind::tf32, 3xTF32 split
// products, FP32 accumulation in tensor memory), fed by TMA.  Used by the
// tensor-core form's two-site merge (src/tn/mps.rs:484-514, 812-866) and
// exposed alone as wqc_tc_zgemm.  The layout of operands and tiles is
// described in tc_gemm.cuh.
//
// Every wait on an mbarrier is bounded (ptx::kWaitNs); a wait that gives up sets
// kStatusDeviceTimeout, the thread stops issuing work, and the block still
// waits (bounded) for what it issued and frees its tensor memory.
#include <cudaTypedefs.h>

#include <mutex>
#include <string>

#include "../../include/wqc_cuda.h"
#include "split_kernels.cuh"
#include "tc_gemm.cuh"
#include "tc_ptx.cuh"

namespace wqc {

namespace {

using namespace ptx;

// Instruction descriptor of kind::tf32: FP32 accumulator (bits 4-5 = 1), A
// and B TF32 (bits 7-9, 10-12 = 2), both K-major, N >> 3 at bits 17-22, M >> 4
// at bits 24-28.
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(kTcTileN >> 3) << 17) |
                              (uint32_t(kTcTileM >> 4) << 24);

__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t addr) { return umma_desc_kmajor<128>(addr); }

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate)
        : "memory");
}

// Tensor-memory columns: the even-K-block hi*hi accumulator at 0, the odd
// one at kTcAccOdd, the lo*hi + hi*lo accumulator at kTcAccSmall (the
// allocation is a power of two of at least 32 columns).
constexpr uint32_t kTcAccOdd = kTcTileN, kTcAccSmall = 2 * kTcTileN;
constexpr uint32_t kTcTmemCols = 512;

__device__ __forceinline__ void tmem_ld16f(uint32_t taddr, float* v) {
    uint32_t r[16];
    tmem_ld16(taddr, r);
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Sixteen accumulator columns at `taddr`, the three accumulators summed in
// FP64 (`odd`: the second hi*hi accumulator holds a part).
__device__ __forceinline__ void tmem_sum16(uint32_t taddr, bool odd, double* v) {
    float a[16], b[16];
    tmem_ld16f(taddr + kTcAccSmall, a);
    tmem_ld16f(taddr, b);
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = double(b[i]) + double(a[i]);
    if (odd) {
        tmem_ld16f(taddr + kTcAccOdd, b);
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] += double(b[i]);
    }
}

// TF32 value of x, rounded to nearest (ties away), in an FP32 container.
__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// hi + lo split of an FP64 value into two TF32 values.
__device__ __forceinline__ void split_tf32(double x, float& hi, float& lo) {
    hi = tf32_rna(float(x));
    lo = tf32_rna(float(x - double(hi)));
}

}  // namespace

// ---------------------------------------------------------------------------
// Operand staging.  A planes: row r of job j is theta's row r (L's (a,s) row),
// column 2g+c the real (c = 0) or imaginary (c = 1) part of L[r][g].  B planes:
// row R' is the real output column; within tile nt (b in [32 nt, 32 nt + 32)),
// R' = 128 nt + 2 q + p with q = 32 t + (b - 32 nt) and p the part of the
// output (0 re, 1 im); column 2g+c holds B2[2g+c][p] of R[g][t][b].
// ---------------------------------------------------------------------------
__device__ __forceinline__ double b2_entry(double2 v, int p, int c) {
    // [[Br, Bi], [-Bi, Br]]: row part c of A, column part p of C
    return p == 0 ? (c == 0 ? v.x : -v.y) : (c == 0 ? v.y : v.x);
}

// Both operands of every job of a wave in one launch (grid: a_blocks +
// N tiles x kpad / 32, jobs).  The first a_blocks blocks stage A: L's rows
// are K-contiguous already, one thread per complex value writes its re/im
// pair into both planes.  Each later block stages one (N tile, 32 K values)
// of B: R[g][t][b] for 16 values of g, both t and 32 values of b read row
// by row into shared memory, then the tile's 128 plane rows written as
// 128-byte runs of K.
__global__ void __launch_bounds__(256) tc_prep_merge_kernel(const SplitJob* jobs, const SplitState* st,
                                                            DeviceMps mps, float* a_planes, float* b_planes,
                                                            int rpad, int npad, int kpad, int a_blocks) {
    const int j = blockIdx.y;
    const SplitState S = st[j];
    if (S.skip) return;
    const SplitJob& J = jobs[j];
    const int k = S.k, tid = threadIdx.x;
    const int kx_end = tc_kpad(k) < kpad ? tc_kpad(k) : kpad;
    if (int(blockIdx.x) < a_blocks) {
        const double2* L = mps.site[J.p];
        const int ldl = mps.dr[J.p], rows = S.rows;
        const int mrows = ((rows + kTcTileM - 1) / kTcTileM) * kTcTileM, gpad = kx_end / 2;
        const size_t plane_a = size_t(rpad) * kpad;
        float* ahi = a_planes + size_t(2 * j) * plane_a;
        float* alo = ahi + plane_a;
        const long na = long(mrows) * gpad;
        for (long e = long(blockIdx.x) * blockDim.x + tid; e < na; e += long(a_blocks) * blockDim.x) {
            const int r = int(e / gpad), g = int(e % gpad);
            const double2 v = (r < rows && g < k) ? L[size_t(r) * ldl + g] : cmake(0, 0);
            float hr, lr, hi, li;
            split_tf32(v.x, hr, lr);
            split_tf32(v.y, hi, li);
            const size_t off = size_t(r) * kpad + 2 * g;
            *reinterpret_cast<float2*>(ahi + off) = make_float2(hr, hi);
            *reinterpret_cast<float2*>(alo + off) = make_float2(lr, li);
        }
        return;
    }
    const int kchunks = kpad / kTcKBlock;
    const int bx = int(blockIdx.x) - a_blocks;
    const int nt = bx / kchunks, kc = bx % kchunks;
    const int dr = S.dr;
    if (nt * 32 >= dr || kc * kTcKBlock >= kx_end) return;  // uniform over the block
    const double2* R = mps.site[J.p + 1];
    __shared__ double2 tile[2][kTcKBlock / 2][33];  // [t][g - g0][b - b0]
    const int g0 = kc * (kTcKBlock / 2), b0 = nt * 32;
    for (int e = tid; e < 2 * (kTcKBlock / 2) * 32; e += blockDim.x) {
        const int t = e / (16 * 32), gi = (e / 32) % 16, bi = e % 32;
        const int g = g0 + gi, b = b0 + bi;
        tile[t][gi][bi] = (g < k && b < dr) ? R[(size_t(g) * 2 + t) * dr + b] : cmake(0, 0);
    }
    __syncthreads();
    const size_t plane_b = size_t(npad) * kpad;
    float* bhi = b_planes + size_t(2 * j) * plane_b;
    float* blo = bhi + plane_b;
    for (int e = tid; e < kTcTileN * (kTcKBlock / 4); e += blockDim.x) {
        const int w = e / (kTcKBlock / 4), c4 = e % (kTcKBlock / 4);  // plane row w, K values 4 c4 .. 4 c4 + 3
        const int q = w >> 1, p = w & 1, t = q >> 5, bi = q & 31;
        float h[4], l[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) split_tf32(b2_entry(tile[t][2 * c4 + (i >> 1)][bi], p, i & 1), h[i], l[i]);
        const size_t off = size_t(nt * kTcTileN + w) * kpad + size_t(kc) * kTcKBlock + 4 * c4;
        *reinterpret_cast<float4*>(bhi + off) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4*>(blo + off) = make_float4(l[0], l[1], l[2], l[3]);
    }
}

// Plain problems: B's rows in natural order, R' = 2 col + p.
__global__ void tc_prep_plain_kernel(const double2* A, const double2* B, int m, int n, int k, float* a_planes,
                                     float* b_planes, int rpad, int npad, int kpad) {
    const size_t plane_a = size_t(rpad) * kpad, plane_b = size_t(npad) * kpad;
    float* ahi = a_planes;
    float* alo = ahi + plane_a;
    float* bhi = b_planes;
    float* blo = bhi + plane_b;
    const long na = long(rpad) * kpad, nb = long(npad) * kpad;
    const long stride = long(gridDim.x) * blockDim.x;
    for (long e = long(blockIdx.x) * blockDim.x + threadIdx.x; e < na + nb; e += stride) {
        if (e < na) {
            const int r = int(e / kpad), kx = int(e % kpad);
            const int g = kx >> 1;
            double x = 0.0;
            if (r < m && g < k) {
                const double2 v = A[size_t(r) * k + g];
                x = (kx & 1) ? v.y : v.x;
            }
            float hi, lo;
            split_tf32(x, hi, lo);
            ahi[e] = hi;
            alo[e] = lo;
        } else {
            const long f = e - na;
            const int rr = int(f / kpad), kx = int(f % kpad);
            const int col = rr >> 1, p = rr & 1, g = kx >> 1;
            double x = 0.0;
            if (col < n && g < k) x = b2_entry(B[size_t(g) * n + col], p, kx & 1);
            float hi, lo;
            split_tf32(x, hi, lo);
            bhi[f] = hi;
            blo[f] = lo;
        }
    }
}

// ---------------------------------------------------------------------------
// The GEMM: one CTA per 128 x 128 real tile of one job (grid: N tiles, M
// tiles, jobs).  Warp 0 allocates 128 tensor-memory columns; its lane 0 then
// runs the TMA producer over kTcStages stages, warp 1's lane 0 the MMA issuer
// (three MMAs per K step of 8: lo*hi, hi*lo, hi*hi); all four warps read the
// accumulator (warp w owns TMEM lanes 32w..32w+31, i.e. tile rows) for the
// epilogue.
// ---------------------------------------------------------------------------
template <bool kMerge, class Args>
__global__ void __launch_bounds__(kTcThreads, 1)
    tc_zgemm_kernel(const __grid_constant__ CUtensorMap ma, const __grid_constant__ CUtensorMap mb, Args args,
                    int* status) {
    const int j = blockIdx.z;
    int rows, k, ntiles;
    if constexpr (kMerge) {
        const SplitState& S = args.st[j];
        if (S.skip) return;
        rows = S.rows;
        k = S.k;
        ntiles = (S.dr + 31) / 32;
    } else {
        rows = args.m;
        k = args.k;
        ntiles = (2 * args.n + kTcTileN - 1) / kTcTileN;
    }
    const int row0 = blockIdx.y * kTcTileM, nt = blockIdx.x;
    if (row0 >= rows || nt >= ntiles || k <= 0) return;  // uniform over the block
    const int nk = tc_kpad(k) / kTcKBlock;

    extern __shared__ uint8_t tc_smem_raw[];
    __shared__ __align__(8) uint64_t bars[2 * kTcStages + 1];
    __shared__ uint32_t tmem_slot;
    const uint32_t tiles = (smem_u32(tc_smem_raw) + 1023u) & ~1023u;  // the swizzle repeats every 1024 bytes
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[kTcStages]),
                   done = smem_u32(&bars[2 * kTcStages]);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kTcStages; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tmem_alloc(smem_u32(&tmem_slot), kTcTmemCols);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    bool ok = true;
    if (warp == 0 && lane == 0) {
        const int z = 2 * j, yb = nt * kTcTileN;
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % kTcStages;
            if (kb >= kTcStages && !mbar_wait(empty0 + 8 * s, ((kb / kTcStages) & 1) ^ 1)) {
                ok = false;
                break;
            }
            const uint32_t base = tiles + uint32_t(s) * kTcStageBytes, fb = full0 + 8 * s;
            const int x = kb * kTcKBlock;
            mbar_expect_tx(fb, kTcStageBytes);
            tma_load_3d(base, &ma, x, row0, z, fb);
            tma_load_3d(base + kTcBoxBytes, &ma, x, row0, z + 1, fb);
            tma_load_3d(base + 2 * kTcBoxBytes, &mb, x, yb, z, fb);
            tma_load_3d(base + 3 * kTcBoxBytes, &mb, x, yb, z + 1, fb);
        }
    } else if (warp == 1 && lane == 0) {
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % kTcStages;
            if (!mbar_wait(full0 + 8 * s, (kb / kTcStages) & 1)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t base = tiles + uint32_t(s) * kTcStageBytes;
#pragma unroll
            for (int kk = 0; kk < kTcKBlock / 8; ++kk) {
                const uint32_t off = uint32_t(kk) * 32;  // 8 TF32 values along K
                const uint64_t ahi = umma_desc_sw128(base + off), alo = umma_desc_sw128(base + kTcBoxBytes + off);
                const uint64_t bhi = umma_desc_sw128(base + 2 * kTcBoxBytes + off),
                               blo = umma_desc_sw128(base + 3 * kTcBoxBytes + off);
                // small terms into their own accumulator; hi*hi alternates
                // between two by K block, so each FP32 accumulator takes a
                // third of the updates (they are summed in FP64 below)
                umma_tf32(tmem + kTcAccSmall, alo, bhi, (kb | kk) != 0 ? 1u : 0u);
                umma_tf32(tmem + kTcAccSmall, ahi, blo, 1u);
                umma_tf32(tmem + ((kb & 1) ? kTcAccOdd : 0u), ahi, bhi, (kb > 1 || kk > 0) ? 1u : 0u);
            }
            umma_commit(empty0 + 8 * s);  // the stage is free once these MMAs have read it
        }
        umma_commit(done);  // also after a timeout: `done` then waits for what was issued
    }
    if (!ok) atomicOr(status, kStatusDeviceTimeout);
    __syncthreads();
    bool ready = mbar_wait(done, 0);
    ready = __all_sync(0xffffffffu, ready);
    if (!ready && lane == 0) atomicOr(status, kStatusDeviceTimeout);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (ready) {
        const uint32_t tl = tmem + (uint32_t(warp * 32) << 16);
        const bool odd = nk > 1;  // the second hi*hi accumulator was written
        const int row = row0 + warp * 32 + lane;
        if constexpr (kMerge) {
            const SplitJob& J = args.jobs[j];
            const SplitState& S = args.st[j];
            const int s_own = row & 1;  // row = 2a + s (row0 is even)
            const int dr = S.dr, cols = S.cols;
            double2 u[2][4];
#pragma unroll
            for (int to = 0; to < 2; ++to)
#pragma unroll
                for (int q = 0; q < 4; ++q) u[to][q] = J.u[(s_own * 2 + to) * 4 + q];
            double2* th = args.slots[J.slot].theta;
            const bool row_ok = row < S.rows;
#pragma unroll 1
            for (int c = 0; c < 4; ++c) {
                double v0[16], v1[16];
                tmem_sum16(tl + 16 * c, odd, v0);       // t = 0: b = 32 nt + 8 c + i
                tmem_sum16(tl + 64 + 16 * c, odd, v1);  // t = 1
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const double2 o0 = cmake(v0[2 * i], v0[2 * i + 1]), o1 = cmake(v1[2 * i], v1[2 * i + 1]);
                    const double2 p0 = cmake(__shfl_xor_sync(0xffffffffu, v0[2 * i], 1),
                                             __shfl_xor_sync(0xffffffffu, v0[2 * i + 1], 1));
                    const double2 p1 = cmake(__shfl_xor_sync(0xffffffffu, v1[2 * i], 1),
                                             __shfl_xor_sync(0xffffffffu, v1[2 * i + 1], 1));
                    // theta[s][t] of this (a, b), s = 0 on even rows
                    const double2 t00 = s_own ? p0 : o0, t01 = s_own ? p1 : o1;
                    const double2 t10 = s_own ? o0 : p0, t11 = s_own ? o1 : p1;
                    const int b = nt * 32 + 8 * c + i;
                    if (row_ok && b < dr) {
#pragma unroll
                        for (int to = 0; to < 2; ++to) {
                            double2 v = cmake(0, 0);
                            cfma(v, u[to][0], t00);
                            cfma(v, u[to][1], t01);
                            cfma(v, u[to][2], t10);
                            cfma(v, u[to][3], t11);
                            th[size_t(row) * cols + to * dr + b] = v;
                        }
                    }
                }
            }
        } else {
            const bool row_ok = row < args.m;
#pragma unroll 1
            for (int c = 0; c < kTcTileN / 16; ++c) {
                double v[16];
                tmem_sum16(tl + 16 * c, odd, v);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int col = nt * (kTcTileN / 2) + 8 * c + i;
                    if (row_ok && col < args.n) args.C[size_t(row) * args.ldc + col] = cmake(v[2 * i], v[2 * i + 1]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        tmem_dealloc(tmem, kTcTmemCols);
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
bool tc_encode_planes(CUtensorMap* map, void* base, int kpad, int rows, int planes) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!encode || !base || kpad % kTcKBlock || rows % kTcTileM || planes < 1) return false;
    const cuuint64_t dims[3] = {cuuint64_t(kpad), cuuint64_t(rows), cuuint64_t(planes)};
    const cuuint64_t strides[2] = {cuuint64_t(kpad) * 4, cuuint64_t(kpad) * 4 * cuuint64_t(rows)};
    const cuuint32_t box[3] = {cuuint32_t(kTcKBlock), cuuint32_t(kTcTileM), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <bool kMerge, class Args>
static cudaError_t launch_tc(const CUtensorMap& ma, const CUtensorMap& mb, dim3 grid, cudaStream_t s,
                             const Args& args, int* status) {
    auto* fn = tc_zgemm_kernel<kMerge, Args>;
    if (cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmemBytes)) return e;
    fn<<<grid, kTcThreads, kTcSmemBytes, s>>>(ma, mb, args, status);
    return cudaGetLastError();
}

cudaError_t launch_tc_merge(const CUtensorMap& ma, const CUtensorMap& mb, dim3 grid, cudaStream_t s,
                            const TcMergeArgs& args, int* status) {
    return launch_tc<true>(ma, mb, grid, s, args, status);
}

cudaError_t launch_tc_plain(const CUtensorMap& ma, const CUtensorMap& mb, dim3 grid, cudaStream_t s,
                            const TcPlainArgs& args, int* status) {
    return launch_tc<false>(ma, mb, grid, s, args, status);
}

}  // namespace wqc

// ---------------------------------------------------------------------------
// C ABI: the tensor-core complex GEMM alone.
// ---------------------------------------------------------------------------
namespace wqc {
wqc_status record_error(wqc_status code, const std::string& msg);  // executor.cu
wqc_status record_oom(uint64_t required, uint64_t available);
int context_device(const wqc_cuda_ctx* ctx);
}  // namespace wqc

extern "C" {

WQC_API wqc_status wqc_tc_zgemm(wqc_cuda_ctx* ctx, uint32_t m, uint32_t n, uint32_t k, const double* a,
                                const double* b, double* c, uint32_t reps, double* kernel_ms) {
    using namespace wqc;
    if (!ctx || !a || !b || !c) return record_error(WQC_ERR_INVALID, "null argument");
    constexpr uint32_t kMax = 16384;
    if (m == 0 || n == 0 || k == 0 || m > kMax || n > kMax || k > kMax)
        return record_error(WQC_ERR_INVALID, "tensor-core GEMM sizes must lie in 1..16384");
    if (reps == 0) reps = 1;
    if (cudaError_t e = cudaSetDevice(context_device(ctx)))
        return record_error(WQC_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    const int rpad = tc_rpad(int(m)), npad = tc_npad(int(n)), kpad = tc_kpad(int(k));
    const size_t bytes_a = size_t(m) * k * sizeof(double2), bytes_b = size_t(k) * n * sizeof(double2),
                 bytes_c = size_t(m) * n * sizeof(double2);
    const size_t bytes_pa = size_t(2) * rpad * kpad * sizeof(float), bytes_pb = size_t(2) * npad * kpad * sizeof(float);
    const size_t need = bytes_a + bytes_b + bytes_c + bytes_pa + bytes_pb + 256;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return record_error(WQC_ERR_CUDA, "cudaMemGetInfo");
    if (need > fr) return record_oom(need, fr);

    void *dA = nullptr, *dB = nullptr, *dC = nullptr, *dPA = nullptr, *dPB = nullptr, *dSt = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto release = [&] {
        if (s) cudaStreamSynchronize(s);
        for (void* p : {dA, dB, dC, dPA, dPB, dSt})
            if (p) cudaFree(p);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (s) cudaStreamDestroy(s);
    };
    auto cuda_fail = [&](const char* what, cudaError_t e) {
        const std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
        cudaGetLastError();
        release();
        return record_error(WQC_ERR_CUDA, msg);
    };
    cudaError_t e = cudaSuccess;
    if ((e = cudaMalloc(&dA, bytes_a)) || (e = cudaMalloc(&dB, bytes_b)) || (e = cudaMalloc(&dC, bytes_c)) ||
        (e = cudaMalloc(&dPA, bytes_pa)) || (e = cudaMalloc(&dPB, bytes_pb)) || (e = cudaMalloc(&dSt, 256)))
        return cuda_fail("cudaMalloc(tensor-core GEMM)", e);
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) || (e = cudaEventCreate(&e0)) ||
        (e = cudaEventCreate(&e1)))
        return cuda_fail("stream", e);
    if ((e = cudaMemcpyAsync(dA, a, bytes_a, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(dB, b, bytes_b, cudaMemcpyHostToDevice, s)) || (e = cudaMemsetAsync(dSt, 0, 256, s)))
        return cuda_fail("cudaMemcpyAsync(tensor-core GEMM operands)", e);
    tc_prep_plain_kernel<<<1184, 256, 0, s>>>(static_cast<const double2*>(dA), static_cast<const double2*>(dB),
                                              int(m), int(n), int(k), static_cast<float*>(dPA),
                                              static_cast<float*>(dPB), rpad, npad, kpad);
    if ((e = cudaGetLastError())) return cuda_fail("tensor-core GEMM staging", e);
    CUtensorMap ma, mb;
    if (!tc_encode_planes(&ma, dPA, kpad, rpad, 2) || !tc_encode_planes(&mb, dPB, kpad, npad, 2)) {
        release();
        return record_error(WQC_ERR_CUDA, "cuTensorMapEncodeTiled refused the operand planes");
    }
    const TcPlainArgs args{int(m), int(n), int(k), static_cast<double2*>(dC), int(n)};
    const dim3 grid(npad / kTcTileN, rpad / kTcTileM, 1);
    if ((e = cudaEventRecord(e0, s))) return cuda_fail("cudaEventRecord", e);
    for (uint32_t r = 0; r < reps; ++r)
        if ((e = launch_tc_plain(ma, mb, grid, s, args, static_cast<int*>(dSt))))
            return cuda_fail("tensor-core GEMM launch", e);
    if ((e = cudaEventRecord(e1, s))) return cuda_fail("cudaEventRecord", e);
    int status = 0;
    if ((e = cudaMemcpyAsync(c, dC, bytes_c, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(&status, dSt, sizeof(int), cudaMemcpyDeviceToHost, s)) || (e = cudaStreamSynchronize(s)))
        return cuda_fail("tensor-core GEMM", e);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (kernel_ms) *kernel_ms = double(ms) / reps;
    release();
    if (status & kStatusDeviceTimeout)
        return record_error(WQC_ERR_DEVICE_TIMEOUT, "tensor-core GEMM gave up waiting on its operands");
    return WQC_OK;
}

}  // extern "C"
