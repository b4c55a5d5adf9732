// FP64-accurate complex GEMM on the tcgen05 tensor cores from int8 slices
// (the Ozaki scheme: exact integer products of fixed-point digit slices),
// kind::i8 with int32 accumulation in tensor memory, fed by TMA.  Used by the
// two-site merge (src/tn/mps.rs:484-514, 812-866) when a state selects
// WQC_MERGE_TC_INT8, and exposed alone as wqc_tc_zgemm_int8.  The scheme and
// the staging layout are described in tc_gemm.cuh.
//
// Every wait on an mbarrier is bounded (ptx::kWaitNs); a wait that gives up
// sets kStatusDeviceTimeout, the thread stops issuing work, and the block
// still waits (bounded) for what it issued and frees its tensor memory.
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/wqc_cuda.h"
#include "split_kernels.cuh"
#include "tc_gemm.cuh"
#include "tc_ptx.cuh"

namespace wqc {

namespace {

using namespace ptx;

// Instruction descriptor of kind::i8: S32 accumulator (bits 4-5 = 2), A and B
// signed 8-bit (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bits 17-22,
// M >> 4 at bits 24-28.
constexpr uint32_t kOzIdesc = (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(kOzTileN >> 3) << 17) |
                              (uint32_t(kOzTileM >> 4) << 24);
constexpr uint32_t kOzTmemCols = 512;  // kOzSlices accumulators of kOzTileN columns

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kOzIdesc), "r"(accumulate)
        : "memory");
}

// Largest |re|, |im| over the lanes of a warp.
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Exponent of a row or column holding a NaN or an infinity: no finite
// exponent comes near it, and the epilogue turns its entries into NaN, so a
// non-finite site still reaches the SVD's non-finite check.
constexpr int kOzNonFinite = 1 << 20;

// Exponent e with max * 2^-e in [1/2, 1) (0 for max = 0).
__device__ __forceinline__ int scale_exponent(double mx, bool nonfinite) {
    if (nonfinite) return kOzNonFinite;
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);
    return e;
}

__device__ __forceinline__ bool nonfinite2(double2 v) { return !(isfinite(v.x) && isfinite(v.y)); }

// The kOzSlices digits of x * 2^-e (|x| 2^-e < 1), by truncation: exact
// (all zero for a non-finite row or column).
__device__ __forceinline__ void digits(double x, int e, int* d) {
    double v = e == kOzNonFinite ? 0.0 : ldexp(x, -e);
#pragma unroll
    for (int p = 0; p < kOzSlices; ++p) {
        v *= 128.0;
        const double t = trunc(v);
        d[p] = int(t);
        v -= t;
    }
}

__device__ __forceinline__ double b2_value(double2 v, int p, int c) {
    // [[Br, Bi], [-Bi, Br]]: row part c of A, column part p of C
    return p == 0 ? (c == 0 ? v.x : -v.y) : (c == 0 ? v.y : v.x);
}

// Source of one job's operands: the merge's L and R sites, or a plain A, B.
// A(r, g) is row r, complex K index g; B(g, nt, q) is complex K index g,
// N tile nt, complex column q of the tile (merge: q = 8 t + b - 8 nt).
struct OzSource {
    const double2* A;
    const double2* B;
    int lda, rows, k;
    int n;  // plain: complex columns of B; merge: dr
    bool merge;
    __device__ __forceinline__ double2 a(int r, int g) const {
        return (r < rows && g < k) ? A[size_t(r) * lda + g] : make_double2(0.0, 0.0);
    }
    __device__ __forceinline__ double2 b(int g, int nt, int q) const {
        if (g >= k) return make_double2(0.0, 0.0);
        if (merge) {
            const int t = q >> 3, bb = nt * 8 + (q & 7);
            return bb < n ? B[(size_t(g) * 2 + t) * n + bb] : make_double2(0.0, 0.0);
        }
        const int col = nt * kOzTileC + q;
        return col < n ? B[size_t(g) * n + col] : make_double2(0.0, 0.0);
    }
    __device__ __forceinline__ int ntiles() const { return merge ? (n + 7) / 8 : (n + kOzTileC - 1) / kOzTileC; }
};

// Stage one job: blocks [0, a_blocks) take rows of A (one warp per row, 8
// rows a block in turn); block a_blocks + nt * (kpad / 64) + kc takes K
// chunk kc (32 values of g) of N tile nt of B: the tile's column maxima over
// all K first (every chunk's block computes them: R is small and in L2),
// then its chunk through shared memory, written as 4-byte runs of K per
// plane row.
__device__ void oz_stage(const OzSource& src, const OzPlanes& P, int j, int a_blocks) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int kx_end = min(oz_kpad(src.k), P.kpad);
    const size_t a_plane = size_t(P.rpad) * P.kpad, b_plane = size_t(P.npad) * P.kpad;
    if (int(blockIdx.x) < a_blocks) {
        const int mrows = oz_rpad(src.rows), gpad = kx_end / 2;
        int8_t* A = P.a + size_t(j) * kOzSlices * a_plane;
        for (int r = blockIdx.x * (blockDim.x / 32) + warp; r < mrows; r += a_blocks * (blockDim.x / 32)) {
            double mx = 0.0;
            bool bad = false;
            for (int g = lane; g < gpad; g += 32) {
                const double2 v = src.a(r, g);
                mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
                bad |= nonfinite2(v);
            }
            const int e = scale_exponent(warp_max(mx), __any_sync(0xffffffffu, bad));
            if (lane == 0) P.ea[size_t(j) * P.rpad + r] = e;
            for (int g = lane; g < gpad; g += 32) {
                const double2 v = src.a(r, g);
                int dr[kOzSlices], di[kOzSlices];
                digits(v.x, e, dr);
                digits(v.y, e, di);
#pragma unroll
                for (int p = 0; p < kOzSlices; ++p) {
                    const uint16_t pair = uint16_t(uint8_t(int8_t(dr[p]))) | (uint16_t(uint8_t(int8_t(di[p]))) << 8);
                    *reinterpret_cast<uint16_t*>(A + size_t(p) * a_plane + size_t(r) * P.kpad + 2 * g) = pair;
                }
            }
        }
        return;
    }
    const int kchunks = P.kpad / kOzKBlock;
    const int nt = (int(blockIdx.x) - a_blocks) / kchunks, kc = (int(blockIdx.x) - a_blocks) % kchunks;
    if (nt >= src.ntiles() || kc * kOzKBlock >= kx_end) return;  // uniform over the block
    constexpr int kSub = 256 / kOzTileC;  // threads splitting g per column in the maxima pass
    __shared__ double colmax[kSub][kOzTileC];
    __shared__ int colbad[kSub][kOzTileC];
    __shared__ int fexp[kOzTileC];
    __shared__ double2 tile[kOzKBlock / 2][kOzTileC + 1];  // [g - g0][q]
    {
        const int q = tid % kOzTileC, gsub = tid / kOzTileC;
        double mx = 0.0;
        bool bad = false;
        for (int g = gsub; g < src.k; g += kSub) {
            const double2 v = src.b(g, nt, q);
            mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
            bad |= nonfinite2(v);
        }
        colmax[gsub][q] = mx;
        colbad[gsub][q] = bad ? 1 : 0;
    }
    __syncthreads();
    if (tid < kOzTileC) {
        double mx = 0.0;
        bool bad = false;
        for (int w = 0; w < kSub; ++w) {
            mx = fmax(mx, colmax[w][tid]);
            bad |= colbad[w][tid] != 0;
        }
        const int f = scale_exponent(mx, bad);
        fexp[tid] = f;
        if (kc == 0) P.eb[size_t(j) * (P.npad / 2) + nt * kOzTileC + tid] = f;
    }
    __syncthreads();
    int8_t* B = P.b + size_t(j) * kOzSlices * b_plane;
    {
        const int g0 = kc * (kOzKBlock / 2);
        for (int e = tid; e < (kOzKBlock / 2) * kOzTileC; e += blockDim.x)
            tile[e / kOzTileC][e % kOzTileC] = src.b(g0 + e / kOzTileC, nt, e % kOzTileC);
        __syncthreads();
        for (int it = tid; it < kOzTileN * (kOzKBlock / 4); it += blockDim.x) {
            const int w = it / (kOzKBlock / 4), kq = it % (kOzKBlock / 4);  // plane row w, K bytes 4 kq .. 4 kq + 3
            const int q = w >> 1, pp = w & 1, f = fexp[q];
            uint32_t packed[kOzSlices];
#pragma unroll
            for (int p = 0; p < kOzSlices; ++p) packed[p] = 0u;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int kx = 4 * kq + i;
                int d[kOzSlices];
                digits(b2_value(tile[kx >> 1][q], pp, kx & 1), f, d);
#pragma unroll
                for (int p = 0; p < kOzSlices; ++p) packed[p] |= uint32_t(uint8_t(int8_t(d[p]))) << (8 * i);
            }
            const size_t off = size_t(nt * kOzTileN + w) * P.kpad + size_t(kc) * kOzKBlock + 4 * kq;
#pragma unroll
            for (int p = 0; p < kOzSlices; ++p) *reinterpret_cast<uint32_t*>(B + size_t(p) * b_plane + off) = packed[p];
        }
        __syncthreads();
    }
}

}  // namespace

__global__ void __launch_bounds__(256) oz_prep_merge_kernel(const SplitJob* jobs, const SplitState* st, DeviceMps mps,
                                                            OzPlanes P, int a_blocks) {
    const int j = blockIdx.y;
    const SplitState S = st[j];
    if (S.skip) return;
    const SplitJob& J = jobs[j];
    const OzSource src{mps.site[J.p], mps.site[J.p + 1], mps.dr[J.p], S.rows, S.k, S.dr, true};
    oz_stage(src, P, j, a_blocks);
}

__global__ void __launch_bounds__(256) oz_prep_plain_kernel(const double2* A, const double2* B, int m, int n, int k,
                                                            OzPlanes P, int a_blocks) {
    const OzSource src{A, B, k, m, k, n, false};
    oz_stage(src, P, 0, a_blocks);
}

// ---------------------------------------------------------------------------
// The GEMM: one CTA per 128 x 32 real tile of one job (grid: N tiles, M
// tiles, jobs).  Warp 0 allocates 512 tensor-memory columns; its lane 0
// runs the TMA producer (18 boxes a stage: the 9 slices of A and of B), warp
// 1's lane 0 the MMA issuer: per 32-byte K step, A_p times B_q for every
// p + q < kOzSlices into accumulator p + q (45 MMAs).  All four warps then
// combine the accumulators of their rows in FP64.
// ---------------------------------------------------------------------------
template <bool kMerge, class Args>
__global__ void __launch_bounds__(kOzThreads, 1)
    oz_zgemm_kernel(const __grid_constant__ CUtensorMap ma, const __grid_constant__ CUtensorMap mb, Args args,
                    const int* __restrict__ ea_all, const int* __restrict__ eb_all, int rpad, int npad, int* status) {
    const int j = blockIdx.z;
    int rows, k, ntiles;
    if constexpr (kMerge) {
        const SplitState& S = args.st[j];
        if (S.skip) return;
        rows = S.rows;
        k = S.k;
        ntiles = (S.dr + 7) / 8;
    } else {
        rows = args.m;
        k = args.k;
        ntiles = (args.n + kOzTileC - 1) / kOzTileC;
    }
    const int row0 = blockIdx.y * kOzTileM, nt = blockIdx.x;
    if (row0 >= rows || nt >= ntiles || k <= 0) return;  // uniform over the block
    const int nk = oz_kpad(k) / kOzKBlock;

    extern __shared__ uint8_t oz_smem_raw[];
    __shared__ __align__(8) uint64_t bars[2 * kOzStages + 1];
    __shared__ uint32_t tmem_slot;
    const uint32_t tiles = (smem_u32(oz_smem_raw) + 1023u) & ~1023u;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[kOzStages]),
                   done = smem_u32(&bars[2 * kOzStages]);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kOzStages; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tmem_alloc(smem_u32(&tmem_slot), kOzTmemCols);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_slot;
    constexpr uint32_t kBOff = kOzSlices * kOzABox;  // B slices follow A's within a stage

    bool ok = true;
    if (warp == 0 && lane == 0) {
        const int z0 = j * kOzSlices, yb = nt * kOzTileN;
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % kOzStages;
            if (kb >= kOzStages && !mbar_wait(empty0 + 8 * s, ((kb / kOzStages) & 1) ^ 1)) {
                ok = false;
                break;
            }
            const uint32_t base = tiles + uint32_t(s) * kOzStageBytes, fb = full0 + 8 * s;
            const int x = kb * kOzKBlock;
            mbar_expect_tx(fb, kOzStageBytes);
            for (int p = 0; p < kOzSlices; ++p) tma_load_3d(base + p * kOzABox, &ma, x, row0, z0 + p, fb);
            for (int q = 0; q < kOzSlices; ++q) tma_load_3d(base + kBOff + q * kOzBBox, &mb, x, yb, z0 + q, fb);
        }
    } else if (warp == 1 && lane == 0) {
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % kOzStages;
            if (!mbar_wait(full0 + 8 * s, (kb / kOzStages) & 1)) {
                ok = false;
                break;
            }
            fence_after_sync();
            const uint32_t base = tiles + uint32_t(s) * kOzStageBytes;
#pragma unroll
            for (int kk = 0; kk < kOzKBlock / 32; ++kk) {
#pragma unroll
                for (int p = 0; p < kOzSlices; ++p) {
                    const uint64_t adesc = umma_desc_kmajor<64>(base + p * kOzABox + kk * 32);
#pragma unroll
                    for (int q = 0; q + p < kOzSlices; ++q) {
                        const uint64_t bdesc = umma_desc_kmajor<64>(base + kBOff + q * kOzBBox + kk * 32);
                        // accumulator p + q is first written by (p = 0, q) at the first K step
                        umma_i8(tmem + uint32_t(p + q) * kOzTileN, adesc, bdesc, (kb | kk | p) != 0 ? 1u : 0u);
                    }
                }
            }
            umma_commit(empty0 + 8 * s);
        }
        umma_commit(done);
    }
    if (!ok) atomicOr(status, kStatusDeviceTimeout);
    __syncthreads();
    bool ready = mbar_wait(done, 0);
    ready = __all_sync(0xffffffffu, ready);
    if (!ready && lane == 0) atomicOr(status, kStatusDeviceTimeout);
    fence_after_sync();

    if (ready) {
        const uint32_t tl = tmem + (uint32_t(warp * 32) << 16);
        const int row = row0 + warp * 32 + lane;
        const int er = row < rows ? ea_all[size_t(j) * rpad + row] : 0;
        const int* eb = eb_all + size_t(j) * (npad / 2) + nt * kOzTileC;
        // 2^(e_r + f_c - 14) x, or NaN where the row or column held a non-finite value
        auto scaled = [&](double x, int f) {
            return (er == kOzNonFinite || f == kOzNonFinite) ? __longlong_as_double(0x7ff8000000000000ll)
                                                             : ldexp(x, er + f - 14);
        };
        // sum_d acc_d 2^-7d over 16 columns from `col`, by Horner from the last d
        auto combine = [&](int col, double* v) {
            uint32_t r[16];
            tmem_ld16(tl + uint32_t(kOzSlices - 1) * kOzTileN + col, r);
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = double(int(r[i]));
#pragma unroll 1
            for (int d = kOzSlices - 2; d >= 0; --d) {
                tmem_ld16(tl + uint32_t(d) * kOzTileN + col, r);
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = v[i] * (1.0 / 128.0) + double(int(r[i]));
            }
        };
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
            // b = 8 nt + i: complex column i (t = 0) and 8 + i (t = 1) of the tile
            double v0[16], v1[16];
            combine(0, v0);
            combine(16, v1);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int f0 = eb[i], f1 = eb[8 + i];
                const double2 o0 = cmake(scaled(v0[2 * i], f0), scaled(v0[2 * i + 1], f0));
                const double2 o1 = cmake(scaled(v1[2 * i], f1), scaled(v1[2 * i + 1], f1));
                const double2 p0 = cmake(__shfl_xor_sync(0xffffffffu, o0.x, 1), __shfl_xor_sync(0xffffffffu, o0.y, 1));
                const double2 p1 = cmake(__shfl_xor_sync(0xffffffffu, o1.x, 1), __shfl_xor_sync(0xffffffffu, o1.y, 1));
                const double2 t00 = s_own ? p0 : o0, t01 = s_own ? p1 : o1;
                const double2 t10 = s_own ? o0 : p0, t11 = s_own ? o1 : p1;
                const int b = nt * 8 + i;
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
        } else {
            const bool row_ok = row < args.m;
#pragma unroll 1
            for (int c = 0; c < kOzTileN / 16; ++c) {
                double v[16];
                combine(16 * c, v);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int q = 8 * c + i, col = nt * kOzTileC + q;
                    if (row_ok && col < args.n)
                        args.C[size_t(row) * args.ldc + col] = cmake(scaled(v[2 * i], eb[q]), scaled(v[2 * i + 1], eb[q]));
                }
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, kOzTmemCols);
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
static bool oz_encode(CUtensorMap* map, void* base, int kpad, int rows, int planes, int box_rows) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!encode || !base || kpad % kOzKBlock || rows % box_rows || planes < 1) return false;
    const cuuint64_t dims[3] = {cuuint64_t(kpad), cuuint64_t(rows), cuuint64_t(planes)};
    const cuuint64_t strides[2] = {cuuint64_t(kpad), cuuint64_t(kpad) * cuuint64_t(rows)};
    const cuuint32_t box[3] = {cuuint32_t(kOzKBlock), cuuint32_t(box_rows), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

size_t oz_planes_bytes(int jobs, int rpad, int npad, int kpad) {
    return align256(size_t(jobs) * kOzSlices * rpad * kpad) + align256(size_t(jobs) * kOzSlices * npad * kpad) +
           align256(size_t(jobs) * rpad * sizeof(int)) + align256(size_t(jobs) * (npad / 2) * sizeof(int));
}

bool oz_planes_init(OzPlanes* P, void* base, int jobs, int rpad, int npad, int kpad) {
    char* c = static_cast<char*>(base);
    P->jobs = jobs;
    P->rpad = rpad;
    P->npad = npad;
    P->kpad = kpad;
    P->a = reinterpret_cast<int8_t*>(c);
    c += align256(size_t(jobs) * kOzSlices * rpad * kpad);
    P->b = reinterpret_cast<int8_t*>(c);
    c += align256(size_t(jobs) * kOzSlices * npad * kpad);
    P->ea = reinterpret_cast<int*>(c);
    c += align256(size_t(jobs) * rpad * sizeof(int));
    P->eb = reinterpret_cast<int*>(c);
    return oz_encode(&P->map_a, P->a, kpad, rpad, jobs * kOzSlices, kOzTileM) &&
           oz_encode(&P->map_b, P->b, kpad, npad, jobs * kOzSlices, kOzTileN);
}

template <bool kMerge, class Args>
static cudaError_t launch_oz(const OzPlanes& P, dim3 grid, cudaStream_t s, const Args& args, int* status) {
    auto* fn = oz_zgemm_kernel<kMerge, Args>;
    if (cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kOzSmemBytes)) return e;
    fn<<<grid, kOzThreads, kOzSmemBytes, s>>>(P.map_a, P.map_b, args, P.ea, P.eb, P.rpad, P.npad, status);
    return cudaGetLastError();
}

cudaError_t launch_oz_merge(const OzPlanes& P, dim3 grid, cudaStream_t s, const TcMergeArgs& args, int* status) {
    return launch_oz<true>(P, grid, s, args, status);
}

cudaError_t launch_oz_plain(const OzPlanes& P, dim3 grid, cudaStream_t s, const TcPlainArgs& args, int* status) {
    return launch_oz<false>(P, grid, s, args, status);
}

}  // namespace wqc

// ---------------------------------------------------------------------------
// C ABI: the int8-slice complex GEMM alone.
// ---------------------------------------------------------------------------
namespace wqc {
wqc_status record_error(wqc_status code, const std::string& msg);  // executor.cu
wqc_status record_oom(uint64_t required, uint64_t available);
int context_device(const wqc_cuda_ctx* ctx);
}  // namespace wqc

extern "C" {

WQC_API wqc_status wqc_tc_zgemm_int8(wqc_cuda_ctx* ctx, uint32_t m, uint32_t n, uint32_t k, const double* a,
                                     const double* b, double* c, uint32_t reps, double* kernel_ms) {
    using namespace wqc;
    if (!ctx || !a || !b || !c) return record_error(WQC_ERR_INVALID, "null argument");
    constexpr uint32_t kMax = 8192;
    if (m == 0 || n == 0 || k == 0 || m > kMax || n > kMax || k > 4096)
        return record_error(WQC_ERR_INVALID, "int8-slice GEMM sizes must lie in 1..8192 (m, n) and 1..4096 (k)");
    if (reps == 0) reps = 1;
    if (cudaError_t e = cudaSetDevice(context_device(ctx)))
        return record_error(WQC_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    const int rpad = oz_rpad(int(m)), npad = oz_npad(int(n)), kpad = oz_kpad(int(k));
    const size_t bytes_a = size_t(m) * k * sizeof(double2), bytes_b = size_t(k) * n * sizeof(double2),
                 bytes_c = size_t(m) * n * sizeof(double2), bytes_p = oz_planes_bytes(1, rpad, npad, kpad);
    const size_t need = bytes_a + bytes_b + bytes_c + bytes_p + 256;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return record_error(WQC_ERR_CUDA, "cudaMemGetInfo");
    if (need > fr) return record_oom(need, fr);

    void *dA = nullptr, *dB = nullptr, *dC = nullptr, *dP = nullptr, *dSt = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto release = [&] {
        if (s) cudaStreamSynchronize(s);
        for (void* p : {dA, dB, dC, dP, dSt})
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
        (e = cudaMalloc(&dP, bytes_p)) || (e = cudaMalloc(&dSt, 256)))
        return cuda_fail("cudaMalloc(int8-slice GEMM)", e);
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) || (e = cudaEventCreate(&e0)) ||
        (e = cudaEventCreate(&e1)))
        return cuda_fail("stream", e);
    OzPlanes P;
    if (!oz_planes_init(&P, dP, 1, rpad, npad, kpad)) {
        release();
        return record_error(WQC_ERR_CUDA, "cuTensorMapEncodeTiled refused the digit planes");
    }
    if ((e = cudaMemcpyAsync(dA, a, bytes_a, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(dB, b, bytes_b, cudaMemcpyHostToDevice, s)) || (e = cudaMemsetAsync(dSt, 0, 256, s)))
        return cuda_fail("cudaMemcpyAsync(int8-slice GEMM operands)", e);
    const int a_blocks = std::min(1184, (rpad + 7) / 8);
    const int ntiles = (int(n) + kOzTileC - 1) / kOzTileC;
    oz_prep_plain_kernel<<<a_blocks + ntiles * (kpad / kOzKBlock), 256, 0, s>>>(static_cast<const double2*>(dA),
                                                           static_cast<const double2*>(dB), int(m), int(n), int(k), P,
                                                           a_blocks);
    if ((e = cudaGetLastError())) return cuda_fail("int8-slice GEMM staging", e);
    const TcPlainArgs args{int(m), int(n), int(k), static_cast<double2*>(dC), int(n)};
    const dim3 grid(ntiles, rpad / kOzTileM, 1);
    if ((e = cudaEventRecord(e0, s))) return cuda_fail("cudaEventRecord", e);
    for (uint32_t r = 0; r < reps; ++r)
        if ((e = launch_oz_plain(P, grid, s, args, static_cast<int*>(dSt)))) return cuda_fail("int8-slice GEMM launch", e);
    if ((e = cudaEventRecord(e1, s))) return cuda_fail("cudaEventRecord", e);
    int status = 0;
    if ((e = cudaMemcpyAsync(c, dC, bytes_c, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(&status, dSt, sizeof(int), cudaMemcpyDeviceToHost, s)) || (e = cudaStreamSynchronize(s)))
        return cuda_fail("int8-slice GEMM", e);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (kernel_ms) *kernel_ms = double(ms) / reps;
    release();
    if (status & kStatusDeviceTimeout)
        return record_error(WQC_ERR_DEVICE_TIMEOUT, "int8-slice GEMM gave up waiting on its operands");
    return WQC_OK;
}

}  // extern "C"
