// PTX building blocks of the tcgen05 GEMMs (tc_gemm.cu, tc_ozaki.cu):
// mbarriers with bounded waits, 3-D TMA loads, shared-memory matrix
// descriptors, MMA completion, tensor-memory loads.  Device code only.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace wqc {
namespace ptx {

constexpr unsigned long long kWaitNs = 1000000000ull;  // 1 s per mbarrier wait

static __device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

static __device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

static __device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

static __device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

static __device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait until the phase of parity `parity` has completed; false after kWaitNs
// (or an iteration bound) without it.
static __device__ inline bool mbar_wait(uint32_t bar, uint32_t parity) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (int i = 0; i < (1 << 26); ++i) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 63) == 63 && globaltimer_ns() - t0 > kWaitNs) return false;
    }
    return false;
}

// 3-D tiled TMA load of one box into shared memory, completing on `bar`.
static __device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z,
                                                   uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
            "r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

// Shared-memory matrix descriptor of a K-major operand tile whose rows are
// `row_bytes` long (128 with the 128-byte swizzle, layout type 2; 64 with the
// 64-byte swizzle, layout type 4): 8-row groups 8 * row_bytes apart (stride
// byte offset), leading byte offset unused by these layouts (1), descriptor
// version 1 (bits 46-47), layout type at bits 61-63.
template <int kRowBytes>
static __device__ __forceinline__ uint64_t umma_desc_kmajor(uint32_t addr) {
    static_assert(kRowBytes == 128 || kRowBytes == 64, "128- or 64-byte swizzle");
    constexpr uint64_t layout = kRowBytes == 128 ? 2 : 4;
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t(1) << 16) | (uint64_t((8 * kRowBytes) >> 4) << 32) |
           (uint64_t(1) << 46) | (layout << 61);
}

// Arrive on `bar` once every tcgen05 operation this thread issued so far has
// completed.
static __device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// Sixteen 32-bit tensor-memory columns of this thread's lane, from `taddr`.
static __device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

static __device__ __forceinline__ void tmem_alloc(uint32_t slot_smem, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_smem), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

static __device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

static __device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
static __device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

}  // namespace ptx
}  // namespace wqc
