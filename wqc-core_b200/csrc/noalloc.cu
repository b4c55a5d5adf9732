// wqc_expectation_pauli_noalloc: Pauli expectation values of an MPS that the
// caller keeps in its own device memory, computed without allocating any.
//
// Some callers cannot let a library call cudaMalloc.  A host that owns the
// GPU's memory through its own allocator (a PyTorch process whose caching
// allocator has reserved most of HBM, or a service that carves a fixed
// budget per tenant out of the device up front) may see cudaMalloc fail
// although its own pool has room, and cudaFree synchronises the whole device,
// stalling the caller's other streams.  Such a caller passes its inputs and
// outputs, and this entry point takes its working memory from one fixed
// array in this file instead.
//
// The scratch array is g_noalloc_scratch below: 16 MiB of transfer-matrix
// workspace plus 128 KiB for the bond dimensions, the labels and the
// per-term results of one launch.  Every GPU on which this library's code
// for this file is loaded holds it until the process exits.  Host code may
// not use the array's name as a device address (on the host it names a
// stand-in object), so the first call on each device looks the address up
// with cudaGetSymbolAddress while that device is current, and passes it to
// the kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/wqc_cuda.h"
#include "common.cuh"

namespace wqc {
wqc_status record_error(wqc_status code, const std::string& msg);  // executor.cu
}

using namespace wqc;

namespace {

constexpr int kNaMaxBond = 256;     // largest bond dimension accepted
constexpr int kNaMaxQubits = 1024;  // longest label accepted
constexpr int kNaMaxTermsPerLaunch = 64;
constexpr int kNaMaxDevices = 64;
constexpr size_t kNaResultsOffset = 0;                // double2 per term of a launch
constexpr size_t kNaDimsOffset = 1024;                // int32 right bond per site
constexpr size_t kNaLabelsOffset = 8192;              // one label per term of a launch
constexpr size_t kNaHeaderBytes = size_t(128) << 10;  // holds the three above
constexpr size_t kNaEnvBytes = size_t(16) << 20;      // 4 terms at bond 256
constexpr size_t kNaScratchBytes = kNaHeaderBytes + kNaEnvBytes;
static_assert(kNaResultsOffset + kNaMaxTermsPerLaunch * sizeof(double2) <= kNaDimsOffset, "results overlap dims");
static_assert(kNaDimsOffset + kNaMaxQubits * sizeof(int) <= kNaLabelsOffset, "dims overlap labels");
static_assert(kNaLabelsOffset + size_t(kNaMaxTermsPerLaunch) * kNaMaxQubits <= kNaHeaderBytes, "labels overflow");
static_assert(4 * size_t(kNaMaxBond) * kNaMaxBond * sizeof(double2) <= kNaEnvBytes, "one term must fit");

static __device__ __align__(256) double2 g_noalloc_scratch[kNaScratchBytes / sizeof(double2)];

std::mutex g_setup_mu;
void* g_scratch_addr[kNaMaxDevices] = {};

// Device address of g_noalloc_scratch on `device`, which must be current.
// Looked up once per device; the first lookup may load this file's device
// code onto that GPU.
wqc_status scratch_address(int device, char** out) {
    if (device < 0 || device >= kNaMaxDevices)
        return record_error(WQC_ERR_INVALID, "device " + std::to_string(device) + " is beyond the " +
                                                 std::to_string(kNaMaxDevices) + " devices this entry point serves");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_addr[device]) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return record_error(WQC_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_scratch_addr[device] = ptr;
    }
    *out = static_cast<char*>(g_scratch_addr[device]);
    return WQC_OK;
}

// <psi|P_t|psi> by transfer matrices, one CTA per term: the computation of
// pauli_expectation_kernel (site_kernels.cu) on sites that the caller packs
// at a fixed stride, with the bond dimensions, labels, environments and
// results all in the scratch array that `scratch` points to.
__global__ void __launch_bounds__(256) pauli_expectation_noalloc_kernel(const double2* sites, size_t stride, int n,
                                                                        int nterms, char* scratch, int env_cap) {
    const int t = blockIdx.x;
    if (t >= nterms) return;
    double2* results = reinterpret_cast<double2*>(scratch + kNaResultsOffset);
    const int* dr = reinterpret_cast<const int*>(scratch + kNaDimsOffset);
    const char* lab = scratch + kNaLabelsOffset + size_t(t) * n;
    const size_t E = size_t(env_cap) * env_cap;
    double2* env = reinterpret_cast<double2*>(scratch + kNaHeaderBytes) + size_t(t) * 4 * E;
    double2* nxt = env + E;
    double2* tmp = env + 2 * E;  // [l_bra][s][r], up to env_cap * 2 * env_cap
    if (threadIdx.x == 0) env[0] = cmake(1.0, 0.0);
    __syncthreads();
    int lk = 1;
    for (int q = 0; q < n; ++q) {
        const int l = q == 0 ? 1 : dr[q - 1], r = dr[q];
        const double2* s = sites + size_t(q) * stride;
        const char ch = lab[n - 1 - q];
        for (long e = threadIdx.x; e < long(lk) * 2 * r; e += blockDim.x) {
            const int lp = int(e / (2 * r)), rem = int(e % (2 * r));
            double2 acc = cmake(0, 0);
            for (int a = 0; a < min(lk, l); ++a) cfma(acc, env[size_t(a) * lk + lp], s[size_t(a) * 2 * r + rem]);
            tmp[e] = acc;
        }
        __syncthreads();
        for (long e = threadIdx.x; e < long(r) * r; e += blockDim.x) {
            const int b = int(e / r), bp = int(e % r);
            double2 acc = cmake(0, 0);
            for (int lp = 0; lp < min(lk, l); ++lp) {
                const double2 t0 = tmp[(size_t(lp) * 2 + 0) * r + b];
                const double2 t1 = tmp[(size_t(lp) * 2 + 1) * r + b];
                const double2 k0 = s[(size_t(lp) * 2 + 0) * r + bp];
                const double2 k1 = s[(size_t(lp) * 2 + 1) * r + bp];
                double2 y0, y1;
                if (ch == 'X') { y0 = t1; y1 = t0; }
                else if (ch == 'Y') { y0 = cmake(t1.y, -t1.x); y1 = cmake(-t0.y, t0.x); }
                else if (ch == 'Z') { y0 = t0; y1 = cmake(-t1.x, -t1.y); }
                else { y0 = t0; y1 = t1; }
                cfma_conj(acc, k0, y0);
                cfma_conj(acc, k1, y1);
            }
            nxt[e] = acc;
        }
        __syncthreads();
        double2* sw = env;
        env = nxt;
        nxt = sw;
        lk = r;
    }
    if (threadIdx.x == 0) results[t] = env[0];
}

wqc_status cuda_fail(const char* what, cudaError_t e) {
    return record_error(WQC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" wqc_status wqc_expectation_pauli_noalloc(const double* sites, uint64_t site_stride,
                                                    const uint32_t* bond_dims, uint32_t qubit_count,
                                                    const char* labels, const double* coeffs, uint32_t nterms,
                                                    void* stream, double out[2]) {
    if (!out || !bond_dims || (nterms > 0 && (!labels || !coeffs)))
        return record_error(WQC_ERR_INVALID, "null argument");
    if (qubit_count == 0) return record_error(WQC_ERR_INVALID_QUBIT_COUNT, "qubit_count must be at least 1");
    if (qubit_count > uint32_t(kNaMaxQubits))
        return record_error(WQC_ERR_INVALID_QUBIT_COUNT,
                            "qubit_count " + std::to_string(qubit_count) + " exceeds the maximum of " +
                                std::to_string(kNaMaxQubits) + " of the allocation-free expectation");
    int env_cap = 1;
    for (uint32_t q = 0; q < qubit_count; ++q) {
        const uint32_t l = q == 0 ? 1 : bond_dims[q - 1], r = bond_dims[q];
        if (r == 0 || r > uint32_t(kNaMaxBond))
            return record_error(WQC_ERR_INVALID, "bond dimension " + std::to_string(r) + " at site " +
                                                     std::to_string(q) + " is outside 1.." +
                                                     std::to_string(kNaMaxBond) +
                                                     " of the allocation-free expectation");
        if (uint64_t(l) * 2 * r > site_stride)
            return record_error(WQC_ERR_INVALID, "site " + std::to_string(q) + " of shape " + std::to_string(l) +
                                                     "x2x" + std::to_string(r) + " does not fit the site stride " +
                                                     std::to_string(site_stride));
        env_cap = std::max(env_cap, int(r));
    }
    // The transfer-matrix recursion ends on the right environment's (0, 0)
    // entry, which is the expectation only for a closed chain.
    if (bond_dims[qubit_count - 1] != 1)
        return record_error(WQC_ERR_INVALID, "the last site's right bond is " +
                                                 std::to_string(bond_dims[qubit_count - 1]) +
                                                 "; the allocation-free expectation needs a closed chain (1)");
    for (size_t i = 0; i < size_t(nterms) * qubit_count; ++i) {
        const char ch = labels[i];
        if (ch != 'I' && ch != 'X' && ch != 'Y' && ch != 'Z')
            return record_error(WQC_ERR_INVALID, "invalid pauli character in label");
    }
    if (!sites) return record_error(WQC_ERR_INVALID, "null argument");
    if (reinterpret_cast<uintptr_t>(sites) % alignof(double2) != 0)
        return record_error(WQC_ERR_INVALID, "sites must be 16-byte aligned");
    if (nterms == 0) {
        out[0] = out[1] = 0;
        return WQC_OK;
    }

    int device = -1;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return record_error(WQC_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    cudaPointerAttributes attr{};
    e = cudaPointerGetAttributes(&attr, sites);
    if (e != cudaSuccess) return cuda_fail("cudaPointerGetAttributes(sites)", e);
    if ((attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) || attr.device != device)
        return record_error(WQC_ERR_INVALID, "sites is not device memory of the current device " +
                                                 std::to_string(device));
    char* scratch = nullptr;
    if (wqc_status s = scratch_address(device, &scratch)) return s;

    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    // Every call waits for its results on the host (cudaStreamSynchronize
    // below), which a stream under capture does not allow.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) return cuda_fail("cudaStreamIsCapturing", e);
    if (cap != cudaStreamCaptureStatusNone)
        return record_error(WQC_ERR_INVALID, "the allocation-free expectation is synchronous and cannot be called "
                                             "while its stream is being captured");
    const size_t per_term = 4 * size_t(env_cap) * env_cap * sizeof(double2);
    const int chunk = int(std::min<size_t>(kNaMaxTermsPerLaunch, kNaEnvBytes / per_term));
    int dims[kNaMaxQubits];
    for (uint32_t q = 0; q < qubit_count; ++q) dims[q] = int(bond_dims[q]);
    e = cudaMemcpyAsync(scratch + kNaDimsOffset, dims, qubit_count * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail("cudaMemcpyAsync(bond dims)", e);

    double2 vals[kNaMaxTermsPerLaunch];
    double re = 0, im = 0;
    for (uint32_t first = 0; first < nterms; first += uint32_t(chunk)) {
        const int count = int(std::min<uint32_t>(uint32_t(chunk), nterms - first));
        e = cudaMemcpyAsync(scratch + kNaLabelsOffset, labels + size_t(first) * qubit_count,
                            size_t(count) * qubit_count, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_fail("cudaMemcpyAsync(labels)", e);
        // The results of an earlier call are still in the array: clear them so
        // that nothing of that call can be read back as this call's.
        e = cudaMemsetAsync(scratch + kNaResultsOffset, 0, kNaMaxTermsPerLaunch * sizeof(double2), st);
        if (e != cudaSuccess) return cuda_fail("cudaMemsetAsync(results)", e);
        pauli_expectation_noalloc_kernel<<<count, 256, 0, st>>>(reinterpret_cast<const double2*>(sites),
                                                                size_t(site_stride), int(qubit_count), count,
                                                                scratch, env_cap);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail("pauli_expectation_noalloc_kernel", e);
        e = cudaMemcpyAsync(vals, scratch + kNaResultsOffset, size_t(count) * sizeof(double2),
                            cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) return cuda_fail("cudaMemcpyAsync(results)", e);
        e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail("cudaStreamSynchronize", e);
        for (int t = 0; t < count; ++t) {  // coeff * Re<P>, summed in term order
            const double v = vals[t].x;
            re += coeffs[2 * (first + t)] * v;
            im += coeffs[2 * (first + t) + 1] * v;
        }
    }
    out[0] = re;
    out[1] = im;
    return WQC_OK;
}
