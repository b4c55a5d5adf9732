// Host side of the cuda MPS backend: the C ABI of include/wqc_cuda.h.
//
// A gate list is expanded into the reference's MpsState operations (one-qubit
// applies and adjacent two-site splits, with SWAP routing and the CCNOT
// decomposition of src/tn/mps.rs:353-375, 657-677), scheduled into levels so
// that splits on disjoint sites share a wave, and enqueued on the state's
// stream without waiting for the device.  Bond dimensions live on the device;
// the host only tracks upper bounds to size launches.
#include <cuda_runtime.h>

#include <sys/stat.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/wqc_cuda.h"
#include "common.cuh"
#include "split_kernels.cuh"
#include "tc_gemm.cuh"

using namespace wqc;

namespace {

thread_local std::string g_err;
// Byte counts of the last WQC_ERR_OOM on this thread, for
// EngineError::InsufficientMemory { required, available } (src/engine.rs:72).
thread_local uint64_t g_oom_required = 0, g_oom_available = 0;

wqc_status fail(wqc_status code, const std::string& msg) {
    g_err = msg;
    return code;
}

wqc_status fail_oom(uint64_t required, uint64_t available) {
    g_oom_required = required;
    g_oom_available = available;
    return fail(WQC_ERR_OOM, "Insufficient memory: need " + std::to_string(required) + " bytes, only " +
                                 std::to_string(available) + " bytes free on the device");
}

#define CUDA_TRY(expr)                                                                                    \
    do {                                                                                                  \
        cudaError_t e_ = (expr);                                                                          \
        if (e_ != cudaSuccess) return fail(WQC_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr int kMaxSweeps = 60;
constexpr int kDenseMaxQubits = 28;  // 2^28 complex128 = 4 GiB on the host
constexpr size_t kSlotBudget = size_t(1) << 30;  // split workspace per chi_max bucket
constexpr size_t kSmemLimit = 232448 - 1024;  // 227 KB opt-in per block, minus static shared memory

struct Mat2 {
    double2 u[4];  // row-major
};
struct Mat4 {
    double2 u[16];  // [c_out][t_out][c_in][t_in] flattened: ((co*2+to)*2+ci)*2+ti
};

double2 C(double r, double i = 0.0) { return make_double2(r, i); }

// src/tn/gates.rs:10-66 and mps.rs:1173-1180.
Mat2 unary_matrix(int kind, double theta) {
    const double r2 = 0.70710678118654752440;
    switch (kind) {
        case WQC_GATE_H: {
            const double k = 1.0 / std::sqrt(2.0);
            return {{C(k), C(k), C(k), C(-k)}};
        }
        case WQC_GATE_X: return {{C(0), C(1), C(1), C(0)}};
        case WQC_GATE_Y: return {{C(0), C(0, -1), C(0, 1), C(0)}};
        case WQC_GATE_Z: return {{C(1), C(0), C(0), C(-1)}};
        case WQC_GATE_S: return {{C(1), C(0), C(0), C(0, 1)}};
        case WQC_GATE_T: return {{C(1), C(0), C(0), C(r2, r2)}};
        case WQC_GATE_RX: {
            const double s = std::sin(theta / 2.0), c = std::cos(theta / 2.0);
            return {{C(c), C(0, -s), C(0, -s), C(c)}};
        }
        case WQC_GATE_RY: {
            const double s = std::sin(theta / 2.0), c = std::cos(theta / 2.0);
            return {{C(c), C(-s), C(s), C(c)}};
        }
        default: {  // RZ
            const double s = std::sin(theta / 2.0), c = std::cos(theta / 2.0);
            return {{C(c, -s), C(0), C(0), C(c, s)}};
        }
    }
}
Mat2 tdg_matrix() {
    const double r2 = 0.70710678118654752440;
    return {{C(1), C(0), C(0), C(r2, -r2)}};
}
int i4(int co, int to, int ci, int ti) { return ((co * 2 + to) * 2 + ci) * 2 + ti; }
Mat4 cnot_matrix() {
    Mat4 m{};
    m.u[i4(0, 0, 0, 0)] = C(1);
    m.u[i4(0, 1, 0, 1)] = C(1);
    m.u[i4(1, 0, 1, 1)] = C(1);
    m.u[i4(1, 1, 1, 0)] = C(1);
    return m;
}
Mat4 cz_matrix() {
    Mat4 m{};
    m.u[i4(0, 0, 0, 0)] = C(1);
    m.u[i4(0, 1, 0, 1)] = C(1);
    m.u[i4(1, 0, 1, 0)] = C(1);
    m.u[i4(1, 1, 1, 1)] = C(-1);
    return m;
}
Mat4 swap_matrix() {
    Mat4 m{};
    m.u[i4(0, 0, 0, 0)] = C(1);
    m.u[i4(0, 1, 1, 0)] = C(1);
    m.u[i4(1, 0, 0, 1)] = C(1);
    m.u[i4(1, 1, 1, 1)] = C(1);
    return m;
}
Mat2 adjoint2(const Mat2& a) {
    return {{make_double2(a.u[0].x, -a.u[0].y), make_double2(a.u[2].x, -a.u[2].y),
             make_double2(a.u[1].x, -a.u[1].y), make_double2(a.u[3].x, -a.u[3].y)}};
}
Mat4 adjoint4(const Mat4& a) {
    Mat4 o{};
    for (int co = 0; co < 2; ++co)
        for (int to = 0; to < 2; ++to)
            for (int ci = 0; ci < 2; ++ci)
                for (int ti = 0; ti < 2; ++ti) {
                    const double2 v = a.u[i4(ci, ti, co, to)];
                    o.u[i4(co, to, ci, ti)] = make_double2(v.x, -v.y);
                }
    return o;
}

// Effective 4x4 acting on theta[a][s][t][b] (mps.rs:396-421, split.rs:808-831).
void effective(const Mat4& u, bool ctrl_is_first, double2* out) {
    for (int so = 0; so < 2; ++so)
        for (int to = 0; to < 2; ++to)
            for (int si = 0; si < 2; ++si)
                for (int ti = 0; ti < 2; ++ti) {
                    const int co = ctrl_is_first ? so : to, tgo = ctrl_is_first ? to : so;
                    const int ci = ctrl_is_first ? si : ti, tgi = ctrl_is_first ? ti : si;
                    out[(so * 2 + to) * 4 + si * 2 + ti] = u.u[i4(co, tgo, ci, tgi)];
                }
}

struct Op {
    bool two;
    int site;        // 1q: site; 2q: left site (global site index)
    int slice = 0;   // batch slice the operation belongs to
    int gate = -1;   // index of the gate (in the caller's list) this operation comes from
    Mat2 m2;
    double2 ueff[16];
};

// Launch shape of one Jacobi phase for a group of jobs.
struct PhaseCfg {
    int C = 0;            // cluster size
    size_t smem = 0;
    int threads = 0;      // one warp per column pair of a block, at most kJacobiThreads
    bool staged = false;  // jacobi_staged_kernel with blocks of b columns
    bool reg = false;     // cluster Jacobi variant with register-resident top columns
    int b = 0;
};

// Jobs of one wave whose SVDs share launch shapes: one phase in the plain
// form; the complex64 first phase and the FP64 finish in the precision form.
struct Group {
    int mode, idx_off, count;
    int nph = 1;
    PhaseCfg ph[2];
};

struct Wave {
    int oq_off = 0, oq_count = 0;  // OneQubitOp entries
    int jobs_off = 0, njobs = 0;   // SplitJob entries
    int max_dl = 1, max_dr = 1, max_rows = 2, max_cols = 2, max_ell = 1;
    bool any_rsvd = false;
    std::vector<Group> groups;
};

struct Arena {
    void* d = nullptr;
    size_t cap = 0;
};

}  // namespace

struct wqc_cuda_ctx {
    int device = 0;
    int sm_count = 0;
    int max_cluster = 8;
    std::mutex mu;
    // Jacobi cluster sizes measured by wqc_cuda_autotune, by working-matrix
    // shape (M x N, rows stored per column, bytes per complex entry) and by
    // kind of wave (one latency-bound split, or a throughput-bound batch).
    struct Tuned {
        int M, N, len, elem, throughput, C;
    };
    std::vector<Tuned> tuned;
    int force_C = 0;  // set by the tuner while it measures one cluster size
};

struct wqc_mps {
    wqc_cuda_ctx* ctx = nullptr;
    int n = 0, chi = 0;
    bool reject = false;
    bool exact_only = false;  // WQC_SPLIT_RULE_EXACT
    bool fp32 = false;        // WQC_PRECISION_FP32 or _TF32X3: complex64 Jacobi columns
    // WQC_PRECISION_TF32X3: merges on the tensor cores (tc_gemm.cu), their
    // operands staged per wave job as TF32 hi/lo planes under two tensor maps
    bool tc = false;
    float* tc_a = nullptr;
    float* tc_b = nullptr;
    int tc_rpad = 0, tc_npad = 0, tc_kpad = 0;
    CUtensorMap tc_map_a{}, tc_map_b{};
    // WQC_MERGE_TC_INT8 (wqc_mps_set_merge): merges from int8 digit slices
    // on the tensor cores (tc_ozaki.cu), staged per wave job
    bool oz = false;
    void* oz_pool = nullptr;
    size_t oz_bytes = 0;
    OzPlanes oz_planes;
    bool batch = false;       // made by wqc_batch_create: Jacobi clusters sized for throughput
    cudaStream_t stream = nullptr;
    // Second stream of a wave: the exact-path SVDs run there while the range
    // finder runs on `stream`; fork after the merge, join before the absorb.
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    // device state
    double2* site_pool = nullptr;
    std::vector<double2*> site_ptr;  // device address of every site (capacity chi_slice * 2 * chi_slice)
    DeviceMps dev{};
    double2** d_site_ptr = nullptr;
    int* d_dl = nullptr;
    int* d_dr = nullptr;
    int* d_status = nullptr;
    volatile int* h_cancel = nullptr;  // mapped pinned
    int* d_cancel = nullptr;
    // split workspace
    int nslots = 0;
    // Slots come in buckets, one per distinct chi_max of the slices, each
    // slot sized for its bucket's largest two-site matrix (R = 2 chi_max).
    std::vector<int> bucket_chi, bucket_base, bucket_cap;
    std::vector<int> slot_R, slot_E;
    int bucket_of(int chi) const {
        for (size_t b = 0; b < bucket_chi.size(); ++b)
            if (bucket_chi[b] == chi) return int(b);
        return 0;
    }
    char* slot_pool = nullptr;
    SlotBuffers* d_slots = nullptr;
    SplitState* d_state = nullptr;
    // per-call plan
    char* h_stage = nullptr;
    size_t h_stage_cap = 0;
    cudaEvent_t stage_done = nullptr;
    Arena d_stage;
    wqc_split_info* d_records = nullptr;
    size_t rec_cap = 0;
    uint32_t rec_count = 0;
    double2* d_small = nullptr;  // results of amplitude / site kernels
    unsigned long long* d_counters = nullptr;  // Jacobi tasks, Jacobi sweeps
    // host bounds: ub[i] = upper bound of the bond between sites i and i+1
    std::vector<int> ub;
    // slices: a single state is one slice; a batch concatenates its slices'
    // sites, and no split ever crosses a slice boundary
    std::vector<int> seg_first, seg_n, seg_chi;
    std::vector<int> site_chi, site_slice;
    int* d_seg = nullptr;  // (first, count) per slice for the amplitude kernel
    // per-slice completion times of the last call (batch, profiling on)
    std::vector<int> slice_last_wave;
    std::vector<cudaEvent_t> wave_done;
    cudaEvent_t call_start = nullptr;
    // Cached environments of the trace feeders (single states): L_0..L_lvalid
    // and R_rvalid..R_{n-1} are current; an operation on sites [a, b] leaves
    // lvalid <= a and rvalid >= b.
    double2* d_envL = nullptr;
    double2* d_envR = nullptr;
    int* d_targets = nullptr;     // targets of one wqc_mps_site_amplitudes_many call
    double2* d_env_out = nullptr; // its (a0, a1) pairs
    int lvalid = 0, rvalid = 0;
    void touch(int a, int b) {
        lvalid = std::min(lvalid, a);
        rvalid = std::max(rvalid, b);
    }
    // Set by wqc_mps_upload_site: the bonds of the chain are checked once
    // before the next call that computes on it.
    bool uploaded = false;
    // accounting
    uint64_t bytes_now = 0, bytes_peak = 0;
    bool profiling = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> events;
    std::vector<cudaEvent_t> event_pool;
    wqc_kernel_stats stats{};

    int left_bond(int site) const { return site == 0 ? 1 : ub[site - 1]; }
    int right_bond(int site) const { return site + 1 >= n ? 1 : ub[site]; }
};

namespace {

wqc_status dmalloc(wqc_mps* m, void** p, size_t bytes);

// Digit planes of the int8-slice merges for every split slot of the state.
size_t oz_state_bytes(const wqc_mps* m) {
    return oz_planes_bytes(m->nslots, oz_rpad(2 * m->chi), oz_npad(2 * m->chi), oz_kpad(m->chi));
}

}  // namespace

// Merges from int8 digit slices from now on: allocate the digit planes of
// every split slot the first time (WQC_ERR_OOM if they do not fit).
static wqc_status oz_enable(wqc_mps* m) {
    if (!m->oz_pool) {
        const int rpad = oz_rpad(2 * m->chi), npad = oz_npad(2 * m->chi), kpad = oz_kpad(m->chi);
        const size_t bytes = oz_state_bytes(m);
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return fail(WQC_ERR_CUDA, "cudaMemGetInfo");
        if (bytes > fr) return fail_oom(bytes, fr);
        void* p = nullptr;
        if (wqc_status st = dmalloc(m, &p, bytes)) return st;
        if (!oz_planes_init(&m->oz_planes, p, m->nslots, rpad, npad, kpad)) {
            cudaFree(p);
            m->bytes_now -= bytes;
            return fail(WQC_ERR_CUDA, "cuTensorMapEncodeTiled refused the merge digit planes");
        }
        m->oz_pool = p;
        m->oz_bytes = bytes;
    }
    m->oz = true;
    return WQC_OK;
}

namespace {

wqc_status dmalloc(wqc_mps* m, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        return fail_oom(bytes, fr);
    }
    m->bytes_now += bytes;
    m->bytes_peak = std::max(m->bytes_peak, m->bytes_now);
    return WQC_OK;
}
void dfree(wqc_mps* m, void* p, size_t bytes) {
    if (!p) return;
    cudaFree(p);
    m->bytes_now -= bytes;
}

std::once_flag g_attr_once;
cudaError_t g_attr_err = cudaSuccess;

void set_kernel_attributes() {
    for (const void* f : {jacobi_kernel(false, false), jacobi_kernel(true, false), jacobi_kernel(false, true),
                          jacobi_kernel(true, true), jacobi_staged(false), jacobi_staged(true)}) {
        if (g_attr_err == cudaSuccess)
            g_attr_err = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemLimit));
        if (g_attr_err == cudaSuccess)
            g_attr_err = cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    }
    for (const void* f : {qr_cluster(false), qr_cluster(true)}) {
        if (g_attr_err == cudaSuccess)
            g_attr_err = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemLimit));
        if (g_attr_err == cudaSuccess)
            g_attr_err = cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    }
    if (g_attr_err == cudaSuccess)
        g_attr_err = cudaFuncSetAttribute(amplitude_zero_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
}

int round_up(int x, int q) { return ((x + q - 1) / q) * q; }

// Cluster size for a Jacobi SVD of an M x N working matrix.  Every sweep has
// N'-1 steps (N' = N padded to a multiple of 4C) whatever C is; a larger C
// gives each CTA fewer column pairs per step (b = N'/2C) but adds 2C-1 block
// exchanges per sweep.  The model below (FP64 work per step and CTA, a floor
// for one pair's latency, a fixed cost per exchange plus its DSMEM traffic)
// picks the fastest sweep when the wave's splits cannot fill the GPU, and the
// least SM-time per split when they can.
// Cluster size of a Jacobi group, from clock64 measurements of the kernel.
// A single state is latency-bound (a few splits per level): a round costs
// its shared-memory traffic at 64 B/clk (at least ~0.3 us) and a block
// exchange ~2 us plus its DSMEM stores; blocks wider than the register
// variant's 12 warps are not considered for columns it can hold, and once
// the wave's clusters would fill the GPU the cost counts SM time.  A batch
// is throughput-bound (its waves fill the GPU), so SM time (sweep time x C)
// decides for every wave, with the round cost of the variant that runs it:
// the dependent rotation chain (~1900 cycles with the top column in
// registers, ~1300 without) or 3 or 6 passes of the partner columns at
// 128 B/clk, whichever is larger, and ~4600 cycles per exchange.  That
// choice depends on the shape alone, so a slice's results do not depend on
// the other slices of its batch.
bool jacobi_reg_variant(int M, int b) { return M <= kJacobiRegMaxRows && b <= kJacobiRegThreads / 32; }

// len: rows stored per column (M, or M + N when the precision form's first
// phase carries V).
int choose_cluster(const wqc_cuda_ctx* ctx, int M, int N, int max_c, int njobs, int sm_count, size_t elem,
                   bool throughput, int len = 0) {
    if (len <= 0) len = M;
    if (ctx) {
        auto fits = [&](int Cc) { return Cc >= 1 && Cc <= max_c && jacobi_smem_bytes(len, N, Cc, elem) <= kSmemLimit; };
        if (ctx->force_C > 0 && fits(ctx->force_C)) return ctx->force_C;
        for (const auto& t : ctx->tuned)
            if (t.M == M && t.N == N && t.len == len && t.elem == int(elem) && t.throughput == int(throughput) &&
                fits(t.C))
                return t.C;
    }
    int best = -1;
    double best_cost = 1e300;
    for (int Cc = 1; Cc <= max_c; ++Cc) {
        if (jacobi_smem_bytes(len, N, Cc, elem) > kSmemLimit) continue;
        const int Np = round_up(N, 4 * Cc), b = Np / (2 * Cc);
        const int max_b = throughput ? kJacobiThreads / 32 : jacobi_max_warps(M);
        if (b > max_b && Cc < max_c) continue;  // more pairs than warps
        double cost;
        if (throughput) {
            const bool reg = jacobi_reg_variant(M, b);
            const double traffic = (reg ? 3.0 : 6.0) * double(elem) * b * len / 128.0;
            const double round = std::max(reg ? 1900.0 : 1300.0, traffic);
            const double cycles = Np * round + (Cc > 1 ? (2 * Cc - 1) * 4600.0 : 0.0);
            cost = cycles / 1900.0 * Cc;  // SM-microseconds at ~1.9 GHz
        } else {
            const double step = std::max(0.3, b * (8.0 * M + 12.0 * len) / 64.0 / 1900.0);
            const double exch = Cc > 1 ? 2.0 + 2.0 * b * len * 16.0 / 1.0e5 : 0.0;
            cost = (Np - 1) * step + (2 * Cc - 1) * exch;
            if (double(njobs) * Cc >= 1.5 * sm_count) cost *= Cc;
        }
        if (cost < best_cost) {
            best_cost = cost;
            best = Cc;
        }
    }
    return best;
}

cudaEvent_t get_event(wqc_mps* m) {
    if (!m->event_pool.empty()) {
        cudaEvent_t e = m->event_pool.back();
        m->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

struct Timed {
    wqc_mps* m;
    int kind;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t s;
    Timed(wqc_mps* mm, int k, cudaStream_t on = nullptr) : m(mm), kind(k), s(on ? on : mm->stream) {
        if (m->profiling) {
            a = get_event(m);
            b = get_event(m);
            cudaEventRecord(a, s);
        }
    }
    ~Timed() {
        if (m->profiling) {
            cudaEventRecord(b, s);
            m->events.push_back({kind, {a, b}});
        }
    }
};

void count_launch(wqc_mps* m, int kind) {
    m->stats.total_launches++;
    if (kind >= 0) m->stats.launches[kind]++;
}

// ---------------------------------------------------------------------------
// Expansion of gates into MpsState operations.
// ---------------------------------------------------------------------------
struct Expander {
    std::vector<Op> ops;
    int cur = -1;  // gate being expanded
    void one(int q, const Mat2& u) {
        Op o{};
        o.two = false;
        o.site = q;
        o.m2 = u;
        o.gate = cur;
        ops.push_back(o);
    }
    void two_at(int p, const Mat4& u, bool cf) {
        Op o{};
        o.two = true;
        o.site = p;
        o.gate = cur;
        effective(u, cf, o.ueff);
        ops.push_back(o);
    }
    void two_routed(int ctrl, int tgt, const Mat4& u) {  // mps.rs:353-375
        const int left = std::min(ctrl, tgt), right = std::max(ctrl, tgt);
        const int span = right - left;
        const Mat4 sw = swap_matrix();
        if (span > 1)
            for (int pos = right - 1; pos >= left + 1; --pos) two_at(pos, sw, true);
        two_at(left, u, ctrl < tgt);
        if (span > 1)
            for (int pos = left + 1; pos < right; ++pos) two_at(pos, sw, true);
    }
    void ccnot(int c1, int c2, int t) {  // mps.rs:657-677
        const Mat2 tdg = tdg_matrix(), h = unary_matrix(WQC_GATE_H, 0), tt = unary_matrix(WQC_GATE_T, 0);
        const Mat4 cx = cnot_matrix();
        one(t, h);
        two_routed(c2, t, cx);
        one(t, tdg);
        two_routed(c1, t, cx);
        one(t, tt);
        two_routed(c2, t, cx);
        one(t, tdg);
        two_routed(c1, t, cx);
        one(t, tt);
        one(t, h);
        one(c2, tt);
        two_routed(c1, c2, cx);
        one(c1, tt);
        one(c2, tdg);
        two_routed(c1, c2, cx);
    }
};

wqc_status check_gate(int n, const wqc_gate& g) {
    auto chk = [&](int q) -> wqc_status {
        if (q < 0 || q >= n)
            return fail(WQC_ERR_QUBIT_OUT_OF_RANGE,
                        "Qubit index " + std::to_string(q) + " out of bounds (limit: " + std::to_string(n) + ")");
        return WQC_OK;
    };
    wqc_status s = WQC_OK;
    switch (g.kind) {
        case WQC_GATE_H: case WQC_GATE_X: case WQC_GATE_Y: case WQC_GATE_Z: case WQC_GATE_S: case WQC_GATE_T:
        case WQC_GATE_RX: case WQC_GATE_RY: case WQC_GATE_RZ:
            return chk(g.q0);
        case WQC_GATE_CNOT: case WQC_GATE_CZ:
            if ((s = chk(g.q0)) || (s = chk(g.q1))) return s;
            if (g.q0 == g.q1) return fail(WQC_ERR_INVALID, "two-qubit gate on one qubit");
            return WQC_OK;
        case WQC_GATE_CCNOT:
            if ((s = chk(g.q0)) || (s = chk(g.q1)) || (s = chk(g.q2))) return s;
            if (g.q0 == g.q1 || g.q0 == g.q2 || g.q1 == g.q2) return fail(WQC_ERR_INVALID, "CCNOT needs three qubits");
            return WQC_OK;
        case WQC_GATE_MEASURE: case WQC_GATE_RESET: case WQC_GATE_IF:
            return WQC_OK;
        default:
            return fail(WQC_ERR_INVALID, "unknown gate kind " + std::to_string(g.kind));
    }
}

wqc_status expand(int n, const wqc_gate* gates, uint32_t count, bool adjoint, Expander& ex) {
    for (uint32_t i = 0; i < count; ++i) {
        const wqc_gate& g = gates[adjoint ? count - 1 - i : i];
        ex.cur = int(adjoint ? count - 1 - i : i);
        if (wqc_status s = check_gate(n, g)) return s;
        switch (g.kind) {
            case WQC_GATE_CNOT:
                ex.two_routed(g.q0, g.q1, adjoint ? adjoint4(cnot_matrix()) : cnot_matrix());
                break;
            case WQC_GATE_CZ:
                ex.two_routed(g.q0, g.q1, adjoint ? adjoint4(cz_matrix()) : cz_matrix());
                break;
            case WQC_GATE_CCNOT:
                ex.ccnot(g.q0, g.q1, g.q2);
                break;
            case WQC_GATE_MEASURE: case WQC_GATE_RESET: case WQC_GATE_IF:
                if (adjoint) return fail(WQC_ERR_INVALID, "time-split overlap does not apply measurement or reset");
                break;
            default: {
                const Mat2 u = unary_matrix(g.kind, g.angle);
                ex.one(g.q0, adjoint ? adjoint2(u) : u);
                break;
            }
        }
    }
    return WQC_OK;
}

// ---------------------------------------------------------------------------
// Plan: levels -> waves, staged in one pinned buffer and copied once.
// ---------------------------------------------------------------------------
struct Plan {
    std::vector<Wave> waves;
    std::vector<OneQubitOp> oq;
    std::vector<double2> mats;
    std::vector<SplitJob> jobs;
    std::vector<int> idx;
    std::vector<int> slice_last_wave;  // last wave holding an operation of each slice
    uint32_t first_seq = 0, nsplits = 0;
};

// Level of every operation: a split on (p, p+1) goes one level after the last
// split that touched p or p+1; a one-qubit gate goes one level after the last
// split on its site and runs before that level's splits.  Each site therefore
// sees its operations in program order, and the splits of one level touch
// disjoint sites.
void assign_levels(int n, const std::vector<Op>& ops, std::vector<int>& level_of) {
    std::vector<int> last2q(n, -1);
    level_of.resize(ops.size());
    for (size_t i = 0; i < ops.size(); ++i) {
        const Op& o = ops[i];
        if (!o.two) {
            level_of[i] = last2q[o.site] + 1;
        } else {
            const int L = std::max(last2q[o.site], last2q[o.site + 1]) + 1;
            level_of[i] = L;
            last2q[o.site] = last2q[o.site + 1] = L;
        }
    }
}

void build_plan(wqc_mps* m, const std::vector<Op>& ops, Plan& plan) {
    struct LevelBuild {
        std::vector<std::pair<int, std::vector<Mat2>>> oq;  // site -> matrices in order
        std::vector<int> oq_index;                          // site -> entry in oq (built lazily)
        std::vector<SplitJob> jobs;
        std::vector<std::pair<int, int>> bounds;  // (ub left of p, ub right of p+1) at the job
        std::vector<int> job_slice;
        std::vector<int> oq_slices;
    };
    std::vector<LevelBuild> levels;
    std::vector<int> level_of;
    assign_levels(m->n, ops, level_of);
    auto level = [&](int L) -> LevelBuild& {
        while (int(levels.size()) <= L) levels.emplace_back();
        return levels[L];
    };
    uint32_t seq = m->rec_count;
    plan.first_seq = seq;
    for (size_t oi = 0; oi < ops.size(); ++oi) {
        const Op& o = ops[oi];
        m->touch(o.site, o.two ? o.site + 1 : o.site);
        if (!o.two) {
            LevelBuild& lb = level(level_of[oi]);
            if (lb.oq_index.empty()) lb.oq_index.assign(m->n, -1);
            int& e = lb.oq_index[o.site];
            if (e < 0) {
                e = int(lb.oq.size());
                lb.oq.push_back({o.site, {}});
                lb.oq_slices.push_back(o.slice);
            }
            lb.oq[e].second.push_back(o.m2);
        } else {
            const int p = o.site;
            LevelBuild& lb = level(level_of[oi]);
            SplitJob J{};
            J.p = p;
            J.seq = int(seq++);
            J.reject = m->reject ? 1 : 0;
            J.exact_only = m->exact_only ? 1 : 0;
            J.chi_max = m->site_chi[p];
            std::memcpy(J.u, o.ueff, sizeof(J.u));
            const int bl = m->left_bond(p), br = m->right_bond(p + 1);
            lb.jobs.push_back(J);
            lb.bounds.push_back({bl, br});
            lb.job_slice.push_back(o.slice);
            m->ub[p] = std::min(std::min(2 * bl, 2 * br), J.chi_max);
        }
    }
    plan.nsplits = seq - plan.first_seq;
    plan.slice_last_wave.assign(m->seg_first.size(), -1);
    for (LevelBuild& lb : levels) {
        // one-qubit ops run first, in one wave with no splits when needed
        std::vector<char> taken(lb.jobs.size(), 0);
        size_t remaining = lb.jobs.size();
        bool first = true;
        do {
            Wave w;
            const int wave_index = int(plan.waves.size());
            if (first) {
                w.oq_off = int(plan.oq.size());
                for (auto& e : lb.oq) {
                    OneQubitOp op;
                    op.site = e.first;
                    op.first = int(plan.mats.size() / 4);
                    op.count = int(e.second.size());
                    for (const Mat2& u : e.second)
                        for (int k = 0; k < 4; ++k) plan.mats.push_back(u.u[k]);
                    plan.oq.push_back(op);
                }
                for (int sl : lb.oq_slices) plan.slice_last_wave[sl] = std::max(plan.slice_last_wave[sl], wave_index);
                w.oq_count = int(lb.oq.size());
                first = false;
            }
            // Jacobi groups: key (mode, shape of phase 1, shape of phase 2);
            // a shape is a cluster size, or -b for the staged kernel with
            // blocks of b columns.
            struct GKey {
                int mode, k1, k2;
            };
            std::vector<std::pair<GKey, std::vector<int>>> groups;
            auto add = [&](int mode, int k1, int k2, int local) {
                for (auto& g : groups)
                    if (g.first.mode == mode && g.first.k1 == k1 && g.first.k2 == k2) {
                        g.second.push_back(local);
                        return;
                    }
                groups.push_back({{mode, k1, k2}, {local}});
            };
            auto shape = [&](size_t k, int& rows, int& cols, int& ell) {
                rows = 2 * lb.bounds[k].first;
                cols = 2 * lb.bounds[k].second;
                ell = std::min(std::min(lb.jobs[k].chi_max + kRsvdOversample, rows), cols);
            };
            // Working matrix of a job in a mode: M x N, M >= N.
            auto dims = [&](size_t k, int mode, int& M, int& N) {
                int rows, cols, ell;
                shape(k, rows, cols, ell);
                M = mode != kJacobiRsvd ? std::max(rows, cols) : cols;
                N = mode != kJacobiRsvd ? std::min(rows, cols) : ell;
            };
            // The wave takes the level's next jobs while their bucket has a
            // free slot (every job of a level is independent of the others).
            std::vector<size_t> sel;
            std::vector<int> sel_slot;
            {
                std::vector<int> used(m->bucket_chi.size(), 0);
                for (size_t k = 0; k < lb.jobs.size(); ++k) {
                    if (taken[k]) continue;
                    const int bk = m->bucket_of(lb.jobs[k].chi_max);
                    if (used[bk] >= m->bucket_cap[bk]) continue;
                    taken[k] = 1;
                    sel.push_back(k);
                    sel_slot.push_back(m->bucket_base[bk] + used[bk]++);
                }
                remaining -= sel.size();
            }
            const int nj_wave = int(sel.size());
            // A shape beyond every cluster's shared memory goes to the staged
            // kernel (0: no kernel takes it).
            auto cluster_or_staged = [&](int M, int N, size_t elem, int len) {
                const int c =
                    choose_cluster(m->ctx, M, N, m->ctx->max_cluster, nj_wave, m->ctx->sm_count, elem, m->batch, len);
                return c >= 1 ? c : -jacobi_staged_b(len, N, elem, kSmemLimit, nullptr);
            };
            auto keys = [&](int M, int N, int& k1, int& k2) {
                if (m->fp32) {
                    k1 = cluster_or_staged(M, N, sizeof(float2), M + N);
                    k2 = cluster_or_staged(M, N, sizeof(double2), M);
                } else {
                    k1 = cluster_or_staged(M, N, sizeof(double2), M);
                    k2 = 0;
                }
            };
            w.jobs_off = int(plan.jobs.size());
            w.njobs = nj_wave;
            for (int local = 0; local < nj_wave; ++local) {
                const size_t k = sel[local];
                SplitJob J = lb.jobs[k];
                J.slot = sel_slot[local];
                plan.jobs.push_back(J);
                plan.slice_last_wave[lb.job_slice[k]] = std::max(plan.slice_last_wave[lb.job_slice[k]], wave_index);
                int rows, cols, ell;
                shape(k, rows, cols, ell);
                const unsigned long long f = (unsigned long long)rows * cols * ell;
                const bool rs = !m->reject && !m->exact_only && ell < std::min(rows, cols) &&
                                f >= (unsigned long long)kRsvdMinSide * kRsvdMinSide * kRsvdMinSide;
                w.max_dl = std::max(w.max_dl, lb.bounds[k].first);
                w.max_dr = std::max(w.max_dr, lb.bounds[k].second);
                w.max_rows = std::max(w.max_rows, rows);
                w.max_cols = std::max(w.max_cols, cols);
                w.max_ell = std::max(w.max_ell, ell);
                int M, N, k1, k2;
                dims(k, kJacobiExact, M, N);
                keys(M, N, k1, k2);
                add(kJacobiExact, k1, k2, local);
                if (rs) {
                    w.any_rsvd = true;
                    add(kJacobiFallback, k1, k2, local);
                    dims(k, kJacobiRsvd, M, N);
                    keys(M, N, k1, k2);
                    add(kJacobiRsvd, k1, k2, local);
                }
            }
            // Launch shape of one phase for the jobs of a group.
            auto fill = [&](PhaseCfg& pc, int key, int mode, const std::vector<int>& locals, size_t elem, bool with_v) {
                size_t sm = 0;
                int bmax = 1, mmax = 1;
                if (key < 0) {
                    pc.staged = true;
                    pc.b = -key;
                    pc.C = m->ctx->max_cluster;
                    for (int local : locals) {
                        int M, N;
                        dims(sel[local], mode, M, N);
                        sm = std::max(sm, size_t(2) * pc.b * size_t(with_v ? M + N : M) * elem);
                    }
                    pc.smem = sm;
                    pc.threads = 32 * std::min(kJacobiStagedThreads / 32, std::max(4, pc.b));
                    return;
                }
                pc.C = key;
                for (int local : locals) {
                    int M, N;
                    dims(sel[local], mode, M, N);
                    sm = std::max(sm, jacobi_smem_bytes(with_v ? M + N : M, N, std::max(pc.C, 1), elem));
                    bmax = std::max(bmax, round_up(N, 4 * std::max(pc.C, 1)) / (2 * std::max(pc.C, 1)));
                    mmax = std::max(mmax, M);
                }
                pc.smem = sm;
                // Register-resident variant when every job of the group fits it.
                pc.reg = jacobi_reg_variant(mmax, bmax);
                pc.threads = 32 * std::min((pc.reg ? kJacobiRegThreads : kJacobiThreads) / 32, std::max(2, bmax));
            };
            for (auto& g : groups) {
                Group gr;
                gr.mode = g.first.mode;
                gr.idx_off = int(plan.idx.size());
                gr.count = int(g.second.size());
                if (m->fp32) {
                    gr.nph = 2;
                    fill(gr.ph[0], g.first.k1, gr.mode, g.second, sizeof(float2), true);
                    fill(gr.ph[1], g.first.k2, gr.mode, g.second, sizeof(double2), false);
                } else {
                    gr.nph = 1;
                    fill(gr.ph[0], g.first.k1, gr.mode, g.second, sizeof(double2), false);
                }
                for (int local : g.second) plan.idx.push_back(local);
                w.groups.push_back(gr);
            }
            plan.waves.push_back(std::move(w));
        } while (remaining > 0);
    }
}

template <class T>
size_t stage_section(size_t& off, const std::vector<T>& v) {
    off = (off + 255) & ~size_t(255);
    const size_t at = off;
    off += v.size() * sizeof(T);
    return at;
}

wqc_status ensure_records(wqc_mps* m, size_t need) {
    if (need <= m->rec_cap) return WQC_OK;
    size_t cap = std::max<size_t>(need, m->rec_cap * 2 + 1024);
    void* p = nullptr;
    if (wqc_status s = dmalloc(m, &p, cap * sizeof(wqc_split_info))) return s;
    if (m->d_records) {
        CUDA_TRY(cudaStreamSynchronize(m->stream));
        CUDA_TRY(cudaMemcpy(p, m->d_records, m->rec_cap * sizeof(wqc_split_info), cudaMemcpyDeviceToDevice));
        dfree(m, m->d_records, m->rec_cap * sizeof(wqc_split_info));
    }
    m->d_records = static_cast<wqc_split_info*>(p);
    m->rec_cap = cap;
    return WQC_OK;
}

wqc_status launch_plan(wqc_mps* m, Plan& plan) {
    if (plan.waves.empty()) return WQC_OK;
    if (wqc_status s = ensure_records(m, size_t(plan.first_seq) + plan.nsplits)) return s;
    size_t off = 0;
    const size_t o_oq = stage_section(off, plan.oq);
    const size_t o_mats = stage_section(off, plan.mats);
    const size_t o_jobs = stage_section(off, plan.jobs);
    const size_t o_idx = stage_section(off, plan.idx);
    const size_t bytes = std::max<size_t>(off, 256);
    // host staging: wait for the previous copy out of it
    CUDA_TRY(cudaEventSynchronize(m->stage_done));
    if (bytes > m->h_stage_cap) {
        if (m->h_stage) cudaFreeHost(m->h_stage);
        m->h_stage = nullptr;
        CUDA_TRY(cudaHostAlloc(reinterpret_cast<void**>(&m->h_stage), bytes * 2, cudaHostAllocDefault));
        m->h_stage_cap = bytes * 2;
    }
    if (bytes > m->d_stage.cap) {
        CUDA_TRY(cudaStreamSynchronize(m->stream));
        dfree(m, m->d_stage.d, m->d_stage.cap);
        m->d_stage.d = nullptr;
        m->d_stage.cap = 0;
        if (wqc_status s = dmalloc(m, &m->d_stage.d, bytes * 2)) return s;
        m->d_stage.cap = bytes * 2;
    }
    std::memcpy(m->h_stage + o_oq, plan.oq.data(), plan.oq.size() * sizeof(OneQubitOp));
    std::memcpy(m->h_stage + o_mats, plan.mats.data(), plan.mats.size() * sizeof(double2));
    std::memcpy(m->h_stage + o_jobs, plan.jobs.data(), plan.jobs.size() * sizeof(SplitJob));
    std::memcpy(m->h_stage + o_idx, plan.idx.data(), plan.idx.size() * sizeof(int));
    CUDA_TRY(cudaMemcpyAsync(m->d_stage.d, m->h_stage, bytes, cudaMemcpyHostToDevice, m->stream));
    m->stats.h2d_bytes += bytes;
    CUDA_TRY(cudaEventRecord(m->stage_done, m->stream));
    char* dbase = static_cast<char*>(m->d_stage.d);
    const OneQubitOp* d_oq = reinterpret_cast<const OneQubitOp*>(dbase + o_oq);
    const double2* d_mats = reinterpret_cast<const double2*>(dbase + o_mats);
    const SplitJob* d_jobs_all = reinterpret_cast<const SplitJob*>(dbase + o_jobs);
    const int* d_idx = reinterpret_cast<const int*>(dbase + o_idx);

    const bool track = m->profiling && !plan.slice_last_wave.empty();
    if (track) {
        while (m->wave_done.size() < plan.waves.size()) {
            cudaEvent_t e = nullptr;
            CUDA_TRY(cudaEventCreate(&e));
            m->wave_done.push_back(e);
        }
        if (!m->call_start) CUDA_TRY(cudaEventCreate(&m->call_start));
        CUDA_TRY(cudaEventRecord(m->call_start, m->stream));
        m->slice_last_wave = plan.slice_last_wave;
    }
    for (size_t wi = 0; wi < plan.waves.size(); ++wi) {
        const Wave& w = plan.waves[wi];
        if (w.oq_count > 0) {
            Timed t(m, 3);
            const int gx = std::min(64, std::max(1, (m->chi * m->chi + 1023) / 1024));
            apply_1q_kernel<<<dim3(gx, w.oq_count), 256, 0, m->stream>>>(d_oq + w.oq_off, d_mats, m->dev);
            count_launch(m, 3);
        }
        if (w.njobs == 0) {
            if (track) CUDA_TRY(cudaEventRecord(m->wave_done[wi], m->stream));
            continue;
        }
        const SplitJob* d_jobs = d_jobs_all + w.jobs_off;
        const int nj = w.njobs;
        // The plain and precision forms end on FP64 columns of an FP64 theta:
        // no singular value is FP32 noise.  The tensor-core form's theta
        // carries FP32-level error (~1e-7 of its norm), which shows as
        // singular values of ~1e-8 of the largest where theta has none; those
        // below 1e-6 of the largest count as zero.
        const double noise_rel = m->tc ? 1e-6 : 0.0;
        {
            Timed t(m, 1);
            prepare_kernel<<<(nj + 127) / 128, 128, 0, m->stream>>>(d_jobs, m->d_state, nj, m->dev);
            count_launch(m, 1);
            if (m->oz) {
                // rows of L by warps, N tiles of R (8 values of b) by blocks
                const int a_blocks = std::max(1, (w.max_rows + 7) / 8);
                const int ntiles = (w.max_dr + 7) / 8;
                const int b_blocks = ntiles * (m->oz_planes.kpad / kOzKBlock);
                oz_prep_merge_kernel<<<dim3(a_blocks + b_blocks, nj), 256, 0, m->stream>>>(d_jobs, m->d_state, m->dev,
                                                                                           m->oz_planes, a_blocks);
                count_launch(m, 1);
                const dim3 g(ntiles, (w.max_rows + kOzTileM - 1) / kOzTileM, nj);
                CUDA_TRY(launch_oz_merge(m->oz_planes, g, m->stream, TcMergeArgs{d_jobs, m->d_state, m->d_slots},
                                         m->d_status));
                count_launch(m, 1);
            } else if (m->tc) {
                // one thread per complex value of L, one block per 32 K values of an N tile of R
                const int a_blocks = std::max(1, (w.max_rows * m->chi + 255) / 256);
                const dim3 gp(a_blocks + ((w.max_dr + 31) / 32) * (m->tc_kpad / kTcKBlock), nj);
                tc_prep_merge_kernel<<<gp, 256, 0, m->stream>>>(d_jobs, m->d_state, m->dev, m->tc_a, m->tc_b,
                                                                m->tc_rpad, m->tc_npad, m->tc_kpad, a_blocks);
                count_launch(m, 1);
                const dim3 g((w.max_dr + 31) / 32, (w.max_rows + kTcTileM - 1) / kTcTileM, nj);
                CUDA_TRY(launch_tc_merge(m->tc_map_a, m->tc_map_b, g, m->stream,
                                         TcMergeArgs{d_jobs, m->d_state, m->d_slots}, m->d_status));
                count_launch(m, 1);
            } else {
                dim3 g((w.max_dr + 15) / 16, (w.max_dl + 15) / 16, nj);
                merge_gate_kernel<<<g, 256, 0, m->stream>>>(d_jobs, m->d_state, m->d_slots, m->dev);
                count_launch(m, 1);
            }
        }
        auto launch_phase = [&](const Group& gr, const PhaseCfg& pc, int mode, int phase, bool fp32,
                                cudaStream_t on) -> wqc_status {
            if (pc.C < 1) return fail(WQC_ERR_INVALID, "two-site matrix too large for the cluster-resident Jacobi SVD");
            Timed t(m, 0, on);
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(gr.count * pc.C);
            cfg.blockDim = dim3(pc.threads);
            cfg.dynamicSmemBytes = pc.smem;
            cfg.stream = on;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = pc.C;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            if (pc.staged)
                CUDA_TRY(launch_jacobi_staged(fp32, cfg, d_jobs, m->d_state, m->d_slots, d_idx + gr.idx_off, mode, phase,
                                              kMaxSweeps, pc.b, m->d_status, m->d_counters));
            else
                CUDA_TRY(launch_jacobi(fp32, pc.reg, cfg, d_jobs, m->d_state, m->d_slots, d_idx + gr.idx_off, mode,
                                       phase, kMaxSweeps, m->d_status, m->d_counters));
            count_launch(m, 0);
            return WQC_OK;
        };
        auto jacobi = [&](int mode, cudaStream_t on) -> wqc_status {
            bool any = false;
            for (const Group& gr : w.groups) {
                if (gr.mode != mode) continue;
                any = true;
                if (gr.nph == 1) {
                    if (wqc_status s = launch_phase(gr, gr.ph[0], mode, kPhasePlain, false, on)) return s;
                } else if (wqc_status s = launch_phase(gr, gr.ph[0], mode, kPhaseFp32V, true, on)) {
                    return s;
                }
            }
            if (!any) return WQC_OK;
            if (m->fp32) {
                // V orthonormalised (two Newton-Schulz steps), X V for every job of the mode, then the FP64 finish.
                Timed t(m, 0, on);
                const int side = std::max(w.max_rows, w.max_cols);
                const dim3 g((side + 31) / 32, (side + 31) / 32, nj);
                for (int stage = 0; stage < kPrecondStages; ++stage) {
                    precond_gemm_kernel<<<g, 256, 0, on>>>(d_jobs, m->d_state, m->d_slots, mode, stage);
                    count_launch(m, 0);
                }
            }
            for (const Group& gr : w.groups)
                if (gr.mode == mode && gr.nph == 2)
                    if (wqc_status s = launch_phase(gr, gr.ph[1], mode, kPhaseFinish, false, on)) return s;
            {
                Timed t(m, 4, on);
                svd_probe_kernel<<<dim3(nj, 2), 256, 0, on>>>(d_jobs, m->d_state, m->d_slots, mode, 0, m->d_status);
                count_launch(m, 4);
            }
            return WQC_OK;
        };
        // Exact-path SVDs on the side stream, concurrently with the range
        // finder below (different jobs, different slots and records).
        const bool fork = w.any_rsvd;
        cudaStream_t xs = fork ? m->side : m->stream;
        if (fork) {
            CUDA_TRY(cudaEventRecord(m->fork_ev, m->stream));
            CUDA_TRY(cudaStreamWaitEvent(m->side, m->fork_ev, 0));
        }
        if (wqc_status s = jacobi(kJacobiExact, xs)) return s;
        {
            Timed t(m, 4, xs);
            finalize_kernel<<<nj, 256, 0, xs>>>(d_jobs, m->d_state, m->d_slots, kJacobiExact, m->chi, noise_rel,
                                                m->d_records, m->d_status);
            count_launch(m, 4);
        }
        if (fork) CUDA_TRY(cudaEventRecord(m->join_ev, m->side));
        if (w.any_rsvd) {
            {
                Timed t(m, 2);
                omega_kernel<<<dim3(32, nj), 256, 0, m->stream>>>(d_jobs, m->d_state, m->d_slots);
                const int tr = (w.max_rows + 31) / 32, tc = (w.max_cols + 31) / 32, te = (w.max_ell + 31) / 32;
                rsvd_gemm_kernel<<<dim3(te, tr, nj), 256, 0, m->stream>>>(d_jobs, m->d_state, m->d_slots, kStageY0);
                rsvd_gemm_kernel<<<dim3(te, tc, nj), 256, 0, m->stream>>>(d_jobs, m->d_state, m->d_slots, kStageZ);
                rsvd_gemm_kernel<<<dim3(te, tr, nj), 256, 0, m->stream>>>(d_jobs, m->d_state, m->d_slots, kStageY);
                // Columns in shared memory on the smallest cluster that holds
                // them; else in global memory on the largest cluster; Y taller
                // than the cluster kernel's reflector registers hold: one CTA.
                int cq = 0;
                bool qglobal = false;
                const bool qfits = w.max_rows <= kQrRowsPerThread * kQrClusterThreads;
                for (int c = 8; qfits && c <= m->ctx->max_cluster; c *= 2)
                    if (qr_cluster_smem_bytes(w.max_rows, w.max_ell, c) <= kSmemLimit) {
                        cq = c;
                        break;
                    }
                if (qfits && !cq &&
                    qr_cluster_smem_bytes(w.max_rows, w.max_ell, m->ctx->max_cluster, true) <= kSmemLimit) {
                    cq = m->ctx->max_cluster;
                    qglobal = true;
                }
                if (cq) {
                    cudaLaunchConfig_t cfg = {};
                    cfg.gridDim = dim3(nj * cq);
                    cfg.blockDim = dim3(kQrClusterThreads);
                    cfg.dynamicSmemBytes = qr_cluster_smem_bytes(w.max_rows, w.max_ell, cq, qglobal);
                    cfg.stream = m->stream;
                    cudaLaunchAttribute attr[1];
                    attr[0].id = cudaLaunchAttributeClusterDimension;
                    attr[0].val.clusterDim.x = cq;
                    attr[0].val.clusterDim.y = 1;
                    attr[0].val.clusterDim.z = 1;
                    cfg.attrs = attr;
                    cfg.numAttrs = 1;
                    CUDA_TRY(launch_qr_cluster(qglobal, cfg, d_jobs, m->d_state, m->d_slots));
                } else {
                    householder_qr_kernel<<<nj, 512, 0, m->stream>>>(d_jobs, m->d_state, m->d_slots);
                }
                rsvd_gemm_kernel<<<dim3(tc, te, nj), 256, 0, m->stream>>>(d_jobs, m->d_state, m->d_slots, kStageB);
                for (int k = 0; k < 6; ++k) count_launch(m, 2);
            }
            if (wqc_status s = jacobi(kJacobiRsvd, m->stream)) return s;
            {
                Timed t(m, 4);
                finalize_kernel<<<nj, 256, 0, m->stream>>>(d_jobs, m->d_state, m->d_slots, kJacobiRsvd, m->chi, noise_rel,
                                                            m->d_records, m->d_status);
                count_launch(m, 4);
            }
            if (wqc_status s = jacobi(kJacobiFallback, m->stream)) return s;
            {
                Timed t(m, 4);
                finalize_kernel<<<nj, 256, 0, m->stream>>>(d_jobs, m->d_state, m->d_slots, kJacobiFallback, m->chi, noise_rel,
                                                            m->d_records, m->d_status);
                count_launch(m, 4);
            }
        }
        if (fork) CUDA_TRY(cudaStreamWaitEvent(m->stream, m->join_ev, 0));
        {
            Timed t(m, 4);
            // The side the Jacobi does not accumulate, as tiled GEMMs over the
            // kept columns (chi <= min(chi_max, rows, cols)).
            const int kmax = std::min(m->chi, std::min(w.max_rows, w.max_cols));
            auto tiles = [](int x) { return (x + 31) / 32; };
            if (w.any_rsvd) {
                recover_gemm_kernel<<<dim3(tiles(kmax), tiles(w.max_ell), nj), 256, 0, m->stream>>>(
                    d_jobs, m->d_state, m->d_slots, m->dev, kRecoverBW);
                recover_gemm_kernel<<<dim3(tiles(kmax), tiles(w.max_rows), nj), 256, 0, m->stream>>>(
                    d_jobs, m->d_state, m->d_slots, m->dev, kRecoverQT);
                count_launch(m, 4);
                count_launch(m, 4);
            }
            recover_gemm_kernel<<<dim3(tiles(std::max(w.max_cols, kmax)), tiles(std::max(w.max_rows, kmax)), nj), 256,
                                  0, m->stream>>>(d_jobs, m->d_state, m->d_slots, m->dev, kRecoverExact);
            count_launch(m, 4);
            const int per = std::max(w.max_rows, w.max_cols) * std::min(m->chi, std::max(w.max_rows, w.max_cols));
            const int gx = std::max(1, std::min(128, per / 256));
            absorb_kernel<<<dim3(gx, nj), 256, 0, m->stream>>>(d_jobs, m->d_state, m->d_slots, m->dev);
            count_launch(m, 4);
        }
        if (track) CUDA_TRY(cudaEventRecord(m->wave_done[wi], m->stream));
    }
    CUDA_TRY(cudaGetLastError());
    m->rec_count = plan.first_seq + plan.nsplits;
    return WQC_OK;
}

// After uploads: every site's left bond must equal its left neighbour's right
// bond, and each slice must start and end on a bond of 1.  An upload is one
// site at a time, so the chain can only be checked once the caller computes
// on it; a broken chain is refused instead of giving wrong results.
wqc_status check_uploaded_chain(wqc_mps* m) {
    if (!m->uploaded) return WQC_OK;
    CUDA_TRY(cudaStreamSynchronize(m->stream));
    std::vector<int> dl(m->n), dr(m->n);
    CUDA_TRY(cudaMemcpy(dl.data(), m->d_dl, m->n * sizeof(int), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(dr.data(), m->d_dr, m->n * sizeof(int), cudaMemcpyDeviceToHost));
    for (size_t sl = 0; sl < m->seg_first.size(); ++sl) {
        const int first = m->seg_first[sl], last = first + m->seg_n[sl] - 1;
        for (int q = first; q <= last; ++q) {
            const int want = q == first ? 1 : dr[q - 1];
            if (dl[q] != want)
                return fail(WQC_ERR_INVALID, "uploaded sites do not chain: site " + std::to_string(q - first) +
                                                 " has left bond " + std::to_string(dl[q]) + ", expected " +
                                                 std::to_string(want));
        }
        if (dr[last] != 1)
            return fail(WQC_ERR_INVALID, "uploaded sites do not chain: the last site's right bond is " +
                                             std::to_string(dr[last]) + ", expected 1");
    }
    m->uploaded = false;
    return WQC_OK;
}

wqc_status run_ops(wqc_mps* m, const std::vector<Op>& ops) {
    if (*m->h_cancel) return fail(WQC_ERR_CANCELLED, "computation cancelled: the client has gone");
    if (wqc_status s = check_uploaded_chain(m)) return s;
    Plan plan;
    build_plan(m, ops, plan);
    return launch_plan(m, plan);
}

// |0> on every site, all bonds 1, status cleared (mps.rs:101-109).
wqc_status reset_sites(wqc_mps* m) {
    reset_sites_kernel<<<(m->n + 255) / 256, 256, 0, m->stream>>>(m->dev);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(m->stream));
    return WQC_OK;
}

wqc_status sync_status(wqc_mps* m) {
    CUDA_TRY(cudaStreamSynchronize(m->stream));
    int stv[5] = {0, 0, 0, 0, 0};
    CUDA_TRY(cudaMemcpy(stv, m->d_status, sizeof(stv), cudaMemcpyDeviceToHost));
    const int st = stv[0];
    if (*m->h_cancel) return fail(WQC_ERR_CANCELLED, "computation cancelled: the client has gone");
    if (st & kStatusCancelled) return fail(WQC_ERR_CANCELLED, "computation cancelled: the client has gone");
    if (st & kStatusTruncationRejected) return fail(WQC_ERR_TRUNCATION_REJECTED, "mps bond exceeded chi");
    if (st & kStatusNonFinite) return fail(WQC_ERR_SVD_FAILED, "SVD of a two-site matrix produced non-finite values");
    if (st & kStatusSvdCheck) return fail(WQC_ERR_SVD_FAILED, "SVD of a two-site matrix failed its check");
    if (st & kStatusDeviceTimeout) return fail(WQC_ERR_DEVICE_TIMEOUT, "a tensor-core merge gave up waiting on its operands");
    if (st & kStatusJacobiNoConvergence) {
        const unsigned long long bits = (static_cast<unsigned long long>(static_cast<unsigned>(stv[3])) << 32) |
                                        static_cast<unsigned>(stv[4]);
        double rel2;
        std::memcpy(&rel2, &bits, sizeof(rel2));
        char buf[200];
        std::snprintf(buf, sizeof(buf),
                      "Jacobi SVD of a two-site matrix did not converge in 60 sweeps (split %d: last sweep %d "
                      "rotations, max |gamma|/sqrt(alpha beta) %.3e)",
                      stv[1] - 1, stv[2], std::sqrt(rel2));
        return fail(WQC_ERR_SVD_FAILED, buf);
    }
    if (st & kStatusBadShape) return fail(WQC_ERR_INVALID, "two-site matrix without a Jacobi workspace");
    return WQC_OK;
}

}  // namespace

// Lets entry points defined in other files of the library set the message
// that wqc_cuda_last_error returns.
namespace wqc {
wqc_status record_error(wqc_status code, const std::string& msg) { return fail(code, msg); }
wqc_status record_oom(uint64_t required, uint64_t available) { return fail_oom(required, available); }
wqc_status check_circuit_gate(int n, const wqc_gate& g) { return check_gate(n, g); }
void gate_matrix_2x2(int kind, double theta, double2 out[4]) {
    const Mat2 m = unary_matrix(kind, theta);
    for (int i = 0; i < 4; ++i) out[i] = m.u[i];
}
int context_device(const wqc_cuda_ctx* ctx) { return ctx->device; }
int context_sm_count(const wqc_cuda_ctx* ctx) { return ctx->sm_count; }
}  // namespace wqc

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* wqc_cuda_last_error(void) { return g_err.c_str(); }

void wqc_cuda_last_oom(uint64_t* required, uint64_t* available) {
    if (required) *required = g_oom_required;
    if (available) *available = g_oom_available;
}

wqc_status wqc_cuda_open(int device, wqc_cuda_ctx** out) {
    if (!out) return fail(WQC_ERR_INVALID, "null output pointer");
    if (device < 0) {
        const char* env = std::getenv("WQC_CUDA_DEVICE");
        device = env ? std::atoi(env) : 0;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(WQC_ERR_NO_DEVICE, "CUDA device not found");
    }
    if (device >= count) return fail(WQC_ERR_NO_DEVICE, "CUDA device index out of range");
    CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop{};
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return fail(WQC_ERR_NO_DEVICE, "the cuda MPS backend is built for sm_100a (B200)");
    std::call_once(g_attr_once, set_kernel_attributes);
    if (g_attr_err != cudaSuccess) return fail(WQC_ERR_CUDA, std::string("kernel attributes: ") + cudaGetErrorString(g_attr_err));
    auto* ctx = new wqc_cuda_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    // Largest cluster the device schedules with a full shared-memory CTA.
    ctx->max_cluster = 8;
    {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(16);
        cfg.blockDim = dim3(kJacobiThreads);
        cfg.dynamicSmemBytes = 200 * 1024;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 16;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, jacobi_kernel(false, false), &cfg) == cudaSuccess && clusters > 0)
            ctx->max_cluster = 16;
        cudaGetLastError();
    }
    *out = ctx;
    return WQC_OK;
}

void wqc_cuda_close(wqc_cuda_ctx* ctx) { delete ctx; }

wqc_status wqc_cuda_device_info(wqc_cuda_ctx* ctx, uint64_t* total_bytes, uint64_t* free_bytes, int32_t* sm_count) {
    if (!ctx) return fail(WQC_ERR_INVALID, "null context");
    CUDA_TRY(cudaSetDevice(ctx->device));
    size_t fr = 0, tot = 0;
    CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    if (total_bytes) *total_bytes = tot;
    if (free_bytes) *free_bytes = fr;
    if (sm_count) *sm_count = ctx->sm_count;
    return WQC_OK;
}

uint64_t wqc_mps_workspace_bytes(uint32_t n, uint32_t chi) {
    const unsigned __int128 v = (unsigned __int128)n * chi * chi * 32;
    return v > ~uint64_t(0) ? ~uint64_t(0) : uint64_t(v);
}

static wqc_status create_state(wqc_cuda_ctx* ctx, const std::vector<int>& ns, const std::vector<int>& chis,
                               int32_t precision, bool reject, int nslots_req, wqc_mps** out,
                               bool single_state = false) {
    if (!ctx || !out) return fail(WQC_ERR_INVALID, "null argument");
    if (ns.empty()) return fail(WQC_ERR_INVALID, "no slices");
    long total_n = 0;
    int chi_cap = 0;
    for (size_t i = 0; i < ns.size(); ++i) {
        if (ns[i] <= 0)
            return fail(WQC_ERR_INVALID_QUBIT_COUNT, "Invalid qubit count: " + std::to_string(ns[i]) + ". Max limit is 40.");
        if (chis[i] <= 0) return fail(WQC_ERR_INVALID, "MPS max bond dimension must be > 0");
        if (chis[i] > 256) return fail(WQC_ERR_INVALID, "the cuda backend supports max_bond_dim <= 256");
        total_n += ns[i];
        chi_cap = std::max(chi_cap, chis[i]);
    }
    if (precision != WQC_PRECISION_FP64 && precision != WQC_PRECISION_FP32 && precision != WQC_PRECISION_TF32X3)
        return fail(WQC_ERR_INVALID, "unsupported precision form");
    if (total_n > (1L << 24)) return fail(WQC_ERR_INVALID, "too many sites");
    CUDA_TRY(cudaSetDevice(ctx->device));
    auto* m = new wqc_mps();
    const int n = int(total_n);
    m->ctx = ctx;
    m->n = n;
    m->chi = chi_cap;
    m->reject = reject;
    m->fp32 = precision != WQC_PRECISION_FP64;
    m->tc = precision == WQC_PRECISION_TF32X3;
    m->ub.assign(n > 0 ? n - 1 : 0, 1);
    m->site_chi.resize(n);
    m->site_slice.resize(n);
    std::vector<size_t> site_off(n + 1, 0);
    for (size_t sl = 0, g = 0; sl < ns.size(); ++sl) {
        m->seg_first.push_back(int(g));
        m->seg_n.push_back(ns[sl]);
        m->seg_chi.push_back(chis[sl]);
        for (int q = 0; q < ns[sl]; ++q, ++g) {
            m->site_chi[g] = chis[sl];
            m->site_slice[g] = int(sl);
            site_off[g + 1] = site_off[g] + size_t(chis[sl]) * 2 * chis[sl];
        }
    }
    auto bail = [&](wqc_status st) {
        wqc_mps_destroy(m);
        return st;
    };
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(fail(WQC_ERR_CUDA, "stream"));
    if (cudaStreamCreateWithFlags(&m->side, cudaStreamNonBlocking) != cudaSuccess) return bail(fail(WQC_ERR_CUDA, "stream"));
    if (cudaEventCreateWithFlags(&m->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&m->join_ev, cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(WQC_ERR_CUDA, "event"));
    if (cudaEventCreateWithFlags(&m->stage_done, cudaEventDisableTiming) != cudaSuccess) return bail(fail(WQC_ERR_CUDA, "event"));
    cudaEventRecord(m->stage_done, m->stream);
    // Split workspace: one bucket of slots per distinct chi_max, each slot
    // holding theta, w, z, the range finder's buffers and tau for two-site
    // matrices up to R x R, R = 2 chi_max (plus the staged Jacobi's workspace
    // when such a matrix can exceed a cluster's shared memory).  A bucket
    // gets a slot per two sites of its slices, at most kSlotBudget bytes of
    // them: waves take as many splits of a bucket as it has slots.
    // The staged Jacobi's workspace holds (R + 32) x R complex128 values: the
    // padded FP64 columns, or the precision form's complex64 columns with V
    // under them ((R + 32) x 2R complex64 values, the same bytes).
    const bool fp32 = precision != WQC_PRECISION_FP64;
    auto no_cluster = [&](int M, int N) {
        return choose_cluster(nullptr, M, N, ctx->max_cluster, 1, ctx->sm_count, sizeof(double2), false) < 1 ||
               (fp32 &&
                choose_cluster(nullptr, M, N, ctx->max_cluster, 1, ctx->sm_count, sizeof(float2), false, M + N) < 1);
    };
    std::vector<size_t> bucket_bytes, bucket_gs;
    {
        std::vector<int> cs(chis);
        std::sort(cs.begin(), cs.end());
        cs.erase(std::unique(cs.begin(), cs.end()), cs.end());
        m->nslots = 0;
        for (int c : cs) {
            const int R = 2 * c, E = std::min(c + kRsvdOversample, R);
            const bool staged = no_cluster(R, R) || no_cluster(R, E);
            const size_t gs_c = staged ? jacobi_staged_elems(R) : 0;
            const size_t slot_c = size_t(R) * R * 3 + size_t(R) * E * 6 + E + gs_c;
            const size_t bytes = ((slot_c * sizeof(double2) + size_t(R) * (sizeof(double) + sizeof(int)) + 4095) / 4096) * 4096;
            long count = 0;
            for (size_t sl = 0; sl < ns.size(); ++sl)
                if (chis[sl] == c) count += ns[sl] / 2;
            long cap = std::max<long>(1, std::min<long>(std::max<long>(count, 1), long(kSlotBudget / bytes)));
            if (nslots_req > 0) cap = std::min<long>(cap, nslots_req);
            m->bucket_chi.push_back(c);
            m->bucket_base.push_back(m->nslots);
            m->bucket_cap.push_back(int(cap));
            bucket_bytes.push_back(bytes);
            bucket_gs.push_back(gs_c);
            m->nslots += int(cap);
        }
    }
    size_t slot_pool_bytes = 0;
    for (size_t b = 0; b < m->bucket_chi.size(); ++b) slot_pool_bytes += bucket_bytes[b] * size_t(m->bucket_cap[b]);
    const size_t site_bytes = site_off[n] * sizeof(double2);
    // Tensor-core form: TF32 hi/lo planes of both merge operands for every job
    // a wave can hold (one per slot), padded to whole tiles of the largest
    // two-site matrix.
    size_t tc_a_bytes = 0, tc_b_bytes = 0;
    if (m->tc) {
        m->tc_rpad = tc_rpad(2 * chi_cap);
        m->tc_kpad = tc_kpad(chi_cap);
        m->tc_npad = tc_npad(2 * chi_cap);
        tc_a_bytes = size_t(2) * m->nslots * m->tc_rpad * m->tc_kpad * sizeof(float);
        tc_b_bytes = size_t(2) * m->nslots * m->tc_npad * m->tc_kpad * sizeof(float);
    }
    // States from wqc_mps_create merge from int8 digit slices on the tensor
    // cores by default (FP64-level, wqc_mps_set_merge); batches (a batch of
    // one included) keep FMA merges, whose many slots would each need digit
    // planes.
    const bool oz_default = single_state && !m->tc;
    const uint64_t need = site_bytes + uint64_t(slot_pool_bytes) + tc_a_bytes + tc_b_bytes +
                          (oz_default ? oz_state_bytes(m) : 0);
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return bail(fail(WQC_ERR_CUDA, "cudaMemGetInfo"));
    if (need > fr) return bail(fail_oom(need, fr));
    void* p = nullptr;
    if (wqc_status st = dmalloc(m, &p, site_bytes)) return bail(st);
    m->site_pool = static_cast<double2*>(p);
    if (wqc_status st = dmalloc(m, &p, size_t(n) * sizeof(double2*))) return bail(st);
    m->d_site_ptr = static_cast<double2**>(p);
    if (wqc_status st = dmalloc(m, &p, 2 * size_t(n) * sizeof(int) + 64)) return bail(st);
    m->d_dl = static_cast<int*>(p);
    m->d_dr = m->d_dl + n;
    m->d_status = m->d_dr + n;
    if (wqc_status st = dmalloc(m, &p, 2 * ns.size() * sizeof(int))) return bail(st);
    m->d_seg = static_cast<int*>(p);
    if (wqc_status st = dmalloc(m, &p, slot_pool_bytes)) return bail(st);
    m->slot_pool = static_cast<char*>(p);
    if (m->tc) {
        if (wqc_status st = dmalloc(m, &p, tc_a_bytes)) return bail(st);
        m->tc_a = static_cast<float*>(p);
        if (wqc_status st = dmalloc(m, &p, tc_b_bytes)) return bail(st);
        m->tc_b = static_cast<float*>(p);
        if (!tc_encode_planes(&m->tc_map_a, m->tc_a, m->tc_kpad, m->tc_rpad, 2 * m->nslots) ||
            !tc_encode_planes(&m->tc_map_b, m->tc_b, m->tc_kpad, m->tc_npad, 2 * m->nslots))
            return bail(fail(WQC_ERR_CUDA, "cuTensorMapEncodeTiled refused the merge operand planes"));
    }
    if (wqc_status st = dmalloc(m, &p, m->nslots * sizeof(SlotBuffers))) return bail(st);
    m->d_slots = static_cast<SlotBuffers*>(p);
    if (wqc_status st = dmalloc(m, &p, m->nslots * sizeof(SplitState))) return bail(st);
    m->d_state = static_cast<SplitState*>(p);
    const size_t small = std::max<size_t>(64, 2 * ns.size() + 8);
    if (wqc_status st = dmalloc(m, &p, small * sizeof(double2))) return bail(st);
    m->d_small = static_cast<double2*>(p);
    m->d_counters = reinterpret_cast<unsigned long long*>(m->d_small + small - 4);
    if (cudaMemset(m->d_small, 0, small * sizeof(double2)) != cudaSuccess) return bail(fail(WQC_ERR_CUDA, "memset"));
    if (oz_default)
        if (wqc_status st = oz_enable(m)) return bail(st);
    if (ns.size() == 1) {  // the trace feeders' environment cache (single states)
        const size_t env_bytes = 2 * size_t(n) * chi_cap * sizeof(double2) + size_t(n) * 2 * sizeof(double2) +
                                 size_t(n) * sizeof(int);
        if (wqc_status st = dmalloc(m, &p, env_bytes)) return bail(st);
        m->d_envL = static_cast<double2*>(p);
        m->d_envR = m->d_envL + size_t(n) * chi_cap;
        m->d_env_out = m->d_envR + size_t(n) * chi_cap;
        m->d_targets = reinterpret_cast<int*>(m->d_env_out + size_t(n) * 2);
    }
    m->lvalid = 0;
    m->rvalid = n - 1;
    int* hc = nullptr;
    if (cudaHostAlloc(reinterpret_cast<void**>(&hc), sizeof(int), cudaHostAllocMapped) != cudaSuccess)
        return bail(fail(WQC_ERR_CUDA, "cudaHostAlloc"));
    *hc = 0;
    m->h_cancel = hc;
    if (cudaHostGetDevicePointer(reinterpret_cast<void**>(&m->d_cancel), hc, 0) != cudaSuccess)
        return bail(fail(WQC_ERR_CUDA, "cudaHostGetDevicePointer"));
    m->site_ptr.resize(n);
    for (int i = 0; i < n; ++i) m->site_ptr[i] = m->site_pool + site_off[i];
    std::vector<int> seg(2 * ns.size());
    for (size_t sl = 0; sl < ns.size(); ++sl) {
        seg[2 * sl] = m->seg_first[sl];
        seg[2 * sl + 1] = m->seg_n[sl];
    }
    if (cudaMemcpy(m->d_site_ptr, m->site_ptr.data(), size_t(n) * sizeof(double2*), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m->d_seg, seg.data(), seg.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(WQC_ERR_CUDA, "initial upload"));
    std::vector<SlotBuffers> slots(m->nslots);
    m->slot_R.assign(m->nslots, 0);
    m->slot_E.assign(m->nslots, 0);
    char* base = m->slot_pool;
    for (int sl = 0; sl < m->nslots; ++sl) {
        size_t bk = 0;
        while (bk + 1 < m->bucket_chi.size() && sl >= m->bucket_base[bk + 1]) ++bk;
        const int R = 2 * m->bucket_chi[bk], E = std::min(m->bucket_chi[bk] + kRsvdOversample, R);
        const size_t gs_c = bucket_gs[bk];
        m->slot_R[sl] = R;
        m->slot_E[sl] = E;
        double2* c = reinterpret_cast<double2*>(base);
        base += bucket_bytes[bk];
        SlotBuffers& bf = slots[sl];
        bf.theta = c; c += size_t(R) * R;
        bf.w = c; c += size_t(R) * R;
        bf.z = c; c += size_t(R) * R;
        bf.omega = c; c += size_t(R) * E;
        bf.y0 = c; c += size_t(R) * E;
        bf.zr = c; c += size_t(R) * E;
        bf.y = c; c += size_t(R) * E;
        bf.q = c; c += size_t(R) * E;
        bf.b = c; c += size_t(R) * E;
        bf.tau = c; c += E;
        bf.gs = gs_c ? static_cast<void*>(c) : nullptr;
        c += gs_c;
        bf.sigma = reinterpret_cast<double*>(c);
        bf.perm = reinterpret_cast<int*>(bf.sigma + R);
    }
    if (cudaMemcpy(m->d_slots, slots.data(), slots.size() * sizeof(SlotBuffers), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(WQC_ERR_CUDA, "slot table upload"));
    m->dev.site = m->d_site_ptr;
    m->dev.dl = m->d_dl;
    m->dev.dr = m->d_dr;
    m->dev.n = n;
    m->dev.chi_max = chi_cap;
    m->dev.status = m->d_status;
    m->dev.cancel = m->d_cancel;
    if (wqc_status st = ensure_records(m, 1024)) return bail(st);
    if (wqc_status st = reset_sites(m)) return bail(st);
    *out = m;
    return WQC_OK;
}

wqc_status wqc_mps_create(wqc_cuda_ctx* ctx, uint32_t n, uint32_t chi, int32_t precision, uint8_t reject,
                          wqc_mps** out) {
    return create_state(ctx, {int(n)}, {int(chi)}, precision, reject != 0, 0, out, true);
}

wqc_status wqc_batch_create(wqc_cuda_ctx* ctx, uint32_t count, const uint32_t* qubit_counts,
                            const uint32_t* max_bond_dims, int32_t precision, uint32_t max_concurrent_splits,
                            wqc_mps** out) {
    if (!qubit_counts || !max_bond_dims || count == 0) return fail(WQC_ERR_INVALID, "null argument");
    std::vector<int> ns(count), chis(count);
    for (uint32_t i = 0; i < count; ++i) {
        ns[i] = int(qubit_counts[i]);
        chis[i] = int(max_bond_dims[i]);
    }
    const wqc_status st = create_state(ctx, ns, chis, precision, false, int(max_concurrent_splits), out);
    if (st == WQC_OK) (*out)->batch = true;
    return st;
}

wqc_status wqc_mps_reset(wqc_mps* m) {
    if (!m) return fail(WQC_ERR_INVALID, "null argument");
    // A reset starts the next request whatever the last one ended with (an
    // error status, a cancellation): the queue drains, the cancel word and the
    // device status word are cleared and the sites return to |0...0>.
    CUDA_TRY(cudaStreamSynchronize(m->stream));
    *m->h_cancel = 0;
    if (wqc_status st = reset_sites(m)) return st;
    std::fill(m->ub.begin(), m->ub.end(), 1);
    m->rec_count = 0;
    m->lvalid = 0;
    m->rvalid = m->n - 1;
    return WQC_OK;
}

void wqc_mps_destroy(wqc_mps* m) {
    if (!m) return;
    if (m->stream) cudaStreamSynchronize(m->stream);
    dfree(m, m->site_pool, 0);
    dfree(m, m->d_site_ptr, 0);
    dfree(m, m->d_dl, 0);
    dfree(m, m->slot_pool, 0);
    dfree(m, m->tc_a, 0);
    dfree(m, m->tc_b, 0);
    dfree(m, m->oz_pool, 0);
    dfree(m, m->d_slots, 0);
    dfree(m, m->d_state, 0);
    dfree(m, m->d_small, 0);
    dfree(m, m->d_records, 0);
    dfree(m, m->d_seg, 0);
    dfree(m, m->d_envL, 0);
    for (auto e : m->wave_done) cudaEventDestroy(e);
    if (m->call_start) cudaEventDestroy(m->call_start);
    dfree(m, m->d_stage.d, 0);
    if (m->h_stage) cudaFreeHost(m->h_stage);
    if (m->h_cancel) cudaFreeHost(const_cast<int*>(m->h_cancel));
    for (auto& e : m->events) {
        cudaEventDestroy(e.second.first);
        cudaEventDestroy(e.second.second);
    }
    for (auto e : m->event_pool) cudaEventDestroy(e);
    if (m->stage_done) cudaEventDestroy(m->stage_done);
    if (m->fork_ev) cudaEventDestroy(m->fork_ev);
    if (m->join_ev) cudaEventDestroy(m->join_ev);
    if (m->side) cudaStreamDestroy(m->side);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
}

wqc_status wqc_schedule_gates(uint32_t n, const wqc_gate* gates, uint32_t count, int32_t* split_site,
                              int32_t* split_level, uint32_t max, uint32_t* nsplits, uint32_t* nlevels) {
    if (n == 0 || (!gates && count) || !nsplits || !nlevels) return fail(WQC_ERR_INVALID, "null argument");
    Expander ex;
    if (wqc_status s = expand(int(n), gates, count, false, ex)) return s;
    std::vector<int> level_of;
    assign_levels(int(n), ex.ops, level_of);
    uint32_t k = 0;
    int top = -1;
    for (size_t i = 0; i < ex.ops.size(); ++i) {
        top = std::max(top, level_of[i]);
        if (!ex.ops[i].two) continue;
        if (k < max) {
            if (split_site) split_site[k] = ex.ops[i].site;
            if (split_level) split_level[k] = level_of[i];
        }
        ++k;
    }
    *nsplits = k;
    *nlevels = uint32_t(top + 1);
    return WQC_OK;
}

wqc_status wqc_mps_apply_gates(wqc_mps* m, const wqc_gate* gates, uint32_t count) {
    if (!m || (!gates && count)) return fail(WQC_ERR_INVALID, "null argument");
    Expander ex;
    if (wqc_status s = expand(m->n, gates, count, false, ex)) return s;
    return run_ops(m, ex.ops);
}

wqc_status wqc_mps_apply_gates_adjoint(wqc_mps* m, const wqc_gate* gates, uint32_t count) {
    if (!m || (!gates && count)) return fail(WQC_ERR_INVALID, "null argument");
    Expander ex;
    if (wqc_status s = expand(m->n, gates, count, true, ex)) return s;
    return run_ops(m, ex.ops);
}

wqc_status wqc_batch_apply_gates(wqc_mps* m, const wqc_gate* gates, const uint32_t* offsets) {
    if (!m || !offsets) return fail(WQC_ERR_INVALID, "null argument");
    Expander all;
    for (size_t sl = 0; sl < m->seg_first.size(); ++sl) {
        const uint32_t g0 = offsets[sl], g1 = offsets[sl + 1];
        if (g1 < g0) return fail(WQC_ERR_INVALID, "gate offsets must not decrease");
        if (g1 == g0) continue;
        if (!gates) return fail(WQC_ERR_INVALID, "null gates");
        Expander ex;
        if (wqc_status s = expand(m->seg_n[sl], gates + g0, g1 - g0, false, ex)) return s;
        for (Op& o : ex.ops) {
            o.site += m->seg_first[sl];
            o.slice = int(sl);
            all.ops.push_back(o);
        }
    }
    return run_ops(m, all.ops);
}

wqc_status wqc_batch_amplitudes(wqc_mps* m, double* out) {
    if (!m || !out) return fail(WQC_ERR_INVALID, "null argument");
    if (wqc_status st = check_uploaded_chain(m)) return st;
    const int nseg = int(m->seg_first.size());
    amplitude_zero_kernel<<<nseg, 512, 2 * m->chi * sizeof(double2), m->stream>>>(m->dev, m->d_seg, m->d_small);
    count_launch(m, -1);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(out, m->d_small, nseg * sizeof(double2), cudaMemcpyDeviceToHost, m->stream));
    m->stats.d2h_bytes += nseg * sizeof(double2);
    return sync_status(m);
}

wqc_status wqc_batch_expectation_pauli(wqc_mps* m, const char* labels, const double* coeffs, uint32_t nterms,
                                       double* out) {
    if (!m || !labels || !coeffs || !out) return fail(WQC_ERR_INVALID, "null argument");
    const int nseg = int(m->seg_first.size());
    const int width = nseg > 0 ? (m->n / nseg) : 0;
    for (int s = 0; s < nseg; ++s) {
        const int first = m->seg_first[s], last = s + 1 < nseg ? m->seg_first[s + 1] : m->n;
        if (last - first != width) return fail(WQC_ERR_INVALID, "batch expectation needs slices of one width");
    }
    for (size_t i = 0; i < size_t(nterms) * width; ++i) {
        const char ch = labels[i];
        if (ch != 'I' && ch != 'X' && ch != 'Y' && ch != 'Z')
            return fail(WQC_ERR_INVALID, std::string("invalid pauli character in label"));
    }
    if (nterms == 0 || nseg == 0) {
        for (int s = 0; s < 2 * nseg; ++s) out[s] = 0;
        return WQC_OK;
    }
    const size_t E = size_t(m->chi) * m->chi;
    const size_t scratch = size_t(nterms) * 4 * E * sizeof(double2);
    const size_t lab_bytes = size_t(nterms) * width + 16;
    const size_t out_bytes = size_t(nterms) * nseg * sizeof(double2);
    void* d_lab = nullptr;
    void* d_scr = nullptr;
    void* d_out = nullptr;
    if (wqc_status s = dmalloc(m, &d_lab, lab_bytes)) return s;
    if (wqc_status s = dmalloc(m, &d_scr, scratch)) {
        dfree(m, d_lab, lab_bytes);
        return s;
    }
    if (wqc_status s = dmalloc(m, &d_out, out_bytes)) {
        dfree(m, d_lab, lab_bytes);
        dfree(m, d_scr, scratch);
        return s;
    }
    wqc_status rc = WQC_OK;
    std::vector<double2> vals(size_t(nterms) * nseg);
    cudaError_t e = cudaMemcpyAsync(d_lab, labels, size_t(nterms) * width, cudaMemcpyHostToDevice, m->stream);
    // One launch per slice on a view of its sites; launches share the scratch
    // in stream order.
    for (int s = 0; s < nseg && e == cudaSuccess; ++s) {
        DeviceMps view = m->dev;
        const int first = m->seg_first[s];
        view.site += first;
        view.dl += first;
        view.dr += first;
        view.n = width;
        pauli_expectation_kernel<<<nterms, 256, 0, m->stream>>>(view, static_cast<const char*>(d_lab), int(nterms),
                                                                  static_cast<double2*>(d_scr), m->chi,
                                                                  static_cast<double2*>(d_out) + size_t(s) * nterms);
        count_launch(m, -1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(vals.data(), d_out, out_bytes, cudaMemcpyDeviceToHost, m->stream);
    if (e != cudaSuccess) rc = fail(WQC_ERR_CUDA, cudaGetErrorString(e));
    if (rc == WQC_OK) rc = sync_status(m);
    dfree(m, d_lab, lab_bytes);
    dfree(m, d_scr, scratch);
    dfree(m, d_out, out_bytes);
    if (rc != WQC_OK) return rc;
    for (int s = 0; s < nseg; ++s) {
        double re = 0, im = 0;
        for (uint32_t t = 0; t < nterms; ++t) {  // coeff * Re<P> (expectation.rs:177-185), term order
            const double v = vals[size_t(s) * nterms + t].x;
            re += coeffs[2 * t] * v;
            im += coeffs[2 * t + 1] * v;
        }
        out[2 * s] = re;
        out[2 * s + 1] = im;
    }
    return WQC_OK;
}

wqc_status wqc_batch_slice_times(wqc_mps* m, double* out_ms) {
    if (!m || !out_ms) return fail(WQC_ERR_INVALID, "null argument");
    if (wqc_status s = sync_status(m)) return s;
    const size_t nseg = m->seg_first.size();
    for (size_t sl = 0; sl < nseg; ++sl) {
        const int w = sl < m->slice_last_wave.size() ? m->slice_last_wave[sl] : -1;
        float ms = -1.0f;
        if (w >= 0 && m->call_start && size_t(w) < m->wave_done.size())
            CUDA_TRY(cudaEventElapsedTime(&ms, m->call_start, m->wave_done[w]));
        out_ms[sl] = double(ms);
    }
    return WQC_OK;
}

wqc_status wqc_mps_apply_1q(wqc_mps* m, uint32_t site, const double u[8]) {
    if (!m || !u) return fail(WQC_ERR_INVALID, "null argument");
    if (site >= uint32_t(m->n)) return fail(WQC_ERR_QUBIT_OUT_OF_RANGE, "site out of range");
    Expander ex;
    Mat2 mm;
    for (int i = 0; i < 4; ++i) mm.u[i] = make_double2(u[2 * i], u[2 * i + 1]);
    ex.one(int(site), mm);
    return run_ops(m, ex.ops);
}

static Mat4 mat4_from(const double u[32]) {
    Mat4 mm;
    for (int i = 0; i < 16; ++i) mm.u[i] = make_double2(u[2 * i], u[2 * i + 1]);
    return mm;
}

wqc_status wqc_mps_apply_2q(wqc_mps* m, uint32_t left, const double u[32], uint8_t cf, wqc_split_info* info) {
    if (!m || !u) return fail(WQC_ERR_INVALID, "null argument");
    if (uint64_t(left) + 1 >= uint64_t(m->n)) return fail(WQC_ERR_QUBIT_OUT_OF_RANGE, "two-site apply needs adjacent positions");
    Expander ex;
    ex.two_at(int(left), mat4_from(u), cf != 0);
    const uint32_t seq = m->rec_count;
    if (wqc_status s = run_ops(m, ex.ops)) return s;
    if (info) {
        if (wqc_status s = sync_status(m)) return s;
        CUDA_TRY(cudaMemcpy(info, m->d_records + seq, sizeof(wqc_split_info), cudaMemcpyDeviceToHost));
    }
    return WQC_OK;
}

wqc_status wqc_mps_apply_2q_routed(wqc_mps* m, uint32_t ctrl, uint32_t tgt, const double u[32]) {
    if (!m || !u) return fail(WQC_ERR_INVALID, "null argument");
    if (ctrl >= uint32_t(m->n) || tgt >= uint32_t(m->n) || ctrl == tgt) return fail(WQC_ERR_QUBIT_OUT_OF_RANGE, "bad qubit pair");
    Expander ex;
    ex.two_routed(int(ctrl), int(tgt), mat4_from(u));
    return run_ops(m, ex.ops);
}

wqc_status wqc_mps_apply_layer(wqc_mps* m, const wqc_gate* gates, uint32_t count) {
    if (!m || (!gates && count)) return fail(WQC_ERR_INVALID, "null argument");
    if (count >= 2) {
        std::vector<int> seen;
        for (uint32_t i = 0; i < count; ++i) {
            const wqc_gate& g = gates[i];
            if (g.kind != WQC_GATE_CNOT && g.kind != WQC_GATE_CZ)
                return fail(WQC_ERR_INVALID, "disjoint layer contains a gate that is not CNOT or CZ");
        }
    }
    return wqc_mps_apply_gates(m, gates, count);
}

wqc_status wqc_mps_set_split_rule(wqc_mps* m, int32_t rule) {
    if (!m) return fail(WQC_ERR_INVALID, "null argument");
    if (rule != WQC_SPLIT_RULE_REFERENCE && rule != WQC_SPLIT_RULE_EXACT) return fail(WQC_ERR_INVALID, "unknown split rule");
    m->exact_only = rule == WQC_SPLIT_RULE_EXACT;
    return WQC_OK;
}

wqc_status wqc_mps_set_merge(wqc_mps* m, int32_t merge) {
    if (!m) return fail(WQC_ERR_INVALID, "null argument");
    if (merge != WQC_MERGE_FFMA && merge != WQC_MERGE_TC_INT8) return fail(WQC_ERR_INVALID, "unknown merge");
    if (m->tc) return fail(WQC_ERR_INVALID, "the tensor-core form merges on its own TF32 path");
    CUDA_TRY(cudaSetDevice(m->ctx->device));
    CUDA_TRY(cudaStreamSynchronize(m->stream));  // no enqueued merge still reads the planes
    if (merge == WQC_MERGE_TC_INT8) return oz_enable(m);
    m->oz = false;
    return WQC_OK;
}

wqc_status wqc_mps_synchronize(wqc_mps* m) {
    if (!m) return fail(WQC_ERR_INVALID, "null argument");
    return sync_status(m);
}

void wqc_mps_cancel(wqc_mps* m) {
    if (m && m->h_cancel) *const_cast<volatile int*>(m->h_cancel) = 1;
}

wqc_status wqc_mps_amplitude_zero(wqc_mps* m, double out[2]) {
    if (!m || !out) return fail(WQC_ERR_INVALID, "null argument");
    if (wqc_status st = check_uploaded_chain(m)) return st;
    amplitude_zero_kernel<<<1, 512, 2 * m->chi * sizeof(double2), m->stream>>>(m->dev, m->d_seg, m->d_small);
    count_launch(m, -1);
    CUDA_TRY(cudaGetLastError());
    double2 h;
    CUDA_TRY(cudaMemcpyAsync(&h, m->d_small, sizeof(double2), cudaMemcpyDeviceToHost, m->stream));
    m->stats.d2h_bytes += sizeof(double2);
    if (wqc_status s = sync_status(m)) return s;
    out[0] = h.x;
    out[1] = h.y;
    return WQC_OK;
}

wqc_status wqc_mps_site_amplitudes_many(wqc_mps* m, const uint32_t* targets, uint32_t count, double* out) {
    if (!m || (count && (!targets || !out))) return fail(WQC_ERR_INVALID, "null argument");
    if (!m->d_envL) return fail(WQC_ERR_INVALID, "site amplitudes take a single state, not a batch");
    if (count == 0) return WQC_OK;
    if (count > uint32_t(m->n)) return fail(WQC_ERR_INVALID, "more targets than sites");
    std::vector<int> t(count);
    int lo = m->n, hi = -1;
    for (uint32_t k = 0; k < count; ++k) {
        if (targets[k] >= uint32_t(m->n)) return fail(WQC_ERR_QUBIT_OUT_OF_RANGE, "target out of range");
        t[k] = int(targets[k]);
        lo = std::min(lo, t[k]);
        hi = std::max(hi, t[k]);
    }
    if (wqc_status st = check_uploaded_chain(m)) return st;
    const int lfrom = m->lvalid, lto = std::max(m->lvalid, hi);
    const int rfrom = m->rvalid, rto = std::min(m->rvalid, lo);
    CUDA_TRY(cudaMemcpyAsync(m->d_targets, t.data(), count * sizeof(int), cudaMemcpyHostToDevice, m->stream));
    m->stats.h2d_bytes += count * sizeof(int);
    site_envs_kernel<<<1, 512, 0, m->stream>>>(m->dev, m->d_envL, m->d_envR, lfrom, lto, rfrom, rto, m->d_targets,
                                               int(count), m->d_env_out);
    count_launch(m, -1);
    CUDA_TRY(cudaGetLastError());
    std::vector<double2> h(2 * size_t(count));
    CUDA_TRY(cudaMemcpyAsync(h.data(), m->d_env_out, h.size() * sizeof(double2), cudaMemcpyDeviceToHost, m->stream));
    m->stats.d2h_bytes += h.size() * sizeof(double2);
    if (wqc_status s = sync_status(m)) return s;
    m->lvalid = lto;
    m->rvalid = rto;
    for (size_t k = 0; k < h.size(); ++k) {
        out[2 * k] = h[k].x;
        out[2 * k + 1] = h[k].y;
    }
    return WQC_OK;
}

wqc_status wqc_mps_site_amplitudes(wqc_mps* m, uint32_t target, double out[4]) {
    if (!m || !out) return fail(WQC_ERR_INVALID, "null argument");
    if (target >= uint32_t(m->n)) return fail(WQC_ERR_QUBIT_OUT_OF_RANGE, "target out of range");
    return wqc_mps_site_amplitudes_many(m, &target, 1, out);
}

wqc_status wqc_mps_to_dense(wqc_mps* m, int32_t mode, double* out) {
    if (!m || !out) return fail(WQC_ERR_INVALID, "null argument");
    if (m->seg_first.size() != 1) return fail(WQC_ERR_INVALID, "the dense state takes a single state, not a batch");
    if (mode != WQC_DENSE_TO_DENSE_STATE && mode != WQC_DENSE_STATEVECTOR)
        return fail(WQC_ERR_INVALID, "unknown dense mode");
    const int n = m->n;
    if (mode == WQC_DENSE_STATEVECTOR && n > 20)  // mps.rs:217-221
        return fail(WQC_ERR_INVALID, "full statevector projection requires qubit_count <= 20");
    if (n > kDenseMaxQubits)
        return fail(WQC_ERR_INVALID_QUBIT_COUNT, "the dense state is limited to " + std::to_string(kDenseMaxQubits) +
                                                     " qubits");
    if (wqc_status st = check_uploaded_chain(m)) return st;
    if (wqc_status s = sync_status(m)) return s;
    std::vector<int> dl(n), dr(n);
    CUDA_TRY(cudaMemcpy(dl.data(), m->d_dl, n * sizeof(int), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(dr.data(), m->d_dr, n * sizeof(int), cudaMemcpyDeviceToHost));
    size_t most = 1;
    for (int q = 0; q < n; ++q) {
        if (dl[q] != (q ? dr[q - 1] : 1))  // mps.rs:229-234
            return fail(WQC_ERR_INVALID, "MPS bond layout mismatch during statevector projection");
        most = std::max(most, (size_t(2) << q) * size_t(dr[q]));
    }
    if (dr[n - 1] != 1) return fail(WQC_ERR_INVALID, "MPS bond layout mismatch during statevector projection");
    void *d_a = nullptr, *d_b = nullptr;
    if (wqc_status st = dmalloc(m, &d_a, most * sizeof(double2))) return st;
    if (wqc_status st = dmalloc(m, &d_b, most * sizeof(double2))) {
        dfree(m, d_a, most * sizeof(double2));
        return st;
    }
    double2* cur = static_cast<double2*>(d_a);
    double2* nxt = static_cast<double2*>(d_b);
    const double2 one = cmake(1.0, 0.0);
    cudaError_t e = cudaMemcpyAsync(cur, &one, sizeof(double2), cudaMemcpyHostToDevice, m->stream);
    const int prune = mode == WQC_DENSE_TO_DENSE_STATE ? 1 : 0;
    for (int q = 0; q < n && e == cudaSuccess; ++q) {
        const long prefix = 1L << q;
        const long total = 2 * prefix * dr[q];
        const int grid = int(std::min<long>((total + 255) / 256, 8L * m->ctx->sm_count));
        dense_step_kernel<<<grid, 256, 0, m->stream>>>(cur, m->site_ptr[q], dl[q], dr[q], prefix, prune, nxt);
        count_launch(m, -1);
        e = cudaGetLastError();
        std::swap(cur, nxt);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, cur, (size_t(1) << n) * sizeof(double2), cudaMemcpyDeviceToHost, m->stream);
    m->stats.d2h_bytes += (size_t(1) << n) * sizeof(double2);
    wqc_status rc = e == cudaSuccess ? sync_status(m) : fail(WQC_ERR_CUDA, cudaGetErrorString(e));
    dfree(m, d_a, most * sizeof(double2));
    dfree(m, d_b, most * sizeof(double2));
    return rc;
}

wqc_status wqc_mps_bond_dims(wqc_mps* m, uint32_t* out) {
    if (!m || !out) return fail(WQC_ERR_INVALID, "null argument");
    if (wqc_status s = sync_status(m)) return s;
    std::vector<int> dr(m->n);
    CUDA_TRY(cudaMemcpy(dr.data(), m->d_dr, m->n * sizeof(int), cudaMemcpyDeviceToHost));
    for (int i = 0; i < m->n; ++i) out[i] = uint32_t(dr[i]);
    return WQC_OK;
}

wqc_status wqc_mps_download_site(wqc_mps* m, uint32_t site, uint32_t* l, uint32_t* r, double* buf) {
    if (!m || !l || !r) return fail(WQC_ERR_INVALID, "null argument");
    if (site >= uint32_t(m->n)) return fail(WQC_ERR_QUBIT_OUT_OF_RANGE, "site out of range");
    if (wqc_status s = sync_status(m)) return s;
    int dl = 0, dr = 0;
    CUDA_TRY(cudaMemcpy(&dl, m->d_dl + site, sizeof(int), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(&dr, m->d_dr + site, sizeof(int), cudaMemcpyDeviceToHost));
    *l = uint32_t(dl);
    *r = uint32_t(dr);
    if (buf)
        CUDA_TRY(cudaMemcpy(buf, m->site_ptr[site], size_t(dl) * 2 * dr * sizeof(double2),
                            cudaMemcpyDeviceToHost));
    return WQC_OK;
}

wqc_status wqc_mps_upload_site(wqc_mps* m, uint32_t site, uint32_t l, uint32_t r, const double* buf) {
    if (!m || !buf) return fail(WQC_ERR_INVALID, "null argument");
    if (site >= uint32_t(m->n)) return fail(WQC_ERR_QUBIT_OUT_OF_RANGE, "site out of range");
    // Against the site's own capacity (a batch slice may have a smaller chi_max than the state).
    const uint32_t cap = uint32_t(m->site_chi[site]);
    if (l == 0 || r == 0 || l > cap || r > cap) return fail(WQC_ERR_INVALID, "site shape exceeds max_bond_dim");
    if (wqc_status s = sync_status(m)) return s;
    CUDA_TRY(cudaMemcpy(m->site_ptr[site], buf, size_t(l) * 2 * r * sizeof(double2), cudaMemcpyHostToDevice));
    const int il = int(l), ir = int(r);
    CUDA_TRY(cudaMemcpy(m->d_dl + site, &il, sizeof(int), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(m->d_dr + site, &ir, sizeof(int), cudaMemcpyHostToDevice));
    if (site > 0) m->ub[site - 1] = std::max(m->ub[site - 1], il);
    if (int(site) + 1 < m->n) m->ub[site] = std::max(m->ub[site], ir);
    m->uploaded = true;
    m->touch(int(site), int(site));
    return WQC_OK;
}

wqc_status wqc_mps_overlap(wqc_mps* ket, wqc_mps* bra, uint32_t env_limit, double out[2]) {
    if (!ket || !bra || !out) return fail(WQC_ERR_INVALID, "null argument");
    if (ket->seg_first.size() != 1 || bra->seg_first.size() != 1)
        return fail(WQC_ERR_INVALID, "the overlap takes single states, not batches");
    if (ket->n != bra->n) return fail(WQC_ERR_INVALID, "mismatched register");  // EngineError::MismatchedRegister
    if (ket->ctx != bra->ctx) return fail(WQC_ERR_INVALID, "the two states live on different contexts");
    if (wqc_status s = sync_status(bra)) return s;
    if (wqc_status s = sync_status(ket)) return s;
    const int n = ket->n;
    std::vector<int> kdl(n), kdr(n), bdl(n), bdr(n);
    CUDA_TRY(cudaMemcpy(kdl.data(), ket->d_dl, n * sizeof(int), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(kdr.data(), ket->d_dr, n * sizeof(int), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(bdl.data(), bra->d_dl, n * sizeof(int), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(bdr.data(), bra->d_dr, n * sizeof(int), cudaMemcpyDeviceToHost));
    for (int q = 0; q < n; ++q) {
        if (kdl[q] != (q ? kdr[q - 1] : 1) || bdl[q] != (q ? bdr[q - 1] : 1))
            return fail(WQC_ERR_INVALID, "mps site shape does not match the overlap");
        if (env_limit && (unsigned long long)kdr[q] * bdr[q] > env_limit)  // mps.rs:1443-1448
            return fail(WQC_ERR_INVALID, "mps overlap environment exceeds " + std::to_string(env_limit));
    }
    const size_t env_bytes = size_t(ket->chi) * bra->chi * sizeof(double2);
    const size_t tmp_bytes = 2 * env_bytes;
    void *d_a = nullptr, *d_b = nullptr, *d_t = nullptr;
    auto release = [&]() {
        if (d_a) dfree(ket, d_a, env_bytes);
        if (d_b) dfree(ket, d_b, env_bytes);
        if (d_t) dfree(ket, d_t, tmp_bytes);
    };
    for (auto& pr : {std::make_pair(&d_a, env_bytes), std::make_pair(&d_b, env_bytes), std::make_pair(&d_t, tmp_bytes)})
        if (wqc_status st = dmalloc(ket, pr.first, pr.second)) {
            release();
            return st;
        }
    double2* env = static_cast<double2*>(d_a);
    double2* nxt = static_cast<double2*>(d_b);
    double2* tmp = static_cast<double2*>(d_t);
    const double2 one = cmake(1.0, 0.0);
    cudaError_t e = cudaMemcpyAsync(env, &one, sizeof(double2), cudaMemcpyHostToDevice, ket->stream);
    int kl = 1, bl = 1;
    for (int q = 0; q < n && e == cudaSuccess; ++q) {
        if (kdl[q] != kl || bdl[q] != bl) {
            e = cudaErrorInvalidValue;
            break;
        }
        const int kr = kdr[q], br = bdr[q];
        const long cap = 4L * ket->ctx->sm_count;
        overlap_half_kernel<<<int(std::min<long>((2L * bl * kr + 255) / 256, cap)), 256, 0, ket->stream>>>(
            env, kl, bl, ket->site_ptr[q], kr, tmp);
        overlap_next_kernel<<<int(std::min<long>((long(kr) * br + 255) / 256, cap)), 256, 0, ket->stream>>>(
            tmp, bl, kr, bra->site_ptr[q], br, nxt);
        count_launch(ket, -1);
        count_launch(ket, -1);
        std::swap(env, nxt);
        kl = kr;
        bl = br;
        e = cudaGetLastError();
    }
    double2 res = cmake(0, 0);
    wqc_status rc = WQC_OK;
    if (e == cudaErrorInvalidValue)
        rc = fail(WQC_ERR_INVALID, "mps site shape does not match the overlap");
    else if (e == cudaSuccess && (kl != 1 || bl != 1))
        rc = fail(WQC_ERR_INVALID, "mps overlap left an open bond");
    else if (e == cudaSuccess)
        e = cudaMemcpyAsync(&res, env, sizeof(double2), cudaMemcpyDeviceToHost, ket->stream);
    if (rc == WQC_OK) rc = e == cudaSuccess ? sync_status(ket) : fail(WQC_ERR_CUDA, cudaGetErrorString(e));
    release();
    if (rc != WQC_OK) return rc;
    out[0] = res.x;
    out[1] = res.y;
    return WQC_OK;
}

wqc_status wqc_mps_sample(wqc_mps* m, const uint32_t* qubits, uint32_t count, uint32_t shots, uint64_t seed,
                          uint64_t* out) {
    if (!m || (!qubits && count) || (!out && shots)) return fail(WQC_ERR_INVALID, "null argument");
    if (m->seg_first.size() != 1) return fail(WQC_ERR_INVALID, "sampling takes a single state, not a batch");
    if (count > 64) return fail(WQC_ERR_INVALID, "at most 64 measured qubits per shot");
    std::vector<int> bitpos(m->n, -1);
    for (uint32_t j = 0; j < count; ++j) {
        if (qubits[j] >= uint32_t(m->n)) return fail(WQC_ERR_QUBIT_OUT_OF_RANGE, "measured qubit out of range");
        if (bitpos[qubits[j]] >= 0) return fail(WQC_ERR_INVALID, "a qubit is listed twice");
        bitpos[qubits[j]] = int(j);
    }
    if (shots == 0) return WQC_OK;
    if (wqc_status s = check_uploaded_chain(m)) return s;
    if (wqc_status s = sync_status(m)) return s;
    const int n = m->n;
    std::vector<int> dl(n), dr(n);
    CUDA_TRY(cudaMemcpy(dl.data(), m->d_dl, n * sizeof(int), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(dr.data(), m->d_dr, n * sizeof(int), cudaMemcpyDeviceToHost));
    // E_q (dl[q] x dl[q]) at env_off[q]; E_n = 1 at env_off[n].
    std::vector<unsigned long long> env_off(n + 1);
    unsigned long long total = 0;
    for (int q = 0; q < n; ++q) {
        env_off[q] = total;
        total += (unsigned long long)dl[q] * dl[q];
    }
    env_off[n] = total;
    total += 1;
    const size_t env_bytes = total * sizeof(double2);
    const size_t tmp_bytes = size_t(2) * m->chi * m->chi * sizeof(double2);
    const size_t aux_bytes = (n + 1) * sizeof(unsigned long long) + n * sizeof(int) + 64;
    const size_t out_bytes = size_t(shots) * sizeof(uint64_t);
    void *d_env = nullptr, *d_tmp = nullptr, *d_aux = nullptr, *d_out = nullptr;
    auto release = [&]() {
        if (d_env) dfree(m, d_env, env_bytes);
        if (d_tmp) dfree(m, d_tmp, tmp_bytes);
        if (d_aux) dfree(m, d_aux, aux_bytes);
        if (d_out) dfree(m, d_out, out_bytes);
    };
    for (auto& pr : {std::make_pair(&d_env, env_bytes), std::make_pair(&d_tmp, tmp_bytes),
                     std::make_pair(&d_aux, aux_bytes), std::make_pair(&d_out, out_bytes)})
        if (wqc_status st = dmalloc(m, pr.first, pr.second)) {
            release();
            return st;
        }
    double2* env = static_cast<double2*>(d_env);
    double2* tmp = static_cast<double2*>(d_tmp);
    unsigned long long* d_off = static_cast<unsigned long long*>(d_aux);
    int* d_bitpos = reinterpret_cast<int*>(d_off + n + 1);
    const double2 one = cmake(1.0, 0.0);
    cudaError_t e = cudaMemcpyAsync(env + env_off[n], &one, sizeof(double2), cudaMemcpyHostToDevice, m->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_off, env_off.data(), (n + 1) * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                            m->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_bitpos, bitpos.data(), n * sizeof(int), cudaMemcpyHostToDevice, m->stream);
    // Right environments, from the last site down to site 1 (E_0 is not drawn from).
    for (int q = n - 1; q >= 1 && e == cudaSuccess; --q) {
        const int l = dl[q], r = dr[q];
        const int g1 = int(std::min<long>((2L * l * r + 255) / 256, 4L * m->ctx->sm_count));
        const int g2 = int(std::min<long>((long(l) * l + 255) / 256, 4L * m->ctx->sm_count));
        sample_env_half_kernel<<<g1, 256, 0, m->stream>>>(m->site_ptr[q], l, r, env + env_off[q + 1], tmp);
        sample_env_kernel<<<g2, 256, 0, m->stream>>>(m->site_ptr[q], l, r, tmp, env + env_off[q]);
        count_launch(m, -1);
        count_launch(m, -1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        const int grid = int(std::min<long>(long(shots), 8L * m->ctx->sm_count));
        sample_shots_kernel<<<grid, 256, 3 * m->chi * sizeof(double2), m->stream>>>(
            m->dev, env, d_off, d_bitpos, (unsigned long long)seed, int(shots), static_cast<unsigned long long*>(d_out));
        count_launch(m, -1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, out_bytes, cudaMemcpyDeviceToHost, m->stream);
    m->stats.d2h_bytes += out_bytes;
    wqc_status rc = e == cudaSuccess ? sync_status(m) : fail(WQC_ERR_CUDA, cudaGetErrorString(e));
    release();
    return rc;
}

wqc_status wqc_mps_expectation_pauli(wqc_mps* m, const char* labels, const double* coeffs, uint32_t nterms,
                                     double out[2]) {
    if (!m || !labels || !coeffs || !out) return fail(WQC_ERR_INVALID, "null argument");
    for (size_t i = 0; i < size_t(nterms) * m->n; ++i) {
        const char ch = labels[i];
        if (ch != 'I' && ch != 'X' && ch != 'Y' && ch != 'Z')
            return fail(WQC_ERR_INVALID, std::string("invalid pauli character in label"));
    }
    if (nterms == 0) {
        out[0] = out[1] = 0;
        return WQC_OK;
    }
    if (wqc_status st = check_uploaded_chain(m)) return st;
    const size_t E = size_t(m->chi) * m->chi;
    const size_t scratch = size_t(nterms) * 4 * E * sizeof(double2);
    void* d_lab = nullptr;
    void* d_scr = nullptr;
    void* d_out = nullptr;
    if (wqc_status s = dmalloc(m, &d_lab, size_t(nterms) * m->n + 16)) return s;
    if (wqc_status s = dmalloc(m, &d_scr, scratch)) {
        dfree(m, d_lab, size_t(nterms) * m->n + 16);
        return s;
    }
    if (wqc_status s = dmalloc(m, &d_out, nterms * sizeof(double2))) {
        dfree(m, d_lab, size_t(nterms) * m->n + 16);
        dfree(m, d_scr, scratch);
        return s;
    }
    wqc_status rc = WQC_OK;
    std::vector<double2> vals(nterms);
    cudaError_t e = cudaMemcpyAsync(d_lab, labels, size_t(nterms) * m->n, cudaMemcpyHostToDevice, m->stream);
    if (e == cudaSuccess) {
        pauli_expectation_kernel<<<nterms, 256, 0, m->stream>>>(m->dev, static_cast<const char*>(d_lab), int(nterms),
                                                                  static_cast<double2*>(d_scr), m->chi,
                                                                  static_cast<double2*>(d_out));
        count_launch(m, -1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(vals.data(), d_out, nterms * sizeof(double2), cudaMemcpyDeviceToHost, m->stream);
    if (e != cudaSuccess) rc = fail(WQC_ERR_CUDA, cudaGetErrorString(e));
    if (rc == WQC_OK) rc = sync_status(m);
    dfree(m, d_lab, size_t(nterms) * m->n + 16);
    dfree(m, d_scr, scratch);
    dfree(m, d_out, nterms * sizeof(double2));
    if (rc != WQC_OK) return rc;
    double re = 0, im = 0;
    for (uint32_t t = 0; t < nterms; ++t) {  // coeff * Re<P> (expectation.rs:177-185)
        const double v = vals[t].x;
        re += coeffs[2 * t] * v;
        im += coeffs[2 * t + 1] * v;
    }
    out[0] = re;
    out[1] = im;
    return WQC_OK;
}

wqc_status wqc_mps_debug_workspace(wqc_mps* m, uint32_t slot, int32_t which, void* out, uint64_t bytes) {
    if (!m || !out) return fail(WQC_ERR_INVALID, "null argument");
    if (slot >= uint32_t(m->nslots)) return fail(WQC_ERR_INVALID, "slot out of range");
    if (wqc_status s = sync_status(m)) return s;
    SlotBuffers b;
    CUDA_TRY(cudaMemcpy(&b, m->d_slots + slot, sizeof(b), cudaMemcpyDeviceToHost));
    const void* src = nullptr;
    const int R = m->slot_R[slot], E = m->slot_E[slot];
    size_t cap = 0;
    switch (which) {
        case 0: src = b.theta; cap = size_t(R) * R * sizeof(double2); break;
        case 1: src = b.omega; cap = size_t(R) * E * sizeof(double2); break;
        case 2: src = b.y0; cap = size_t(R) * E * sizeof(double2); break;
        case 3: src = b.zr; cap = size_t(R) * E * sizeof(double2); break;
        case 4: src = b.y; cap = size_t(R) * E * sizeof(double2); break;
        case 5: src = b.q; cap = size_t(R) * E * sizeof(double2); break;
        case 6: src = b.b; cap = size_t(R) * E * sizeof(double2); break;
        case 7: src = b.w; cap = size_t(R) * R * sizeof(double2); break;
        case 8: src = b.z; cap = size_t(R) * R * sizeof(double2); break;
        case 9: src = b.sigma; cap = size_t(R) * sizeof(double); break;
        case 10: src = b.perm; cap = size_t(R) * sizeof(int); break;
        case 11: src = b.tau; cap = size_t(E) * sizeof(double2); break;
        case 12: src = m->d_state + slot; cap = sizeof(SplitState); break;
        default: return fail(WQC_ERR_INVALID, "unknown workspace buffer");
    }
    CUDA_TRY(cudaMemcpy(out, src, std::min<size_t>(cap, bytes), cudaMemcpyDeviceToHost));
    return WQC_OK;
}

uint32_t wqc_mps_split_count(wqc_mps* m) { return m ? m->rec_count : 0; }

wqc_status wqc_mps_split_records(wqc_mps* m, wqc_split_info* out, uint32_t max, uint32_t* written) {
    if (!m || (!out && max)) return fail(WQC_ERR_INVALID, "null argument");
    if (wqc_status s = sync_status(m)) return s;
    const uint32_t k = std::min(max, m->rec_count);
    if (k) CUDA_TRY(cudaMemcpy(out, m->d_records, k * sizeof(wqc_split_info), cudaMemcpyDeviceToHost));
    if (written) *written = k;
    return WQC_OK;
}

uint64_t wqc_mps_peak_vram_bytes(wqc_mps* m) { return m ? m->bytes_peak : 0; }

const char* wqc_mps_backend_label(wqc_mps*) { return "cuda"; }

wqc_status wqc_mps_set_profiling(wqc_mps* m, int32_t on) {
    if (!m) return fail(WQC_ERR_INVALID, "null argument");
    m->profiling = on != 0;
    return WQC_OK;
}

wqc_status wqc_mps_kernel_stats(wqc_mps* m, wqc_kernel_stats* out) {
    if (!m || !out) return fail(WQC_ERR_INVALID, "null argument");
    CUDA_TRY(cudaStreamSynchronize(m->stream));
    for (auto& e : m->events) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, e.second.first, e.second.second) == cudaSuccess) m->stats.milliseconds[e.first] += ms;
        m->event_pool.push_back(e.second.first);
        m->event_pool.push_back(e.second.second);
    }
    m->events.clear();
    unsigned long long c[3] = {0, 0, 0};
    CUDA_TRY(cudaMemcpy(c, m->d_counters, sizeof(c), cudaMemcpyDeviceToHost));
    m->stats.jacobi_tasks = c[0];
    m->stats.jacobi_sweeps = c[1];
    m->stats.jacobi_sweeps_first = c[2];
    *out = m->stats;
    return WQC_OK;
}

void wqc_mps_reset_stats(wqc_mps* m) {
    if (!m) return;
    cudaStreamSynchronize(m->stream);
    for (auto& e : m->events) {
        m->event_pool.push_back(e.second.first);
        m->event_pool.push_back(e.second.second);
    }
    m->events.clear();
    m->stats = wqc_kernel_stats{};
    cudaMemset(m->d_counters, 0, 3 * sizeof(unsigned long long));
}

void* wqc_mps_stream(wqc_mps* m) { return m ? static_cast<void*>(m->stream) : nullptr; }

}  // extern "C"

// ===========================================================================
// Differentiation form: the adjoint (reverse-mode) gradient of a Pauli-sum
// observable with respect to the rotation angles of the gate list.
//
// Forward: the gate list runs on the state from |0...0> in segments; the
// sites (and bonds) at the start of every segment but the first, and at the
// end, are copied to checkpoints.  Backward: the site cotangents of the end
// state come from the observable's environments; then, segment by segment
// from the last, the segment's state is restored from its checkpoint and its
// operations are recomputed one at a time, the inputs each needs in reverse
// (the site before a one-qubit gate; the sites, theta and the Jacobi's W,
// singular values and order of a split) copied to a tape, and the tape is
// swept in reverse (adjoint_kernels.cu).  The split rule is the exact one on
// every split (a range finder seeded by a rank-48 test matrix has no
// meaningful derivative), and the plain FP64 form is required.
// ===========================================================================
struct wqc_adjoint {
    wqc_mps* m = nullptr;
    std::vector<wqc_gate> gates;
    std::vector<uint32_t> starts;  // segment starts; segment s is [starts[s], starts[s + 1] or count)
    size_t pool_bytes = 0;         // the state's site pool
    // checkpoint c (1 .. nseg - 1: segment starts; nseg: the end state):
    // site pool, then dl and dr
    std::vector<char*> cp;
    std::vector<std::vector<int>> cp_ub;
    uint32_t end_records = 0;
    bool forward_done = false;
};

namespace {

// d u / d angle of the rotations of gates.rs:10-66.
bool rotation_derivative(const wqc_gate& g, double2* du) {
    const double s = 0.5 * std::sin(g.angle / 2.0), c = 0.5 * std::cos(g.angle / 2.0);
    switch (g.kind) {
        case WQC_GATE_RX:
            du[0] = C(-s); du[1] = C(0, -c); du[2] = C(0, -c); du[3] = C(-s);
            return true;
        case WQC_GATE_RY:
            du[0] = C(-s); du[1] = C(-c); du[2] = C(c); du[3] = C(-s);
            return true;
        case WQC_GATE_RZ:
            du[0] = C(-s, -c); du[1] = C(0); du[2] = C(0); du[3] = C(-s, c);
            return true;
        default:
            return false;
    }
}

size_t adj_pool_bytes(const wqc_mps* m) { return size_t(m->n) * m->chi * 2 * m->chi * sizeof(double2); }

wqc_status adj_save(wqc_adjoint* a, size_t c) {
    wqc_mps* m = a->m;
    const size_t bytes = a->pool_bytes + 2 * size_t(m->n) * sizeof(int);
    if (!a->cp[c]) {
        void* p = nullptr;
        if (wqc_status st = dmalloc(m, &p, bytes)) return st;
        a->cp[c] = static_cast<char*>(p);
    }
    CUDA_TRY(cudaMemcpyAsync(a->cp[c], m->site_pool, a->pool_bytes, cudaMemcpyDeviceToDevice, m->stream));
    CUDA_TRY(cudaMemcpyAsync(a->cp[c] + a->pool_bytes, m->d_dl, size_t(m->n) * sizeof(int), cudaMemcpyDeviceToDevice,
                             m->stream));
    CUDA_TRY(cudaMemcpyAsync(a->cp[c] + a->pool_bytes + size_t(m->n) * sizeof(int), m->d_dr,
                             size_t(m->n) * sizeof(int), cudaMemcpyDeviceToDevice, m->stream));
    a->cp_ub[c] = m->ub;
    return WQC_OK;
}

wqc_status adj_restore(wqc_adjoint* a, size_t c) {
    wqc_mps* m = a->m;
    if (c == 0) {
        reset_sites_kernel<<<(m->n + 255) / 256, 256, 0, m->stream>>>(m->dev);
        CUDA_TRY(cudaGetLastError());
        std::fill(m->ub.begin(), m->ub.end(), 1);
    } else {
        CUDA_TRY(cudaMemcpyAsync(m->site_pool, a->cp[c], a->pool_bytes, cudaMemcpyDeviceToDevice, m->stream));
        CUDA_TRY(cudaMemcpyAsync(m->d_dl, a->cp[c] + a->pool_bytes, size_t(m->n) * sizeof(int),
                                 cudaMemcpyDeviceToDevice, m->stream));
        CUDA_TRY(cudaMemcpyAsync(m->d_dr, a->cp[c] + a->pool_bytes + size_t(m->n) * sizeof(int),
                                 size_t(m->n) * sizeof(int), cudaMemcpyDeviceToDevice, m->stream));
        m->ub = a->cp_ub[c];
    }
    m->lvalid = 0;
    m->rvalid = m->n - 1;
    return WQC_OK;
}

// Device buffers of one backward pass, freed together.
struct AdjBuffers {
    wqc_mps* m;
    std::vector<std::pair<void*, size_t>> owned;
    explicit AdjBuffers(wqc_mps* mm) : m(mm) {}
    ~AdjBuffers() {
        if (m->stream) cudaStreamSynchronize(m->stream);
        for (auto& p : owned) dfree(m, p.first, p.second);
    }
    template <class T>
    wqc_status get(T** out, size_t count) {
        void* p = nullptr;
        const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
        if (wqc_status st = dmalloc(m, &p, bytes)) return st;
        owned.push_back({p, bytes});
        *out = static_cast<T*>(p);
        return WQC_OK;
    }
    void release(void* p) {
        for (size_t i = 0; i < owned.size(); ++i)
            if (owned[i].first == p) {
                cudaStreamSynchronize(m->stream);
                dfree(m, p, owned[i].second);
                owned.erase(owned.begin() + long(i));
                return;
            }
    }
};

// One recomputed operation on the tape.
struct TapeEntry {
    bool two;
    int site;
    int gate;
    double2 u[16];
    size_t off;  // byte offset of its data in the tape arena
};

}  // namespace

extern "C" {

wqc_status wqc_adjoint_forward(wqc_mps* m, const wqc_gate* gates, uint32_t count, const uint32_t* checkpoints,
                               uint32_t ncheckpoints, wqc_adjoint** out) {
    if (!m || !out || (!gates && count) || (ncheckpoints && !checkpoints)) return fail(WQC_ERR_INVALID, "null argument");
    if (m->seg_first.size() != 1) return fail(WQC_ERR_INVALID, "the adjoint takes a single state, not a batch");
    if (m->fp32) return fail(WQC_ERR_INVALID, "the adjoint differentiates the plain FP64 form");
    Expander check;
    if (wqc_status st = expand(m->n, gates, count, false, check)) return st;
    auto* a = new wqc_adjoint();
    a->m = m;
    a->gates.assign(gates, gates + count);
    a->starts.push_back(0);
    std::vector<uint32_t> cps(checkpoints, checkpoints + ncheckpoints);
    std::sort(cps.begin(), cps.end());
    for (uint32_t c : cps)
        if (c > a->starts.back() && c < count) a->starts.push_back(c);
    a->pool_bytes = adj_pool_bytes(m);
    a->cp.assign(a->starts.size() + 1, nullptr);
    a->cp_ub.resize(a->starts.size() + 1);
    const bool rule = m->exact_only;
    m->exact_only = true;
    wqc_status st = wqc_mps_reset(m);
    for (size_t sgi = 0; sgi < a->starts.size() && st == WQC_OK; ++sgi) {
        if (sgi > 0) st = adj_save(a, sgi);
        const uint32_t g0 = a->starts[sgi], g1 = sgi + 1 < a->starts.size() ? a->starts[sgi + 1] : count;
        if (st == WQC_OK && g1 > g0) {
            Expander ex;
            st = expand(m->n, a->gates.data() + g0, g1 - g0, false, ex);
            if (st == WQC_OK) st = run_ops(m, ex.ops);
        }
    }
    if (st == WQC_OK) st = adj_save(a, a->starts.size());
    if (st == WQC_OK) st = sync_status(m);
    m->exact_only = rule;
    a->end_records = m->rec_count;
    if (st != WQC_OK) {
        wqc_adjoint_destroy(a);
        return st;
    }
    a->forward_done = true;
    *out = a;
    return WQC_OK;
}

wqc_status wqc_adjoint_backward(wqc_adjoint* a, const char* labels, const double* coeffs, uint32_t nterms,
                                double value[2], double* grad) {
    if (!a || !a->forward_done || !labels || !coeffs || !value || (!grad && !a->gates.empty()))
        return fail(WQC_ERR_INVALID, "null argument");
    wqc_mps* m = a->m;
    const int n = m->n, chi = m->chi, R = 2 * chi;
    for (size_t i = 0; i < size_t(nterms) * n; ++i) {
        const char ch = labels[i];
        if (ch != 'I' && ch != 'X' && ch != 'Y' && ch != 'Z')
            return fail(WQC_ERR_INVALID, std::string("invalid pauli character in label"));
    }
    if (nterms == 0) return fail(WQC_ERR_INVALID, "the adjoint needs at least one Pauli term");
    CUDA_TRY(cudaSetDevice(m->ctx->device));
    const bool rule = m->exact_only;
    m->exact_only = true;
    struct RuleGuard {
        wqc_mps* m;
        bool rule;
        ~RuleGuard() { m->exact_only = rule; }
    } guard{m, rule};
    AdjBuffers buf(m);
    const size_t site_cap = size_t(chi) * 2 * chi;
    // Cotangent sites, one per site at the state's capacity, and their pointers.
    double2* bar_pool = nullptr;
    double2** d_bars = nullptr;
    if (wqc_status st = buf.get(&bar_pool, site_cap * n)) return st;
    if (wqc_status st = buf.get(&d_bars, n)) return st;
    std::vector<double2*> bars(n);
    for (int q = 0; q < n; ++q) bars[q] = bar_pool + site_cap * q;
    CUDA_TRY(cudaMemcpyAsync(d_bars, bars.data(), n * sizeof(double2*), cudaMemcpyHostToDevice, m->stream));
    // The end state and the observable's environments, values and cotangents.
    if (wqc_status st = adj_restore(a, a->starts.size())) return st;
    {
        const size_t E = size_t(chi) * chi;
        char* d_lab = nullptr;
        double* d_cre = nullptr;
        double2 *envs = nullptr, *tmp = nullptr, *vals = nullptr;
        if (wqc_status st = buf.get(&d_lab, size_t(nterms) * n + 16)) return st;
        if (wqc_status st = buf.get(&d_cre, nterms)) return st;
        if (wqc_status st = buf.get(&envs, size_t(nterms) * (2 * n + 1) * E)) return st;
        if (wqc_status st = buf.get(&tmp, size_t(nterms) * 2 * E)) return st;
        if (wqc_status st = buf.get(&vals, nterms)) return st;
        std::vector<double> cre(nterms);
        for (uint32_t t = 0; t < nterms; ++t) cre[t] = coeffs[2 * t];
        CUDA_TRY(cudaMemcpyAsync(d_lab, labels, size_t(nterms) * n, cudaMemcpyHostToDevice, m->stream));
        CUDA_TRY(cudaMemcpyAsync(d_cre, cre.data(), nterms * sizeof(double), cudaMemcpyHostToDevice, m->stream));
        adj_pauli_envs_kernel<<<nterms, 256, 0, m->stream>>>(m->dev, d_lab, int(nterms), chi, envs, tmp, vals);
        count_launch(m, -1);
        // Holes in chunks of terms, accumulated in term order.
        const size_t per_term = 2 * size_t(n) * site_cap * sizeof(double2);
        const int chunk = int(std::max<size_t>(1, std::min<size_t>(16, (size_t(1) << 30) / per_term)));
        double2 *holes = nullptr, *htmp = nullptr;
        if (wqc_status st = buf.get(&holes, size_t(chunk) * n * site_cap)) return st;
        if (wqc_status st = buf.get(&htmp, size_t(chunk) * n * site_cap)) return st;
        const int agrid = int(std::max<size_t>(1, std::min<size_t>((site_cap + 255) / 256, 64)));
        for (uint32_t t0 = 0; t0 < nterms; t0 += uint32_t(chunk)) {
            const int cnt = int(std::min<uint32_t>(uint32_t(chunk), nterms - t0));
            adj_pauli_holes_kernel<<<dim3(n, cnt), 256, 0, m->stream>>>(m->dev, d_lab, int(t0), chi, envs, htmp, holes);
            adj_pauli_accumulate_kernel<<<dim3(agrid, n), 256, 0, m->stream>>>(m->dev, d_bars, holes, d_cre, int(t0),
                                                                             cnt, chi, t0 == 0 ? 1 : 0);
            count_launch(m, -1);
            count_launch(m, -1);
        }
        CUDA_TRY(cudaGetLastError());
        std::vector<double2> hv(nterms);
        CUDA_TRY(cudaMemcpyAsync(hv.data(), vals, nterms * sizeof(double2), cudaMemcpyDeviceToHost, m->stream));
        CUDA_TRY(cudaStreamSynchronize(m->stream));
        double re = 0, im = 0;
        for (uint32_t t = 0; t < nterms; ++t) {  // coeff * Re<P> (expectation.rs:177-185), term order
            re += coeffs[2 * t] * hv[t].x;
            im += coeffs[2 * t + 1] * hv[t].x;
        }
        value[0] = re;
        value[1] = im;
        buf.release(envs);
        buf.release(tmp);
        buf.release(holes);
        buf.release(htmp);
    }
    // Gradient slots: one per one-qubit operation of the whole list.
    Expander all;
    if (wqc_status st = expand(n, a->gates.data(), uint32_t(a->gates.size()), false, all)) return st;
    size_t n1q = 0;
    for (const Op& o : all.ops) n1q += o.two ? 0 : 1;
    double* d_grad = nullptr;
    if (wqc_status st = buf.get(&d_grad, n1q + 1)) return st;
    CUDA_TRY(cudaMemsetAsync(d_grad, 0, (n1q + 1) * sizeof(double), m->stream));
    std::vector<int> slot_gate;  // gate of each gradient slot
    // Split workspace (column-major R x R matrices) and the slot-0 buffers.
    double2* ws = nullptr;
    double* wsd = nullptr;
    if (wqc_status st = buf.get(&ws, 10 * size_t(R) * R)) return st;
    if (wqc_status st = buf.get(&wsd, 2 * size_t(R))) return st;
    SlotBuffers slot0;
    CUDA_TRY(cudaMemcpy(&slot0, m->d_slots, sizeof(slot0), cudaMemcpyDeviceToHost));
    // Tape layout of one operation (bytes, 256-aligned parts).
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t site_b = al(site_cap * sizeof(double2));
    const size_t mat_b = al(size_t(R) * R * sizeof(double2));
    const size_t one_b = site_b + al(2 * sizeof(int));
    const size_t two_b = 2 * site_b + 2 * mat_b + al(R * sizeof(double)) + al(R * sizeof(int)) + al(sizeof(SplitState));
    char* tape = nullptr;
    size_t tape_cap = 0;
    // First gradient slot of each segment (one-qubit operations in program order).
    std::vector<size_t> seg_slot0(a->starts.size());
    {
        size_t acc = 0;
        for (size_t sgi = 0; sgi < a->starts.size(); ++sgi) {
            seg_slot0[sgi] = acc;
            const uint32_t g1 = sgi + 1 < a->starts.size() ? a->starts[sgi + 1] : uint32_t(a->gates.size());
            for (const Op& o : all.ops)
                if (!o.two && o.gate >= int(a->starts[sgi]) && o.gate < int(g1)) ++acc;
        }
        for (const Op& o : all.ops)
            if (!o.two) slot_gate.push_back(o.gate);
    }
    const int eg = int(std::min<long>((long(R) * R + 255) / 256, 4L * m->ctx->sm_count));
    const dim3 gg((R + 31) / 32, (R + 31) / 32);
    for (size_t sgi = a->starts.size(); sgi-- > 0;) {
        const uint32_t g0 = a->starts[sgi];
        const uint32_t g1 = sgi + 1 < a->starts.size() ? a->starts[sgi + 1] : uint32_t(a->gates.size());
        if (g1 <= g0) continue;
        Expander ex;
        if (wqc_status st = expand(n, a->gates.data() + g0, g1 - g0, false, ex)) return st;
        std::vector<TapeEntry> ents;
        size_t need = 0;
        for (const Op& o : ex.ops) {
            TapeEntry t{};
            t.two = o.two;
            t.site = o.site;
            t.gate = o.gate + int(g0);
            if (o.two)
                std::memcpy(t.u, o.ueff, sizeof(t.u));
            else
                std::memcpy(t.u, o.m2.u, sizeof(o.m2.u));
            t.off = need;
            need += o.two ? two_b : one_b;
            ents.push_back(t);
        }
        if (need > tape_cap) {
            if (tape) buf.release(tape);
            tape = nullptr;
            if (wqc_status st = buf.get(&tape, need)) return st;
            tape_cap = need;
        }
        // Recompute the segment one operation at a time, taping each one's inputs.
        if (wqc_status st = adj_restore(a, sgi)) return st;
        for (size_t k = 0; k < ex.ops.size(); ++k) {
            const Op& o = ex.ops[k];
            char* base = tape + ents[k].off;
            if (!o.two) {
                CUDA_TRY(cudaMemcpyAsync(base, m->site_ptr[o.site], site_cap * sizeof(double2),
                                         cudaMemcpyDeviceToDevice, m->stream));
                CUDA_TRY(cudaMemcpyAsync(base + site_b, m->d_dl + o.site, sizeof(int), cudaMemcpyDeviceToDevice,
                                         m->stream));
                CUDA_TRY(cudaMemcpyAsync(base + site_b + sizeof(int), m->d_dr + o.site, sizeof(int),
                                         cudaMemcpyDeviceToDevice, m->stream));
            } else {
                CUDA_TRY(cudaMemcpyAsync(base, m->site_ptr[o.site], site_cap * sizeof(double2),
                                         cudaMemcpyDeviceToDevice, m->stream));
                CUDA_TRY(cudaMemcpyAsync(base + site_b, m->site_ptr[o.site + 1], site_cap * sizeof(double2),
                                         cudaMemcpyDeviceToDevice, m->stream));
            }
            std::vector<Op> one{o};
            if (wqc_status st = run_ops(m, one)) return st;
            if (o.two) {
                char* p = base + 2 * site_b;
                CUDA_TRY(cudaMemcpyAsync(p, slot0.theta, size_t(R) * R * sizeof(double2), cudaMemcpyDeviceToDevice,
                                         m->stream));
                CUDA_TRY(cudaMemcpyAsync(p + mat_b, slot0.w, size_t(R) * R * sizeof(double2),
                                         cudaMemcpyDeviceToDevice, m->stream));
                CUDA_TRY(cudaMemcpyAsync(p + 2 * mat_b, slot0.sigma, R * sizeof(double), cudaMemcpyDeviceToDevice,
                                         m->stream));
                CUDA_TRY(cudaMemcpyAsync(p + 2 * mat_b + al(R * sizeof(double)), slot0.perm, R * sizeof(int),
                                         cudaMemcpyDeviceToDevice, m->stream));
                CUDA_TRY(cudaMemcpyAsync(p + 2 * mat_b + al(R * sizeof(double)) + al(R * sizeof(int)), m->d_state,
                                         sizeof(SplitState), cudaMemcpyDeviceToDevice, m->stream));
            }
        }
        // Reverse sweep over the segment.
        size_t slot = seg_slot0[sgi];
        for (const TapeEntry& t : ents) slot += t.two ? 0 : 1;
        for (size_t k = ents.size(); k-- > 0;) {
            const TapeEntry& t = ents[k];
            const char* base = tape + t.off;
            if (!t.two) {
                --slot;
                Adj1q g{};
                std::memcpy(g.u, t.u, sizeof(g.u));
                g.has_du = rotation_derivative(a->gates[t.gate], g.du) ? 1 : 0;
                g.slot = int(slot);
                adj_one_qubit_kernel<<<1, 256, 0, m->stream>>>(bars[t.site], reinterpret_cast<const double2*>(base),
                                                               reinterpret_cast<const int*>(base + site_b), g, d_grad);
                count_launch(m, -1);
                continue;
            }
            AdjSplit A{};
            const char* p = base + 2 * site_b;
            A.site_l = reinterpret_cast<const double2*>(base);
            A.site_r = reinterpret_cast<const double2*>(base + site_b);
            A.theta = reinterpret_cast<const double2*>(p);
            A.w = reinterpret_cast<const double2*>(p + mat_b);
            A.sigma = reinterpret_cast<const double*>(p + 2 * mat_b);
            A.perm = reinterpret_cast<const int*>(p + 2 * mat_b + al(R * sizeof(double)));
            A.st = reinterpret_cast<const SplitState*>(p + 2 * mat_b + al(R * sizeof(double)) + al(R * sizeof(int)));
            A.bar_l = bars[t.site];
            A.bar_r = bars[t.site + 1];
            std::memcpy(A.u, t.u, sizeof(A.u));
            double2* w = ws;
            const size_t RR = size_t(R) * R;
            A.U = w; A.V = w + RR; A.Ub = w + 2 * RR; A.Vb = w + 3 * RR; A.M = w + 4 * RR; A.Nm = w + 5 * RR;
            A.Z = w + 6 * RR; A.T1 = w + 7 * RR; A.tb = w + 8 * RR; A.tb0 = w + 9 * RR;
            A.inv = wsd;
            A.sq = wsd + R;
            A.R = R;
            adj_split_prep_kernel<<<eg, 256, 0, m->stream>>>(A);
            adj_split_gemm_kernel<<<gg, 256, 0, m->stream>>>(A, kAdjStageOther);
            adj_split_gemm_kernel<<<gg, 256, 0, m->stream>>>(A, kAdjStageM);
            adj_split_gemm_kernel<<<gg, 256, 0, m->stream>>>(A, kAdjStageN);
            adj_split_assemble_kernel<<<eg, 256, 0, m->stream>>>(A);
            adj_split_gemm_kernel<<<gg, 256, 0, m->stream>>>(A, kAdjStageT1);
            adj_split_gemm_kernel<<<gg, 256, 0, m->stream>>>(A, kAdjStageTb);
            adj_split_gemm_kernel<<<gg, 256, 0, m->stream>>>(A, kAdjStageTb2);
            adj_split_gate_kernel<<<eg, 256, 0, m->stream>>>(A);
            adj_split_gemm_kernel<<<gg, 256, 0, m->stream>>>(A, kAdjStageBarL);
            adj_split_gemm_kernel<<<gg, 256, 0, m->stream>>>(A, kAdjStageBarR);
            for (int c = 0; c < 11; ++c) count_launch(m, -1);
        }
        CUDA_TRY(cudaGetLastError());
    }
    std::vector<double> hg(n1q + 1);
    CUDA_TRY(cudaMemcpyAsync(hg.data(), d_grad, (n1q + 1) * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    if (wqc_status st = sync_status(m)) return st;
    for (size_t i = 0; i < a->gates.size(); ++i) grad[i] = 0.0;
    for (size_t sl = 0; sl < n1q; ++sl) grad[slot_gate[sl]] += hg[sl];
    // The state holds the end state again; its records are the forward's.
    if (wqc_status st = adj_restore(a, a->starts.size())) return st;
    m->rec_count = a->end_records;
    return sync_status(m);
}

void wqc_adjoint_destroy(wqc_adjoint* a) {
    if (!a) return;
    if (a->m) {
        if (a->m->stream) cudaStreamSynchronize(a->m->stream);
        const size_t bytes = a->pool_bytes + 2 * size_t(a->m->n) * sizeof(int);
        for (char* p : a->cp) dfree(a->m, p, bytes);
    }
    delete a;
}

}  // extern "C"

// ===========================================================================
// Autotuner of the Jacobi SVD's cluster size, with a fingerprinted cache (the
// pattern of the reference's GEMM side calibration, src/tn/gpu/gemm.rs:
// 495-543, 649-702: measure once per machine, keep the result in a file keyed
// by what the measurement depends on, reuse it on later starts).
//
// For every saturated shape of the configured chi_max values (2 chi x 2 chi,
// chi in 16, 32, 64, 128), in the plain form and in the precision form's
// first phase, and for both kinds of wave -- one latency-bound split, and a
// batch of 32 splits that fills the device -- each cluster size whose shared
// memory fits is timed on seeded random sites (Jacobi kernel time from the
// state's CUDA events, best of three) and the fastest is kept.  Shapes the
// table does not hold keep the cost model of choose_cluster.
// ===========================================================================
namespace {

constexpr int kTuneVersion = 1;

std::string tune_fingerprint(const wqc_cuda_ctx* ctx) {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, ctx->device);
    int drv = 0, rt = 0;
    cudaDriverGetVersion(&drv);
    cudaRuntimeGetVersion(&rt);
    std::string name(prop.name);
    for (char& c : name)
        if (c == '|' || c == '\n' || c == '\r') c = ' ';
    return "wqc-jacobi-clusters v" + std::to_string(kTuneVersion) + "|" + name + "|sm=" +
           std::to_string(prop.multiProcessorCount) + "|cc=" + std::to_string(prop.major) + "." +
           std::to_string(prop.minor) + "|driver=" + std::to_string(drv) + "|runtime=" + std::to_string(rt) +
           "|max_cluster=" + std::to_string(ctx->max_cluster);
}

std::string tune_cache_path(const char* path) {
    if (path && *path) return path;
    if (const char* p = std::getenv("WQC_TUNE_PATH")) return p;
    std::string base;
    if (const char* x = std::getenv("XDG_CACHE_HOME"))
        base = x;
    else if (const char* h = std::getenv("HOME"))
        base = std::string(h) + "/.cache";
    else
        base = ".";
    return base + "/wqc/jacobi-clusters";
}

bool tune_read(const std::string& path, const std::string& fp, std::vector<wqc_cuda_ctx::Tuned>& out) {
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    char line[512];
    bool ok = std::fgets(line, sizeof(line), f) != nullptr;
    if (ok) {
        std::string first(line);
        while (!first.empty() && (first.back() == '\n' || first.back() == '\r')) first.pop_back();
        ok = first == fp;
    }
    std::vector<wqc_cuda_ctx::Tuned> t;
    while (ok && std::fgets(line, sizeof(line), f)) {
        wqc_cuda_ctx::Tuned e{};
        if (std::sscanf(line, "%d %d %d %d %d %d", &e.M, &e.N, &e.len, &e.elem, &e.throughput, &e.C) == 6 && e.C >= 1)
            t.push_back(e);
    }
    std::fclose(f);
    if (ok) out = t;
    return ok;
}

bool tune_write(const std::string& path, const std::string& fp, const std::vector<wqc_cuda_ctx::Tuned>& t) {
    const size_t slash = path.find_last_of('/');
    if (slash != std::string::npos) {  // create the parent directories
        std::string dir = path.substr(0, slash);
        for (size_t i = 1; i <= dir.size(); ++i)
            if (i == dir.size() || dir[i] == '/') {
                const std::string part = dir.substr(0, i);
                if (!part.empty()) mkdir(part.c_str(), 0755);
            }
    }
    const std::string tmp = path + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "w");
    if (!f) return false;
    std::fprintf(f, "%s\n", fp.c_str());
    for (const auto& e : t) std::fprintf(f, "%d %d %d %d %d %d\n", e.M, e.N, e.len, e.elem, e.throughput, e.C);
    const bool ok = std::fclose(f) == 0;
    return ok && std::rename(tmp.c_str(), path.c_str()) == 0;
}

// Seeded random complex entries in [-1, 1) (xorshift64*).
void fill_random(std::vector<double>& v, unsigned long long& state) {
    for (double& x : v) {
        state ^= state >> 12;
        state ^= state << 25;
        state ^= state >> 27;
        x = double((state * 2685821657736338717ull) >> 11) * (2.0 / 9007199254740992.0) - 1.0;
    }
}

// Jacobi milliseconds of one wave of `count` exact 2chi x 2chi splits at the
// cluster size the context forces (best of `reps`); < 0 on failure.
double tune_measure(wqc_cuda_ctx* ctx, int chi, int precision, int count, int reps) {
    std::vector<uint32_t> qs(count, 4), chis(count, uint32_t(chi));
    wqc_mps* m = nullptr;
    if (wqc_batch_create(ctx, uint32_t(count), qs.data(), chis.data(), precision, 0, &m) != WQC_OK) return -1.0;
    if (count == 1) m->batch = false;  // one split: the latency-bound kind of wave
    m->exact_only = true;
    unsigned long long rng = 0x9E3779B97F4A7C15ull ^ (unsigned long long)(chi * 131 + count);
    const int dims[4][2] = {{1, chi}, {chi, chi}, {chi, chi}, {chi, 1}};
    std::vector<double> buf;
    double best = -1.0;
    for (int rep = 0; rep <= reps; ++rep) {
        wqc_mps_reset(m);
        for (int sl = 0; sl < count; ++sl)
            for (int q = 0; q < 4; ++q) {
                buf.assign(size_t(dims[q][0]) * 2 * dims[q][1] * 2, 0.0);
                fill_random(buf, rng);
                if (wqc_mps_upload_site(m, uint32_t(sl * 4 + q), uint32_t(dims[q][0]), uint32_t(dims[q][1]),
                                        buf.data()) != WQC_OK) {
                    wqc_mps_destroy(m);
                    return -1.0;
                }
            }
        std::vector<wqc_gate> gates(count);
        std::vector<uint32_t> offs(count + 1);
        for (int sl = 0; sl < count; ++sl) {
            gates[sl] = wqc_gate{WQC_GATE_CZ, 1, 2, 0, 0.0};
            offs[sl] = uint32_t(sl);
        }
        offs[count] = uint32_t(count);
        wqc_mps_reset_stats(m);
        wqc_mps_set_profiling(m, rep > 0 ? 1 : 0);  // rep 0 warms up
        wqc_status st = wqc_batch_apply_gates(m, gates.data(), offs.data());
        wqc_kernel_stats ks{};
        if (st == WQC_OK) st = wqc_mps_synchronize(m);
        if (st == WQC_OK) st = wqc_mps_kernel_stats(m, &ks);
        if (st != WQC_OK) {
            wqc_mps_destroy(m);
            return -1.0;
        }
        if (rep > 0 && (best < 0 || ks.milliseconds[0] < best)) best = ks.milliseconds[0];
    }
    wqc_mps_destroy(m);
    return best;
}

}  // namespace

extern "C" {

wqc_status wqc_cuda_autotune(wqc_cuda_ctx* ctx, const char* cache_path, double budget_seconds, uint32_t* entries) {
    if (!ctx) return fail(WQC_ERR_INVALID, "null context");
    CUDA_TRY(cudaSetDevice(ctx->device));
    const std::string fp = tune_fingerprint(ctx);
    const std::string path = tune_cache_path(cache_path);
    std::vector<wqc_cuda_ctx::Tuned> table;
    if (tune_read(path, fp, table)) {
        ctx->tuned = table;
        if (entries) *entries = uint32_t(table.size());
        return WQC_OK;
    }
    const auto t0 = std::chrono::steady_clock::now();
    auto elapsed = [&]() {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    };
    ctx->tuned.clear();
    for (int precision : {WQC_PRECISION_FP64, WQC_PRECISION_FP32}) {
        for (int chi : {16, 32, 64, 128}) {
            for (int throughput : {0, 1}) {
                if (budget_seconds > 0 && elapsed() > budget_seconds) break;
                const int M = 2 * chi, N = 2 * chi;
                const size_t elem = precision == WQC_PRECISION_FP32 ? sizeof(float2) : sizeof(double2);
                const int len = precision == WQC_PRECISION_FP32 ? M + N : M;
                int best_c = 0;
                double best_ms = 0.0;
                for (int c = 1; c <= ctx->max_cluster; ++c) {
                    if (jacobi_smem_bytes(len, N, c, elem) > kSmemLimit) continue;
                    const int b = round_up(N, 4 * c) / (2 * c);
                    if (b > kJacobiThreads / 32) continue;  // more column pairs than warps
                    ctx->force_C = c;
                    const double ms = tune_measure(ctx, chi, precision, throughput ? 32 : 1, 3);
                    ctx->force_C = 0;
                    if (ms < 0) {
                        ctx->tuned.clear();
                        return fail(WQC_ERR_CUDA, std::string("autotune measurement failed: ") + g_err);
                    }
                    // A batch is throughput-bound: SM time (ms x C) decides.
                    const double cost = throughput ? ms * c : ms;
                    if (!best_c || cost < best_ms) {
                        best_c = c;
                        best_ms = cost;
                    }
                }
                if (best_c) ctx->tuned.push_back({M, N, len, int(elem), throughput, best_c});
            }
        }
    }
    tune_write(path, fp, ctx->tuned);  // a cache that cannot be written only costs the next start a measurement
    if (entries) *entries = uint32_t(ctx->tuned.size());
    return WQC_OK;
}

}  // extern "C"
