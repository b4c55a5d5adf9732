/* wqc_cuda.h - C ABI of the `WQC_TN_BACKEND=cuda` MPS backend (B200, sm_100a).
 *
 * The entry points are what the reference's MpsState backend hooks would bind
 * through `extern "C"` (src/tn/mps.rs:62-67, 128-212, 431-482, 489-495,
 * 567-590, 937-1079 are the webgpu hooks this backend sits beside).  Plain
 * pointers and sizes only; every call returns a status and never unwinds.
 *
 * Threading: a wqc_cuda_ctx is process-wide (one per device, like the shared
 * device OnceLock at src/tn/engine_status.rs:27).  A wqc_mps is used from one
 * thread at a time (the request's spawn_blocking thread, src/api.rs:342) and
 * owns one CUDA stream; calls enqueue device work and return, and the calls
 * that hand results to the host synchronise that stream.
 */
#ifndef WQC_CUDA_H
#define WQC_CUDA_H

#include <stddef.h>
#include <stdint.h>

#include "wqc_types.h"

#if defined(__GNUC__)
#define WQC_API __attribute__((visibility("default")))
#else
#define WQC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t wqc_status;

/* Status codes and the EngineError each maps to on the Rust side
 * (src/engine.rs:67-77). */
enum wqc_status_code {
    WQC_OK = 0,
    WQC_ERR_INVALID = 1,              /* ExecutionFailed(msg) */
    WQC_ERR_OOM = 2,                  /* InsufficientMemory { required, available } */
    WQC_ERR_TRUNCATION_REJECTED = 3,  /* ExecutionFailed("mps bond exceeded chi"), mps.rs:1143 */
    WQC_ERR_SVD_FAILED = 4,           /* ExecutionFailed("SVD ... failed its check"), svd_guard.rs:134-138 */
    WQC_ERR_CANCELLED = 5,            /* ExecutionFailed(cancel::CANCELLED), src/cancel.rs:20 */
    WQC_ERR_DEVICE_TIMEOUT = 6,       /* ExecutionFailed: a bounded device wait gave up */
    WQC_ERR_CUDA = 7,                 /* ExecutionFailed: CUDA runtime error */
    WQC_ERR_NO_DEVICE = 8,            /* backend probe note: no CUDA device (engine_status.rs:74-81) */
    WQC_ERR_QUBIT_OUT_OF_RANGE = 9,   /* QubitIndexOutOfBounds { index, limit } */
    WQC_ERR_INVALID_QUBIT_COUNT = 10  /* InvalidQubitCount(n), mps.rs:83-85 */
};

/* Arithmetic of the split path. */
enum wqc_precision {
    WQC_PRECISION_FP64 = 0, /* plain form: complex128 throughout */
    WQC_PRECISION_FP32 = 1, /* precision form: each Jacobi SVD runs in two phases.  The
                               first sweeps complex64 columns (FP32 dot products and
                               rotation updates, FP64 rotation parameters, tolerance and
                               convergence tests) that carry X V and the accumulated V;
                               V is then made orthonormal to FP64 rounding (two
                               Newton-Schulz steps) and X V formed in FP64, and FP64
                               sweeps finish from there (quadratic convergence: a few
                               sweeps).  Sites, range finder, sort and cut stay FP64 and
                               merges FP64-level (wqc_mps_set_merge), so results carry
                               FP64-level error. */
    WQC_PRECISION_TF32X3 = 2 /* tensor-core form: the precision form's Jacobi, with every
                               two-site merge (theta = L R and the 4x4 gate) on the tcgen05
                               tensor cores: operands split into TF32 hi and lo parts, the
                               three products lo*hi + hi*lo + hi*hi accumulated in FP32
                               in tensor memory, the gate applied in FP64 to the FP32
                               product.  Each theta carries FP32-level error (about 1e-7
                               relative), which the splits after it carry on. */
};

typedef struct wqc_cuda_ctx wqc_cuda_ctx;
typedef struct wqc_mps wqc_mps;

/* Message of the last failing call on this thread (thread-local, never NULL). */
WQC_API const char* wqc_cuda_last_error(void);

/* Byte counts of the last call on this thread that returned WQC_ERR_OOM:
 * the device memory it needed and the free device memory it saw (0, 0
 * before any).  They fill EngineError::InsufficientMemory { required,
 * available } (src/engine.rs:72), which the reference raises from
 * ensure_mps_workspace_budget (src/tn/mps.rs:36-48).  Either pointer may be
 * NULL. */
WQC_API void wqc_cuda_last_oom(uint64_t* required, uint64_t* available);

/* Open the process-wide context on `device` (-1: WQC_CUDA_DEVICE or 0).
 * Replaces the shared device probe (engine_status.rs:40-102). */
WQC_API wqc_status wqc_cuda_open(int device, wqc_cuda_ctx** out);
WQC_API void wqc_cuda_close(wqc_cuda_ctx* ctx);

/* Measure the Jacobi SVD's cluster size for the saturated shapes of chi_max
 * 16, 32, 64 and 128 (plain form and the precision form's first phase; one
 * latency-bound split and a 32-split batch), or load the measurement from
 * `cache_path` (NULL: $WQC_TUNE_PATH, else $XDG_CACHE_HOME or ~/.cache,
 * /wqc/jacobi-clusters) when its first line matches this machine's
 * fingerprint (device name, SM count, compute capability, driver and
 * runtime versions).  A fresh measurement is written back there.  States
 * created on `ctx` afterwards use the measured sizes for those shapes and
 * the cost model for the rest.  The calibration-plus-cache pattern of the
 * reference's GEMM side (src/tn/gpu/gemm.rs:495-543, 649-702); budget_seconds
 * > 0 stops measuring once spent.  *entries (nullable) receives the number
 * of tuned shapes. */
WQC_API wqc_status wqc_cuda_autotune(wqc_cuda_ctx* ctx, const char* cache_path, double budget_seconds,
                                     uint32_t* entries);

/* Device memory for /sysinfo's vram_budget_bytes (engine_status.rs:105-117)
 * and the SM count.  Any out pointer may be NULL. */
WQC_API wqc_status wqc_cuda_device_info(wqc_cuda_ctx* ctx, uint64_t* total_bytes, uint64_t* free_bytes, int32_t* sm_count);

/* Device bytes of the site tensors at bond chi: N * chi^2 * 32, the same
 * estimate as mps_workspace_bytes (mps.rs:27-32). */
WQC_API uint64_t wqc_mps_workspace_bytes(uint32_t qubit_count, uint32_t max_bond_dim);

/* MpsState::try_new_with_bond (mps.rs:82-126): N sites of |0>, each stored at
 * chi_max capacity in device memory.  reject_truncation marks a time-split
 * half (mps.rs:1270): a split that would drop a singular value above the
 * cutoff fails with WQC_ERR_TRUNCATION_REJECTED instead of cutting.  Fails
 * with WQC_ERR_OOM when the sites plus split workspace exceed free device
 * memory (the device analogue of ensure_mps_workspace_budget, mps.rs:36-48). */
WQC_API wqc_status wqc_mps_create(wqc_cuda_ctx* ctx, uint32_t qubit_count, uint32_t max_bond_dim, int32_t precision,
                          uint8_t reject_truncation, wqc_mps** out);
WQC_API void wqc_mps_destroy(wqc_mps* mps);

/* Batching form: `count` independent slices (the orchestrator's tensor-network
 * slices, each its own register and chi_max) held in one state.  The slices'
 * sites are concatenated, so every wave of splits mixes ready splits from all
 * slices; each slice still sees exactly its own MpsState sequence.
 * max_concurrent_splits bounds the split workspace (0: one slot per two
 * sites).  SVD launch shapes are sized for throughput and depend on each
 * split's shape only, so a slice gives bit for bit the same results in any
 * batch (a batch of one included); against a single-state run of the same
 * circuit they agree to rounding.  No reference counterpart: the reference
 * runs one slice per request (src/api.rs:336-697); this is how one B200
 * takes many at once. */
WQC_API wqc_status wqc_batch_create(wqc_cuda_ctx* ctx, uint32_t count, const uint32_t* qubit_counts,
                                    const uint32_t* max_bond_dims, int32_t precision, uint32_t max_concurrent_splits,
                                    wqc_mps** out);
/* Gates of slice s are gates[offsets[s] .. offsets[s+1]); qubits are local to
 * the slice.  Semantics per slice as wqc_mps_apply_gates.  Returns once the
 * work is queued on the state's stream (a submit); wqc_mps_synchronize, or
 * any call that hands results to the host, waits for it. */
WQC_API wqc_status wqc_batch_apply_gates(wqc_mps* batch, const wqc_gate* gates, const uint32_t* offsets);
/* <0...0|psi_s> of every slice: out[2s], out[2s+1]. */
WQC_API wqc_status wqc_batch_amplitudes(wqc_mps* batch, double* out);
/* With profiling on: milliseconds from the start of the last
 * wqc_batch_apply_gates call to the completion of each slice's last split
 * (CUDA events on the state's stream); -1 for a slice without operations. */
WQC_API wqc_status wqc_batch_slice_times(wqc_mps* batch, double* out_ms);
/* compute_expectations (src/expectation.rs:98-200) on every slice: the same
 * Pauli sum (labels as for wqc_mps_expectation_pauli; every slice must have
 * the labels' width), out[2s], out[2s+1] for slice s.  The batching form's
 * route to parameter-shift gradients: each shifted circuit is one slice. */
WQC_API wqc_status wqc_batch_expectation_pauli(wqc_mps* batch, const char* labels, const double* coeffs,
                                               uint32_t nterms, double* out);

/* Back to |0...0> with the split records cleared, keeping the device memory
 * (a fresh MpsState for the next request without reallocating); also after
 * a cancelled or failed request, whose cancel word and status it clears. */
WQC_API wqc_status wqc_mps_reset(wqc_mps* mps);

/* MpsState::apply_gate (mps.rs:278-297) for each gate in order: 1q gates,
 * CNOT/CZ with SWAP routing and undo (mps.rs:353-375), CCNOT as the
 * reference's 15-gate decomposition (mps.rs:657-677); MEASURE/RESET/IF are
 * no-ops.  Splits on disjoint sites run concurrently; each site sees exactly
 * the reference's sequence of operations. */
WQC_API wqc_status wqc_mps_apply_gates(wqc_mps* mps, const wqc_gate* gates, uint32_t count);

/* MpsState::apply_gate_adjoint (mps.rs:301-331) for each gate in order. */
WQC_API wqc_status wqc_mps_apply_gates_adjoint(wqc_mps* mps, const wqc_gate* gates, uint32_t count);

/* apply_one_qubit / apply_unary_at / apply_tdg_at (mps.rs:333-351, 621-629):
 * u is the 2x2 as re,im pairs in row-major order [u00,u01,u10,u11]. */
WQC_API wqc_status wqc_mps_apply_1q(wqc_mps* mps, uint32_t site, const double u[8]);

/* apply_two_qubit_at_positions / apply_pair_at / apply_cnot_at /
 * apply_swap_at (mps.rs:377-429, 631-655): u is a Mat4 [c_out][t_out][c_in]
 * [t_in] (gates.rs:7-8) as 16 re,im pairs; ctrl_is_first says whether the
 * control is at left_site.  `info` (nullable) receives the split record
 * (synchronises the stream). */
WQC_API wqc_status wqc_mps_apply_2q(wqc_mps* mps, uint32_t left_site, const double u[32], uint8_t ctrl_is_first,
                            wqc_split_info* info);

/* apply_two_qubit_gate (mps.rs:353-375): SWAP the right operand down to the
 * left one, apply, SWAP back; the same split sequence as the reference. */
WQC_API wqc_status wqc_mps_apply_2q_routed(wqc_mps* mps, uint32_t ctrl, uint32_t tgt, const double u[32]);

/* apply_adjacent_disjoint_gates (mps.rs:520-565): a layer of adjacent,
 * qubit-disjoint CNOT/CZ, merged from the current sites then split. */
WQC_API wqc_status wqc_mps_apply_layer(wqc_mps* mps, const wqc_gate* gates, uint32_t count);

/* Which split the state performs (applies to splits enqueued afterwards).
 * REFERENCE: the reference's rule, an exact SVD or the seeded range finder
 * when the split is large (mps.rs:929-981).  EXACT: an exact SVD on every
 * split.  The range finder's test matrix has rank 48 for every shape (its
 * signs are bits 8 and 9 of a power-of-two LCG, period 1024), so on a split
 * of rank above 48 part of its basis is set by rounding; EXACT gives a
 * reproducible truncation at those shapes. */
enum wqc_split_rule { WQC_SPLIT_RULE_REFERENCE = 0, WQC_SPLIT_RULE_EXACT = 1 };
WQC_API wqc_status wqc_mps_set_split_rule(wqc_mps* mps, int32_t rule);

/* How the state performs its merges (merge_two_site_tensors / cpu_merge,
 * mps.rs:484-514, 812-831, with the 4x4 of mps.rs:833-866; applies to merges
 * enqueued afterwards).  FFMA: tiled FP64 FMA (the default of batches).
 * TC_INT8 (the default of states from wqc_mps_create, except the tensor-core
 * form): on the
 * tcgen05 tensor cores from int8 digit slices (the Ozaki scheme): each row of
 * L and each column of R scaled by a power of two, cut into 9 signed 7-bit
 * digits (63 bits), the digit products exact in int32 in tensor memory and
 * summed in FP64 -- FP64-level results (the dropped slice products lie below
 * 2^-60 of the row and column maxima) from the integer tensor pipe.  The
 * digit planes of every split slot are allocated with the state when
 * TC_INT8 is its default, else by the first TC_INT8 call (WQC_ERR_OOM if
 * they do not fit).  Not for the tensor-core form, whose merges are its TF32
 * path. */
enum wqc_merge { WQC_MERGE_FFMA = 0, WQC_MERGE_TC_INT8 = 1 };
WQC_API wqc_status wqc_mps_set_merge(wqc_mps* mps, int32_t merge);

/* Host-only: how wqc_mps_apply_gates would schedule `gates` on n sites,
 * without a device.  For each split in program order, its left site and its
 * level (splits of one level run concurrently); *nsplits and *nlevels
 * receive the totals, and at most `max` entries are written.  The split
 * sequence is the reference's (mps.rs:353-375 routing, 657-677 CCNOT). */
WQC_API wqc_status wqc_schedule_gates(uint32_t n, const wqc_gate* gates, uint32_t count, int32_t* split_site,
                                      int32_t* split_level, uint32_t max, uint32_t* nsplits, uint32_t* nlevels);

/* Wait for the enqueued work; reports device-side failures. */
WQC_API wqc_status wqc_mps_synchronize(wqc_mps* mps);

/* Ask the running work to stop (src/cancel.rs:38-63): splits not yet started
 * are skipped and the next synchronising call returns WQC_ERR_CANCELLED.
 * Safe to call from another thread. */
WQC_API void wqc_mps_cancel(wqc_mps* mps);

/* amplitude_at_compact_zero (mps.rs:262-276): <0...0|psi> as re, im. */
WQC_API wqc_status wqc_mps_amplitude_zero(wqc_mps* mps, double out[2]);

/* site_amplitudes (mps.rs:679-693), the trace feeder of trace.rs:401:
 * out = a0.re, a0.im, a1.re, a1.im.  control_probability is |a1|^2.
 * Single states only.  The left and right environments (left_environment,
 * right_environment, mps.rs:700-740) stay cached on the device between
 * calls: a call recomputes only the ones that operations since the last
 * call have touched, so the per-gate reads of trace.rs cost one chain over
 * the sites an operation changed rather than over the whole register. */
WQC_API wqc_status wqc_mps_site_amplitudes(wqc_mps* mps, uint32_t target, double out[4]);

/* site_amplitudes for `count` targets in one call (one launch, one
 * synchronisation): out[4k .. 4k+3] for targets[k].  resolve_pre_amps
 * (trace.rs:375-411) reads the control probabilities and the target's
 * amplitudes of one step; a disjoint layer (emit_disjoint_layer,
 * trace.rs:264-315) reads every gate's before applying any. */
WQC_API wqc_status wqc_mps_site_amplitudes_many(wqc_mps* mps, const uint32_t* targets, uint32_t count, double* out);

/* The dense state, 2^n complex values (re,im pairs) with basis bit q =
 * qubit q, contracted on the device.  WQC_DENSE_TO_DENSE_STATE follows
 * to_dense_state (mps.rs:742-780), which skips site entries with |x|^2 <
 * 1e-30; WQC_DENSE_STATEVECTOR follows contract_to_statevector
 * (mps.rs:215-260): every entry, and qubit_count <= 20 or the reference's
 * error.  At most 28 qubits; single states only. */
enum wqc_dense_mode { WQC_DENSE_TO_DENSE_STATE = 0, WQC_DENSE_STATEVECTOR = 1 };
WQC_API wqc_status wqc_mps_to_dense(wqc_mps* mps, int32_t mode, double* out);

/* Right bond of every site (out has qubit_count entries). */
WQC_API wqc_status wqc_mps_bond_dims(wqc_mps* mps, uint32_t* out);

/* Read / write one site tensor [l][2][r] as re,im pairs (used for
 * to_dense_state, overlap and tests; mps.rs:742-780, 1421-1474).  With
 * buf == NULL only the shape is returned.  Uploads are taken one site at a
 * time; the next call that computes on the state first checks that the
 * chain closes (each left bond equals the left neighbour's right bond, the
 * first left and last right bonds are 1) and fails with WQC_ERR_INVALID
 * ("uploaded sites do not chain") otherwise. */
WQC_API wqc_status wqc_mps_download_site(wqc_mps* mps, uint32_t site, uint32_t* l, uint32_t* r, double* buf);
WQC_API wqc_status wqc_mps_upload_site(wqc_mps* mps, uint32_t site, uint32_t l, uint32_t r, const double* buf);

/* <bra|ket> = sum over all indices of ket sites times conjugated bra sites
 * (overlap, mps.rs:1423-1474; the time split's final step,
 * contract_time_split, mps.rs:1241-1281), by a left environment on the
 * device.  Fails like the reference on registers of different width
 * (EngineError::MismatchedRegister), mismatched site shapes and, with
 * env_limit > 0, an environment of more than env_limit entries (the
 * reference passes 256, its STARK witness limit, "mps overlap environment
 * exceeds 256"); env_limit = 0 bounds it only by chi_ket x chi_bra.  Both
 * states must come from the same context; single states only. */
WQC_API wqc_status wqc_mps_overlap(wqc_mps* ket, wqc_mps* bra, uint32_t env_limit, double out[2]);

/* `shots` draws from |<b|psi>|^2 / <psi|psi>, computed on the device from
 * the MPS (site-by-site conditional sampling against right environments), so
 * not limited to 20 qubits as the reference's dense route is
 * (sample_terminal_measurements, src/sample.rs:192-211, which builds the
 * outcome table of compute_outcome_probabilities, src/sample.rs:85-131).
 * out[k] bit j is the outcome of qubits[j] in shot k (count <= 64 distinct
 * qubits); the host forms the reference's Qiskit-order keys from them.  The
 * draws come from SplitMix64 keyed by (seed, shot, qubit): deterministic for
 * a seed, but not the reference's StdRng stream.  Single states only. */
WQC_API wqc_status wqc_mps_sample(wqc_mps* mps, const uint32_t* qubits, uint32_t count, uint32_t shots, uint64_t seed,
                                  uint64_t* out);

/* Sum_t coeff_t <psi|P_t|psi> for Pauli strings (labels: nterms strings of
 * qubit_count characters in IXYZ, character n-1-q acting on qubit q as in
 * src/expectation.rs:98-132; coeffs: re,im pairs).  Computed on the device
 * with transfer matrices, so it is not limited to 20 qubits. */
WQC_API wqc_status wqc_mps_expectation_pauli(wqc_mps* mps, const char* labels, const double* coeffs, uint32_t nterms,
                                     double out[2]);

/* The same sum for an MPS held in the caller's own device memory, computed
 * without allocating any device memory.  This entry point has no
 * counterpart in the reference.  It is for callers that cannot let a
 * library call cudaMalloc: hosts whose allocator already owns the GPU's
 * memory (a PyTorch caching allocator, a fixed per-tenant budget), where
 * cudaMalloc may fail although their pool has room and cudaFree would
 * synchronise the whole device.
 *
 * sites: device memory of the current device, 16-byte aligned, holding
 * qubit_count * site_stride complex128 values (re,im pairs); site q starts at
 * complex element q * site_stride and is [l][2][r] row-major, r =
 * bond_dims[q] and l = bond_dims[q - 1] (1 for q = 0), the layout that
 * wqc_mps_download_site returns.  The chain must be closed: the last right
 * bond, bond_dims[qubit_count - 1], is 1 (else WQC_ERR_INVALID).  bond_dims,
 * labels, coeffs and out are host memory; labels holds nterms *
 * qubit_count characters and coeffs 2 * nterms doubles.  stream: a
 * cudaStream_t of the current device (NULL = the legacy default stream).
 *
 * The call is synchronous: it returns once its work on `stream` has
 * finished and the result is in `out`.  It must not be called while
 * `stream` is being captured into a CUDA graph (it then returns
 * WQC_ERR_INVALID without enqueuing anything).
 *
 * Working memory is one array of 16 MiB + 128 KiB that the library holds in
 * every GPU where this code is loaded, until the process exits.  Limits:
 * bond dimensions 1..256 and at most 1024 qubits; larger sizes are rejected
 * with WQC_ERR_INVALID or WQC_ERR_INVALID_QUBIT_COUNT and a message naming
 * the limit.  The first call on a device looks up that device's address of
 * the array (and may load this code onto the GPU).  All calls on a device
 * share the array, which keeps the last call's contents; calls that overlap
 * on the GPU (from two host threads at once) race on it, so serialise them. */
WQC_API wqc_status wqc_expectation_pauli_noalloc(const double* sites, uint64_t site_stride, const uint32_t* bond_dims,
                                                 uint32_t qubit_count, const char* labels, const double* coeffs,
                                                 uint32_t nterms, void* stream, double out[2]);

/* Differentiation form: the adjoint (reverse-mode) gradient of a Pauli-sum
 * observable f = sum_t Re(c_t) <psi|P_t|psi> (compute_expectations,
 * src/expectation.rs:98-200) with respect to the angle of every RX/RY/RZ
 * gate, through the reference's truncated forward path: one-qubit gates,
 * SWAP-routed two-site applies and the truncated SVD split with sqrt(S)
 * absorbed on both sides (mps.rs:333-429, 1124-1171).  The reference has no
 * reverse mode; this pair is the forward/backward op a Rust caller binds.
 *
 * wqc_adjoint_forward resets `mps` to |0...0>, runs `gates` on it and keeps
 * a checkpoint of the sites at each gate index in `checkpoints` (for
 * instance the first gate of every second layer) and at the end; the state
 * then holds the circuit's output.  Every split takes the exact SVD (the
 * range finder's rank-48 test matrix has no meaningful derivative); single
 * states in the plain FP64 form only.
 *
 * wqc_adjoint_backward: value[0] = f, value[1] = sum_t Im(c_t) <P_t>;
 * grad[i] = d f / d angle of gate i (0 for gates without an angle).  The
 * sweep restores each segment from its checkpoint, recomputes it and runs
 * it in reverse: a split's reverse is the complex SVD's reverse mode with
 * the cotangents of the dropped singular vectors zero (the truncation term)
 * and 1/(s_j^2 - s_i^2) Lorentzian-broadened for near-degenerate values.
 * This is the derivative of the truncated map, which differs from a
 * parameter-shift estimate by the truncation's own effect.  `adj` can be
 * swept again with other observables; the state holds the forward's output
 * afterwards. */
typedef struct wqc_adjoint wqc_adjoint;
WQC_API wqc_status wqc_adjoint_forward(wqc_mps* mps, const wqc_gate* gates, uint32_t count,
                                       const uint32_t* checkpoints, uint32_t ncheckpoints, wqc_adjoint** out);
WQC_API wqc_status wqc_adjoint_backward(wqc_adjoint* adj, const char* labels, const double* coeffs, uint32_t nterms,
                                        double value[2], double* grad);
WQC_API void wqc_adjoint_destroy(wqc_adjoint* adj);

/* Diagnostics: copy one split-workspace buffer of `slot` (the last wave's
 * job in that slot) to host memory, at most `bytes`.  which: 0 theta
 * (rows x cols, row-major), 1 Omega, 2 A*Omega, 3 A^H*(A*Omega), 4 Y then
 * Householder vectors (column-major), 5 thin Q (column-major), 6 Q^H A,
 * 7 Jacobi W, 8 the range finder's B W (kept columns; column-major), 9 column norms, 10 sort
 * permutation, 11 Householder scalars, 12 the split's device state. */
WQC_API wqc_status wqc_mps_debug_workspace(wqc_mps* mps, uint32_t slot, int32_t which, void* out, uint64_t bytes);

/* Split records in program order (one per merge + gate + split). */
WQC_API uint32_t wqc_mps_split_count(wqc_mps* mps);
WQC_API wqc_status wqc_mps_split_records(wqc_mps* mps, wqc_split_info* out, uint32_t max, uint32_t* written);

/* WorkReport.vram_peak_bytes (mps.rs:158-166, api.rs:657): high-water mark of
 * this state's device allocations. */
WQC_API uint64_t wqc_mps_peak_vram_bytes(wqc_mps* mps);

/* WorkReport.tn_backend (mps.rs:147-155): "cuda". */
WQC_API const char* wqc_mps_backend_label(wqc_mps* mps);

/* Per-kernel timing, taken with CUDA events on this state's stream while
 * profiling is on.  kind: 0 Jacobi SVD, 1 merge+gate, 2 range finder
 * (GEMMs + QR), 3 one-qubit, 4 cut + absorb. */
typedef struct wqc_kernel_stats {
    uint64_t launches[5];
    double milliseconds[5];
    uint64_t total_launches; /* every kernel this state launched */
    uint64_t h2d_bytes;      /* host-to-device bytes copied by the calls (gate plans, sites) */
    uint64_t d2h_bytes;      /* device-to-host bytes of results (amplitudes, ...) */
    uint64_t jacobi_tasks;   /* SVDs run by the Jacobi kernel */
    uint64_t jacobi_sweeps;  /* FP64 sweeps those SVDs took in total */
    uint64_t jacobi_sweeps_first; /* precision form: sweeps of the complex64 first phase */
} wqc_kernel_stats;
WQC_API wqc_status wqc_mps_set_profiling(wqc_mps* mps, int32_t on);
WQC_API wqc_status wqc_mps_kernel_stats(wqc_mps* mps, wqc_kernel_stats* out);
WQC_API void wqc_mps_reset_stats(wqc_mps* mps);

/* The CUDA stream this state enqueues on (cudaStream_t), for callers that
 * time or order work around it. */
WQC_API void* wqc_mps_stream(wqc_mps* mps);

/* ---------------------------------------------------------------------------
 * Exact contraction trees (src/tn/exact.rs): a ContractionTree whose nodes
 * are all Contract { left, right } (src/tn/tree.rs), walked with its state
 * tensors in device memory.  A node joins two states with no wire in common
 * by an outer product, or applies a gate to the state that holds all of the
 * gate's wires; gates are consumed in circuit order; at most 26 open legs per
 * tensor and a declared peak of at most 1 GiB (exact.rs:25-27).
 * ------------------------------------------------------------------------- */

/* TensorRef (src/tn/tree.rs).  Only KET0, GATE and NODE are leaves of an exact
 * tree; the others are rejected with the reference's messages
 * (exact.rs:243-258). */
enum wqc_tree_ref_kind {
    WQC_TREE_KET0 = 0,    /* Ket0(wire): |0> on one wire */
    WQC_TREE_GATE = 1,    /* Gate(index): gates[index] */
    WQC_TREE_NODE = 2,    /* Node(index): result of nodes[index] */
    WQC_TREE_LEFT = 3,    /* Left(_)    -> "exact contraction has no split" */
    WQC_TREE_RIGHT = 4,   /* Right(_)   -> "exact contraction has no split" */
    WQC_TREE_BRA0 = 5,    /* Bra0(_)    -> "exact contraction has no bra0" */
    WQC_TREE_CONTROL = 6, /* Control(_) -> "exact contraction has no gate halves" */
    WQC_TREE_TARGET = 7   /* Target(_)  -> "exact contraction has no gate halves" */
};
typedef struct wqc_tree_ref {
    int32_t kind; /* enum wqc_tree_ref_kind */
    uint32_t index;
} wqc_tree_ref;

/* ContractionNode: op 0 is Contract { left, right }; any other op is a sweep
 * step (Site, Swap, Pair, ...), which an exact tree may not hold
 * ("contraction tree mixes sweep steps and exact contractions"). */
typedef struct wqc_tree_node {
    int32_t op;
    wqc_tree_ref left, right;
} wqc_tree_node;

/* ContractionTree { kind, site_order, nodes, peak_bytes } (src/tn/tree.rs).
 * The site order must be empty or the identity (exact and network trees keep
 * the parent's wire numbers); has_peak 0 stands for peak_bytes: None; kind 1
 * is ContractionKind::Network, 0 an absent kind (the caller's dispatch picks
 * wqc_exact_* or wqc_network_* by it, tree.rs:178-205). */
typedef struct wqc_tree {
    const wqc_tree_node* nodes;
    uint32_t node_count;
    const uint32_t* site_order;
    uint32_t site_order_len;
    int32_t has_peak;
    uint64_t peak_bytes;
    int32_t kind;
} wqc_tree;

typedef struct wqc_exact wqc_exact;

/* An executor of exact trees on ctx's device: its own stream, a device arena
 * that holds the live tensors (reused, grown on demand) and the pass tables. */
WQC_API wqc_status wqc_exact_create(wqc_cuda_ctx* ctx, wqc_exact** out);
WQC_API void wqc_exact_destroy(wqc_exact* ex);

/* exact::validate (exact.rs:48-58): the declared peak and the tree's shape,
 * host only.  mps_site_order may be NULL (None); otherwise it must be the
 * identity over qubit_count wires. */
WQC_API wqc_status wqc_exact_validate(uint32_t qubit_count, const wqc_gate* gates, uint32_t gate_count,
                                      const wqc_tree* tree, const uint64_t* mps_site_order, uint32_t mps_site_order_len);

/* The peak of the walk without evaluating (exact.rs:650-658, `measured_peak`):
 * the value a tree declares.  Host only; the declared peak is not read. */
WQC_API wqc_status wqc_exact_measured_peak(uint32_t qubit_count, const wqc_gate* gates, uint32_t gate_count,
                                           const wqc_tree* tree, uint64_t* peak);

/* contract_exact_at (exact.rs:70-85) for `count` basis vectors at once: the
 * tree is contracted once and out[2k], out[2k+1] receive the amplitude of
 * bits[k] (bit q of bits[k] is wire q).  count 1 is the reference's call;
 * bits 0 is contract_exact (exact.rs:60-68).  Every failure the reference
 * reports (tree shape, circuit order, shared wires, legs, peak, declared
 * peak mismatch) is returned before any device work, with its message in
 * wqc_cuda_last_error.  Synchronous. */
WQC_API wqc_status wqc_exact_contract(wqc_exact* ex, uint32_t qubit_count, const wqc_gate* gates, uint32_t gate_count,
                                      const wqc_tree* tree, const uint64_t* mps_site_order,
                                      uint32_t mps_site_order_len, const uint64_t* bits, uint32_t count, double* out);

/* Size of the register tiles that states of at least `bits` legs are swept
 * in: 2^bits amplitudes per block, bits 12 (256 threads, the default) or 13
 * (512 threads).  A tuning knob: results do not depend on it. */
WQC_API wqc_status wqc_exact_set_tile_bits(wqc_exact* ex, int32_t bits);

/* Stop a contraction in progress (the reference's cancel::check per gate,
 * exact.rs:419-421): the running call returns WQC_ERR_CANCELLED at its next
 * launch; a cancel that arrives between calls stops the next call.  Safe to
 * call from another thread. */
WQC_API void wqc_exact_cancel(wqc_exact* ex);

/* What the last wqc_exact_contract did on the device. */
typedef struct wqc_exact_stats {
    uint32_t launches;       /* kernels launched */
    uint32_t passes;         /* gate passes (each: one sweep of a tensor through shared memory) */
    uint32_t outer_products; /* outer-product joins */
    uint32_t gates;          /* gates applied */
    double device_ms;        /* CUDA-event time of the device work, first launch to last */
    double pass_ms;          /* part of device_ms in passes over tensors of at least 2^20 amplitudes */
    uint64_t pass_bytes;     /* bytes those passes read and wrote (16 B per amplitude, both ways) */
    uint64_t bytes_moved;    /* bytes every launch read and wrote, by its access pattern */
    uint64_t arena_bytes;    /* device arena the tensors were placed in */
    uint32_t exchanges;      /* register-tile exchanges through shared memory, over all passes */
} wqc_exact_stats;
WQC_API wqc_status wqc_exact_last_stats(wqc_exact* ex, wqc_exact_stats* out);

/* ---------------------------------------------------------------------------
 * Network contraction trees (src/tn/network.rs): <0...0|U|0...0> of the
 * circuit as one tensor network.  Wire w starts at a ket0(w) leaf and ends
 * at a bra0(w) leaf; unitary gate i is a gate(i) leaf with an input and an
 * output leg per wire, or, for CNOT and CZ, two halves control(i) and
 * target(i) joined by a bond.  A node contracts two tensors over the legs
 * they share (a permutation of each operand, then a complex GEMM), at most
 * 26 legs per tensor and a declared peak of at most 1 GiB, with the
 * reference's byte accounting (network.rs:17-27).  The tree's kind must be 1.
 * ------------------------------------------------------------------------- */
typedef struct wqc_network wqc_network;
WQC_API wqc_status wqc_network_create(wqc_cuda_ctx* ctx, wqc_network** out);
WQC_API void wqc_network_destroy(wqc_network* net);

/* network::validate (network.rs:128-143): the declared peak against the
 * walk's, host only. */
WQC_API wqc_status wqc_network_validate(uint32_t qubit_count, const wqc_gate* gates, uint32_t gate_count,
                                        const wqc_tree* tree, const uint64_t* mps_site_order,
                                        uint32_t mps_site_order_len);

/* measured_peak (network.rs:162-169): the walk's peak, host only. */
WQC_API wqc_status wqc_network_measured_peak(uint32_t qubit_count, const wqc_gate* gates, uint32_t gate_count,
                                             const wqc_tree* tree, uint64_t* peak);

/* contract_network (network.rs:145-160): out[0], out[1] = <0...0|U|0...0>.
 * Every failure the reference reports is returned before any device work.
 * Synchronous. */
WQC_API wqc_status wqc_network_contract(wqc_network* net, uint32_t qubit_count, const wqc_gate* gates,
                                        uint32_t gate_count, const wqc_tree* tree, const uint64_t* mps_site_order,
                                        uint32_t mps_site_order_len, double out[2]);

/* As wqc_exact_cancel (network.rs:202-204 checks per node). */
WQC_API void wqc_network_cancel(wqc_network* net);

typedef struct wqc_network_stats {
    uint32_t nodes;          /* contractions */
    uint32_t permutes;       /* operands reordered on the device */
    uint32_t gemms;          /* complex GEMMs (cuBLAS ZGEMM) of the large contractions */
    uint32_t launches;       /* device launches, the GEMMs' included */
    double device_ms;        /* CUDA-event time of the device work */
    double permute_ms;       /* part of it in the large contractions' permutations (each timed) */
    double gemm_ms;          /* part of it in their GEMMs (each timed) */
    uint64_t permute_bytes;  /* bytes the permutations read and wrote */
    double gemm_flops;       /* real flops of the GEMMs (8 m n k each) */
    uint64_t arena_bytes;    /* device arena of the tensors */
    uint32_t small;          /* small contractions, run one block each in level-batched launches */
} wqc_network_stats;
WQC_API wqc_status wqc_network_last_stats(wqc_network* net, wqc_network_stats* out);

/* ------------------------------------------------------------------------
 * Complex GEMM on the tcgen05 tensor cores: the product of the tensor-core
 * form's two-site merge (mps.rs:812-831, the cpu_merge product; the webgpu
 * backend's gemm.wgsl is its GPU counterpart), here on its own.
 * C = A B with A m x k, B k x n, C m x n, row-major complex FP64 in host
 * memory (re, im interleaved).  Each operand is split into two TF32 values
 * (hi, lo = x - hi) and the three products lo*hi + hi*lo + hi*hi accumulate
 * in FP32 in tensor memory (kind::tf32, operands TMA-loaded with the 128-byte
 * swizzle): results carry FP32-level error, each entry within
 * 2^-24 max(16, k/4) |A_i| |B_j| (row and column 2-norms): the FP32
 * accumulation in tensor memory grows with k (measured 3.4e-7 relative at
 * k = 128, 2.4e-6 at k = 1000).  The GEMM kernel runs
 * `reps` times (0 counts as 1) on operands staged on the device once;
 * *kernel_ms (may be NULL) receives the mean CUDA-event time of one launch.
 * Sizes 1..16384. */
WQC_API wqc_status wqc_tc_zgemm(wqc_cuda_ctx* ctx, uint32_t m, uint32_t n, uint32_t k, const double* a,
                                const double* b, double* c, uint32_t reps, double* kernel_ms);

/* The same product from int8 digit slices on the tensor cores (kind::i8,
 * the scheme of WQC_MERGE_TC_INT8).  Each entry lies within 2^-49 2k of the
 * product of its row's largest |re|, |im| in A and its column's in B: FP64
 * level wherever the terms of a dot product are not far below those maxima.
 * Where a row's large entries meet a column's small ones along k, the result
 * is small against the maxima and loses relative accuracy (FP64 FMA would
 * not); the merge's operands, L = U sqrt(S) and R = sqrt(S) V^H, shrink
 * together along k and keep FP64-level relative error.  m, n in 1..8192,
 * k in 1..4096 (the int32 accumulators' bound). */
WQC_API wqc_status wqc_tc_zgemm_int8(wqc_cuda_ctx* ctx, uint32_t m, uint32_t n, uint32_t k, const double* a,
                                     const double* b, double* c, uint32_t reps, double* kernel_ms);

#ifdef __cplusplus
}
#endif

#endif /* WQC_CUDA_H */
