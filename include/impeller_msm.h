/*
 * impeller_msm.h -- C ABI of libimpeller_msm.so, the B200 (sm_100a) BN254 G1
 * multi-scalar multiplication.
 *
 * Data layout everywhere (the reference's, core/src/msm/src/msm.h and
 * core/src/msm.rs:319-341): a field element is 8 little-endian uint32 limbs in
 * Montgomery form (R = 2^256); an affine point is 16 uint32 (x then y),
 * byte-identical to halo2curves' G1Affine; the identity point is (0, 0).
 * Scalars are Fr elements in Montgomery form.  Results are canonical affine
 * points in the same form.
 *
 * Return values are cudaError_t codes; argument errors return
 * cudaErrorInvalidValue and impeller_last_error() says why.
 */
#ifndef IMPELLER_MSM_H
#define IMPELLER_MSM_H

#include <cuda_runtime_api.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------
 * Drop-in replacements of the reference's two symbols.
 *
 * Replaces core/src/msm/src/msm.h:4-9 (defined in core/src/msm/src/msm.cu:9-41),
 * bound by core/src/msm.rs:116-133 and called at core/src/msm.rs:282-302
 * (size query) and :349-365 (run).  Same two-phase protocol: with
 * buffers == NULL the per-card scratch byte sizes are written to
 * buffer_sizes[0..num_cards) and nothing runs; otherwise buffers[i] is a
 * device allocation of at least that size on card cards[i].  h_points holds
 * n_precompute host arrays of len points (table j = 2^(j*n_windows*c) * P),
 * h_scaler_batch holds `batches` host arrays of len scalars, h_result
 * `batches` host arrays of 16 uint32.  Blocking, like the reference.
 *
 * The window size c and target window count of this symbol are those of the
 * library it is loaded from: 16 and 16 for libimpeller_msm.so (the
 * reference's MsmConfig::default, common/src/msm_config.rs:52-55), or the
 * values baked into a per-configuration shim named like the reference's
 * libmsm_bn254_{c}_{alpha}_{debug}.so (core/src/msm.rs:101-112).
 */
cudaError_t msm(void *const *buffers, unsigned long *buffer_sizes, unsigned long long len,
                unsigned int batch_per_run, unsigned int parts, unsigned int stage_scalers,
                unsigned int stage_points, unsigned int num_cards, const unsigned int *cards,
                unsigned int const *const *h_points, unsigned int batches,
                unsigned int const *const *h_scaler_batch, unsigned int *const *h_result);

/* Replaces core/src/msm/src/msm.h:11 (core/src/msm/src/msm.cu:43-49,
 * MSMPrecompute::precompute at core/src/msm/src/msm_impl.cuh:803-829), bound
 * by core/src/msm.rs:139-146.  Fills h_points[1..n_precompute) from
 * h_points[0] on up to max_cards devices. */
cudaError_t msm_precompute(unsigned long long len, unsigned int *const *h_points, unsigned int max_cards);

/* The same two entry points with the configuration as arguments (the
 * reference bakes window_size / target_window into the library name,
 * core/src/msm.rs:101-112; per-configuration shims forward here). */
cudaError_t impeller_msm_cfg(unsigned int window_size, unsigned int target_window, int debug,
                             void *const *buffers, unsigned long *buffer_sizes, unsigned long long len,
                             unsigned int batch_per_run, unsigned int parts, unsigned int stage_scalers,
                             unsigned int stage_points, unsigned int num_cards, const unsigned int *cards,
                             unsigned int const *const *h_points, unsigned int batches,
                             unsigned int const *const *h_scaler_batch, unsigned int *const *h_result);
cudaError_t impeller_msm_precompute_cfg(unsigned int window_size, unsigned int target_window,
                                        unsigned long long len, unsigned int *const *h_points,
                                        unsigned int max_cards);

/* Curves: the reference builds one MSM library per curve, MSM_CURVE = bn254
 * or bls12381 (utils/expand_targets.py:40-41; Rust side core/src/msm.rs:24-34).
 * BLS12-381 G1 points are 24 uint32 (x then y, 12 little-endian limbs each,
 * Montgomery form), scalars 8 uint32 (Montgomery Fr), results 24 uint32. */
#define IMPELLER_CURVE_BN254 0u
#define IMPELLER_CURVE_BLS12381 1u

/* msm() / msm_precompute() for a given curve (the per-curve libraries'
 * symbols; the BLS12-381 shims libmsm_bls12381_{c}_{alpha}_{debug}.so forward
 * here).  Configurations whose window count differs from the reference's
 * table layout on that curve are refused (cudaErrorInvalidValue). */
cudaError_t impeller_msm_cfg_curve(unsigned int curve, unsigned int window_size, unsigned int target_window,
                                   int debug, void *const *buffers, unsigned long *buffer_sizes,
                                   unsigned long long len, unsigned int batch_per_run, unsigned int parts,
                                   unsigned int stage_scalers, unsigned int stage_points, unsigned int num_cards,
                                   const unsigned int *cards, unsigned int const *const *h_points,
                                   unsigned int batches, unsigned int const *const *h_scaler_batch,
                                   unsigned int *const *h_result);
cudaError_t impeller_msm_precompute_cfg_curve(unsigned int curve, unsigned int window_size,
                                              unsigned int target_window, unsigned long long len,
                                              unsigned int *const *h_points, unsigned int max_cards);
unsigned int impeller_msm_n_precompute_curve(unsigned int curve, unsigned int window_size,
                                             unsigned int target_window);

/* Number of window tables the reference derives from (window_size,
 * target_window) for a 254-bit scalar (common/src/msm_config.rs:17-25). */
unsigned int impeller_msm_n_precompute(unsigned int window_size, unsigned int target_window);

/* ------------------------------------------------------------------------
 * Resident-SRS context (additive; no reference counterpart -- the reference
 * re-uploads its points on every call, core/src/msm/src/msm_impl.cuh:478-499).
 */
typedef struct impeller_ctx impeller_ctx;

/* Upload (or adopt) `len` affine points to `device`.  points_on_device != 0
 * means `points` is already a device pointer on that device; the context then
 * borrows it and the caller keeps it alive. */
cudaError_t impeller_ctx_create(impeller_ctx **out, int device, const uint32_t *points, uint64_t len,
                                int points_on_device);
/* The same on a given curve (IMPELLER_CURVE_*); every MSM, batch and server
 * on the context then runs on that curve. */
cudaError_t impeller_ctx_create_curve(impeller_ctx **out, int device, const uint32_t *points, uint64_t len,
                                      int points_on_device, unsigned int curve);
cudaError_t impeller_ctx_destroy(impeller_ctx *ctx);
/* Device pointer of the resident points (len x 16 uint32; len x 24 on
 * BLS12-381). */
const uint32_t *impeller_ctx_points(const impeller_ctx *ctx);
uint64_t impeller_ctx_len(const impeller_ctx *ctx);

/* Resident window tables for window size c (additive; the device-resident
 * counterpart of msm_precompute with one bucket set): W(c) signed-digit
 * windows (ceil(254/c) on BN254) tables of len points, table j = 2^(j*c) * P, kept in HBM next to the points.
 * MSMs on this context that use window c then accumulate every digit window
 * into one bucket set: no per-window reduction and no window doublings.
 * Replaces any previous tables.  Blocks until the tables are built. */
cudaError_t impeller_ctx_precompute(impeller_ctx *ctx, unsigned int c);
/* Window an MSM of n points uses on this context when c == 0 is passed. */
unsigned int impeller_ctx_window(const impeller_ctx *ctx, uint64_t n);

/* Window size the autotune table picks for a plain MSM of n points. */
unsigned int impeller_default_window(uint64_t n);
/* The same on a curve (IMPELLER_CURVE_*): on BLS12-381 a pick that would
 * need an extra signed-digit window holding only carries (c = 3, 5, 15, 17)
 * moves to its neighbour (4, 6, 16, 16). */
unsigned int impeller_default_window_curve(uint64_t n, unsigned int curve);
/* Window of resident tables the autotune table recommends for MSMs of n
 * points (0: the plain path is faster at that size). */
unsigned int impeller_table_window(uint64_t n);
/* Replace the autotune table (the library starts with the table measured by
 * impeller_b200/autotune.py and compiled in): `count` entries (log2 n, plain
 * window c, tables window or 0); the entry with the nearest log2 n applies.
 * tables_c may be NULL.  count == 0 falls back to the built-in cost model. */
cudaError_t impeller_set_window_table(const uint32_t *log2n, const uint32_t *c, const uint32_t *tables_c,
                                      uint32_t count);

/* One MSM over the first n resident points.  d_scalars: device, n x 8
 * uint32 (Montgomery Fr); d_result: device, 16 uint32.  c == 0 picks the
 * window from the table.  Asynchronous on `stream`. */
cudaError_t impeller_msm_device(impeller_ctx *ctx, const uint32_t *d_scalars, uint64_t n, unsigned int c,
                                uint32_t *d_result, cudaStream_t stream);
/* Same with host scalars and result: copies in, runs, copies out, waits. */
cudaError_t impeller_msm_host(impeller_ctx *ctx, const uint32_t *h_scalars, uint64_t n, unsigned int c,
                              uint32_t *h_result, cudaStream_t stream);

/* Per-phase timing of a context's MSMs: when enabled, each run records CUDA
 * events on its stream between phases (tables, histogram, scan, scatter,
 * accumulate, fixup, reduce, final).  profile_read waits for the recorded
 * runs, writes the summed milliseconds of each phase (nphase >= 8) and the
 * number of runs, and clears the record. */
cudaError_t impeller_ctx_profile(impeller_ctx *ctx, int enable);
cudaError_t impeller_ctx_profile_read(impeller_ctx *ctx, double *ms_per_phase, uint32_t nphase, uint32_t *runs);
const char *impeller_phase_name(uint32_t i);
/* Kernel launches of one MSM of n points with window c (0: the context's
 * choice) on this context; 0 for invalid arguments. */
uint32_t impeller_ctx_launches(impeller_ctx *ctx, uint64_t n, unsigned int c);

/* ------------------------------------------------------------------------
 * Batched MSMs of uneven sizes over prefixes of the resident points: one
 * plan, every phase one launch for the whole batch, optionally captured in a
 * CUDA graph and replayed.  sizes[i] <= ctx len; windows[i] == 0 picks the
 * table's window; windows may be NULL.
 */
typedef struct impeller_batch impeller_batch;
#define IMPELLER_BATCH_GRAPH 1u
cudaError_t impeller_batch_create(impeller_batch **out, impeller_ctx *ctx, const uint64_t *sizes,
                                  const unsigned int *windows, uint32_t count, uint32_t flags);
cudaError_t impeller_batch_destroy(impeller_batch *b);
/* d_scalars[i]: device scalars of MSM i; d_results: device, count x 16. */
cudaError_t impeller_batch_run(impeller_batch *b, const uint32_t *const *d_scalars, uint32_t *d_results,
                               cudaStream_t stream);
/* Kernel launches one run of the batch issues (for launch accounting). */
uint32_t impeller_batch_launches(const impeller_batch *b);
/* Per-phase timing of a batch created without IMPELLER_BATCH_GRAPH (same
 * phases and semantics as impeller_ctx_profile / impeller_ctx_profile_read). */
cudaError_t impeller_batch_profile(impeller_batch *b, int enable);
cudaError_t impeller_batch_profile_read(impeller_batch *b, double *ms_per_phase, uint32_t nphase, uint32_t *runs);

/* ------------------------------------------------------------------------
 * Continuous-batching server over a context (additive; the reference serves
 * whole proofs through its scheduler, scheduler/src/scheduler/core.rs:419-580,
 * and has no MSM-level serving).  Jobs are admitted in arrival order while
 * one of max_inflight batch slots is free and their device footprint fits the
 * HBM budget (0: free memory at creation minus 1 GiB); each admitted group
 * (at most max_batch jobs) runs as one batch on its own stream, so batches on
 * the GPU at the same time overlap.  Each job uses the window (and resident
 * table set) the context would use alone, so its result is the same alone and
 * in any mix.  Batch scratch comes from a memory pool of the server's own,
 * mapped at creation (16 GiB, or the budget if smaller) and kept mapped.  The
 * caller keeps h_scalars alive and unchanged until the job's result has been
 * taken.
 */
typedef struct impeller_server impeller_server;
typedef struct impeller_server_stats {
    uint64_t submitted, completed, rejected, failed, batches, points, peak_bytes, budget_bytes;
    double mean_batch; /* jobs per batch */
    double span_s;     /* first submission to last completion */
    double p50_ms, p99_ms, mean_ms, max_ms; /* submission-to-result latency */
    uint64_t max_concurrent;                /* most batches on the GPU at once */
} impeller_server_stats;

cudaError_t impeller_server_create(impeller_server **out, impeller_ctx *ctx, uint32_t max_batch,
                                   uint32_t max_inflight, uint64_t hbm_budget);
/* Queue one MSM over the first n resident points.  Refuses (and counts) n == 0,
 * n > SRS length, NULL scalars (cudaErrorInvalidValue) and jobs whose device
 * footprint exceeds the budget (cudaErrorMemoryAllocation). */
cudaError_t impeller_server_submit(impeller_server *s, const uint32_t *h_scalars, uint64_t n, uint64_t *job_id);
/* Block until the job is done; copy its 16-word result; return its status.
 * A job is taken once: a second wait (or poll) on the same id, concurrent or
 * later, returns cudaErrorInvalidValue. */
cudaError_t impeller_server_wait(impeller_server *s, uint64_t job_id, uint32_t *h_result, double *latency_ms);
/* Like wait, but cudaErrorNotReady while the job is pending. */
cudaError_t impeller_server_poll(impeller_server *s, uint64_t job_id, uint32_t *h_result, double *latency_ms);
cudaError_t impeller_server_get_stats(impeller_server *s, impeller_server_stats *out);
/* Fail the next `batches` batches on the host, without GPU work (failure
 * handling tests: their jobs complete with cudaErrorLaunchFailure). */
cudaError_t impeller_server_inject_failures(impeller_server *s, uint32_t batches);
/* Test hook: the next impeller_server_create fails at setup step `step`
 * (1 memory pool, 2 streams, 3 pinned buffers, 4 pool reserve; 0 clears)
 * with cudaErrorMemoryAllocation, releasing what it had made; the message of
 * impeller_last_error() names the step. */
cudaError_t impeller_server_fail_setup_step(uint32_t step);
/* Drain queued and running jobs, then stop. */
cudaError_t impeller_server_destroy(impeller_server *s);

/* ------------------------------------------------------------------------
 * Seeded synthetic inputs, computed on the device (definitions shared with
 * the CPU oracle: splitmix64 counter streams, uniform Fr, the skewed
 * witness-like mix, P_i = r_i * G). */
cudaError_t impeller_gen_scalars(uint32_t *d_out, uint64_t n, uint64_t seed, uint64_t stream, int dist,
                                 uint64_t start, int mont, cudaStream_t s);
cudaError_t impeller_gen_points(uint32_t *d_out, uint64_t n, uint64_t seed, uint64_t start, cudaStream_t s);
/* The same streams on a given curve (IMPELLER_CURVE_*): scalars are 8 u32
 * on both curves, points PW u32 (16 BN254, 24 BLS12-381), G the curve's
 * generator. */
cudaError_t impeller_gen_scalars_curve(int curve, uint32_t *d_out, uint64_t n, uint64_t seed, uint64_t stream,
                                       int dist, uint64_t start, int mont, cudaStream_t s);
cudaError_t impeller_gen_points_curve(int curve, uint32_t *d_out, uint64_t n, uint64_t seed, uint64_t start,
                                      cudaStream_t s);

/* Element-wise field / point operations on the device, for parity tests.
 * field: 0 = BN254 Fq, 1 = BN254 Fr, 2 = BLS12-381 Fq (12 u32 per element),
 * 3 = BLS12-381 Fr.  op: 0 add, 1 sub, 2 mul, 3 sqr, 4 neg, 5 to_mont,
 * 6 from_mont, 7 inv (Fermat), 8 pow, 9 inv (binary extended Euclid), 10 inv
 * (Bernstein-Yang divsteps, the one MSM results use).  Point ops (affine in/out): 0 add (madd path),
 * 1 dbl, 2 add via XYZZ+XYZZ, 3 k*P (k plain 256-bit). */
cudaError_t impeller_test_field_op(int field, int op, const uint32_t *d_a, const uint32_t *d_b, uint32_t *d_out,
                                   uint64_t count, cudaStream_t s);
cudaError_t impeller_test_point_op(int op, const uint32_t *d_p, const uint32_t *d_q, uint32_t *d_out,
                                   uint64_t count, cudaStream_t s);
cudaError_t impeller_test_point_op_curve(int curve, int op, const uint32_t *d_p, const uint32_t *d_q, uint32_t *d_out,
                                         uint64_t count, cudaStream_t s);

/* Integer-multiply ceiling of `device`, measured: the throughput of
 * independent Fq Montgomery products (four chains per thread, full
 * occupancy), in 10^9 32x32 -> 64-bit partial products per second (136 per
 * Montgomery product).  Blocks until done. */
cudaError_t impeller_imad_peak(int device, double *gops);
/* The same for a curve's base field (IMPELLER_CURVE_*): BLS12-381's 12-limb
 * products count 300 partial products each. */
cudaError_t impeller_imad_peak_curve(int device, unsigned int curve, double *gops);

/* Single-thread latency, in SM clock cycles, of a dependent chain of one
 * operation: 0 Fq Montgomery product, 1 XYZZ addition (plus the doubling
 * that feeds it), 2 XYZZ doubling, 3 mixed XYZZ + affine addition. */
cudaError_t impeller_op_latency(int op, uint32_t iters, double *cycles_per_op);

/* ------------------------------------------------------------------------
 * MSM that allocates nothing (no counterpart in the reference).
 *
 * For callers that cannot call cudaMalloc when they need an MSM: runtimes
 * whose device memory is planned ahead of time into a fixed arena, paths
 * where cudaMalloc / cudaFree would synchronize the device, processes that
 * must not grow their device footprint after start-up.  All scratch comes
 * from a file-scope __device__ array of IMPELLER_NOALLOC_SCRATCH_BYTES that
 * every GPU loading this library holds until exit; no device or pinned
 * memory is allocated per call.  The caller passes the inputs (d_points:
 * n affine points, d_scalars: n Montgomery Fr scalars, both device memory on
 * the current device) and the output (d_result: 16 uint32, canonical affine).
 * n > IMPELLER_NOALLOC_MAX_N returns cudaErrorInvalidValue.  Every call shares
 * the one array, so calls that overlap on the GPU race: serialize them.  The
 * first call on a device looks up the array's address (cudaGetSymbolAddress)
 * and keeps it for the life of the process; make that first call before any
 * stream capture.  A cudaDeviceReset after that first call is not supported:
 * the kept address would refer to the released module.  Asynchronous on
 * `stream`.
 */
#define IMPELLER_NOALLOC_SCRATCH_BYTES (16u << 20)
#define IMPELLER_NOALLOC_MAX_N (1u << 14)
cudaError_t impeller_msm_device_noalloc(const uint32_t *d_points, const uint32_t *d_scalars, uint64_t n,
                                        uint32_t *d_result, cudaStream_t stream);

/* Last error message of the calling thread ("" if none). */
const char *impeller_last_error(void);
/* Library version string. */
const char *impeller_version(void);

#ifdef __cplusplus
}
#endif

#endif /* IMPELLER_MSM_H */
