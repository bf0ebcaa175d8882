/*
 * libmsm.so: multi-scalar multiplication over BN254 G1.
 *
 * `msm` and `msm_precompute` keep the exact signatures of the reference's library
 * (core/src/msm/src/msm.h:4-11, implemented in core/src/msm/src/msm.cu:9-48) so the Rust
 * wrapper (core/src/msm.rs:136-369) can dlopen this library unchanged.  Scalars are 32-byte
 * Montgomery-form Fr elements; points are 64-byte affine (x, y) Montgomery Fq with (0, 0) the
 * identity; results are written as 64-byte affine points.
 *
 * The reference fixes the window width and the number of precomputed point tables per
 * library build (libmsm_<curve>_<window>_<target_windows>_<debug>.so, core/src/msm.rs:100-111).
 * Installed under such a name this library reads the same two fields from its file name;
 * under any other name it uses one point table and chooses the window per call.
 */
#ifndef ZKP_MSM_H
#define ZKP_MSM_H
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Synchronous MSM over host arrays (replaces msm.h:4-8, msm_impl.cuh:830-909).
 * buffers == NULL: writes the device workspace bytes each card needs into buffer_sizes and
 * returns (size-query protocol, msm.cu:20-22).  Otherwise buffers[k] is a caller-owned
 * device buffer of that size on cards[k]; h_points holds the n_precompute host point tables
 * of length len, h_scaler_batch[b] the len scalars of batch b, and h_result[b] receives the
 * affine result of batch b.  batch_per_run, parts, stage_scalers and stage_points are the
 * reference's host-streaming knobs; with the whole problem resident in HBM they are accepted
 * and ignored.  Several cards each take a contiguous slice of the points; their partial
 * results are added on cards[0]. */
cudaError_t msm(void *const *buffers, unsigned long *buffer_sizes, unsigned long long len, unsigned int batch_per_run,
                unsigned int parts, unsigned int stage_scalers, unsigned int stage_points, unsigned int num_cards,
                const unsigned int *cards, unsigned int const *const *h_points, unsigned int batches,
                unsigned int const *const *h_scaler_batch, unsigned int *const *h_result);

/* Fills the host tables h_points[1 .. n_precompute-1] from h_points[0]: table j holds
 * 2^(j * n_windows * window) * P (replaces msm.h:10 / msm_impl.cuh:776-828).  With one table
 * there is nothing to do. */
cudaError_t msm_precompute(unsigned long long len, unsigned int *const *h_points, unsigned int max_cards);

/* ---- additions (no counterpart in the reference): asynchronous MSM over device memory ---- */

/* Device workspace bytes for zkp_msm_device with n points, window bits `window` (0 = auto)
 * and n_tables point tables (0 = the library's configuration). */
unsigned long long zkp_msm_workspace_size(unsigned long long n, unsigned int window, unsigned int n_tables);

/* Window width the library picks for n points when window == 0. */
unsigned int zkp_msm_default_window(unsigned long long n);

/* Affine pairing rounds for MSMs planned after this call (-1 = chosen by size, the default;
 * else 0..4).  Each round halves every bucket's point list with affine additions whose
 * inverses share one inversion (Montgomery's trick) before the XYZZ bucket walk.  The
 * workspace size depends on it: query sizes and run under the same setting. */
cudaError_t zkp_msm_set_affine_rounds(int rounds);

/* The number of pairing rounds an MSM of n points (window, n_tables as for
 * zkp_msm_workspace_size) runs under the current setting. */
unsigned int zkp_msm_rounds_for(unsigned long long n, unsigned int window, unsigned int n_tables);

/* result_d (64-byte affine) = sum_i scalars_d[i] * points_d[i], asynchronous on `stream`.
 * points_d holds n_tables contiguous tables of n affine points (table j = 2^(j*Wp*window) P
 * with Wp = ceil(ceil(254/window) / n_tables)); workspace_d is caller-owned, at least
 * zkp_msm_workspace_size(n, window, n_tables) bytes, and may be reused once the call's work
 * on `stream` is done. */
cudaError_t zkp_msm_device(void *workspace_d, unsigned long long workspace_bytes, const unsigned int *points_d,
                           unsigned int n_tables, const unsigned int *scalars_d, unsigned long long n,
                           unsigned int window, unsigned int *result_d, cudaStream_t stream);

/* ---- batched form (no counterpart in the reference): up to 32 MSMs of uneven sizes share
 * every stage launch (one counting sort over all their digits, one load-balanced accumulation
 * over all their buckets, one reduction, one combine with a thread per MSM).  The task table
 * travels as a kernel parameter, so zkp_msm_batch allocates nothing, copies nothing from the
 * host and can be captured into a CUDA graph. */
typedef struct ZkpMsmTask {
    const unsigned int *points_d;  /* n_tables tables of n affine points */
    unsigned int n_tables;         /* 0 = the library's configuration */
    const unsigned int *scalars_d; /* n Montgomery scalars */
    unsigned long long n;
    unsigned int window;           /* 0 = choose */
    unsigned int *result_d;        /* 64-byte affine result */
    unsigned long long table_stride; /* points between tables (0 = n): an MSM over the first n
                                        points of longer resident tables */
} ZkpMsmTask;

unsigned long long zkp_msm_batch_workspace_size(const ZkpMsmTask *tasks, unsigned int ntasks);
cudaError_t zkp_msm_batch(const ZkpMsmTask *tasks, unsigned int ntasks, void *workspace_d,
                          unsigned long long workspace_bytes, cudaStream_t stream);

/* Builds the n_tables - 1 extra tables on the device: tables_d holds n_tables * n affine
 * points and its first table is filled by the caller. */
cudaError_t zkp_msm_precompute_device(unsigned int *tables_d, unsigned long long n, unsigned int window,
                                      unsigned int n_tables, cudaStream_t stream);

/* ---- allocation-free MSM (no counterpart in the reference) ----
 * For callers that cannot allocate device memory - a plugin whose host application only hands
 * it input and output buffers and owns every allocator, or a latency-critical loop that must
 * not call cudaMalloc because it synchronises the whole device.  Same result as
 * zkp_msm_device, but the workspace is a fixed 64 MiB array inside the library (every GPU that
 * loads the library holds it until the process exits), which fits MSMs of up to 2^15 points
 * with the default window (2^16 points need 68.8 MiB); larger problems return
 * cudaErrorInvalidValue without touching the device.  The call allocates nothing.  Nothing in
 * the array has to start at zero: each call clears the counters, bucket sums and flags it uses,
 * on its stream, before its kernels read them.  The array has one copy per CUDA context: the
 * first call in each context (the runtime's primary context of a device, or a context the host
 * made current through the driver API) looks up that context's copy and caches it under the
 * context's id, so a new context after cudaDeviceReset gets its own lookup.  Make that first
 * call before any stream capture: a call that would need the lookup while its stream is being
 * captured returns cudaErrorStreamCaptureUnsupported and does nothing.  Every call in a context
 * shares the one array, which keeps the last call's contents: calls that overlap on the GPU
 * (other streams, other host threads) race, so serialise them on one stream. */
cudaError_t zkp_msm_device_noalloc(const unsigned int *points_d, unsigned int n_tables,
                                   const unsigned int *scalars_d, unsigned long long n, unsigned int window,
                                   unsigned int *result_d, cudaStream_t stream);
/* Bytes of the fixed workspace zkp_msm_device_noalloc uses (compare zkp_msm_workspace_size). */
unsigned long long zkp_msm_noalloc_capacity(void);

/* CTA size (64, 128 or 256 threads; 0 = 256) of one MSM stage for MSMs planned from now on:
 * stage 0 the pairing rounds' up pass, 1 their down pass, 2 the XYZZ walk.  Set by the
 * autotuner (no counterpart in the reference); results do not depend on it. */
cudaError_t zkp_msm_set_block(unsigned int stage, unsigned int threads);

/* Benchmark support: per-stage CUDA-event timing of the last MSM (see zkp_ntt_profile_enable). */
void zkp_msm_profile_enable(int on);
int zkp_msm_profile_read(float *ms, const char **names, int max);

/* Integer-multiply throughput probe: blocks x 256 threads x iters x 16 IMAD instructions
 * (out_d: blocks * 256 words).  Used to measure the IMAD peak the MSM roofline divides by. */
cudaError_t zkp_imad_probe(unsigned int blocks, unsigned int iters, unsigned int *out_d, cudaStream_t stream);

/* Montgomery-product throughput probe: blocks x 256 threads x iters x 2 Fq products with the
 * library's own product routine (out_d: blocks * 256 * 8 words).  Its rate is the denominator
 * of the field-product roofline fractions. */
cudaError_t zkp_mont_probe(unsigned int blocks, unsigned int iters, unsigned int *out_d, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif
