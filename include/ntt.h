/*
 * libntt.so: NTT entry points over BN254 Fr (natural order in and out, in place).
 *
 * The first five symbols keep the exact signatures of the reference's libntt.so
 * (core/src/ntt/src/ntt.h:5-16, implemented in core/src/ntt/src/ntt.cu:7-25) so the Rust
 * wrappers (core/src/ntt.rs:97-371) can dlopen this library unchanged.  All device work is
 * asynchronous on `stream`; the precompute helpers are synchronous and write host memory.
 * Errors come back as cudaError_t (cudaErrorInvalidValue for malformed arguments).
 *
 * The zkp_* symbols are additions with the same conventions (no counterpart in the
 * reference): fused inverse scaling, fused coset shift, a coset low-degree extension
 * that reads a shorter coefficient vector, and a second twiddle table format (Shoup pairs,
 * 64 bytes per root) that makes the twiddle products of the register passes cheaper.
 */
#ifndef ZKP_NTT_H
#define ZKP_NTT_H
#include <cuda_runtime.h>
#include "poly_ptr.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Forward DFT of x (len 2^log_len) with the root table twiddle = [w^0 .. w^(n/2-1)] on the
 * device (replaces ntt.h:6 / ssip_ntt.cuh:503-566).  The two thread-cap arguments are the
 * reference's kernel tuning knobs; this implementation plans its own stages and ignores them. */
cudaError_t ssip_ntt(PolyPtr x, const unsigned int *twiddle, unsigned int log_len, cudaStream_t stream,
                     const unsigned int max_threads_stage1_log, const unsigned int max_threads_stage2_log);

/* Host output: twiddle[i] = unit^i for i < len (replaces ntt.h:9 / precompute.cuh:9-87; the
 * reference's Rust caller passes the table length, core/src/ntt.rs:226-233). */
cudaError_t ssip_precompute(unsigned int *twiddle, unsigned int len, const unsigned int *unit);

/* Forward DFT that derives its roots from omegas_d = [w, w^2, w^4, ...] instead of an n/2
 * table (replaces ntt.h:12 / recompute_ntt.cuh:362-438). pq_d / pq_deg are accepted for ABI
 * compatibility; the kernels rebuild every root they need from omegas_d. */
cudaError_t recompute_ntt(PolyPtr x, const unsigned int *pq_d, unsigned int pq_deg, const unsigned int *omegas_d,
                          unsigned int log_len, cudaStream_t stream, const unsigned int max_threads_stage1_log,
                          const unsigned int max_threads_stage2_log);

/* Host: pq[i] = (unit^(len >> pq_deg))^i for i < 2^(pq_deg-1) and omegas[i] = unit^(2^i) for
 * i < 32, byte-identical to the reference (ntt.h:15 / precompute.cuh:89-113). */
void gen_pq_omegas(unsigned int *pq, unsigned int *omegas, unsigned int pq_deg, unsigned int len, unsigned int *unit);

/* x[i] *= powers[i % power_num] (replaces ntt.h:16 / distribute_powers.cuh:5-21). */
cudaError_t distribute_powers(PolyPtr poly, const unsigned int *powers, unsigned long long power_num,
                              cudaStream_t stream);

/* ---- additions ---- */
/* DFT with optional fused pre-shift x[i] *= shift^i (coset) and post-scale by *scale
 * (inverse NTT's n^-1); shift_d / scale_d are device pointers to one element or NULL. */
cudaError_t zkp_ntt_ex(PolyPtr x, const unsigned int *twiddle, unsigned int log_len, const unsigned int *shift_d,
                       const unsigned int *scale_d, cudaStream_t stream);

/* Coset low-degree extension: out (len 2^log_out) = DFT_{2^log_out}(in[i] * shift^i, zero
 * padded), in has length 2^log_in <= 2^log_out; twiddle is the table for 2^log_out. */
cudaError_t zkp_coset_lde(PolyPtr out, ConstPolyPtr in, const unsigned int *twiddle, unsigned int log_in,
                          unsigned int log_out, const unsigned int *shift_d, cudaStream_t stream);

/* Twiddle table for Shoup's product by a fixed factor: entry e (16 words, 64 bytes) holds w^e
 * as a plain value (8 words) and floor(w^e * 2^256 / r) (8 words), for e < 2^(log_len-1),
 * built on the device from the Montgomery table twiddle_d ([w^0 .. w^(n/2-1)], as for
 * ssip_ntt).  table_d: room for 2^(log_len-1) * 16 words.  Asynchronous, no allocation. */
cudaError_t zkp_ntt_shoup_table(const unsigned int *twiddle_d, unsigned int log_len, unsigned int *table_d,
                                cudaStream_t stream);

/* zkp_ntt_ex and zkp_coset_lde whose register passes (the passes of at most 2^6-point pencils
 * that make up the plan of every transform above 2^6 points) multiply by the twiddles of
 * shoup_d, a zkp_ntt_shoup_table of the same twiddle table: 207 multiply instructions per
 * twiddle product instead of the Montgomery product's 256, identical results.  twiddle is
 * still read by the other passes; shoup_d = NULL gives zkp_ntt_ex / zkp_coset_lde. */
cudaError_t zkp_ntt_ex_shoup(PolyPtr x, const unsigned int *twiddle, const unsigned int *shoup_d,
                             unsigned int log_len, const unsigned int *shift_d, const unsigned int *scale_d,
                             cudaStream_t stream);
cudaError_t zkp_coset_lde_shoup(PolyPtr out, ConstPolyPtr in, const unsigned int *twiddle,
                                const unsigned int *shoup_d, unsigned int log_in, unsigned int log_out,
                                const unsigned int *shift_d, cudaStream_t stream);

/* Device twin of ssip_precompute: out_d[i] = unit^i for i < count, unit_d on the device;
 * asynchronous on `stream`, no allocation. */
cudaError_t zkp_ntt_roots_device(unsigned int *out_d, unsigned long long count, const unsigned int *unit_d,
                                 cudaStream_t stream);

/* Plan tuning (no counterpart in the reference): caps the digit width of the passes used for
 * transforms of 2^log_len elements (log_len 0: every size) at max_digit in [4, 12] (0 restores
 * the default 12).  Each pass transforms 2^D-element pencils in shared memory, D <= max_digit;
 * a smaller cap means more passes of smaller CTAs.  Plans made after the call use it. */
cudaError_t zkp_ntt_set_max_digit(unsigned int log_len, unsigned int max_digit);
/* CTA size (32, 64, 128 or 256 threads; 0 = 128) of the register passes of transforms of
 * 2^log_len elements (log_len 0: every size), set by the autotuner (no counterpart in the
 * reference, whose launch shapes follow max_threads_stage*_log).  Results do not depend on it. */
cudaError_t zkp_ntt_set_block(unsigned int log_len, unsigned int threads);

/* The digit widths, top digit first, of the sub-transform passes the current plan for
 * 2^log_len uses (at most max written); returns the number of passes (0 if log_len is 0 or
 * above 28). */
unsigned int zkp_ntt_plan_digits(unsigned int log_len, unsigned int *digits, unsigned int max);

/* Number of sub-transform passes + permutation passes the plan for 2^log_len uses. */
unsigned int zkp_ntt_num_passes(unsigned int log_len);

/* ---- batched form (no counterpart in the reference): many transforms of uneven sizes ----
 * One task per transform, in place; twiddle is the root table of the task's size (use the
 * inverse root's table and scale_d = n^-1 for an inverse NTT, shift_d for a coset); shoup_d
 * optionally the zkp_ntt_shoup_table of that table (or NULL).  A plan uploads the task tables
 * once; running it launches one persistent kernel per pass for the small tasks (every small
 * task's pencils share the launch) and one batched permutation, and runs each task of at least
 * 2^solo_log points (zkp_ntt_batch_set_solo_log) through its own tuned register-pass plan, as
 * zkp_ntt_ex_shoup does.  No allocation or host copy happens at run time, so a run can be
 * captured into a CUDA graph and replayed. */
typedef struct ZkpNttTask {
    PolyPtr x;
    const unsigned int *twiddle;
    unsigned int log_len;
    const unsigned int *shift_d;
    const unsigned int *scale_d;
    const unsigned int *shoup_d;
} ZkpNttTask;

typedef struct ZkpNttBatchPlan ZkpNttBatchPlan;

cudaError_t zkp_ntt_batch_plan_create(const ZkpNttTask *tasks, unsigned int ntasks, ZkpNttBatchPlan **plan);
/* Plans made after the call run tasks of at least 2^log_len points on their own (0: every
 * task shares the persistent launches); the default is 16. */
cudaError_t zkp_ntt_batch_set_solo_log(unsigned int log_len);
cudaError_t zkp_ntt_batch_run(const ZkpNttBatchPlan *plan, cudaStream_t stream);
void zkp_ntt_batch_plan_destroy(ZkpNttBatchPlan *plan);

/* Benchmark support: throughput probe of the Shoup twiddle product (blocks x 256 threads x
 * iters x 2 products; out_d holds blocks * 256 * 8 words). */
cudaError_t zkp_ntt_shoup_probe(unsigned int blocks, unsigned int iters, unsigned int *out_d, cudaStream_t stream);

/* Benchmark support: when enabled, the library records a CUDA event on the call's stream after
 * each launch of its next calls; read returns the per-launch milliseconds of the last call. */
void zkp_ntt_profile_enable(int on);
int zkp_ntt_profile_read(float *ms, const char **names, int max);

#ifdef __cplusplus
}
#endif
#endif
