/*
 * libpoly.so: polynomial kernels over BN254 Fr, same C ABI as the reference's libpoly.so
 * (core/src/poly/src/poly.h:4-28; Rust wrappers core/src/poly.rs:37-784).
 *
 * All calls are asynchronous on `stream`.  Functions taking a temp buffer follow the
 * reference's size-query protocol: with temp == NULL they write the bytes they need into
 * *size and return.  Scalars (x, b, res, target) are device pointers to one 32-byte element.
 */
#ifndef ZKP_POLY_H
#define ZKP_POLY_H
#include <cuda_runtime.h>
#include "poly_ptr.h"

#ifdef __cplusplus
extern "C" {
#endif

/* r[i] = a[i] +/-/* b[i] for i < min(len); the longer operand passes through (negated for
 * b - a) up to max(len) (poly.h:4-8, poly_basic.cu:5-53). */
cudaError_t poly_add(PolyPtr r, ConstPolyPtr a, ConstPolyPtr b, cudaStream_t stream);
cudaError_t poly_sub(PolyPtr r, ConstPolyPtr a, ConstPolyPtr b, cudaStream_t stream);
cudaError_t poly_mul(PolyPtr r, ConstPolyPtr a, ConstPolyPtr b, cudaStream_t stream);

/* r[i] = a[i]^2 (addition, no counterpart in the reference; the dedicated Montgomery squaring) */
cudaError_t zkp_poly_square(PolyPtr r, ConstPolyPtr a, cudaStream_t stream);

/* all ones (Lagrange one), [1, 0, ...] (coefficient one), all zeros (poly.h:10-14) */
cudaError_t poly_one_lagrange(PolyPtr target, cudaStream_t stream);
cudaError_t poly_one_coef(PolyPtr target, cudaStream_t stream);
cudaError_t poly_zero(PolyPtr target, cudaStream_t stream);

/* *res = sum_i poly[i] * x^i (poly.h:16, poly_eval.cuh:8-74) */
cudaError_t poly_eval(void *temp_buf, unsigned long *temp_buf_size, ConstPolyPtr poly, unsigned int *res,
                      const unsigned int *x, cudaStream_t stream);

/* q[i] = sum_{j>i} p[j] b^(j-i-1), i.e. (p - p(b)) / (X - b); q[n-1] = 0 (poly.h:18,
 * kate_division.cuh:57-85) */
cudaError_t kate_division(void *temp_buf, unsigned long *temp_buf_size, unsigned int log_p, ConstPolyPtr p,
                          const unsigned int *b, PolyPtr q, cudaStream_t stream);

/* inclusive product scan in place (poly.h:20, scan_mul.cuh:1-28) */
cudaError_t scan_mul(void *temp_buffer, unsigned long *buffer_size, PolyPtr target, cudaStream_t stream);

/* elementwise inverse in place, zeros stay zero (poly.h:22, batched_invert.cuh:56-93) */
cudaError_t batched_invert(void *temp_buffer, unsigned long *buffer_size, PolyPtr poly, cudaStream_t stream);

/* *target = target^-1, *target = target^exp (poly.h:24-26, poly_basic.cu:61-72) */
cudaError_t inv_scalar(unsigned int *target, cudaStream_t stream);
cudaError_t scalar_pow(unsigned int *target, unsigned long long exp, cudaStream_t stream);

/* lookup permutation over the first `usable` rows (poly.h:28, permute.cuh:74-222): res_input =
 * input sorted ascending by canonical value; res_table = at the first row of each run of equal
 * values that value (taken once from the table), elsewhere the unused table values ascending.
 * Every input value must occur in the table.  temp_buffer == null: *buffer_size = bytes needed. */
cudaError_t permute(void *temp_buffer, unsigned long *buffer_size, unsigned long usable, ConstPolyPtr input,
                    ConstPolyPtr table, PolyPtr res_input, PolyPtr res_table, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif
