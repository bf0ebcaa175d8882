/*
 * CPU oracle for the BN254 hot path: TEST INFRASTRUCTURE ONLY.
 *
 * This library restates, in plain C, the algorithms the reference runs on the CPU for
 * this path so that the CUDA kernels can be checked bit-for-bit against it:
 *   - Montgomery arithmetic over BN254 Fr / Fq (core/src/common/mont/src/field.cuh:29-157
 *     host_arith, params bn254_fr.cuh:9-91, bn254_fq.cuh:6-84);
 *   - G1 XYZZ / affine arithmetic (core/src/common/curve/src/curve_xyzz.cuh:163-419,
 *     curve parameters core/src/common/curve/src/bn254.cuh:13-77);
 *   - halo2 best_fft, multiexp_serial / best_multiexp and eval_polynomial as copied into
 *     core/tests/msm_halo2.rs:63-383 (halo2_proofs v0.3.0 over halo2curves 0.6.0);
 *   - the poly library semantics (core/src/poly/src/poly_eval.cuh, batched_invert.cuh) and the compiler's INTT / coset
 *     composition (compiler/src/transit/type2/intt_mending.rs:11-70,
 *     core/src/ntt/src/distribute_powers.cuh:5-21).
 *
 * Only tests, the smoke check and the CPU-baseline leg of bench.py may load it.  The
 * product path never calls into it.
 *
 * Representation: an element is 4 little-endian u64 limbs == 8 little-endian u32 limbs,
 * the reference's byte layout (core/src/common/mont/src/field.cuh:685-743).  Field
 * elements are in Montgomery form (R = 2^256) and canonical (< modulus).
 */
#ifndef ZKP_ORACLE_H
#define ZKP_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { uint64_t l[4]; } fe_t;          /* field element, 32 B */
typedef struct { fe_t x, y; } g1a_t;              /* affine point, 64 B; identity == (0,0) */
typedef struct { fe_t x, y, zz, zzz; } g1x_t;     /* XYZZ point, 128 B; identity iff zz == 0 */

enum { OR_FR = 0, OR_FQ = 1 };

/* threads used by the parallel routines (0 = all online cores) */
void or_set_threads(int n);
int or_get_threads(void);

/* ---- field (f = OR_FR or OR_FQ) ---- */
void or_field_consts(int f, uint64_t *modulus, uint64_t *r1, uint64_t *r2, uint64_t *minv64);
void or_mul(int f, fe_t *r, const fe_t *a, const fe_t *b);
void or_add(int f, fe_t *r, const fe_t *a, const fe_t *b);
void or_sub(int f, fe_t *r, const fe_t *a, const fe_t *b);
void or_neg(int f, fe_t *r, const fe_t *a);
void or_to_mont(int f, fe_t *r, const fe_t *a);
void or_from_mont(int f, fe_t *r, const fe_t *a);
void or_pow(int f, fe_t *r, const fe_t *a, const uint64_t *e, int elimbs);
void or_inv(int f, fe_t *r, const fe_t *a);
void or_one(int f, fe_t *r);
/* plain 256-bit integer helpers used by the reference's Number tests */
void or_bn_mul(uint64_t r[8], const uint64_t a[4], const uint64_t b[4]);
void or_bn_slr(uint64_t r[4], const uint64_t a[4], unsigned k);

/* elementwise batches over n Fr elements */
void or_vec_mul(fe_t *r, const fe_t *a, const fe_t *b, size_t n);
void or_vec_add(fe_t *r, const fe_t *a, const fe_t *b, size_t n);
void or_vec_sub(fe_t *r, const fe_t *a, const fe_t *b, size_t n);

/* ---- deterministic input generator (counter based, identical on GPU) ---- */
void or_gen_fr(uint64_t seed, uint64_t start, size_t n, fe_t *out);       /* Montgomery form */
void or_gen_fr_raw(uint64_t seed, uint64_t idx, fe_t *canonical);         /* canonical integer */

/* ---- roots of unity ---- */
void or_root_of_unity(unsigned log_n, int inverse, fe_t *omega);          /* Montgomery form */
void or_twiddles(const fe_t *omega, size_t count, fe_t *out);             /* [w^0..w^(count-1)] */

/* ---- NTT family ---- */
void or_best_fft(fe_t *a, const fe_t *omega, unsigned log_n);
void or_intt(fe_t *a, unsigned log_n);                                    /* fft(w^-1) * n^-1 */
void or_ntt(fe_t *a, unsigned log_n);                                     /* fft(w) */
void or_distribute_powers(fe_t *a, size_t n, const fe_t *powers, size_t power_num);
void or_coset_ntt(fe_t *out, const fe_t *coef, unsigned log_in, unsigned log_out, const fe_t *g);
void or_naive_dft(fe_t *out, const fe_t *in, size_t n, const fe_t *omega);

/* ---- poly ---- */
void or_eval(fe_t *res, const fe_t *poly, size_t n, const fe_t *x);
void or_batch_invert(fe_t *a, size_t n);
void or_poly_ptr_gather(fe_t *out, const fe_t *base, size_t len, size_t rotate, size_t offset, size_t whole_len);

/* ---- G1 ---- */
void or_g1_generator(g1a_t *g);
int  or_g1_on_curve(const g1a_t *p);
void or_g1_to_xyzz(g1x_t *r, const g1a_t *p);
void or_g1_to_affine(g1a_t *r, const g1x_t *p);
void or_g1_add(g1x_t *r, const g1x_t *p, const g1x_t *q);
void or_g1_madd(g1x_t *r, const g1x_t *p, const g1a_t *q);
void or_g1_dbl(g1x_t *r, const g1x_t *p);
void or_g1_affine_add(g1a_t *r, const g1a_t *p, const g1a_t *q);
void or_g1_scalar_mul(g1x_t *r, const g1a_t *p, const fe_t *k_canonical);
void or_g1_batch_to_affine(g1a_t *out, const g1x_t *in, size_t n);
void or_gen_points(uint64_t seed, uint64_t start, size_t n, g1a_t *out);  /* P_i = k_i * G */

/* ---- MSM ---- */
/* halo2 best_multiexp: scalars in Montgomery form, bases affine (Montgomery); result affine */
void or_best_multiexp(g1a_t *res, const fe_t *scalars, const g1a_t *bases, size_t n);
void or_naive_msm(g1a_t *res, const fe_t *scalars, const g1a_t *bases, size_t n);

#ifdef __cplusplus
}
#endif
#endif
