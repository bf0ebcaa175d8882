/*
 * Oracle (test infrastructure only): multi-scalar multiplication over G1.
 *
 * or_best_multiexp restates halo2's best_multiexp / multiexp_serial as copied into
 * core/tests/msm_halo2.rs:63-219: scalars are converted out of Montgomery form (to_repr,
 * little-endian), split into c-bit unsigned windows with c = ceil(ln n) (1 below 4 points,
 * 3 below 32), buckets 1..2^c-1 filled with mixed additions, summation by parts from the
 * top bucket down, c doublings between windows, and the input chunked one chunk per thread
 * with the chunk results summed.  The result is normalised to affine, the form the
 * reference's msm returns (core/src/msm/src/msm.cu:38) and the form the parity tests
 * compare (core/tests/msm.rs:228-238).
 */
#include "oracle.h"
#include "util.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

static void xyzz_identity(g1x_t *r) {
    memset(r, 0, sizeof(*r));
    or_one(OR_FQ, &r->zzz);
}

/* get_at: c bits of the little-endian repr starting at bit segment*c */
static size_t get_at(size_t segment, size_t c, const fe_t *repr) {
    size_t skip = segment * c;
    if (skip >= 256) return 0;
    const uint8_t *bytes = (const uint8_t *)repr->l;
    size_t skip_bytes = skip / 8;
    if (skip_bytes >= 32) return 0;
    uint64_t v = 0;
    for (size_t i = 0; i < 8 && skip_bytes + i < 32; i++) v |= (uint64_t)bytes[skip_bytes + i] << (8 * i);
    v >>= (skip - skip_bytes * 8);
    v &= ((uint64_t)1 << c) - 1;
    return (size_t)v;
}

static void multiexp_serial(const fe_t *coeffs, const g1a_t *bases, size_t n, g1x_t *acc) {
    fe_t *repr = (fe_t *)malloc(n * sizeof(fe_t));
    for (size_t i = 0; i < n; i++) or_from_mont(OR_FR, &repr[i], &coeffs[i]);
    size_t c;
    if (n < 4) c = 1;
    else if (n < 32) c = 3;
    else c = (size_t)ceil(log((double)n));
    size_t segments = 254 / c + 1;
    size_t nb = ((size_t)1 << c) - 1;
    g1x_t *buckets = (g1x_t *)malloc(nb * sizeof(g1x_t));
    for (size_t seg = segments; seg-- > 0;) {
        for (size_t k = 0; k < c; k++) or_g1_dbl(acc, acc);
        for (size_t b = 0; b < nb; b++) xyzz_identity(&buckets[b]);
        for (size_t i = 0; i < n; i++) {
            size_t d = get_at(seg, c, &repr[i]);
            if (d) or_g1_madd(&buckets[d - 1], &buckets[d - 1], &bases[i]);
        }
        g1x_t running;
        xyzz_identity(&running);
        for (size_t b = nb; b-- > 0;) {
            or_g1_add(&running, &running, &buckets[b]);
            or_g1_add(acc, acc, &running);
        }
    }
    free(buckets);
    free(repr);
}

typedef struct { const fe_t *s; const g1a_t *p; size_t n, chunk; g1x_t *res; } me_job;

static void me_worker(void *ctx, size_t lo, size_t hi) {
    me_job *j = (me_job *)ctx;
    for (size_t t = lo; t < hi; t++) {
        size_t a = t * j->chunk, b = a + j->chunk;
        if (b > j->n) b = j->n;
        xyzz_identity(&j->res[t]);
        multiexp_serial(j->s + a, j->p + a, b - a, &j->res[t]);
    }
}

void or_best_multiexp(g1a_t *res, const fe_t *scalars, const g1a_t *bases, size_t n) {
    size_t th = (size_t)or_get_threads();
    g1x_t acc;
    xyzz_identity(&acc);
    if (n > th) {
        size_t chunk = n / th;
        size_t nchunks = (n + chunk - 1) / chunk;
        g1x_t *parts = (g1x_t *)malloc(nchunks * sizeof(g1x_t));
        me_job j = {scalars, bases, n, chunk, parts};
        or_parallel_tasks(nchunks, me_worker, &j);
        for (size_t i = 0; i < nchunks; i++) or_g1_add(&acc, &acc, &parts[i]);
        free(parts);
    } else {
        multiexp_serial(scalars, bases, n, &acc);
    }
    or_g1_to_affine(res, &acc);
}

void or_naive_msm(g1a_t *res, const fe_t *scalars, const g1a_t *bases, size_t n) {
    g1x_t acc, t;
    xyzz_identity(&acc);
    for (size_t i = 0; i < n; i++) {
        fe_t k;
        or_from_mont(OR_FR, &k, &scalars[i]);
        or_g1_scalar_mul(&t, &bases[i], &k);
        or_g1_add(&acc, &acc, &t);
    }
    or_g1_to_affine(res, &acc);
}
