/*
 * Oracle (test infrastructure only): the NTT family on the CPU.
 *
 * or_best_fft restates halo2's best_fft as copied into core/tests/msm_halo2.rs:221-325:
 * bit-reverse permutation, twiddle table [w^0 .. w^(n/2-1)], then radix-2 DIT butterflies,
 * recursively split and joined across threads (recursive_butterfly_arithmetic).  Input and
 * output are in natural order, which is what the reference's ssip_ntt produces
 * (core/tests/ntt.rs:83,166-168).
 *
 * or_intt: the compiler composes the inverse NTT as NTT(w^-1) followed by a multiply by
 * n^-1 (compiler/src/utils.rs:51-77, compiler/src/transit/type2/intt_mending.rs:11-70).
 * or_distribute_powers: x[i] *= powers[i % power_num]
 * (core/src/ntt/src/distribute_powers.cuh:5-11).
 * or_coset_ntt: zero-extend (compiler/src/ast/poly_coef.rs:252-255), multiply by g^i, NTT
 * at the extended size.
 */
#include "oracle.h"
#include "util.h"
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

static size_t bitreverse(size_t n, unsigned l) {
    size_t r = 0;
    for (unsigned i = 0; i < l; i++) {
        r = (r << 1) | (n & 1);
        n >>= 1;
    }
    return r;
}

typedef struct { fe_t *tw; const fe_t *omega; size_t count; } tw_job;

static void tw_worker(void *ctx, size_t lo, size_t hi) {
    tw_job *j = (tw_job *)ctx;
    fe_t w;
    uint64_t e[1] = {lo};
    or_pow(OR_FR, &w, j->omega, e, 1);
    for (size_t i = lo; i < hi; i++) {
        j->tw[i] = w;
        or_mul(OR_FR, &w, &w, j->omega);
    }
}

typedef struct {
    fe_t *a;
    size_t n, tc;
    const fe_t *tw;
    int depth;
} rb_args;

static void butterflies(fe_t *a, size_t n, size_t tc, const fe_t *tw) {
    fe_t *left = a, *right = a + n / 2;
    fe_t t = right[0];
    right[0] = left[0];
    or_add(OR_FR, &left[0], &left[0], &t);
    or_sub(OR_FR, &right[0], &right[0], &t);
    for (size_t i = 1; i < n / 2; i++) {
        or_mul(OR_FR, &t, &right[i], &tw[i * tc]);
        right[i] = left[i];
        or_add(OR_FR, &left[i], &left[i], &t);
        or_sub(OR_FR, &right[i], &right[i], &t);
    }
}

static void *rba(void *p);

static void rba_call(fe_t *a, size_t n, size_t tc, const fe_t *tw, int depth) {
    rb_args args = {a, n, tc, tw, depth};
    rba(&args);
}

/* recursive_butterfly_arithmetic (msm_halo2.rs:287-325); the join is a thread while depth > 0 */
static void *rba(void *p) {
    rb_args *r = (rb_args *)p;
    if (r->n == 2) {
        fe_t t = r->a[1];
        r->a[1] = r->a[0];
        or_add(OR_FR, &r->a[0], &r->a[0], &t);
        or_sub(OR_FR, &r->a[1], &r->a[1], &t);
        return NULL;
    }
    size_t h = r->n / 2;
    if (r->depth > 0) {
        rb_args la = {r->a, h, r->tc * 2, r->tw, r->depth - 1};
        pthread_t th;
        pthread_create(&th, NULL, rba, &la);
        rba_call(r->a + h, h, r->tc * 2, r->tw, r->depth - 1);
        pthread_join(th, NULL);
    } else {
        rba_call(r->a, h, r->tc * 2, r->tw, 0);
        rba_call(r->a + h, h, r->tc * 2, r->tw, 0);
    }
    butterflies(r->a, r->n, r->tc, r->tw);
    return NULL;
}

static unsigned log2_floor(size_t x) {
    unsigned r = 0;
    while (x >>= 1) r++;
    return r;
}

void or_best_fft(fe_t *a, const fe_t *omega, unsigned log_n) {
    size_t n = (size_t)1 << log_n;
    if (n <= 1) return;
    unsigned log_threads = log2_floor((size_t)or_get_threads());
    for (size_t k = 0; k < n; k++) {
        size_t rk = bitreverse(k, log_n);
        if (k < rk) {
            fe_t t = a[rk];
            a[rk] = a[k];
            a[k] = t;
        }
    }
    fe_t *tw = (fe_t *)malloc((n / 2) * sizeof(fe_t));
    tw_job tj = {tw, omega, n / 2};
    or_parallel_for(n / 2, 1 << 14, tw_worker, &tj);
    if (log_n <= log_threads) {
        size_t chunk = 2, tc = n / 2;
        for (unsigned s = 0; s < log_n; s++) {
            for (size_t c = 0; c < n; c += chunk) butterflies(a + c, chunk, tc, tw);
            chunk *= 2;
            tc /= 2;
        }
    } else {
        rba_call(a, n, 1, tw, (int)log_threads);
    }
    free(tw);
}

typedef struct { fe_t *a; const fe_t *powers; size_t pn; const fe_t *scale; } dp_job;

static void dp_worker(void *ctx, size_t lo, size_t hi) {
    dp_job *j = (dp_job *)ctx;
    for (size_t i = lo; i < hi; i++) {
        if (j->powers) or_mul(OR_FR, &j->a[i], &j->a[i], &j->powers[i % j->pn]);
        else or_mul(OR_FR, &j->a[i], &j->a[i], j->scale);
    }
}

void or_distribute_powers(fe_t *a, size_t n, const fe_t *powers, size_t power_num) {
    dp_job j = {a, powers, power_num, NULL};
    or_parallel_for(n, 4096, dp_worker, &j);
}

void or_ntt(fe_t *a, unsigned log_n) {
    fe_t w;
    or_root_of_unity(log_n, 0, &w);
    or_best_fft(a, &w, log_n);
}

void or_intt(fe_t *a, unsigned log_n) {
    fe_t w, ninv, nn = {{(uint64_t)1 << log_n, 0, 0, 0}}, nm;
    or_root_of_unity(log_n, 1, &w);
    or_best_fft(a, &w, log_n);
    or_to_mont(OR_FR, &nm, &nn);
    or_inv(OR_FR, &ninv, &nm);
    dp_job j = {a, NULL, 0, &ninv};
    or_parallel_for((size_t)1 << log_n, 4096, dp_worker, &j);
}

typedef struct { fe_t *out; const fe_t *in; size_t n_in; const fe_t *g; } cs_job;

static void cs_worker(void *ctx, size_t lo, size_t hi) {
    cs_job *j = (cs_job *)ctx;
    fe_t p;
    uint64_t e[1] = {lo};
    or_pow(OR_FR, &p, j->g, e, 1);
    for (size_t i = lo; i < hi; i++) {
        if (i < j->n_in) or_mul(OR_FR, &j->out[i], &j->in[i], &p);
        else memset(&j->out[i], 0, sizeof(fe_t));
        or_mul(OR_FR, &p, &p, j->g);
    }
}

void or_coset_ntt(fe_t *out, const fe_t *coef, unsigned log_in, unsigned log_out, const fe_t *g) {
    size_t n_out = (size_t)1 << log_out;
    cs_job j = {out, coef, (size_t)1 << log_in, g};
    or_parallel_for(n_out, 4096, cs_worker, &j);
    or_ntt(out, log_out);
}

void or_naive_dft(fe_t *out, const fe_t *in, size_t n, const fe_t *omega) {
    fe_t wk;
    or_one(OR_FR, &wk);
    for (size_t k = 0; k < n; k++) {
        fe_t acc = {{0, 0, 0, 0}}, w;
        or_one(OR_FR, &w);
        for (size_t j = 0; j < n; j++) {
            fe_t t;
            or_mul(OR_FR, &t, &in[j], &w);
            or_add(OR_FR, &acc, &acc, &t);
            or_mul(OR_FR, &w, &w, &wk);
        }
        out[k] = acc;
        or_mul(OR_FR, &wk, &wk, omega);
    }
}
