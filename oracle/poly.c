/*
 * Oracle (test infrastructure only): polynomial helpers.
 *
 * or_eval restates halo2's eval_polynomial (core/tests/msm_halo2.rs:354-383): Horner per
 * chunk, each chunk scaled by point^start, chunks summed; the reference's GPU poly_eval
 * computes the same sum (core/src/poly/src/poly_eval.cuh:8-74, Horner truth in
 * core/tests/poly.rs:170-176).
 * or_batch_invert: elementwise inverse where zeros stay zero
 * (core/src/poly/src/batched_invert.cuh:13-93).
 * or_poly_ptr_gather: the PolyPtr view, element i at data[(offset + i) % whole_len], with a
 * rotation r turning into offset = len - r (core/src/common/iter/src/iter.cuh:12-26,
 * :308-327).
 */
#include "oracle.h"
#include "util.h"
#include <stdlib.h>
#include <string.h>

typedef struct { const fe_t *poly; size_t n, chunk; const fe_t *x; fe_t *parts; } ev_job;

static void ev_worker(void *ctx, size_t lo, size_t hi) {
    ev_job *j = (ev_job *)ctx;
    for (size_t t = lo; t < hi; t++) {
        size_t a = t * j->chunk, b = a + j->chunk;
        if (a >= j->n) { memset(&j->parts[t], 0, sizeof(fe_t)); continue; }
        if (b > j->n) b = j->n;
        fe_t acc = {{0, 0, 0, 0}};
        for (size_t i = b; i-- > a;) {
            or_mul(OR_FR, &acc, &acc, j->x);
            or_add(OR_FR, &acc, &acc, &j->poly[i]);
        }
        fe_t p;
        uint64_t e[1] = {a};
        or_pow(OR_FR, &p, j->x, e, 1);
        or_mul(OR_FR, &j->parts[t], &acc, &p);
    }
}

void or_eval(fe_t *res, const fe_t *poly, size_t n, const fe_t *x) {
    size_t th = (size_t)or_get_threads();
    fe_t acc = {{0, 0, 0, 0}};
    if (n * 2 < th) {
        for (size_t i = n; i-- > 0;) {
            or_mul(OR_FR, &acc, &acc, x);
            or_add(OR_FR, &acc, &acc, &poly[i]);
        }
    } else {
        size_t chunk = (n + th - 1) / th;
        fe_t *parts = (fe_t *)malloc(th * sizeof(fe_t));
        ev_job j = {poly, n, chunk, x, parts};
        or_parallel_tasks(th, ev_worker, &j);
        for (size_t i = 0; i < th; i++) or_add(OR_FR, &acc, &acc, &parts[i]);
        free(parts);
    }
    *res = acc;
}

void or_batch_invert(fe_t *a, size_t n) {
    fe_t *pref = (fe_t *)malloc((n + 1) * sizeof(fe_t));
    or_one(OR_FR, &pref[0]);
    for (size_t i = 0; i < n; i++) {
        int z = (a[i].l[0] | a[i].l[1] | a[i].l[2] | a[i].l[3]) == 0;
        if (z) pref[i + 1] = pref[i];
        else or_mul(OR_FR, &pref[i + 1], &pref[i], &a[i]);
    }
    fe_t inv;
    or_inv(OR_FR, &inv, &pref[n]);
    for (size_t i = n; i-- > 0;) {
        int z = (a[i].l[0] | a[i].l[1] | a[i].l[2] | a[i].l[3]) == 0;
        if (z) continue;
        fe_t r;
        or_mul(OR_FR, &r, &inv, &pref[i]);
        or_mul(OR_FR, &inv, &inv, &a[i]);
        a[i] = r;
    }
    free(pref);
}

void or_poly_ptr_gather(fe_t *out, const fe_t *base, size_t len, size_t rotate, size_t offset,
                        size_t whole_len) {
    if (whole_len == 0) whole_len = len;
    if (rotate != 0) offset = len - rotate;
    for (size_t i = 0; i < len; i++) out[i] = base[(offset + i) % whole_len];
}
