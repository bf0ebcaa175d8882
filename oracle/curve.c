/*
 * Oracle (test infrastructure only): BN254 G1 arithmetic over Fq.
 *
 * Restates core/src/common/curve/src/curve_xyzz.cuh:163-419 (EFD XYZZ formulas:
 * add-2008-s :325-345, madd-2008-s :352-370, dbl-2008-s-1 :377-391, mdbl-2008-s-1
 * :229-241, scaling to affine :316-322) with a = 0, b = 3 (core/src/common/curve/src/
 * bn254.cuh:13-77).  Affine identity is (0, 0) (is_identity checks y == 0); XYZZ identity
 * is zz == 0.  Points are Montgomery-form Fq coordinates.
 */
#include "oracle.h"
#include "util.h"
#include <stdlib.h>
#include <string.h>

#define F OR_FQ

static int fe_is_zero(const fe_t *a) { return (a->l[0] | a->l[1] | a->l[2] | a->l[3]) == 0; }
static int fe_eq(const fe_t *a, const fe_t *b) { return memcmp(a, b, sizeof(fe_t)) == 0; }
static void mul(fe_t *r, const fe_t *a, const fe_t *b) { or_mul(F, r, a, b); }
static void add(fe_t *r, const fe_t *a, const fe_t *b) { or_add(F, r, a, b); }
static void sub(fe_t *r, const fe_t *a, const fe_t *b) { or_sub(F, r, a, b); }

void or_g1_generator(g1a_t *g) {
    fe_t one = {{1, 0, 0, 0}}, two = {{2, 0, 0, 0}};
    or_to_mont(F, &g->x, &one);
    or_to_mont(F, &g->y, &two);
}

int or_g1_on_curve(const g1a_t *p) {
    if (fe_is_zero(&p->y)) return 1;
    fe_t t0, t1, b, three = {{3, 0, 0, 0}};
    or_to_mont(F, &b, &three);
    mul(&t0, &p->x, &p->x);
    mul(&t0, &t0, &p->x);
    add(&t0, &t0, &b);
    mul(&t1, &p->y, &p->y);
    return fe_eq(&t0, &t1);
}

static void xyzz_identity(g1x_t *r) {
    memset(r, 0, sizeof(*r));
    or_one(F, &r->zzz);
}

void or_g1_to_xyzz(g1x_t *r, const g1a_t *p) {
    if (fe_is_zero(&p->y)) {
        xyzz_identity(r);
        return;
    }
    r->x = p->x;
    r->y = p->y;
    or_one(F, &r->zz);
    or_one(F, &r->zzz);
}

void or_g1_to_affine(g1a_t *r, const g1x_t *p) {
    fe_t a, b;
    or_inv(F, &a, &p->zzz);
    mul(&b, &p->zz, &a);
    mul(&b, &b, &b);
    mul(&r->x, &p->x, &b);
    mul(&r->y, &p->y, &a);
}

void or_g1_dbl(g1x_t *r, const g1x_t *p) {
    if (fe_is_zero(&p->zz)) {
        *r = *p;
        return;
    }
    fe_t u, v, w, s, x2, m, x3, y3, t;
    add(&u, &p->y, &p->y);
    mul(&v, &u, &u);
    mul(&w, &u, &v);
    mul(&s, &p->x, &v);
    mul(&x2, &p->x, &p->x);
    add(&m, &x2, &x2);
    add(&m, &m, &x2);
    mul(&x3, &m, &m);
    sub(&x3, &x3, &s);
    sub(&x3, &x3, &s);
    sub(&t, &s, &x3);
    mul(&y3, &m, &t);
    mul(&t, &w, &p->y);
    sub(&y3, &y3, &t);
    g1x_t o;
    o.x = x3;
    o.y = y3;
    mul(&o.zz, &v, &p->zz);
    mul(&o.zzz, &w, &p->zzz);
    *r = o;
}

static void affine_dbl(g1x_t *r, const g1a_t *p) {
    fe_t u, v, w, s, x2, m, x3, y3, t;
    add(&u, &p->y, &p->y);
    mul(&v, &u, &u);
    mul(&w, &u, &v);
    mul(&s, &p->x, &v);
    mul(&x2, &p->x, &p->x);
    add(&m, &x2, &x2);
    add(&m, &m, &x2);
    mul(&x3, &m, &m);
    sub(&x3, &x3, &s);
    sub(&x3, &x3, &s);
    sub(&t, &s, &x3);
    mul(&y3, &m, &t);
    mul(&t, &w, &p->y);
    sub(&y3, &y3, &t);
    r->x = x3;
    r->y = y3;
    r->zz = v;
    r->zzz = w;
}

void or_g1_add(g1x_t *r, const g1x_t *p, const g1x_t *q) {
    if (fe_is_zero(&p->zz)) { *r = *q; return; }
    if (fe_is_zero(&q->zz)) { *r = *p; return; }
    fe_t u1, u2, s1, s2, P, R, pp, ppp, Q, x3, y3, t;
    mul(&u1, &p->x, &q->zz);
    mul(&u2, &q->x, &p->zz);
    mul(&s1, &p->y, &q->zzz);
    mul(&s2, &q->y, &p->zzz);
    sub(&P, &u2, &u1);
    sub(&R, &s2, &s1);
    if (fe_is_zero(&P) && fe_is_zero(&R)) {
        or_g1_dbl(r, p);
        return;
    }
    mul(&pp, &P, &P);
    mul(&ppp, &P, &pp);
    mul(&Q, &u1, &pp);
    mul(&x3, &R, &R);
    sub(&x3, &x3, &ppp);
    sub(&x3, &x3, &Q);
    sub(&x3, &x3, &Q);
    sub(&t, &Q, &x3);
    mul(&y3, &R, &t);
    mul(&t, &s1, &ppp);
    sub(&y3, &y3, &t);
    g1x_t o;
    o.x = x3;
    o.y = y3;
    mul(&o.zz, &p->zz, &q->zz);
    mul(&o.zz, &o.zz, &pp);
    mul(&o.zzz, &p->zzz, &q->zzz);
    mul(&o.zzz, &o.zzz, &ppp);
    *r = o;
}

void or_g1_madd(g1x_t *r, const g1x_t *p, const g1a_t *q) {
    if (fe_is_zero(&p->zz)) { or_g1_to_xyzz(r, q); return; }
    if (fe_is_zero(&q->y)) { *r = *p; return; }
    fe_t u2, s2, P, R, pp, ppp, Q, x3, y3, t;
    mul(&u2, &q->x, &p->zz);
    mul(&s2, &q->y, &p->zzz);
    sub(&P, &u2, &p->x);
    sub(&R, &s2, &p->y);
    if (fe_is_zero(&P) && fe_is_zero(&R)) {
        affine_dbl(r, q);
        return;
    }
    mul(&pp, &P, &P);
    mul(&ppp, &P, &pp);
    mul(&Q, &p->x, &pp);
    mul(&x3, &R, &R);
    sub(&x3, &x3, &ppp);
    sub(&x3, &x3, &Q);
    sub(&x3, &x3, &Q);
    sub(&t, &Q, &x3);
    mul(&y3, &R, &t);
    mul(&t, &p->y, &ppp);
    sub(&y3, &y3, &t);
    g1x_t o;
    o.x = x3;
    o.y = y3;
    mul(&o.zz, &p->zz, &pp);
    mul(&o.zzz, &p->zzz, &ppp);
    *r = o;
}

void or_g1_affine_add(g1a_t *r, const g1a_t *p, const g1a_t *q) {
    g1x_t t;
    or_g1_to_xyzz(&t, p);
    or_g1_madd(&t, &t, q);
    or_g1_to_affine(r, &t);
}

/* double-and-add over the canonical scalar's bits, MSB first (PointXYZZ::multiple style) */
void or_g1_scalar_mul(g1x_t *r, const g1a_t *p, const fe_t *k) {
    g1x_t acc;
    xyzz_identity(&acc);
    for (int i = 255; i >= 0; i--) {
        or_g1_dbl(&acc, &acc);
        if ((k->l[i / 64] >> (i % 64)) & 1) or_g1_madd(&acc, &acc, p);
    }
    *r = acc;
}

/* Montgomery-trick normalisation; identities map to (0,0) */
void or_g1_batch_to_affine(g1a_t *out, const g1x_t *in, size_t n) {
    fe_t *pref = (fe_t *)malloc((n + 1) * sizeof(fe_t));
    or_one(F, &pref[0]);
    for (size_t i = 0; i < n; i++) {
        if (fe_is_zero(&in[i].zz)) pref[i + 1] = pref[i];
        else mul(&pref[i + 1], &pref[i], &in[i].zzz);
    }
    fe_t inv;
    or_inv(F, &inv, &pref[n]);
    for (size_t i = n; i-- > 0;) {
        if (fe_is_zero(&in[i].zz)) {
            memset(&out[i], 0, sizeof(g1a_t));
            continue;
        }
        fe_t a, b;
        mul(&a, &inv, &pref[i]);           /* zzz_i^-1 */
        mul(&inv, &inv, &in[i].zzz);
        mul(&b, &in[i].zz, &a);
        mul(&b, &b, &b);
        g1a_t o;
        mul(&o.x, &in[i].x, &b);
        mul(&o.y, &in[i].y, &a);
        out[i] = o;
    }
    free(pref);
}

/* ---- synthetic bases P_i = k_i * G with a fixed-base byte table ---- */
static g1a_t *fb_table = NULL;  /* [32][256] affine: d * 2^(8w) * G */

static void build_fb_table(void) {
    if (fb_table) return;
    g1x_t *tmp = (g1x_t *)malloc(32 * 256 * sizeof(g1x_t));
    g1a_t g;
    or_g1_generator(&g);
    g1x_t base;
    or_g1_to_xyzz(&base, &g);
    for (int w = 0; w < 32; w++) {
        g1a_t ba;
        or_g1_to_affine(&ba, &base);
        xyzz_identity(&tmp[w * 256]);
        for (int d = 1; d < 256; d++) or_g1_madd(&tmp[w * 256 + d], &tmp[w * 256 + d - 1], &ba);
        for (int k = 0; k < 8; k++) or_g1_dbl(&base, &base);
    }
    g1a_t *t = (g1a_t *)malloc(32 * 256 * sizeof(g1a_t));
    or_g1_batch_to_affine(t, tmp, 32 * 256);
    free(tmp);
    fb_table = t;
}

typedef struct { uint64_t seed, start; g1a_t *out; } gp_job;

static void gp_worker(void *ctx, size_t lo, size_t hi) {
    gp_job *j = (gp_job *)ctx;
    size_t n = hi - lo;
    g1x_t *acc = (g1x_t *)malloc(n * sizeof(g1x_t));
    for (size_t i = lo; i < hi; i++) {
        fe_t k;
        or_gen_fr_raw(j->seed, j->start + i, &k);
        g1x_t a;
        xyzz_identity(&a);
        for (int w = 0; w < 32; w++) {
            unsigned d = (unsigned)((k.l[w / 8] >> ((w % 8) * 8)) & 0xff);
            if (d) or_g1_madd(&a, &a, &fb_table[w * 256 + d]);
        }
        acc[i - lo] = a;
    }
    or_g1_batch_to_affine(j->out + lo, acc, n);
    free(acc);
}

void or_gen_points(uint64_t seed, uint64_t start, size_t n, g1a_t *out) {
    build_fb_table();
    gp_job j = {seed, start, out};
    or_parallel_for(n, 1024, gp_worker, &j);
}
