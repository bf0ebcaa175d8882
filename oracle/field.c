/*
 * Oracle (test infrastructure only): BN254 Fr / Fq Montgomery arithmetic.
 *
 * Restates the reference's host Montgomery code (core/src/common/mont/src/field.cuh:29-157:
 * schoolbook product, word-serial Montgomery reduction, final conditional subtraction so
 * every result is canonical < m) with 64-bit limbs.  Because results are canonical, the
 * bytes are identical to the reference's 32-bit-limb code.  Moduli follow
 * core/src/common/mont/src/bn254_fr.cuh:18-26 and bn254_fq.cuh:10-18; R mod m, R^2 mod m
 * and -m^-1 are derived here and checked against those constants by the tests.
 */
#include "oracle.h"
#include "util.h"
#include <string.h>

typedef unsigned __int128 u128;

typedef struct {
    uint64_t p[4];
    uint64_t pinv;   /* -p^-1 mod 2^64 */
    uint64_t r1[4];  /* R mod p */
    uint64_t r2[4];  /* R^2 mod p */
} fparams;

static fparams FP[2];
static int inited = 0;

static const uint64_t FR_MOD[4] = {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL,
                                   0xb85045b68181585dULL, 0x30644e72e131a029ULL};
static const uint64_t FQ_MOD[4] = {0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL,
                                   0xb85045b68181585dULL, 0x30644e72e131a029ULL};

static int geq(const uint64_t *a, const uint64_t *b) {
    for (int i = 3; i >= 0; i--) {
        if (a[i] != b[i]) return a[i] > b[i];
    }
    return 1;
}

static uint64_t sub4(uint64_t *r, const uint64_t *a, const uint64_t *b) {
    uint64_t borrow = 0;
    for (int i = 0; i < 4; i++) {
        u128 d = (u128)a[i] - b[i] - borrow;
        r[i] = (uint64_t)d;
        borrow = (uint64_t)(d >> 64) & 1;
    }
    return borrow;
}

static uint64_t add4(uint64_t *r, const uint64_t *a, const uint64_t *b) {
    u128 c = 0;
    for (int i = 0; i < 4; i++) {
        c += (u128)a[i] + b[i];
        r[i] = (uint64_t)c;
        c >>= 64;
    }
    return (uint64_t)c;
}

/* r = 2*a mod p for a < p */
static void dbl_mod(const fparams *F, uint64_t *r, const uint64_t *a) {
    uint64_t t[4];
    uint64_t c = add4(t, a, a);
    if (c || geq(t, F->p)) sub4(t, t, F->p);
    memcpy(r, t, 32);
}

static void init_params(fparams *F, const uint64_t *mod) {
    memcpy(F->p, mod, 32);
    uint64_t inv = 1;
    for (int i = 0; i < 7; i++) inv *= 2 - mod[0] * inv;
    F->pinv = (uint64_t)0 - inv;
    uint64_t x[4] = {1, 0, 0, 0};
    for (int i = 0; i < 256; i++) dbl_mod(F, x, x);
    memcpy(F->r1, x, 32);
    for (int i = 0; i < 256; i++) dbl_mod(F, x, x);
    memcpy(F->r2, x, 32);
}

static void ensure_init(void) {
    if (!inited) {
        init_params(&FP[0], FR_MOD);
        init_params(&FP[1], FQ_MOD);
        inited = 1;
    }
}

void or_field_consts(int f, uint64_t *modulus, uint64_t *r1, uint64_t *r2, uint64_t *minv64) {
    ensure_init();
    memcpy(modulus, FP[f].p, 32);
    memcpy(r1, FP[f].r1, 32);
    memcpy(r2, FP[f].r2, 32);
    *minv64 = FP[f].pinv;
}

/* CIOS Montgomery product; inputs < p, output canonical < p */
static inline void mont_mul(const fparams *F, uint64_t *r, const uint64_t *a, const uint64_t *b) {
    uint64_t t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        u128 c = 0;
        for (int j = 0; j < 4; j++) {
            c += (u128)a[j] * b[i] + t[j];
            t[j] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[4] = (uint64_t)c;
        t[5] = (uint64_t)(c >> 64);
        uint64_t m = t[0] * F->pinv;
        c = (u128)m * F->p[0] + t[0];
        c >>= 64;
        for (int j = 1; j < 4; j++) {
            c += (u128)m * F->p[j] + t[j];
            t[j - 1] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[3] = (uint64_t)c;
        t[4] = t[5] + (uint64_t)(c >> 64);
    }
    if (t[4] || geq(t, F->p)) sub4(t, t, F->p);
    memcpy(r, t, 32);
}

void or_mul(int f, fe_t *r, const fe_t *a, const fe_t *b) {
    ensure_init();
    mont_mul(&FP[f], r->l, a->l, b->l);
}

void or_add(int f, fe_t *r, const fe_t *a, const fe_t *b) {
    ensure_init();
    uint64_t t[4];
    uint64_t c = add4(t, a->l, b->l);
    if (c || geq(t, FP[f].p)) sub4(t, t, FP[f].p);
    memcpy(r->l, t, 32);
}

void or_sub(int f, fe_t *r, const fe_t *a, const fe_t *b) {
    ensure_init();
    uint64_t t[4];
    if (sub4(t, a->l, b->l)) add4(t, t, FP[f].p);
    memcpy(r->l, t, 32);
}

void or_neg(int f, fe_t *r, const fe_t *a) {
    ensure_init();
    if ((a->l[0] | a->l[1] | a->l[2] | a->l[3]) == 0) {
        memset(r, 0, 32);
        return;
    }
    sub4(r->l, FP[f].p, a->l);
}

void or_to_mont(int f, fe_t *r, const fe_t *a) {
    ensure_init();
    uint64_t t[4];
    memcpy(t, a->l, 32);
    while (geq(t, FP[f].p)) sub4(t, t, FP[f].p);  /* reduce a raw number first */
    mont_mul(&FP[f], r->l, t, FP[f].r2);
}

void or_from_mont(int f, fe_t *r, const fe_t *a) {
    ensure_init();
    uint64_t one[4] = {1, 0, 0, 0};
    mont_mul(&FP[f], r->l, a->l, one);
}

void or_one(int f, fe_t *r) {
    ensure_init();
    memcpy(r->l, FP[f].r1, 32);
}

/* Element::pow (field.cuh:1133-1160): square-and-multiply over the exponent's bits, MSB first */
void or_pow(int f, fe_t *r, const fe_t *a, const uint64_t *e, int elimbs) {
    ensure_init();
    fe_t acc;
    or_one(f, &acc);
    for (int i = elimbs * 64 - 1; i >= 0; i--) {
        mont_mul(&FP[f], acc.l, acc.l, acc.l);
        if ((e[i / 64] >> (i % 64)) & 1) mont_mul(&FP[f], acc.l, acc.l, a->l);
    }
    *r = acc;
}

/* Element::invert (field.cuh:1172-1175): a^(m-2) */
void or_inv(int f, fe_t *r, const fe_t *a) {
    ensure_init();
    uint64_t e[4];
    uint64_t two[4] = {2, 0, 0, 0};
    sub4(e, FP[f].p, two);
    or_pow(f, r, a, e, 4);
}

void or_bn_mul(uint64_t r[8], const uint64_t a[4], const uint64_t b[4]) {
    uint64_t t[8] = {0};
    for (int i = 0; i < 4; i++) {
        u128 c = 0;
        for (int j = 0; j < 4; j++) {
            c += (u128)a[j] * b[i] + t[i + j];
            t[i + j] = (uint64_t)c;
            c >>= 64;
        }
        t[i + 4] = (uint64_t)c;
    }
    memcpy(r, t, 64);
}

void or_bn_slr(uint64_t r[4], const uint64_t a[4], unsigned k) {
    uint64_t t[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        unsigned src_bit = i * 64 + k;
        unsigned w = src_bit / 64, s = src_bit % 64;
        if (w < 4) {
            t[i] = a[w] >> s;
            if (s && w + 1 < 4) t[i] |= a[w + 1] << (64 - s);
        }
    }
    memcpy(r, t, 32);
}

/* ---- elementwise Fr batches (threaded) ---- */
typedef struct { fe_t *r; const fe_t *a, *b; int op; } vec_job;

static void vec_worker(void *ctx, size_t lo, size_t hi) {
    vec_job *j = (vec_job *)ctx;
    for (size_t i = lo; i < hi; i++) {
        if (j->op == 0) mont_mul(&FP[0], j->r[i].l, j->a[i].l, j->b[i].l);
        else if (j->op == 1) or_add(OR_FR, &j->r[i], &j->a[i], &j->b[i]);
        else or_sub(OR_FR, &j->r[i], &j->a[i], &j->b[i]);
    }
}

static void vec_run(fe_t *r, const fe_t *a, const fe_t *b, size_t n, int op) {
    ensure_init();
    vec_job j = {r, a, b, op};
    or_parallel_for(n, 4096, vec_worker, &j);
}

void or_vec_mul(fe_t *r, const fe_t *a, const fe_t *b, size_t n) { vec_run(r, a, b, n, 0); }
void or_vec_add(fe_t *r, const fe_t *a, const fe_t *b, size_t n) { vec_run(r, a, b, n, 1); }
void or_vec_sub(fe_t *r, const fe_t *a, const fe_t *b, size_t n) { vec_run(r, a, b, n, 2); }
