/*
 * Oracle (test infrastructure only): deterministic synthetic inputs and roots of unity.
 *
 * Generator: counter based, so element i depends only on (seed, i) and the GPU generator
 * reproduces it exactly.  Candidate limbs come from the SplitMix64 finalizer applied to a
 * per-(seed, i, attempt, limb) counter; the top limb is masked to 62 bits (254-bit
 * candidates) and candidates >= r are rejected (attempt = 0..63), giving uniform elements
 * of Fr.  Field elements are returned in Montgomery form (x * R mod r).
 *
 * Roots of unity follow compiler/src/utils.rs:51-77: omega_k = ROOT^(2^(S-k)) with
 * ROOT = 7^((r-1)/2^S), S = 28 (the 2-adicity of r - 1), inverted for the inverse NTT.
 */
#include "oracle.h"
#include <string.h>

static uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static const uint64_t FR_MOD[4] = {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL,
                                   0xb85045b68181585dULL, 0x30644e72e131a029ULL};

static int lt_mod(const uint64_t *a) {
    for (int i = 3; i >= 0; i--) {
        if (a[i] != FR_MOD[i]) return a[i] < FR_MOD[i];
    }
    return 0;
}

void or_gen_fr_raw(uint64_t seed, uint64_t idx, fe_t *out) {
    uint64_t s = mix64(seed ^ 0x6a09e667f3bcc909ULL);
    for (uint64_t attempt = 0; attempt < 64; attempt++) {
        uint64_t c[4];
        for (uint64_t k = 0; k < 4; k++) {
            uint64_t ctr = (idx << 8) | (attempt << 2) | k;
            c[k] = mix64(s + ctr * 0x9E3779B97F4A7C15ULL);
        }
        c[3] &= 0x3FFFFFFFFFFFFFFFULL;
        if (lt_mod(c)) {
            memcpy(out->l, c, 32);
            return;
        }
    }
    memset(out, 0, sizeof(*out));
}

void or_gen_fr(uint64_t seed, uint64_t start, size_t n, fe_t *out) {
    for (size_t i = 0; i < n; i++) {
        fe_t raw;
        or_gen_fr_raw(seed, start + i, &raw);
        or_to_mont(OR_FR, &out[i], &raw);
    }
}

void or_root_of_unity(unsigned log_n, int inverse, fe_t *omega) {
    /* t = (r - 1) >> 28 */
    uint64_t t[4];
    memcpy(t, FR_MOD, 32);
    t[0] -= 1;
    for (int i = 0; i < 4; i++) {
        t[i] = (t[i] >> 28) | (i < 3 ? (t[i + 1] << 36) : 0);
    }
    fe_t seven = {{7, 0, 0, 0}}, g, root;
    or_to_mont(OR_FR, &g, &seven);
    or_pow(OR_FR, &root, &g, t, 4);
    for (unsigned i = log_n; i < 28; i++) or_mul(OR_FR, &root, &root, &root);
    if (inverse) or_inv(OR_FR, &root, &root);
    *omega = root;
}

void or_twiddles(const fe_t *omega, size_t count, fe_t *out) {
    fe_t w;
    or_one(OR_FR, &w);
    for (size_t i = 0; i < count; i++) {
        out[i] = w;
        or_mul(OR_FR, &w, &w, omega);
    }
}
