// Host-side BN254 Fr / Fq Montgomery arithmetic for set-up work that the reference also
// does on the CPU (gen_pq_omegas, core/src/ntt/src/precompute.cuh:89-113; scalar constants
// such as n^-1 and coset shifts).  Canonical outputs, same bytes as the device code.
#pragma once
#include <cstdint>
#include <cstring>

namespace zkh {

typedef unsigned __int128 u128;

struct Fe {
    uint64_t l[4];
};

struct Params {
    uint64_t p[4];
    uint64_t pinv;
    uint64_t r1[4];
    uint64_t r2[4];
};

inline bool geq(const uint64_t *a, const uint64_t *b) {
    for (int i = 3; i >= 0; i--)
        if (a[i] != b[i]) return a[i] > b[i];
    return true;
}

inline uint64_t sub4(uint64_t *r, const uint64_t *a, const uint64_t *b) {
    uint64_t br = 0;
    for (int i = 0; i < 4; i++) {
        u128 d = (u128)a[i] - b[i] - br;
        r[i] = (uint64_t)d;
        br = (uint64_t)(d >> 64) & 1;
    }
    return br;
}

inline uint64_t add4(uint64_t *r, const uint64_t *a, const uint64_t *b) {
    u128 c = 0;
    for (int i = 0; i < 4; i++) {
        c += (u128)a[i] + b[i];
        r[i] = (uint64_t)c;
        c >>= 64;
    }
    return (uint64_t)c;
}

inline Params make_params(const uint64_t *mod) {
    Params P;
    memcpy(P.p, mod, 32);
    uint64_t inv = 1;
    for (int i = 0; i < 7; i++) inv *= 2 - mod[0] * inv;
    P.pinv = (uint64_t)0 - inv;
    uint64_t x[4] = {1, 0, 0, 0};
    for (int k = 0; k < 512; k++) {
        uint64_t t[4];
        uint64_t c = add4(t, x, x);
        if (c || geq(t, P.p)) sub4(t, t, P.p);
        memcpy(x, t, 32);
        if (k == 255) memcpy(P.r1, x, 32);
    }
    memcpy(P.r2, x, 32);
    return P;
}

inline const Params &fr() {
    static const uint64_t m[4] = {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL,
                                  0x30644e72e131a029ULL};
    static const Params P = make_params(m);
    return P;
}

inline const Params &fq() {
    static const uint64_t m[4] = {0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL,
                                  0x30644e72e131a029ULL};
    static const Params P = make_params(m);
    return P;
}

inline Fe mul(const Params &P, const Fe &a, const Fe &b) {
    uint64_t t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        u128 c = 0;
        for (int j = 0; j < 4; j++) {
            c += (u128)a.l[j] * b.l[i] + t[j];
            t[j] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[4] = (uint64_t)c;
        t[5] = (uint64_t)(c >> 64);
        uint64_t m = t[0] * P.pinv;
        c = (u128)m * P.p[0] + t[0];
        c >>= 64;
        for (int j = 1; j < 4; j++) {
            c += (u128)m * P.p[j] + t[j];
            t[j - 1] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[3] = (uint64_t)c;
        t[4] = t[5] + (uint64_t)(c >> 64);
    }
    if (t[4] || geq(t, P.p)) sub4(t, t, P.p);
    Fe r;
    memcpy(r.l, t, 32);
    return r;
}

inline Fe one(const Params &P) {
    Fe r;
    memcpy(r.l, P.r1, 32);
    return r;
}

inline Fe from_u64(const Params &P, uint64_t v) {
    Fe x = {{v, 0, 0, 0}};
    Fe r2;
    memcpy(r2.l, P.r2, 32);
    return mul(P, x, r2);
}

inline Fe pow(const Params &P, const Fe &a, uint64_t e) {
    Fe r = one(P), b = a;
    while (e) {
        if (e & 1) r = mul(P, r, b);
        b = mul(P, b, b);
        e >>= 1;
    }
    return r;
}

inline Fe inv(const Params &P, const Fe &a) {
    uint64_t e[4];
    uint64_t two[4] = {2, 0, 0, 0};
    sub4(e, P.p, two);
    Fe r = one(P);
    for (int i = 255; i >= 0; i--) {
        r = mul(P, r, r);
        if ((e[i / 64] >> (i % 64)) & 1) r = mul(P, r, a);
    }
    return r;
}

// a^e for a 256-bit exponent (4 little-endian u64 limbs)
inline Fe pow_big(const Params &P, const Fe &a, const uint64_t e[4]) {
    Fe r = one(P);
    for (int i = 255; i >= 0; i--) {
        r = mul(P, r, r);
        if ((e[i / 64] >> (i % 64)) & 1) r = mul(P, r, a);
    }
    return r;
}

// primitive 2^log_n-th root of unity of Fr, Montgomery form: (7^((r-1)/2^28))^(2^(28-log_n)),
// inverted when `inverse` (compiler/src/utils.rs:51-77)
inline Fe fr_root_of_unity(unsigned log_n, bool inverse) {
    const Params &P = fr();
    uint64_t t[4];
    memcpy(t, P.p, 32);
    t[0] -= 1;
    for (int i = 0; i < 4; i++) t[i] = (t[i] >> 28) | (i < 3 ? (t[i + 1] << 36) : 0);
    Fe root = pow_big(P, from_u64(P, 7), t);
    for (unsigned i = log_n; i < 28; i++) root = mul(P, root, root);
    return inverse ? inv(P, root) : root;
}

inline Fe load(const unsigned int *w) {
    Fe r;
    memcpy(r.l, w, 32);
    return r;
}

inline void store(unsigned int *w, const Fe &a) { memcpy(w, a.l, 32); }

}  // namespace zkh
