// BN254 Fr / Fq Montgomery arithmetic for sm_100a.
//
// Semantics follow the reference's mont::Element (core/src/common/mont/src/field.cuh:906-1204):
// an element is 8 little-endian u32 limbs in Montgomery form (R = 2^256), and every value a
// kernel stores is canonical (< m), so bytes match the reference and the oracle exactly.
//
// Inside kernels values are kept "lazy" in [0, 2m): both moduli are below 2^254, so with
// 4m < R the CIOS product of two values below 2m is again below 2m and needs no final
// subtraction; additions and subtractions fold back into [0, 2m) with one conditional
// correction.  `canonical()` maps [0, 2m) to [0, m) before a store.
//
// The multiply is word-serial CIOS with two carry chains per row (low halves, then high
// halves) on mad.lo.cc / madc.hi.cc; the low word of the reduction row is replaced by a
// carry test because it is zero by construction.
#pragma once
#include <cstdint>

namespace zk {

using u32 = uint32_t;
using u64 = uint64_t;

// ------------------------------------------------------------------ PTX carry primitives
#define ZK_DI __device__ __forceinline__

ZK_DI u32 add_cc(u32 a, u32 b) { u32 r; asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
ZK_DI u32 addc_cc(u32 a, u32 b) { u32 r; asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
ZK_DI u32 addc(u32 a, u32 b) { u32 r; asm volatile("addc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
ZK_DI u32 sub_cc(u32 a, u32 b) { u32 r; asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
ZK_DI u32 subc_cc(u32 a, u32 b) { u32 r; asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
ZK_DI u32 subc(u32 a, u32 b) { u32 r; asm volatile("subc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
ZK_DI u32 mad_lo_cc(u32 a, u32 b, u32 c) { u32 r; asm volatile("mad.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }
ZK_DI u32 madc_lo_cc(u32 a, u32 b, u32 c) { u32 r; asm volatile("madc.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }
ZK_DI u32 mad_hi_cc(u32 a, u32 b, u32 c) { u32 r; asm volatile("mad.hi.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }
ZK_DI u32 madc_hi_cc(u32 a, u32 b, u32 c) { u32 r; asm volatile("madc.hi.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }
ZK_DI u32 madc_hi(u32 a, u32 b, u32 c) { u32 r; asm volatile("madc.hi.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }

// ------------------------------------------------------------------ field parameters
// moduli from core/src/common/mont/src/bn254_fr.cuh:18-26 and bn254_fq.cuh:10-18
struct FrParams {
    ZK_DI static constexpr u32 m(int i) {
        constexpr u32 t[8] = {0xf0000001u, 0x43e1f593u, 0x79b97091u, 0x2833e848u,
                                 0x8181585du, 0xb85045b6u, 0xe131a029u, 0x30644e72u};
        return t[i];
    }
    ZK_DI static constexpr u32 m2(int i) {
        constexpr u32 t[8] = {0xe0000002u, 0x87c3eb27u, 0xf372e122u, 0x5067d090u,
                                  0x0302b0bau, 0x70a08b6du, 0xc2634053u, 0x60c89ce5u};
        return t[i];
    }
    ZK_DI static constexpr u32 r1(int i) {
        constexpr u32 t[8] = {0x4ffffffbu, 0xac96341cu, 0x9f60cd29u, 0x36fc7695u,
                                  0x7879462eu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u};
        return t[i];
    }
    ZK_DI static constexpr u32 r2(int i) {
        constexpr u32 t[8] = {0xae216da7u, 0x1bb8e645u, 0xe35c59e3u, 0x53fe3ab1u,
                                  0x53bb8085u, 0x8c49833du, 0x7f4e44a5u, 0x0216d0b1u};
        return t[i];
    }
    static constexpr u32 MPRIME = 4026531839u;  // -m^-1 mod 2^32
    // 2^34 R^3 mod m: the final factor of inv_binary (curve.cuh)
    ZK_DI static constexpr u32 invk(int i) {
        constexpr u32 t[8] = {0xdd8b6d21u, 0x352ff640u, 0x331ce10au, 0x011e8bd1u,
                                 0x55d392c2u, 0x438150aeu, 0x73335b20u, 0x21fe9388u};
        return t[i];
    }
    // 2^256 - m and -m^-1 mod 2^256 (the constants of the Shoup product by a fixed factor)
    ZK_DI static constexpr u32 np(int i) {
        constexpr u32 t[8] = {0x0fffffffu, 0xbc1e0a6cu, 0x86468f6eu, 0xd7cc17b7u,
                                 0x7e7ea7a2u, 0x47afba49u, 0x1ece5fd6u, 0xcf9bb18du};
        return t[i];
    }
    ZK_DI static constexpr u32 minv(int i) {
        constexpr u32 t[8] = {0xefffffffu, 0xc2e1f593u, 0x4c6911b3u, 0x6586864bu,
                                 0x99062391u, 0xe39a9828u, 0x0d8341b2u, 0x73f82f1du};
        return t[i];
    }
};

struct FqParams {
    ZK_DI static constexpr u32 m(int i) {
        constexpr u32 t[8] = {0xd87cfd47u, 0x3c208c16u, 0x6871ca8du, 0x97816a91u,
                                 0x8181585du, 0xb85045b6u, 0xe131a029u, 0x30644e72u};
        return t[i];
    }
    ZK_DI static constexpr u32 m2(int i) {
        constexpr u32 t[8] = {0xb0f9fa8eu, 0x7841182du, 0xd0e3951au, 0x2f02d522u,
                                  0x0302b0bbu, 0x70a08b6du, 0xc2634053u, 0x60c89ce5u};
        return t[i];
    }
    ZK_DI static constexpr u32 r1(int i) {
        constexpr u32 t[8] = {0xc58f0d9du, 0xd35d438du, 0xf5c70b3du, 0x0a78eb28u,
                                  0x7879462cu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u};
        return t[i];
    }
    ZK_DI static constexpr u32 r2(int i) {
        constexpr u32 t[8] = {0x538afa89u, 0xf32cfc5bu, 0xd44501fbu, 0xb5e71911u,
                                  0x0a417ff6u, 0x47ab1effu, 0xcab8351fu, 0x06d89f71u};
        return t[i];
    }
    static constexpr u32 MPRIME = 3834012553u;
    ZK_DI static constexpr u32 invk(int i) {
        constexpr u32 t[8] = {0x13bd45e1u, 0x31d6a0d9u, 0x382c59a2u, 0x45fbf2bcu,
                                 0x1ab31dfbu, 0x5b5fa369u, 0xb36fd339u, 0x24811383u};
        return t[i];
    }
};

template <class P>
struct Fp {
    u32 v[8];

    static constexpr int LIMBS = 8;

    ZK_DI static Fp zero() {
        Fp r;
#pragma unroll
        for (int i = 0; i < 8; i++) r.v[i] = 0;
        return r;
    }
    ZK_DI static Fp one() {
        Fp r;
#pragma unroll
        for (int i = 0; i < 8; i++) r.v[i] = P::r1(i);
        return r;
    }
    ZK_DI static Fp from_words(const u32 *w) {
        Fp r;
#pragma unroll
        for (int i = 0; i < 8; i++) r.v[i] = w[i];
        return r;
    }

    // 128-bit vector load / store of one 32-byte element
    ZK_DI static Fp load(const u32 *p) {
        const uint4 *q = reinterpret_cast<const uint4 *>(p);
        uint4 a = q[0], b = q[1];
        Fp r;
        r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
        r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
        return r;
    }
    ZK_DI static Fp load_nc(const u32 *p) {
        const uint4 *q = reinterpret_cast<const uint4 *>(p);
        uint4 a = __ldg(q), b = __ldg(q + 1);
        Fp r;
        r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
        r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
        return r;
    }
    ZK_DI void store(u32 *p) const {
        uint4 *q = reinterpret_cast<uint4 *>(p);
        q[0] = make_uint4(v[0], v[1], v[2], v[3]);
        q[1] = make_uint4(v[4], v[5], v[6], v[7]);
    }

    ZK_DI bool is_zero() const {
        u32 acc = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) acc |= v[i];
        return acc == 0;
    }
    ZK_DI bool operator==(const Fp &o) const {
        u32 acc = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) acc |= v[i] ^ o.v[i];
        return acc == 0;
    }

    // r = a - b over 256 bits; returns the borrow (0 or 1)
    ZK_DI static u32 sub_raw(u32 *r, const u32 *a, const u32 *b) {
        r[0] = sub_cc(a[0], b[0]);
#pragma unroll
        for (int i = 1; i < 8; i++) r[i] = subc_cc(a[i], b[i]);
        return subc(0u, 0u) & 1u;
    }

    // x in [0, 2k) -> [0, k) for k = m (K2 = false) or k = 2m (K2 = true)
    template <bool K2>
    ZK_DI static void fold(u32 *x) {
        u32 t[8];
        if (K2) {
            t[0] = sub_cc(x[0], P::m2(0));
#pragma unroll
            for (int i = 1; i < 8; i++) t[i] = subc_cc(x[i], P::m2(i));
        } else {
            t[0] = sub_cc(x[0], P::m(0));
#pragma unroll
            for (int i = 1; i < 8; i++) t[i] = subc_cc(x[i], P::m(i));
        }
        u32 borrow = subc(0u, 0u);
        bool keep = borrow != 0;
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = keep ? x[i] : t[i];
    }

    // [0, 2m) -> [0, m)
    ZK_DI Fp canonical() const {
        Fp r = *this;
        fold<false>(r.v);
        return r;
    }

    // lazy add: a, b < 2m -> (a + b) mod 2m in [0, 2m)
    ZK_DI static Fp add(const Fp &a, const Fp &b) {
        Fp r;
        r.v[0] = add_cc(a.v[0], b.v[0]);
#pragma unroll
        for (int i = 1; i < 8; i++) r.v[i] = addc_cc(a.v[i], b.v[i]);
        fold<true>(r.v);  // a + b < 4m < 2^256, no carry out
        return r;
    }

    // lazy sub: a, b < 2m -> (a - b) mod 2m in [0, 2m)
    ZK_DI static Fp sub(const Fp &a, const Fp &b) {
        Fp r;
        u32 borrow = sub_raw(r.v, a.v, b.v);
        u32 mask = 0u - borrow;
        r.v[0] = add_cc(r.v[0], P::m2(0) & mask);
#pragma unroll
        for (int i = 1; i < 8; i++) r.v[i] = addc_cc(r.v[i], P::m2(i) & mask);
        return r;
    }

    // canonical add / sub: inputs < m, outputs < m
    ZK_DI static Fp add_c(const Fp &a, const Fp &b) {
        Fp r;
        r.v[0] = add_cc(a.v[0], b.v[0]);
#pragma unroll
        for (int i = 1; i < 8; i++) r.v[i] = addc_cc(a.v[i], b.v[i]);
        fold<false>(r.v);
        return r;
    }
    ZK_DI static Fp sub_c(const Fp &a, const Fp &b) {
        Fp r;
        u32 borrow = sub_raw(r.v, a.v, b.v);
        u32 mask = 0u - borrow;
        r.v[0] = add_cc(r.v[0], P::m(0) & mask);
#pragma unroll
        for (int i = 1; i < 8; i++) r.v[i] = addc_cc(r.v[i], P::m(i) & mask);
        return r;
    }

    // lazy negation: a < 2m -> 2m - a, mapped so that 0 stays 0 (result in [0, 2m))
    ZK_DI static Fp neg(const Fp &a) {
        Fp r;
        u32 m2[8];
#pragma unroll
        for (int i = 0; i < 8; i++) m2[i] = P::m2(i);
        sub_raw(r.v, m2, a.v);
        bool z = a.is_zero();
#pragma unroll
        for (int i = 0; i < 8; i++) r.v[i] = z ? 0u : r.v[i];
        return r;
    }

    // doubling (lazy)
    ZK_DI static Fp dbl(const Fp &a) { return add(a, a); }

    // CIOS Montgomery product: a, b < 2m -> a * b / R mod m in [0, 2m).  Every 32x32 multiply
    // is emitted as a (low, high) pair on adjacent words: per row, the products of the even
    // limbs a[0], a[2], a[4], a[6] form one carry chain over t[0..7] (their word pairs do not
    // overlap) and the odd limbs a second chain over t[1..8]; the reduction row q * m is split
    // the same way.  Emitting the pairs together runs 28 % faster on B200 than one chain of
    // low halves followed by one chain of high halves per row (57.0 vs 44.6 G products/s,
    // bit-identical results).  Bounds: with a, b < 2m < 2^255 the running sum stays below
    // 2^288 (nine words) inside a row and below 2^256 after each shift.
    ZK_DI static Fp mul(const Fp &a, const Fp &b) {
        u32 t[9];
        {
            const u32 bi = b.v[0];
#pragma unroll
            for (int j = 0; j < 8; j += 2) {
                t[j] = a.v[j] * bi;
                t[j + 1] = __umulhi(a.v[j], bi);
            }
            t[8] = 0;
            t[1] = mad_lo_cc(a.v[1], bi, t[1]);
            t[2] = madc_hi_cc(a.v[1], bi, t[2]);
            t[3] = madc_lo_cc(a.v[3], bi, t[3]);
            t[4] = madc_hi_cc(a.v[3], bi, t[4]);
            t[5] = madc_lo_cc(a.v[5], bi, t[5]);
            t[6] = madc_hi_cc(a.v[5], bi, t[6]);
            t[7] = madc_lo_cc(a.v[7], bi, t[7]);
            t[8] = madc_hi(a.v[7], bi, t[8]);
            reduce_row(t);
        }
#pragma unroll
        for (int i = 1; i < 8; i++) {
            const u32 bi = b.v[i];
            t[0] = mad_lo_cc(a.v[0], bi, t[0]);
            t[1] = madc_hi_cc(a.v[0], bi, t[1]);
            t[2] = madc_lo_cc(a.v[2], bi, t[2]);
            t[3] = madc_hi_cc(a.v[2], bi, t[3]);
            t[4] = madc_lo_cc(a.v[4], bi, t[4]);
            t[5] = madc_hi_cc(a.v[4], bi, t[5]);
            t[6] = madc_lo_cc(a.v[6], bi, t[6]);
            t[7] = madc_hi_cc(a.v[6], bi, t[7]);
            t[8] = addc(t[8], 0u);
            t[1] = mad_lo_cc(a.v[1], bi, t[1]);
            t[2] = madc_hi_cc(a.v[1], bi, t[2]);
            t[3] = madc_lo_cc(a.v[3], bi, t[3]);
            t[4] = madc_hi_cc(a.v[3], bi, t[4]);
            t[5] = madc_lo_cc(a.v[5], bi, t[5]);
            t[6] = madc_hi_cc(a.v[5], bi, t[6]);
            t[7] = madc_lo_cc(a.v[7], bi, t[7]);
            t[8] = madc_hi(a.v[7], bi, t[8]);
            reduce_row(t);
        }
        Fp r;
#pragma unroll
        for (int i = 0; i < 8; i++) r.v[i] = t[i];
        return r;
    }

    // one reduction row: t += q * m with q = t[0] * m' (the low word becomes zero), then
    // t >>= 32.  The even limbs of m pair up over t[0..7] (the low word of q * m[0] is never
    // formed: its carry is t[0] != 0), the odd limbs over t[1..8].
    ZK_DI static void reduce_row(u32 *t) {
        const u32 q = t[0] * P::MPRIME;
        add_cc(t[0], 0xffffffffu);
        t[1] = madc_hi_cc(q, P::m(0), t[1]);
        t[2] = madc_lo_cc(q, P::m(2), t[2]);
        t[3] = madc_hi_cc(q, P::m(2), t[3]);
        t[4] = madc_lo_cc(q, P::m(4), t[4]);
        t[5] = madc_hi_cc(q, P::m(4), t[5]);
        t[6] = madc_lo_cc(q, P::m(6), t[6]);
        t[7] = madc_hi_cc(q, P::m(6), t[7]);
        t[8] = addc(t[8], 0u);
        t[1] = mad_lo_cc(q, P::m(1), t[1]);
        t[2] = madc_hi_cc(q, P::m(1), t[2]);
        t[3] = madc_lo_cc(q, P::m(3), t[3]);
        t[4] = madc_hi_cc(q, P::m(3), t[4]);
        t[5] = madc_lo_cc(q, P::m(5), t[5]);
        t[6] = madc_hi_cc(q, P::m(5), t[6]);
        t[7] = madc_lo_cc(q, P::m(7), t[7]);
        t[8] = madc_hi(q, P::m(7), t[8]);
#pragma unroll
        for (int j = 0; j < 8; j++) t[j] = t[j + 1];
        t[8] = 0;
    }

    // ---- product by a fixed factor (Shoup's method with a truncated quotient estimate)
    // For a factor w < m with ws = floor(w * 2^256 / m) precomputed: q = floor(a * ws / 2^256)
    // is estimated from the partial products that land in columns 7 and up of a * ws (the
    // dropped ones sum to less than 14 * 2^224, so the estimate is q or q - 1); then
    // r = a * w - q * m = a * w + q * (2^256 - m) mod 2^256 lies in [0, 3m), and one
    // conditional subtraction of 2m leaves [0, 2m).  Any 256-bit a is accepted.  With a in
    // Montgomery form (a = x R) and w a plain value, r is the Montgomery form of x * w: the
    // value mul(a, w R) gives, from 207 multiply instructions instead of 256.
    //
    // mul_shoup_table_entry turns a Montgomery-form factor wR into the pair (w, ws):
    // w = REDC(wR), and ws = (w * 2^256 - wR) / m exactly, i.e. ws = wR * (-m^-1) mod 2^256.

    // row i of the truncated high product: the terms a_i * ws_j with i + j = par (mod 2) that
    // land in column 7 or above (h[k] holds column 7 + k); keep_carry leaves the carry of the
    // last term in the flag for the caller
    ZK_DI static void shoup_high_chain(u32 *h, u32 ai, const u32 *ws, int i, int par, bool keep_carry) {
        bool first = true;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (((i + j) & 1) != par) continue;
            const int c = i + j;  // column of the low half
            const bool last = j + 2 > 7;
            if (c >= 7) {
                h[c - 7] = first ? mad_lo_cc(ai, ws[j], h[c - 7]) : madc_lo_cc(ai, ws[j], h[c - 7]);
                first = false;
            }
            if (c >= 6) {
                if (first) h[c - 6] = mad_hi_cc(ai, ws[j], h[c - 6]);
                else if (last && !keep_carry) h[c - 6] = madc_hi(ai, ws[j], h[c - 6]);
                else h[c - 6] = madc_hi_cc(ai, ws[j], h[c - 6]);
                first = false;
            }
        }
    }
    // row i of a low product mod 2^256: the terms a_i * b_j with j = par (mod 2) in columns 0..7
    ZK_DI static void shoup_low_chain(u32 *t, u32 ai, const u32 *b, int i, int par) {
        bool first = true;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if ((j & 1) != par) continue;
            const int c = i + j;
            if (c <= 7) {
                t[c] = first ? mad_lo_cc(ai, b[j], t[c]) : madc_lo_cc(ai, b[j], t[c]);
                first = false;
            }
            if (c + 1 <= 7) t[c + 1] = madc_hi_cc(ai, b[j], t[c + 1]);
        }
    }
    template <class Q = P>
    ZK_DI static Fp mul_shoup(const Fp &a, const Fp &w, const Fp &ws) {
        u32 h[9];
#pragma unroll
        for (int k = 0; k < 9; k++) h[k] = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            // the chain of parity i ends at column i + 7, the other at i + 8 (the row's top)
            shoup_high_chain(h, a.v[i], ws.v, i, i & 1, true);
            h[i + 1] = addc(h[i + 1], 0u);
            shoup_high_chain(h, a.v[i], ws.v, i, (i + 1) & 1, false);
        }
        // q = h[1..8]; r = a * w + q * (2^256 - m) mod 2^256
        u32 t[8], npv[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            t[k] = 0;
            npv[k] = Q::np(k);
        }
#pragma unroll
        for (int i = 0; i < 8; i++) {
            shoup_low_chain(t, a.v[i], w.v, i, 0);
            shoup_low_chain(t, a.v[i], w.v, i, 1);
        }
#pragma unroll
        for (int i = 0; i < 8; i++) {
            shoup_low_chain(t, h[i + 1], npv, i, 0);
            shoup_low_chain(t, h[i + 1], npv, i, 1);
        }
        Fp r;
#pragma unroll
        for (int k = 0; k < 8; k++) r.v[k] = t[k];
        fold<true>(r.v);
        return r;
    }
    // (w, ws) for the Montgomery-form factor wr (any value below 2m)
    template <class Q = P>
    ZK_DI static void mul_shoup_table_entry(const Fp &wr, Fp *w, Fp *ws) {
        Fp c = wr.canonical();
        u32 one[8];
#pragma unroll
        for (int k = 0; k < 8; k++) one[k] = k == 0 ? 1u : 0u;
        *w = mul(c, from_words(one)).canonical();
        u32 t[8], mi[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            t[k] = 0;
            mi[k] = Q::minv(k);
        }
#pragma unroll
        for (int i = 0; i < 8; i++) {
            shoup_low_chain(t, c.v[i], mi, i, 0);
            shoup_low_chain(t, c.v[i], mi, i, 1);
        }
#pragma unroll
        for (int k = 0; k < 8; k++) ws->v[k] = t[k];
    }

    // Montgomery square.  The product routine with both operands equal: on B200 it runs faster
    // (58.6 G/s) than a schoolbook square that forms the 28 off-diagonal products once
    // (52.6 G/s, one low chain and one high chain per row); the results are identical.
    ZK_DI static Fp sqr(const Fp &a) { return mul(a, a); }

    // x in [0, 2m) is 0 mod m exactly when x == 0 or x == m
    ZK_DI bool is_zero_mod() const {
        u32 z = 0, e = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            z |= v[i];
            e |= v[i] ^ P::m(i);
        }
        return z == 0 || e == 0;
    }

    // exponentiation by a 64-bit exponent (Element::pow with a small exponent)
    ZK_DI static Fp pow_u64(const Fp &a, u64 e) {
        Fp r = one();
        Fp base = a;
        while (e) {
            if (e & 1) r = mul(r, base);
            base = mul(base, base);
            e >>= 1;
        }
        return r;
    }

    // inverse by Fermat: a^(m-2) (Element::invert, field.cuh:1172-1175)
    ZK_DI static Fp inv(const Fp &a) {
        Fp r = one();
#pragma unroll 1
        for (int w = 7; w >= 0; w--) {
            const u32 e = (w == 0) ? (P::m(0) - 2u) : P::m(w);
#pragma unroll 1
            for (int b = 31; b >= 0; b--) {
                r = mul(r, r);
                if ((e >> b) & 1u) r = mul(r, a);
            }
        }
        return r;
    }

    // Montgomery form <-> integer
    ZK_DI static Fp to_mont(const Fp &x) {
        Fp r2;
#pragma unroll
        for (int i = 0; i < 8; i++) r2.v[i] = P::r2(i);
        return mul(x, r2).canonical();
    }
    ZK_DI Fp to_number() const {
        Fp o = zero();
        o.v[0] = 1;
        return mul(*this, o).canonical();
    }
};

using Fr = Fp<FrParams>;
using Fq = Fp<FqParams>;

}  // namespace zk
