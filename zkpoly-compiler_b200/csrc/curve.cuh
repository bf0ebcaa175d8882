// BN254 G1 (y^2 = x^3 + 3 over Fq) in XYZZ and affine coordinates, device side.
//
// Formulas are the EFD XYZZ ones the reference uses (core/src/common/curve/src/
// curve_xyzz.cuh:252-391): madd-2008-s, add-2008-s, dbl-2008-s-1 and mdbl-2008-s-1.  Affine
// points are (x, y) Montgomery Fq with (0, 0) the identity (PointAffine::is_identity tests
// y == 0); an XYZZ point is the identity when zz == 0.
//
// Coordinates are lazy ([0, 2q)), so every "is zero" decision is a test for 0 or q.
#pragma once
#include "field.cuh"

namespace zk {

// The curve formulas reach the Fq product and square through fmul / fsqr.  By default they are
// inlined.  With ZK_CURVE_OUTLINE_MUL both call one out-of-line product, which keeps a loop of
// additions inside the instruction cache at the price of a call (and register traffic) per
// product.  On B200 the out-of-line form was 11 % faster for the 2^22 MSM while the product
// ran one low chain and one high chain per row; with the paired product the inlined form is
// faster (15.7 vs 17.9 ms, same results).
#ifdef ZK_CURVE_OUTLINE_MUL
static __device__ __noinline__ Fq fq_mul_call(const Fq a, const Fq b) { return Fq::mul(a, b); }
ZK_DI Fq fmul(const Fq &a, const Fq &b) { return fq_mul_call(a, b); }
ZK_DI Fq fsqr(const Fq &a) { return fq_mul_call(a, a); }
#else
ZK_DI Fq fmul(const Fq &a, const Fq &b) { return Fq::mul(a, b); }
ZK_DI Fq fsqr(const Fq &a) { return Fq::sqr(a); }
#endif

struct G1A {
    Fq x, y;

    ZK_DI static G1A load(const u32 *p) {
        G1A r;
        r.x = Fq::load(p);
        r.y = Fq::load(p + 8);
        return r;
    }
    ZK_DI static G1A load_nc(const u32 *p) {
        G1A r;
        r.x = Fq::load_nc(p);
        r.y = Fq::load_nc(p + 8);
        return r;
    }
    ZK_DI void store(u32 *p) const {
        x.store(p);
        y.store(p + 8);
    }
    ZK_DI bool is_identity() const { return y.is_zero_mod(); }
    ZK_DI G1A neg() const {
        G1A r;
        r.x = x;
        r.y = Fq::neg(y);
        return r;
    }
};

struct G1X {
    Fq x, y, zz, zzz;

    ZK_DI static G1X identity() {
        G1X r;
        r.x = Fq::zero();
        r.y = Fq::zero();
        r.zz = Fq::zero();
        r.zzz = Fq::zero();
        return r;
    }
    ZK_DI static G1X from_affine(const G1A &a) {
        if (a.is_identity()) return identity();
        G1X r;
        r.x = a.x;
        r.y = a.y;
        r.zz = Fq::one();
        r.zzz = Fq::one();
        return r;
    }
    ZK_DI bool is_identity() const { return zz.is_zero_mod(); }

    ZK_DI static G1X load(const u32 *p) {
        G1X r;
        r.x = Fq::load(p);
        r.y = Fq::load(p + 8);
        r.zz = Fq::load(p + 16);
        r.zzz = Fq::load(p + 24);
        return r;
    }
    ZK_DI void store(u32 *p) const {
        x.store(p);
        y.store(p + 8);
        zz.store(p + 16);
        zzz.store(p + 24);
    }
    ZK_DI G1X neg() const {
        G1X r = *this;
        r.y = Fq::neg(y);
        return r;
    }
};

// mdbl-2008-s-1: 2 * (x, y) for an affine point (curve_xyzz.cuh:229-241)
ZK_DI G1X g1_dbl_affine(const G1A &p) {
    Fq u = Fq::dbl(p.y);
    Fq v = fsqr(u);
    Fq w = fmul(u, v);
    Fq s = fmul(p.x, v);
    Fq x2 = fsqr(p.x);
    Fq m = Fq::add(Fq::dbl(x2), x2);
    G1X r;
    r.x = Fq::sub(Fq::sub(fsqr(m), s), s);
    r.y = Fq::sub(fmul(m, Fq::sub(s, r.x)), fmul(w, p.y));
    r.zz = v;
    r.zzz = w;
    return r;
}

// dbl-2008-s-1 (curve_xyzz.cuh:377-391)
ZK_DI G1X g1_dbl(const G1X &p) {
    if (p.is_identity()) return p;
    Fq u = Fq::dbl(p.y);
    Fq v = fsqr(u);
    Fq w = fmul(u, v);
    Fq s = fmul(p.x, v);
    Fq x2 = fsqr(p.x);
    Fq m = Fq::add(Fq::dbl(x2), x2);
    G1X r;
    r.x = Fq::sub(Fq::sub(fsqr(m), s), s);
    r.y = Fq::sub(fmul(m, Fq::sub(s, r.x)), fmul(w, p.y));
    r.zz = fmul(v, p.zz);
    r.zzz = fmul(w, p.zzz);
    return r;
}

// madd-2008-s: XYZZ + affine (curve_xyzz.cuh:352-370)
ZK_DI G1X g1_madd(const G1X &a, const G1A &b) {
    if (b.is_identity()) return a;
    if (a.is_identity()) return G1X::from_affine(b);
    Fq u2 = fmul(b.x, a.zz);
    Fq s2 = fmul(b.y, a.zzz);
    Fq p = Fq::sub(u2, a.x);
    Fq r = Fq::sub(s2, a.y);
    if (p.is_zero_mod() && r.is_zero_mod()) return g1_dbl_affine(b);
    Fq pp = fsqr(p);
    Fq ppp = fmul(p, pp);
    Fq q = fmul(a.x, pp);
    G1X o;
    o.x = Fq::sub(Fq::sub(Fq::sub(fsqr(r), ppp), q), q);
    o.y = Fq::sub(fmul(r, Fq::sub(q, o.x)), fmul(a.y, ppp));
    o.zz = fmul(a.zz, pp);
    o.zzz = fmul(a.zzz, ppp);
    return o;
}

// add-2008-s: XYZZ + XYZZ (curve_xyzz.cuh:325-345)
ZK_DI G1X g1_add(const G1X &a, const G1X &b) {
    if (a.is_identity()) return b;
    if (b.is_identity()) return a;
    Fq u1 = fmul(a.x, b.zz);
    Fq u2 = fmul(b.x, a.zz);
    Fq s1 = fmul(a.y, b.zzz);
    Fq s2 = fmul(b.y, a.zzz);
    Fq p = Fq::sub(u2, u1);
    Fq r = Fq::sub(s2, s1);
    if (p.is_zero_mod() && r.is_zero_mod()) return g1_dbl(a);
    Fq pp = fsqr(p);
    Fq ppp = fmul(p, pp);
    Fq q = fmul(u1, pp);
    G1X o;
    o.x = Fq::sub(Fq::sub(Fq::sub(fsqr(r), ppp), q), q);
    o.y = Fq::sub(fmul(r, Fq::sub(q, o.x)), fmul(s1, ppp));
    o.zz = fmul(fmul(a.zz, b.zz), pp);
    o.zzz = fmul(fmul(a.zzz, b.zzz), ppp);
    return o;
}

// ------------------------------------------------------------------ warp-parallel forms
// For a serial chain of point operations on one point (the window combination of an MSM
// without precomputed tables: about 240 doublings), one thread pays every Fq product's full
// latency in turn.  These forms run the same formulas with every lane of a warp holding the
// same point: the products of one dependency level (at most four) are computed at once, one
// per lane, and broadcast with shuffles.  A doubling then costs three product latencies
// instead of nine, an addition four instead of fourteen; the values are the serial forms'.
ZK_DI Fq lane_pick(u32 lane, const Fq &a0, const Fq &a1, const Fq &a2, const Fq &a3) {
    Fq r;
#pragma unroll
    for (int w = 0; w < 8; w++) r.v[w] = lane == 1 ? a1.v[w] : lane == 2 ? a2.v[w] : lane == 3 ? a3.v[w] : a0.v[w];
    return r;
}
ZK_DI Fq lane_bcast(const Fq &x, int src) {
    Fq r;
#pragma unroll
    for (int w = 0; w < 8; w++) r.v[w] = __shfl_sync(0xffffffffu, x.v[w], src);
    return r;
}

// dbl-2008-s-1 with its nine products in three levels; every lane of the warp passes the same p
ZK_DI G1X g1_dbl_warp(const G1X &p) {
    if (p.is_identity()) return p;
    const u32 lane = threadIdx.x & 31;
    const Fq u = Fq::dbl(p.y);
    // level 1: v = u^2, x2 = x^2
    Fq t = fmul(lane_pick(lane, u, p.x, u, p.x), lane_pick(lane, u, p.x, u, p.x));
    const Fq v = lane_bcast(t, 0), x2 = lane_bcast(t, 1);
    const Fq m = Fq::add(Fq::dbl(x2), x2);
    // level 2: w = u v, s = x v, m^2, zz v
    t = fmul(lane_pick(lane, u, p.x, m, v), lane_pick(lane, v, v, m, p.zz));
    const Fq w = lane_bcast(t, 0), sv = lane_bcast(t, 1), m2 = lane_bcast(t, 2);
    G1X r;
    r.zz = lane_bcast(t, 3);
    r.x = Fq::sub(Fq::sub(m2, sv), sv);
    // level 3: m (s - x3), w y, w zzz
    t = fmul(lane_pick(lane, m, w, w, w), lane_pick(lane, Fq::sub(sv, r.x), p.y, p.zzz, p.zzz));
    r.y = Fq::sub(lane_bcast(t, 0), lane_bcast(t, 1));
    r.zzz = lane_bcast(t, 2);
    return r;
}

// add-2008-s with its fourteen products in four levels; every lane passes the same a and b
ZK_DI G1X g1_add_warp(const G1X &a, const G1X &b) {
    if (a.is_identity()) return b;
    if (b.is_identity()) return a;
    const u32 lane = threadIdx.x & 31;
    // level 1: u1 = x_a zz_b, u2 = x_b zz_a, s1 = y_a zzz_b, s2 = y_b zzz_a
    Fq t = fmul(lane_pick(lane, a.x, b.x, a.y, b.y), lane_pick(lane, b.zz, a.zz, b.zzz, a.zzz));
    const Fq u1 = lane_bcast(t, 0), u2 = lane_bcast(t, 1), s1 = lane_bcast(t, 2), s2 = lane_bcast(t, 3);
    const Fq p = Fq::sub(u2, u1);
    const Fq r = Fq::sub(s2, s1);
    if (p.is_zero_mod() && r.is_zero_mod()) return g1_dbl_warp(a);
    // level 2: pp = p^2, r^2, zz_a zz_b, zzz_a zzz_b
    t = fmul(lane_pick(lane, p, r, a.zz, a.zzz), lane_pick(lane, p, r, b.zz, b.zzz));
    const Fq pp = lane_bcast(t, 0), r2 = lane_bcast(t, 1), zzab = lane_bcast(t, 2), zzzab = lane_bcast(t, 3);
    // level 3: ppp = p pp, q = u1 pp, zz = zz_a zz_b pp
    t = fmul(lane_pick(lane, p, u1, zzab, zzab), lane_pick(lane, pp, pp, pp, pp));
    const Fq ppp = lane_bcast(t, 0), q = lane_bcast(t, 1);
    G1X o;
    o.zz = lane_bcast(t, 2);
    o.x = Fq::sub(Fq::sub(Fq::sub(r2, ppp), q), q);
    // level 4: r (q - x3), s1 ppp, zzz_a zzz_b ppp
    t = fmul(lane_pick(lane, r, s1, zzzab, zzzab), lane_pick(lane, Fq::sub(q, o.x), ppp, ppp, ppp));
    o.y = Fq::sub(lane_bcast(t, 0), lane_bcast(t, 1));
    o.zzz = lane_bcast(t, 2);
    return o;
}

// k * p by double-and-add over the bits of a 64-bit k
ZK_DI G1X g1_mul_u64(const G1X &p, u64 k) {
    G1X acc = G1X::identity();
    if (k == 0) return acc;
    int top = 63 - __clzll(k);
    acc = p;
    for (int i = top - 1; i >= 0; i--) {
        acc = g1_dbl(acc);
        if ((k >> i) & 1) acc = g1_add(acc, p);
    }
    return acc;
}

// ------------------------------------------------------------------ inversion
// Binary extended GCD with batched steps (T. Pornin, "Optimized Binary GCD for Modular
// Inversion", IACR ePrint 2020/972, algorithm 2 with k - 1 = 30).  With a = y, b = m, u = 1,
// v = 0 and t steps taken, a 2^t = y u and b 2^t = y v (mod m).  A step halves a when it is
// even; otherwise it swaps (a, b), (u, v) when a < b and replaces a by (a - b) / 2, u by u - v;
// every step doubles v.  Each of 17 outer iterations takes 30 steps on 62-bit approximations of
// a and b (their low 30 bits below their top 32 bits, at a common bit length n >= 62), collects
// them in signed factors f0, g0, f1, g1 (|f| + |g| <= 2^30 per row), then applies them to the
// full values: a <- (a f0 + b g0) / 2^30, b <- (a f1 + b g1) / 2^30 (exact; a negative result is
// negated with its row), and u, v by one Montgomery step each, (u f + v g) 2^-32 mod m.  After
// 510 steps a = 0 and b = gcd = 1, so y^-1 = v 2^(32 * 17 - 510) = v 2^34.  The iteration counts
// are fixed and every step is a select, so the threads of a warp never diverge.
ZK_DI void mul_small9(const u32 *x, u32 c, u32 *r) {
    u64 carry = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const u64 t = (u64)x[i] * c + carry;
        r[i] = (u32)t;
        carry = t >> 32;
    }
    r[8] = (u32)carry;
}
ZK_DI void neg9_if(u32 *r, bool neg) {
    const u32 mask = neg ? 0xffffffffu : 0u;
    u64 c = neg ? 1u : 0u;
#pragma unroll
    for (int i = 0; i < 9; i++) {
        const u64 t = (u64)(r[i] ^ mask) + c;
        r[i] = (u32)t;
        c = t >> 32;
    }
}
// |x f + y g| / 2^30 into out (x, y < 2^255, |f| + |g| <= 2^30, the sum divisible by 2^30);
// returns whether x f + y g is negative
ZK_DI bool lin_shift30(const u32 *x, int f, const u32 *y, int g, u32 *out) {
    u32 p[9], q[9], s[9];
    mul_small9(x, (u32)(f < 0 ? -f : f), p);
    neg9_if(p, f < 0);
    mul_small9(y, (u32)(g < 0 ? -g : g), q);
    neg9_if(q, g < 0);
    u64 c = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) {
        const u64 t = (u64)p[i] + q[i] + c;
        s[i] = (u32)t;
        c = t >> 32;
    }
    const bool neg = (s[8] >> 31) != 0;
    neg9_if(s, neg);
#pragma unroll
    for (int i = 0; i < 8; i++) out[i] = (s[i] >> 30) | (s[i + 1] << 2);
    return neg;
}
// (u f + v g) 2^-32 mod m into out, for u, v < m and |f| + |g| <= 2^30
template <class P>
ZK_DI void coef_step(const u32 *u, int f, const u32 *v, int g, u32 *out) {
    u32 uu[8], vv[8], p[9], q[9], x[9];
    // a negative factor multiplies m - u instead (m when u = 0, still within the bound)
    {
        u32 bu = 0, bv = 0;
        const u32 mu = f < 0 ? 0xffffffffu : 0u, mv = g < 0 ? 0xffffffffu : 0u;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const u64 tu = (u64)P::m(i) - u[i] - bu;
            const u64 tv = (u64)P::m(i) - v[i] - bv;
            bu = (u32)(tu >> 32) & 1u;
            bv = (u32)(tv >> 32) & 1u;
            uu[i] = ((u32)tu & mu) | (u[i] & ~mu);
            vv[i] = ((u32)tv & mv) | (v[i] & ~mv);
        }
    }
    mul_small9(uu, (u32)(f < 0 ? -f : f), p);
    mul_small9(vv, (u32)(g < 0 ? -g : g), q);
    u64 c = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) {
        const u64 t = (u64)p[i] + q[i] + c;
        x[i] = (u32)t;
        c = t >> 32;
    }
    // x < m 2^30; (x + k m) / 2^32 < 2m with k = x * (-m^-1) mod 2^32
    const u32 k = x[0] * P::MPRIME;
    c = ((u64)P::m(0) * k + x[0]) >> 32;
#pragma unroll
    for (int i = 1; i < 8; i++) {
        const u64 t = (u64)P::m(i) * k + x[i] + c;
        out[i - 1] = (u32)t;
        c = t >> 32;
    }
    out[7] = (u32)((u64)x[8] + c);
    // conditional subtraction of m
    u32 d[8], br = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const u64 t = (u64)out[i] - P::m(i) - br;
        d[i] = (u32)t;
        br = (u32)(t >> 32) & 1u;
    }
#pragma unroll
    for (int i = 0; i < 8; i++) out[i] = br ? out[i] : d[i];
}
// bits [s, s + 32) of the 256-bit x (s < 256), with x's limbs picked by selects, not indexing
ZK_DI u32 bits32_at(const u32 *x, u32 s) {
    const u32 w = s >> 5, sh = s & 31;
    u32 lo = 0, hi = 0;
#pragma unroll
    for (u32 i = 0; i < 8; i++) {
        lo = i == w ? x[i] : lo;
        hi = i == w + 1 ? x[i] : hi;
    }
    return __funnelshift_r(lo, hi, sh);
}

// Input a = x R mod m (Montgomery form, x != 0); returns x^-1 R mod m (0 for 0).
template <class P>
ZK_DI Fp<P> inv_binary(const Fp<P> &a_mont) {
    using F = Fp<P>;
    const F y = a_mont.canonical();
    if (y.is_zero()) return F::zero();
    u32 a[8], b[8], u[8], v[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        a[i] = y.v[i];
        b[i] = P::m(i);
        u[i] = 0;
        v[i] = 0;
    }
    u[0] = 1;
    for (int it = 0; it < 17; it++) {
        // common length n = max(len a, len b, 62)
        u32 n = 62;
#pragma unroll
        for (u32 i = 0; i < 8; i++) {
            const u32 o = a[i] | b[i];
            const u32 len = o ? 32 * i + 32 - __clz(o) : 0u;
            n = len > n ? len : n;
        }
        u64 ab = ((u64)bits32_at(a, n - 32) << 30) | (a[0] & 0x3fffffffu);
        u64 bb = ((u64)bits32_at(b, n - 32) << 30) | (b[0] & 0x3fffffffu);
        int f0 = 1, g0 = 0, f1 = 0, g1 = 1;
#pragma unroll 10
        for (int j = 0; j < 30; j++) {
            const bool odd = (ab & 1u) != 0;
            const bool sw = odd && ab < bb;
            const u64 ta = sw ? bb : ab, tb = sw ? ab : bb;
            const int tf0 = sw ? f1 : f0, tg0 = sw ? g1 : g0, tf1 = sw ? f0 : f1, tg1 = sw ? g0 : g1;
            ab = (odd ? ta - tb : ta) >> 1;
            bb = tb;
            f0 = odd ? tf0 - tf1 : tf0;
            g0 = odd ? tg0 - tg1 : tg0;
            f1 = tf1 * 2;
            g1 = tg1 * 2;
        }
        u32 na[8], nb[8], nu[8], nv[8];
        if (lin_shift30(a, f0, b, g0, na)) {
            f0 = -f0;
            g0 = -g0;
        }
        if (lin_shift30(a, f1, b, g1, nb)) {
            f1 = -f1;
            g1 = -g1;
        }
        coef_step<P>(u, f0, v, g0, nu);
        coef_step<P>(u, f1, v, g1, nv);
#pragma unroll
        for (int i = 0; i < 8; i++) {
            a[i] = na[i];
            b[i] = nb[i];
            u[i] = nu[i];
            v[i] = nv[i];
        }
    }
    // v = y^-1 2^-34, and x^-1 R = y^-1 R^2 = Montgomery product of v and 2^34 R^3
    F k;
#pragma unroll
    for (int i = 0; i < 8; i++) k.v[i] = P::invk(i);
    return F::mul(F::from_words(v), k).canonical();
}

// XYZZ -> affine (scaling-z, curve_xyzz.cuh:316-322); identity -> (0, 0)
ZK_DI G1A g1_to_affine(const G1X &p) {
    G1A r;
    if (p.is_identity()) {
        r.x = Fq::zero();
        r.y = Fq::zero();
        return r;
    }
    Fq a = inv_binary<FqParams>(p.zzz);
    Fq b = fsqr(fmul(p.zz, a));
    r.x = fmul(p.x, b).canonical();
    r.y = fmul(p.y, a).canonical();
    return r;
}

}  // namespace zk
