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

// ------------------------------------------------------------------ inversion for the
// latency-critical single-thread tail: binary extended Euclid on plain integers.
// Input a = x R mod q (Montgomery form, x != 0); returns x^-1 R mod q.
ZK_DI void bn_rshift1(u32 *a) {
#pragma unroll
    for (int i = 0; i < 7; i++) a[i] = (a[i] >> 1) | (a[i + 1] << 31);
    a[7] >>= 1;
}
ZK_DI bool bn_is_one(const u32 *a) {
    u32 acc = a[0] ^ 1u;
#pragma unroll
    for (int i = 1; i < 8; i++) acc |= a[i];
    return acc == 0;
}
ZK_DI bool bn_geq(const u32 *a, const u32 *b) {
    for (int i = 7; i >= 0; i--) {
        if (a[i] != b[i]) return a[i] > b[i];
    }
    return true;
}
// (x + q) / 2 or x / 2 modulo q for x < q
template <class P>
ZK_DI void half_mod(u32 *x) {
    if (x[0] & 1u) {
        u32 c;
        x[0] = add_cc(x[0], P::m(0));
#pragma unroll
        for (int i = 1; i < 8; i++) x[i] = addc_cc(x[i], P::m(i));
        c = addc(0u, 0u);
        bn_rshift1(x);
        x[7] |= c << 31;
    } else {
        bn_rshift1(x);
    }
}

template <class P>
ZK_DI Fp<P> inv_binary(const Fp<P> &a_mont) {
    using F = Fp<P>;
    F a = a_mont.canonical();
    if (a.is_zero()) return F::zero();
    u32 u[8], v[8], x1[8], x2[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        u[i] = a.v[i];
        v[i] = P::m(i);
        x1[i] = 0;
        x2[i] = 0;
    }
    x1[0] = 1;
    // invariant: x1 * a == u, x2 * a == v (mod q)
    while (!bn_is_one(u) && !bn_is_one(v)) {
        while ((u[0] & 1u) == 0) {
            bn_rshift1(u);
            half_mod<P>(x1);
        }
        while ((v[0] & 1u) == 0) {
            bn_rshift1(v);
            half_mod<P>(x2);
        }
        if (bn_geq(u, v)) {
            F::sub_raw(u, u, v);
            F t1 = F::from_words(x1), t2 = F::from_words(x2);
            F d = F::sub_c(t1, t2);
#pragma unroll
            for (int i = 0; i < 8; i++) x1[i] = d.v[i];
        } else {
            F::sub_raw(v, v, u);
            F t1 = F::from_words(x1), t2 = F::from_words(x2);
            F d = F::sub_c(t2, t1);
#pragma unroll
            for (int i = 0; i < 8; i++) x2[i] = d.v[i];
        }
    }
    F r = bn_is_one(u) ? F::from_words(x1) : F::from_words(x2);
    // r = (xR)^-1 = x^-1 R^-1.  Each Montgomery product with R^2 multiplies by R:
    // x^-1 R^-1 -> x^-1 -> x^-1 R (the Montgomery form of x^-1)
    F r2;
#pragma unroll
    for (int i = 0; i < 8; i++) r2.v[i] = P::r2(i);
    r = F::mul(r, r2);
    r = F::mul(r, r2);
    return r.canonical();
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
