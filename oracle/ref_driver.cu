// Test infrastructure only: exports the reference's own host-side arithmetic (compiled from the
// reference's headers where they lie) as C functions, so the oracle restatement can be checked
// against the reference itself on random inputs.  Built by oracle/build_ref.py into
// oracle/_ref/libref.so; never part of the product.
#include <cstdint>
#include <cstring>

#include "bn254.cuh"         // core/src/common/curve/src/bn254.cuh (Fr, Fq, G1)
#include "precompute.cuh"    // core/src/ntt/src/precompute.cuh (gen_pq_omegas)

using u32 = uint32_t;
using Fr = bn254_fr::Element;
using Fq = bn254_fq::Element;

extern "C" {
void ref_fr_mul(u32 *r, const u32 *a, const u32 *b) { (Fr::load(a) * Fr::load(b)).store(r); }
void ref_fr_add(u32 *r, const u32 *a, const u32 *b) { (Fr::load(a) + Fr::load(b)).store(r); }
void ref_fr_sub(u32 *r, const u32 *a, const u32 *b) { (Fr::load(a) - Fr::load(b)).store(r); }
void ref_fr_neg(u32 *r, const u32 *a) { Fr::load(a).neg().store(r); }
void ref_fr_inv(u32 *r, const u32 *a) { Fr::load(a).invert().store(r); }
void ref_fr_pow(u32 *r, const u32 *a, const u32 *e) { Fr::load(a).pow(mont::Number<8>::load(e)).store(r); }
void ref_fr_from_number(u32 *r, const u32 *a) { Fr::from_number(mont::Number<8>::load(a)).store(r); }
void ref_fr_to_number(u32 *r, const u32 *a) { Fr::load(a).to_number().store(r); }
void ref_fq_mul(u32 *r, const u32 *a, const u32 *b) { (Fq::load(a) * Fq::load(b)).store(r); }
void ref_fq_add(u32 *r, const u32 *a, const u32 *b) { (Fq::load(a) + Fq::load(b)).store(r); }
void ref_fq_sub(u32 *r, const u32 *a, const u32 *b) { (Fq::load(a) - Fq::load(b)).store(r); }
void ref_fq_inv(u32 *r, const u32 *a) { Fq::load(a).invert().store(r); }

// affine p + q through XYZZ (PointXYZZ + PointAffine, then to_affine)
void ref_g1_add(u32 *r, const u32 *p, const u32 *q) {
    auto a = bn254::PointAffine::load(p).to_point();
    auto s = a + bn254::PointAffine::load(q);
    s.to_affine().store(r);
}
// k * p via PointXYZZ::multiple
void ref_g1_mul(u32 *r, const u32 *p, u32 k) {
    bn254::PointAffine::load(p).to_point().multiple(k).to_affine().store(r);
}
void ref_gen_pq_omegas(u32 *pq, u32 *omegas, u32 pq_deg, u32 len, const u32 *unit) {
    detail::gen_pq_omegas<Fr>(pq, omegas, pq_deg, len, Fr::load(unit));
}
}
