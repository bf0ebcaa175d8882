"""Cross-check of the oracle restatement (and of this library's host-side gen_pq_omegas)
against the reference's own host arithmetic, compiled from its headers into oracle/_ref
(CPU only).  Skipped where oracle/_ref was not built (no reference checkout)."""
import ctypes
import os

import numpy as np
import pytest

from conftest import ROOT

REF = os.path.join(ROOT, "oracle", "_ref", "libref.so")
pytestmark = pytest.mark.skipif(not os.path.exists(REF), reason="oracle/_ref not built (no reference checkout)")

FR_M = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
FQ_M = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47


@pytest.fixture(scope="module")
def ref():
    return ctypes.CDLL(REF)


def w32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint64).view(np.uint32))


def call(fn, *args, out_words=8):
    out = np.zeros(out_words, dtype=np.uint32)
    fn(out.ctypes.data, *[a.ctypes.data if isinstance(a, np.ndarray) else a for a in args])
    return out.view(np.uint64)


def rand_elems(orc, m, n, seed):
    rng = np.random.default_rng(seed)
    return [orc.int_to_limbs(int.from_bytes(rng.bytes(32), "little") % m) for _ in range(n)]


def test_field_ops_match_reference(orc, ref):
    xs = rand_elems(orc, FR_M, 120, 1)
    ys = rand_elems(orc, FR_M, 120, 2)
    for a, b in zip(xs, ys):
        A, B = w32(a), w32(b)
        assert np.array_equal(call(ref.ref_fr_mul, A, B), orc.mul(a, b))
        assert np.array_equal(call(ref.ref_fr_add, A, B), orc.add(a, b))
        assert np.array_equal(call(ref.ref_fr_sub, A, B), orc.sub(a, b))
        assert np.array_equal(call(ref.ref_fr_neg, A), orc.neg(a))
        assert np.array_equal(call(ref.ref_fr_from_number, A), orc.to_mont(a))
        assert np.array_equal(call(ref.ref_fr_to_number, A), orc.from_mont(a))
    for a in xs[:10]:
        assert np.array_equal(call(ref.ref_fr_inv, w32(a)), orc.inv(a))
        e = orc.limbs_to_int(a)
        assert np.array_equal(call(ref.ref_fr_pow, w32(a), w32(orc.int_to_limbs(e))), orc.pow_(a, e))
    qs = rand_elems(orc, FQ_M, 60, 3)
    rs = rand_elems(orc, FQ_M, 60, 4)
    for a, b in zip(qs, rs):
        A, B = w32(a), w32(b)
        assert np.array_equal(call(ref.ref_fq_mul, A, B), orc.mul(a, b, orc.FQ))
        assert np.array_equal(call(ref.ref_fq_add, A, B), orc.add(a, b, orc.FQ))
        assert np.array_equal(call(ref.ref_fq_sub, A, B), orc.sub(a, b, orc.FQ))
    for a in qs[:5]:
        assert np.array_equal(call(ref.ref_fq_inv, w32(a)), orc.inv(a, orc.FQ))


def test_curve_ops_match_reference(orc, ref):
    pts = orc.gen_points(55, 40)
    for i in range(0, 40, 2):
        p, q = pts[i], pts[i + 1]
        assert np.array_equal(call(ref.ref_g1_add, w32(p), w32(q), out_words=16), orc.g1_affine_add(p, q))
        assert np.array_equal(call(ref.ref_g1_add, w32(p), w32(p), out_words=16), orc.g1_affine_add(p, p))
    for k in (1, 2, 3, 100, 12345, 0xFFFFFFFF):
        assert np.array_equal(call(ref.ref_g1_mul, w32(pts[0]), ctypes.c_uint(k), out_words=16),
                              orc.g1_scalar_mul_affine(pts[0], k))


@pytest.mark.parametrize("log_len,pq_deg", [(16, 8), (20, 7), (24, 6)])
def test_gen_pq_omegas_matches_reference(zk, orc, ref, log_len, pq_deg):
    """This library's host gen_pq_omegas is byte-identical to the reference's."""
    unit = w32(orc.root_of_unity(log_len))
    pq_len = 1 << pq_deg >> 1
    exp_pq = np.zeros(pq_len * 8, dtype=np.uint32)
    exp_om = np.zeros(32 * 8, dtype=np.uint32)
    ref.ref_gen_pq_omegas(exp_pq.ctypes.data, exp_om.ctypes.data, pq_deg, 1 << log_len, unit.ctypes.data)
    lib = zk.native.load("libntt.so")
    got_pq = np.zeros(pq_len * 8, dtype=np.uint32)
    got_om = np.zeros(32 * 8, dtype=np.uint32)
    u = unit.copy()
    lib.gen_pq_omegas(got_pq.ctypes.data, got_om.ctypes.data, pq_deg, 1 << log_len, u.ctypes.data)
    assert np.array_equal(got_pq, exp_pq)
    assert np.array_equal(got_om, exp_om)
