"""Pins the CPU oracle against the reference's own known-answer vectors and against
independent Python big-integer arithmetic (CPU only; no GPU needed)."""
import numpy as np
import pytest

from conftest import u32_to_int, u32_to_u64

FR_M = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
FQ_M = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
R = 1 << 256


def I(orc, v):
    return orc.int_to_limbs(v)


def test_field_params_match_reference_headers(orc, golden):
    for f, name in ((orc.FR, "fr"), (orc.FQ, "fq")):
        m, r1, r2, minv64 = orc.field_consts(f)
        p = golden["params"][name]
        assert m == u32_to_int(p["m"])
        assert r1 == u32_to_int(p["r_mod"])
        assert r2 == u32_to_int(p["r2_mod"])
        assert 2 * m == u32_to_int(p["mm2"])
        assert m - 2 == u32_to_int(p["m_sub2"])
        # the reference's 32-bit m' is the low word of the 64-bit -m^-1
        assert minv64 & 0xFFFFFFFF == p["m_prime"]
    assert orc.field_consts(orc.FR)[0] == FR_M
    assert orc.field_consts(orc.FQ)[0] == FQ_M


@pytest.mark.parametrize("inst", ["instance1", "instance2"])
def test_mont_known_answers(orc, golden, inst):
    g = golden["fr"]
    a = u32_to_u64(g[f"{inst}.a"])
    b = u32_to_u64(g[f"{inst}.b"])
    ai, bi = u32_to_int(g[f"{inst}.a"]), u32_to_int(g[f"{inst}.b"])
    # Number ops (main.cu bn_add / bn_sub / bn_mul / bn_square / bn_slr)
    assert (ai + bi) % R == u32_to_int(g[f"{inst}.sum"])
    assert (ai - bi) % R == u32_to_int(g[f"{inst}.sub"])
    assert orc.limbs_to_int(orc.bn_mul(a, b)) == u32_to_int(g[f"{inst}.prod"])
    assert orc.limbs_to_int(orc.bn_mul(a, a)) == u32_to_int(g[f"{inst}.a_square"])
    assert orc.limbs_to_int(orc.bn_slr(a, 125)) == u32_to_int(g[f"{inst}.a_slr125"])
    # Element ops (main.cu mont_add / mont_sub / mont_mul take a, b as Montgomery reprs)
    assert orc.limbs_to_int(orc.add(a, b)) == u32_to_int(g[f"{inst}.sum_mont"])
    assert orc.limbs_to_int(orc.sub(a, b)) == u32_to_int(g[f"{inst}.sub_mont"])
    assert orc.limbs_to_int(orc.mul(a, b)) == u32_to_int(g[f"{inst}.prod_mont"])
    # from_number(a) then square / pow(b) / invert (main.cu mont_square, mont_pow, mont_inv)
    am = orc.to_mont(a)
    assert orc.limbs_to_int(orc.mul(am, am)) == u32_to_int(g[f"{inst}.a_square_mont"])
    assert orc.limbs_to_int(orc.pow_(am, bi)) == u32_to_int(g[f"{inst}.pow_mont"])
    assert orc.limbs_to_int(orc.inv(am)) == u32_to_int(g[f"{inst}.a_inv_mont"])


def test_mont_conversion_and_lazy_vectors(orc, golden):
    g = golden["fr"]
    x, xm = u32_to_u64(g["x"]), u32_to_u64(g["x_mont"])
    assert orc.limbs_to_int(orc.to_mont(x)) == u32_to_int(g["x_mont"])
    assert orc.limbs_to_int(orc.from_mont(xm)) == u32_to_int(g["x"])
    # instance3: add/sub modulo 2m and reduce modulo m (main.cu:527-548), Python big ints
    xi, yi = u32_to_int(g["instance3.x"]), u32_to_int(g["instance3.y"])
    assert (xi + yi) % (2 * FR_M) == u32_to_int(g["instance3.r_add"])
    assert (xi - yi) % (2 * FR_M) == u32_to_int(g["instance3.r_sub"])
    assert xi % FR_M == u32_to_int(g["instance3.x_mod_m"])
    assert orc.limbs_to_int(orc.neg(orc.zeros(1)[0])) == 0


def test_mont_mul_against_python_bigint(orc):
    rng = np.random.default_rng(7)
    rinv_r = pow(R, -1, FR_M)
    rinv_q = pow(R, -1, FQ_M)
    for _ in range(200):
        a = int.from_bytes(rng.bytes(32), "little") % FR_M
        b = int.from_bytes(rng.bytes(32), "little") % FR_M
        assert orc.limbs_to_int(orc.mul(I(orc, a), I(orc, b))) == a * b * rinv_r % FR_M
        assert orc.limbs_to_int(orc.add(I(orc, a), I(orc, b))) == (a + b) % FR_M
        assert orc.limbs_to_int(orc.sub(I(orc, a), I(orc, b))) == (a - b) % FR_M
        c = int.from_bytes(rng.bytes(32), "little") % FQ_M
        d = int.from_bytes(rng.bytes(32), "little") % FQ_M
        assert orc.limbs_to_int(orc.mul(I(orc, c), I(orc, d), orc.FQ)) == c * d * rinv_q % FQ_M


def test_vec_ops(orc):
    a = orc.gen_fr(11, 1000)
    b = orc.gen_fr(12, 1000)
    prod = orc.vec_mul(a, b)
    for i in (0, 17, 999):
        assert (prod[i] == orc.mul(a[i], b[i])).all()
    s = orc.vec_add(a, b)
    d = orc.vec_sub(s, b)
    assert (d == a).all()


def test_generator_uniform_and_canonical(orc):
    a = orc.gen_fr(0, 4096)
    ints = [orc.limbs_to_int(orc.from_mont(x)) for x in a[:256]]
    assert all(0 <= v < FR_M for v in ints)
    assert len(set(ints)) == 256
    assert all(orc.limbs_to_int(x) < FR_M for x in a)
    # counter based: a window of the stream equals the same elements generated alone
    assert (orc.gen_fr(0, 10, start=100) == a[100:110]).all()
    # top bits are populated (uniform over [0, r))
    tops = np.array([x[3] >> np.uint64(60) for x in orc.gen_fr(5, 2000)])
    assert len(np.unique(tops)) >= 3


def test_root_of_unity(orc):
    w = orc.root_of_unity(28)
    canon = orc.limbs_to_int(orc.from_mont(w))
    assert canon == 0x03DDB9F5166D18B798865EA93DD31F743215CF6DD39329C8D34F1ED960C37C9C
    assert pow(canon, 1 << 28, FR_M) == 1
    assert pow(canon, 1 << 27, FR_M) == FR_M - 1
    for k in (1, 5, 16):
        wk = orc.limbs_to_int(orc.from_mont(orc.root_of_unity(k)))
        assert pow(wk, 1 << k, FR_M) == 1 and pow(wk, 1 << (k - 1), FR_M) == FR_M - 1
        wi = orc.limbs_to_int(orc.from_mont(orc.root_of_unity(k, inverse=True)))
        assert wk * wi % FR_M == 1


@pytest.mark.parametrize("log_n", [1, 2, 3, 5, 8])
def test_best_fft_matches_naive_dft(orc, log_n):
    n = 1 << log_n
    a = orc.gen_fr(100 + log_n, n)
    w = orc.root_of_unity(log_n)
    assert (orc.best_fft(a, w, log_n) == orc.naive_dft(a, w)).all()


@pytest.mark.parametrize("log_n", [4, 10, 14])
def test_ntt_roundtrip(orc, log_n):
    a = orc.gen_fr(log_n, 1 << log_n)
    assert (orc.intt(orc.ntt(a, log_n), log_n) == a).all()


def test_fft_threaded_equals_serial(orc):
    a = orc.gen_fr(3, 1 << 12)
    w = orc.root_of_unity(12)
    orc.set_threads(1)
    try:
        serial = orc.best_fft(a, w, 12)
    finally:
        orc.set_threads(0)
    assert (orc.best_fft(a, w, 12) == serial).all()


def test_coset_ntt_definition(orc):
    log_in, log_out = 3, 5
    coef = orc.gen_fr(9, 1 << log_in)
    g = orc.to_mont(I(orc, 7))
    out = orc.coset_ntt(coef, log_in, log_out, g)
    # evaluation of sum a_i X^i at g * w^j
    w = orc.root_of_unity(log_out)
    x = g.copy()
    for j in range(1 << log_out):
        assert (out[j] == orc.eval_poly(coef, x)).all()
        x = orc.mul(x, w)


def test_distribute_powers(orc):
    a = orc.gen_fr(1, 100)
    p = orc.gen_fr(2, 7)
    r = orc.distribute_powers(a, p)
    for i in (0, 6, 7, 99):
        assert (r[i] == orc.mul(a[i], p[i % 7])).all()


def test_zeta_periodic_powers_are_a_coset(orc):
    """Three periodic powers [1, zeta, zeta^2] of a cube root zeta equal the coset shift by zeta
    (zeta^(i mod 3) = zeta^i): the identity the zeta-coset extension test relies on."""
    r = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
    zeta = orc.to_mont(I(orc, pow(7, (r - 1) // 3, r)))
    assert not (zeta == orc.one()).all() and (orc.pow_(zeta, 3) == orc.one()).all()
    k, ext = 4, 6
    coef = orc.gen_fr(19, 1 << k)
    padded = np.zeros((1 << ext, 4), dtype=np.uint64)
    padded[: 1 << k] = coef
    shifted = orc.distribute_powers(padded, np.stack([orc.one(), zeta, orc.mul(zeta, zeta)]))
    assert np.array_equal(orc.ntt(shifted, ext), orc.coset_ntt(coef, k, ext, zeta))


def test_eval_horner_and_chunked(orc):
    poly = orc.gen_fr(4, 5000)
    x = orc.gen_fr(5, 1)[0]
    xi = orc.limbs_to_int(orc.from_mont(x))
    acc = 0
    for c in reversed(poly):
        acc = (acc * xi + orc.limbs_to_int(orc.from_mont(c))) % FR_M
    assert orc.limbs_to_int(orc.from_mont(orc.eval_poly(poly, x))) == acc


def test_batch_invert(orc):
    a = orc.gen_fr(6, 300)
    a[5] = 0
    a[299] = 0
    inv = orc.batch_invert(a)
    one = orc.one()
    for i in range(300):
        if i in (5, 299):
            assert (inv[i] == 0).all()
        else:
            assert (orc.mul(a[i], inv[i]) == one).all()


def test_poly_ptr_view(orc):
    base = orc.gen_fr(8, 16)
    v = orc.poly_ptr_view(base, 16, rotate=3)
    for i in range(16):
        assert (v[i] == base[(i - 3) % 16]).all()
    v = orc.poly_ptr_view(base, 5, offset=14, whole_len=16)
    for i in range(5):
        assert (v[i] == base[(14 + i) % 16]).all()


# ---------------------------------------------------------------- G1
def _pt(golden, name):
    g = golden["g1"]
    return np.concatenate([u32_to_u64(g[f"{name}_x"]), u32_to_u64(g[f"{name}_y"])])


def test_g1_known_answers(orc, golden):
    p1, p2 = _pt(golden, "p1"), _pt(golden, "p2")
    for name in ("p1", "p2", "pr", "pr100", "p1r128"):
        assert orc.g1_on_curve(_pt(golden, name)), name
    assert (orc.g1_affine_add(p1, p2) == _pt(golden, "pr")).all()
    p100 = orc.g1_scalar_mul_affine(p2, 100)
    assert (orc.g1_affine_add(p1, p100) == _pt(golden, "pr100")).all()
    assert (orc.g1_scalar_mul_affine(p1, 128) == _pt(golden, "p1r128")).all()
    # affine <-> XYZZ round trip and identity handling
    assert (orc.g1_xyzz_to_affine(orc.g1_to_xyzz(p1)) == p1).all()
    ident = np.zeros(8, dtype=np.uint64)
    assert (orc.g1_affine_add(p1, ident) == p1).all()
    neg = p1.copy()
    neg[4:] = orc.neg(p1[4:], orc.FQ)
    assert (orc.g1_affine_add(p1, neg) == ident).all()
    assert (orc.g1_affine_add(p1, p1) == orc.g1_scalar_mul_affine(p1, 2)).all()


def test_gen_points(orc):
    pts = orc.gen_points(2, 40)
    g = orc.g1_generator()
    assert orc.g1_on_curve(g)
    for i in (0, 1, 39):
        assert orc.g1_on_curve(pts[i])
        k = orc.limbs_to_int(orc.from_mont(orc.gen_fr(2, 1, start=i)[0]))
        assert (orc.g1_scalar_mul_affine(g, k) == pts[i]).all()
    assert (orc.gen_points(2, 5, start=35) == pts[35:40]).all()


@pytest.mark.parametrize("n", [1, 3, 5, 31, 64, 200])
def test_best_multiexp_matches_naive(orc, n):
    s = orc.gen_fr(1000 + n, n)
    p = orc.gen_points(2000 + n, n)
    if n > 4:
        s[2] = 0                     # zero scalar
        p[3] = 0                     # identity base
        p[4] = p[1]                  # repeated base
        s[4] = orc.neg(s[1])         # cancelling pair
    assert (orc.best_multiexp(s, p) == orc.naive_msm(s, p)).all()
