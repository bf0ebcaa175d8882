"""Poly library on the GPU through the C ABI, bit-exact against the oracle / big integers."""
import numpy as np
import pytest

from conftest import lookup_case
import torch

pytestmark = pytest.mark.gpu

M = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
R = 1 << 256


def dev(zk, a):
    return zk.ScalarArray.from_numpy(a)


def scal(zk, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int32).reshape(1, 8).copy()).cuda()


def ints(orc, a):
    """canonical integers of Montgomery-form limbs"""
    return [orc.limbs_to_int(x) * pow(R, -1, M) % M for x in a]


@pytest.mark.parametrize("la,lb", [(1000, 1000), (1000, 300), (300, 1000)])
def test_binary_ops_unequal_lengths(zk, orc, la, lb):
    a, b = orc.gen_fr(1, la), orc.gen_fr(2, lb)
    up, lo = max(la, lb), min(la, lb)
    for name, fn in (("add", zk.poly.poly_add), ("sub", zk.poly.poly_sub), ("mul", zk.poly.poly_mul)):
        r = zk.ScalarArray.zeros(up)
        fn(r, dev(zk, a), dev(zk, b))
        got = r.numpy_u64()
        head = {"add": orc.vec_add, "sub": orc.vec_sub, "mul": orc.vec_mul}[name](a[:lo], b[:lo])
        assert np.array_equal(got[:lo], head), name
        longer = a if la >= lb else b
        tail = longer[lo:]
        if name == "sub" and la < lb:
            tail = np.stack([orc.neg(x) for x in tail])
        assert np.array_equal(got[lo:], tail), name


def test_binary_ops_rotated(zk, orc):
    n = 512
    a, b = orc.gen_fr(3, n), orc.gen_fr(4, n)
    xa, xb = dev(zk, a), dev(zk, b)
    xa.rotate(5)
    xb.rotate(n - 7)
    r = zk.ScalarArray.zeros(n)
    r.rotate(11)
    zk.poly.poly_mul(r, xa, xb)
    va = orc.poly_ptr_view(a, n, rotate=5)
    vb = orc.poly_ptr_view(b, n, rotate=n - 7)
    assert np.array_equal(r.numpy_u64(), orc.vec_mul(va, vb))


def test_fills(zk, orc):
    t = dev(zk, orc.gen_fr(5, 100))
    zk.poly.poly_one_lagrange(t)
    assert np.array_equal(t.numpy_u64(), np.repeat(orc.one()[None], 100, 0))
    zk.poly.poly_one_coef(t)
    got = t.numpy_u64()
    assert np.array_equal(got[0], orc.one()) and not got[1:].any()
    zk.poly.poly_zero(t)
    assert not t.numpy_u64().any()


@pytest.mark.parametrize("n", [1, 5, 64, 65, 512, 513, 4097, 32769, 1 << 20])
def test_poly_eval(zk, orc, n):
    a = orc.gen_fr(6, n)
    x = orc.gen_fr(7, 1)[0]
    res = torch.zeros((1, 8), dtype=torch.int32, device="cuda")
    zk.poly.poly_eval(dev(zk, a), scal(zk, x), res)
    assert np.array_equal(res.cpu().numpy().view(np.uint64)[0], orc.eval_poly(a, x))


@pytest.mark.parametrize("n", [1, 63, 64, 65, 512, 513, 5000, 32769, 1 << 20])
def test_batched_invert(zk, orc, n):
    a = orc.gen_fr(8, n)
    if n > 10:
        a[3] = 0
        a[n - 1] = 0
        a[64:128 if n > 128 else n] = 0  # a whole zero chunk
    t = dev(zk, a)
    zk.poly.batched_invert(t)
    assert np.array_equal(t.numpy_u64(), orc.batch_invert(a))


@pytest.mark.parametrize("n", [1, 64, 65, 512, 513, 4100, 32769, 70000])
def test_scan_mul(zk, orc, n):
    a = orc.gen_fr(9, n)
    t = dev(zk, a)
    zk.poly.scan_mul(t)
    got = ints(orc, t.numpy_u64())
    acc, expect = 1, []
    for v in ints(orc, a):
        acc = acc * v % M
        expect.append(acc)
    assert got == expect


@pytest.mark.parametrize("log_n", [0, 1, 4, 6, 7, 9, 10, 12, 15, 16])
def test_kate_division(zk, orc, log_n):
    n = 1 << log_n
    p = orc.gen_fr(10, n)
    b = orc.gen_fr(11, 1)[0]
    q = zk.ScalarArray.zeros(n)
    xp = dev(zk, p)
    xp.rotate(2 % n if n > 1 else 0)
    zk.poly.kate_division(xp, scal(zk, b), q)
    pv = ints(orc, orc.poly_ptr_view(p, n, rotate=2 % n if n > 1 else 0))
    bi = ints(orc, [b])[0]
    expect = [0] * n
    for i in range(n - 2, -1, -1):
        expect[i] = (pv[i + 1] + bi * expect[i + 1]) % M
    assert ints(orc, q.numpy_u64()) == expect


def test_scalar_inv_and_pow(zk, orc):
    x = orc.gen_fr(12, 1)[0]
    t = scal(zk, x)
    zk.poly.inv_scalar(t)
    assert np.array_equal(t.cpu().numpy().view(np.uint64)[0], orc.inv(x))
    t = scal(zk, x)
    zk.poly.scalar_pow(t, 12345678901)
    assert np.array_equal(t.cpu().numpy().view(np.uint64)[0], orc.pow_(x, 12345678901))
    z = scal(zk, np.zeros(4, dtype=np.uint64))
    zk.poly.inv_scalar(z)
    assert not z.cpu().numpy().any()


def test_scalar_inv_edge_words(zk, orc):
    """The inversion (batched binary-GCD steps, fixed 17 x 30 iterations) on the stored words
    it inverts: small values, values next to m and to powers of two, R mod m, R^2 mod m, and
    seeded values; each equals the oracle's Montgomery inverse."""
    words = [1, 2, 3, 5, M - 1, M - 2, (M - 1) // 2, (M + 1) // 2, 1 << 253, (1 << 254) % M, (1 << 128) + 1,
             (1 << 32) - 1, R % M, R * R % M, M - (1 << 200)]
    vals = [orc.int_to_limbs(w) for w in words] + list(orc.gen_fr(13, 48))
    for x in vals:
        t = scal(zk, x)
        zk.poly.inv_scalar(t)
        assert np.array_equal(t.cpu().numpy().view(np.uint64)[0], orc.inv(x)), orc.limbs_to_int(x)


def test_square_matches_mul(zk, orc):
    """The dedicated Montgomery squaring equals a * a bit for bit (edge values included)."""
    n = 20000
    a = orc.gen_fr(13, n)
    M_limbs = orc.int_to_limbs(M - 1)
    a[0] = 0
    a[1] = M_limbs                      # m - 1
    a[2] = orc.int_to_limbs(1)
    a[3] = orc.int_to_limbs((1 << 253) + 12345)
    r = zk.ScalarArray.zeros(n)
    zk.poly.poly_square(r, dev(zk, a))
    assert np.array_equal(r.numpy_u64(), orc.vec_mul(a, a))


@pytest.mark.parametrize("log_n", [6, 10, 14])
def test_permute_matches_oracle(zk, orc, log_n):
    n = 1 << log_n
    usable = n - min(25, n // 4)
    inp, table = lookup_case(zk, n, usable, 70 + log_n)
    ri, rt = zk.ScalarArray.alloc(usable), zk.ScalarArray.alloc(usable)
    zk.poly.permute(inp, table, usable, ri, rt)
    ei, et = orc.permute(inp.numpy_u64(), table.numpy_u64(), usable)
    assert np.array_equal(ri.numpy_u64(), ei)
    assert np.array_equal(rt.numpy_u64(), et)
