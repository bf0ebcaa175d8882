"""NTT family on the GPU through the C ABI, bit-exact against the CPU oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def to_dev(zk, a):
    return zk.ScalarArray.from_numpy(a)


@pytest.mark.parametrize("log_n", list(range(1, 17)) + [18, 20])
def test_ssip_ntt_matches_best_fft(zk, orc, log_n):
    n = 1 << log_n
    a = orc.gen_fr(0 if log_n == 16 else 40 + log_n, n)
    x = to_dev(zk, a)
    zk.ntt.ssip_ntt(x, zk.ntt.twiddle_table(log_n))
    expect = orc.best_fft(a, orc.root_of_unity(log_n), log_n)
    assert np.array_equal(x.numpy_u64(), expect)


@pytest.mark.parametrize("log_n", [1, 5, 12, 13, 16, 25])
def test_intt_roundtrip(zk, orc, log_n):
    n = 1 << log_n
    a = orc.gen_fr(7, n)
    x = to_dev(zk, a)
    zk.ntt.ntt(x)
    zk.ntt.intt(x)
    assert np.array_equal(x.numpy_u64(), a)


def test_intt_matches_oracle(zk, orc):
    log_n = 14
    a = orc.gen_fr(70, 1 << log_n)
    x = to_dev(zk, a)
    zk.ntt.intt(x)
    assert np.array_equal(x.numpy_u64(), orc.intt(a, log_n))


def test_config1_roundtrip_2_16(zk, orc):
    """NTT 2^16 of seed-0 data, bit-exact vs best_fft, then INTT round trip."""
    a = orc.gen_fr(0, 1 << 16)
    x = to_dev(zk, a)
    zk.ntt.ntt(x)
    assert np.array_equal(x.numpy_u64(), orc.ntt(a, 16))
    zk.ntt.intt(x)
    assert np.array_equal(x.numpy_u64(), a)


def test_ntt_2_24_properties(zk, orc):
    """Full metric size: round trip and linearity NTT(a + b) = NTT(a) + NTT(b) at 2^24."""
    import torch
    log_n = 24
    n = 1 << log_n
    a = orc.gen_fr(1, n)
    b = orc.gen_fr(2, n)
    xa, xb = to_dev(zk, a), to_dev(zk, b)
    xs = to_dev(zk, orc.vec_add(a, b))
    for x in (xa, xb, xs):
        zk.ntt.ntt(x)
    # spot-check entries against direct evaluation at w^k
    w = orc.root_of_unity(log_n)
    got = xa.values.cpu().numpy().view(np.uint64).reshape(-1, 4)
    for k in (0, 1, 12345, n - 1):
        assert np.array_equal(got[k], orc.eval_poly(a, orc.pow_(w, k))), k
    sa = orc.vec_add(got, xb.values.cpu().numpy().view(np.uint64).reshape(-1, 4))
    assert np.array_equal(sa, xs.values.cpu().numpy().view(np.uint64).reshape(-1, 4))
    zk.ntt.intt(xa)
    assert np.array_equal(xa.values.cpu().numpy().view(np.uint64).reshape(-1, 4), a)
    del torch


@pytest.mark.parametrize("log_n", [3, 11, 15])
def test_rotated_and_sliced_views(zk, orc, log_n):
    n = 1 << log_n
    base = orc.gen_fr(5, n)
    # rotated whole array
    x = to_dev(zk, base)
    x.rotate(3)
    view = orc.poly_ptr_view(base, n, rotate=3)
    zk.ntt.ssip_ntt(x, zk.ntt.twiddle_table(log_n))
    assert np.array_equal(x.numpy_u64(), orc.ntt(view, log_n))
    # slice of a larger buffer that wraps around its end
    big = orc.gen_fr(6, 2 * n)
    xb = to_dev(zk, big)
    s = xb.set_slice_raw(2 * n - 5, n)
    view = orc.poly_ptr_view(big, n, offset=2 * n - 5, whole_len=2 * n)
    zk.ntt.ssip_ntt(s, zk.ntt.twiddle_table(log_n))
    assert np.array_equal(s.numpy_u64(), orc.ntt(view, log_n))
    # the part of the buffer outside the slice is untouched
    after = xb.values.cpu().numpy().view(np.uint64).reshape(-1, 4)
    untouched = [i for i in range(2 * n) if not (i >= 2 * n - 5 or i < n - 5)]
    assert np.array_equal(after[untouched], big[untouched])


@pytest.mark.parametrize("log_n", [4, 12, 17])
def test_recompute_ntt(zk, orc, log_n):
    n = 1 << log_n
    a = orc.gen_fr(9, n)
    w = zk.field.mont_words(zk.field.root_of_unity(log_n))
    pq_len = zk.ntt.get_pq_len(log_n)
    pq, omegas = zk.ntt.gen_pq_omegas(pq_len, n, w)
    x = to_dev(zk, a)
    zk.ntt.recompute_ntt(x, zk.ScalarArray.from_numpy(pq), zk.ScalarArray.from_numpy(omegas))
    assert np.array_equal(x.numpy_u64(), orc.ntt(a, log_n))


def test_precompute_tables(zk, orc):
    w = orc.root_of_unity(12)
    tab = zk.ntt.ssip_precompute(2048, w.view(np.uint32))
    assert np.array_equal(tab.view(np.uint64).reshape(-1, 4), orc.twiddles(w, 2048))
    assert np.array_equal(zk.ntt.ssip_precompute(1, w.view(np.uint32)).view(np.uint64).reshape(-1, 4)[0],
                          orc.one())


def test_distribute_powers(zk, orc):
    a = orc.gen_fr(10, 1000)
    for pn in (1, 7, 64, 1000, 2000):
        p = orc.gen_fr(11, pn)
        x = to_dev(zk, a)
        zk.ntt.distribute_powers(x, zk.ScalarArray.from_numpy(p))
        assert np.array_equal(x.numpy_u64(), orc.distribute_powers(a, p)), pn


@pytest.mark.parametrize("k", [10, 13, 16])
def test_distribute_zeta_then_recompute_ntt(zk, orc, k):
    """The reference's composed case (core/tests/ntt.rs:262-383): 2^k coefficients zero-extended
    to 2^(k+2) in a view rotated by -2, multiplied periodically by [1, zeta, zeta^2]
    (distribute_powers with three powers), then recompute_ntt at the extended size: halo2's
    coeff_to_extended, the evaluations at zeta * w_ext^j.  halo2curves' ZETA is one of Fr's two
    primitive cube roots; 7^((r-1)/3) is used here, the choice changes only the constant."""
    F = zk.field
    zeta = pow(F.GENERATOR, (F.FR_MODULUS - 1) // 3, F.FR_MODULUS)
    assert zeta != 1 and pow(zeta, 3, F.FR_MODULUS) == 1
    ext = k + 2
    N = 1 << ext
    a = orc.gen_fr(300 + k, 1 << k)
    logical = np.zeros((N, 4), dtype=np.uint64)
    logical[: 1 << k] = a
    # rotate(-2): logical element i is stored at (i + 2) mod N
    x = to_dev(zk, np.roll(logical, 2, axis=0))
    x.rotate(-2)
    assert np.array_equal(x.numpy_u64(), logical)
    zm = orc.to_mont(orc.int_to_limbs(zeta))
    powers = np.stack([orc.one(), zm, orc.mul(zm, zm)])
    zk.ntt.distribute_powers(x, zk.ScalarArray.from_numpy(powers))
    w = F.mont_words(F.root_of_unity(ext))
    pq, omegas = zk.ntt.gen_pq_omegas(zk.ntt.get_pq_len(ext), N, w)
    zk.ntt.recompute_ntt(x, zk.ScalarArray.from_numpy(pq), zk.ScalarArray.from_numpy(omegas))
    assert np.array_equal(x.numpy_u64(), orc.coset_ntt(a, k, ext, zm))


@pytest.mark.parametrize("log_in,log_out", [(2, 5), (10, 13), (13, 16), (16, 19)])
def test_coset_lde(zk, orc, log_in, log_out):
    coef = orc.gen_fr(12, 1 << log_in)
    g = orc.to_mont(orc.int_to_limbs(7))
    out = zk.ScalarArray.zeros(1 << log_out)
    zk.ntt.coset_ntt(out, to_dev(zk, coef))
    assert np.array_equal(out.numpy_u64(), orc.coset_ntt(coef, log_in, log_out, g))


def test_ntt_ex_shift_and_scale(zk, orc):
    log_n = 14
    a = orc.gen_fr(13, 1 << log_n)
    g = orc.to_mont(orc.int_to_limbs(5))
    x = to_dev(zk, a)
    zk.ntt.ntt_ex(x, zk.ntt.twiddle_table(log_n), shift=zk.ntt.scalar_const(5), scale=zk.ntt.scalar_const(3))
    expect = orc.coset_ntt(a, log_n, log_n, g)
    three = orc.to_mont(orc.int_to_limbs(3))
    expect = np.stack([orc.mul(e, three) for e in expect])
    assert np.array_equal(x.numpy_u64(), expect)


def test_invalid_arguments_return_error(zk):
    x = zk.ScalarArray.zeros(16)
    bad = x.poly_ptr()
    bad.len = 15
    lib = zk.native.load("libntt.so")
    tw = zk.ntt.twiddle_table(4)
    assert lib.ssip_ntt(bad, tw.values.data_ptr(), 4, None, 8, 8) == 1  # cudaErrorInvalidValue
    bad = x.poly_ptr()
    bad.rotate = 3
    bad.offset = 2
    assert lib.ssip_ntt(bad, tw.values.data_ptr(), 4, None, 8, 8) == 1


def test_ntt_batch_uneven_sizes(zk, orc):
    """Batched form: transforms of 2^1..2^20 mixing forward, inverse and coset, one plan."""
    rng = np.random.default_rng(3)
    logs = [1, 3, 10, 12, 13, 15, 17, 20, 11, 14, 4, 18]
    kinds = [["ntt", "intt", "coset"][int(k)] for k in rng.integers(0, 3, len(logs))]
    data = [orc.gen_fr(500 + i, 1 << L) for i, L in enumerate(logs)]
    xs = [to_dev(zk, a) for a in data]
    batch = zk.ntt.NttBatch(list(zip(xs, kinds)))
    batch.run()
    g = orc.to_mont(orc.int_to_limbs(7))
    for a, x, L, kind in zip(data, xs, logs, kinds):
        if kind == "ntt":
            expect = orc.ntt(a, L)
        elif kind == "intt":
            expect = orc.intt(a, L)
        else:
            expect = orc.coset_ntt(a, L, L, g)
        assert np.array_equal(x.numpy_u64(), expect), (L, kind)
    # replay through a CUDA graph gives the same as running the plan twice directly
    import torch
    ys = [to_dev(zk, a) for a in data]
    batch2 = zk.ntt.NttBatch(list(zip(ys, kinds)))
    s = torch.cuda.Stream()
    g_ = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g_, stream=s):
        batch2.run(s)
    g_.replay()
    torch.cuda.synchronize()
    for x, y in zip(xs, ys):
        assert np.array_equal(x.numpy_u64(), y.numpy_u64())


@pytest.mark.parametrize("solo_log", [0, 1, 12, 16])
def test_ntt_batch_solo_threshold(zk, orc, solo_log):
    """Every split between shared persistent launches and tasks run on their own plans gives the
    oracle's transforms (0: all shared; 1: all on their own)."""
    lib = zk.native.load("libntt.so")
    logs = [2, 9, 12, 14, 16, 19]
    kinds = ["coset", "intt", "ntt", "coset", "intt", "ntt"]
    data = [orc.gen_fr(700 + i, 1 << L) for i, L in enumerate(logs)]
    xs = [to_dev(zk, a) for a in data]
    try:
        assert lib.zkp_ntt_batch_set_solo_log(solo_log) == 0
        zk.ntt.NttBatch(list(zip(xs, kinds))).run()
    finally:
        assert lib.zkp_ntt_batch_set_solo_log(16) == 0
    g = orc.to_mont(orc.int_to_limbs(7))
    for a, x, L, kind in zip(data, xs, logs, kinds):
        expect = {"ntt": lambda: orc.ntt(a, L), "intt": lambda: orc.intt(a, L),
                  "coset": lambda: orc.coset_ntt(a, L, L, g)}[kind]()
        assert np.array_equal(x.numpy_u64(), expect), (solo_log, L, kind)


@pytest.mark.parametrize("log_n", [9, 13, 17, 20])
def test_digit_caps_give_the_same_transform(zk, orc, log_n):
    """Every plan the tuner can pick (digit cap 4..12: more passes of smaller pencils) computes
    the same transform, forward, coset and inverse."""
    lib = zk.native.load("libntt.so")
    n = 1 << log_n
    a = orc.gen_fr(90 + log_n, n)
    expect = orc.best_fft(a, orc.root_of_unity(log_n), log_n)
    g = orc.to_mont(orc.int_to_limbs(7))
    expect_coset = orc.coset_ntt(a, log_n, log_n, g)
    try:
        for d in (4, 5, 6, 7, 8, 10, 11, 12):
            assert lib.zkp_ntt_set_max_digit(log_n, d) == 0
            x = to_dev(zk, a)
            zk.ntt.ssip_ntt(x, zk.ntt.twiddle_table(log_n))
            assert np.array_equal(x.numpy_u64(), expect), d
            y = to_dev(zk, a)
            zk.ntt.ntt_ex(y, zk.ntt.twiddle_table(log_n), zk.ntt.scalar_const(7))
            assert np.array_equal(y.numpy_u64(), expect_coset), d
            zk.ntt.intt(x)
            assert np.array_equal(x.numpy_u64(), a), d
    finally:
        assert lib.zkp_ntt_set_max_digit(log_n, 0) == 0
        zk.tuner.apply_ntt_plans()  # back to the tuned plan, if one is cached
    assert lib.zkp_ntt_set_max_digit(log_n, 3) != 0 and lib.zkp_ntt_set_max_digit(log_n, 13) != 0


# ---- Shoup twiddle table and the register passes that read it
def test_shoup_table_entries(zk, orc):
    """Entry e = (w^e plain, floor(w^e 2^256 / r)) from the Montgomery root table."""
    log_n = 12
    p = zk.field.FR_MODULUS
    tab = zk.ntt.shoup_table_of(zk.ntt.twiddle_table(log_n)).cpu().numpy().view(np.uint32)
    w = zk.field.root_of_unity(log_n)
    for e in (0, 1, 2, 777, (1 << (log_n - 1)) - 1):
        we = pow(w, e, p)
        got_w = orc.limbs_to_int(tab[e, :8].view(np.uint64))
        got_ws = orc.limbs_to_int(tab[e, 8:].view(np.uint64))
        assert got_w == we, e
        assert got_ws == (we << 256) // p, e


@pytest.mark.parametrize("log_n", [7, 8, 11, 12, 13, 17, 20, 22])
def test_ntt_shoup_matches_best_fft(zk, orc, log_n):
    """zkp_ntt_ex_shoup: bit-identical to the oracle's best_fft at sizes whose plans use register
    passes of every width the tuner may pick."""
    n = 1 << log_n
    a = orc.gen_fr(90 + log_n, n)
    x = to_dev(zk, a)
    tw = zk.ntt.twiddle_table(log_n)
    zk.ntt.ntt_ex(x, tw, shoup=zk.ntt.shoup_table_of(tw))
    assert np.array_equal(x.numpy_u64(), orc.best_fft(a, orc.root_of_unity(log_n), log_n))


@pytest.mark.parametrize("cap", [4, 5, 6])
def test_ntt_shoup_every_pass_width(zk, orc, cap):
    """Digit caps 4..6 route every pass of a 2^16 transform through the Shoup register pass with
    that pencil width; the plan is restored afterwards."""
    lib = zk.native.load("libntt.so")
    log_n = 16
    a = orc.gen_fr(123, 1 << log_n)
    expect = orc.best_fft(a, orc.root_of_unity(log_n), log_n)
    old = zk.ntt.plan_digits(log_n)
    try:
        assert lib.zkp_ntt_set_max_digit(log_n, cap) == 0
        assert max(zk.ntt.plan_digits(log_n)) <= cap
        x = to_dev(zk, a)
        tw = zk.ntt.twiddle_table(log_n)
        zk.ntt.ntt_ex(x, tw, shoup=zk.ntt.shoup_table_of(tw))
        assert np.array_equal(x.numpy_u64(), expect)
    finally:
        assert lib.zkp_ntt_set_max_digit(log_n, max(old)) == 0


def test_ntt_shoup_shift_scale_and_views(zk, orc):
    """Shift and scale fused around Shoup passes, and a rotated view, equal the Montgomery path."""
    log_n = 14
    n = 1 << log_n
    a = orc.gen_fr(131, n)
    tw = zk.ntt.twiddle_table(log_n)
    sh = zk.ntt.shoup_table_of(tw)
    x1, x2 = to_dev(zk, a), to_dev(zk, a)
    five, three = zk.ntt.scalar_const(5), zk.ntt.scalar_const(3)
    zk.ntt.ntt_ex(x1, tw, shift=five, scale=three)
    zk.ntt.ntt_ex(x2, tw, shift=five, scale=three, shoup=sh)
    assert np.array_equal(x1.numpy_u64(), x2.numpy_u64())
    base = to_dev(zk, a)
    view = zk.ScalarArray(base.values, length=n, rotate=5)
    ref = to_dev(zk, orc.poly_ptr_view(a, n, rotate=5))
    zk.ntt.ntt_ex(view, tw, shoup=sh)
    zk.ntt.ssip_ntt(ref, tw)
    assert np.array_equal(view.numpy_u64(), ref.numpy_u64())


def test_coset_lde_shoup_matches_oracle(zk, orc):
    log_in, log_out = 12, 15
    coef = orc.gen_fr(140, 1 << log_in)
    g = orc.to_mont(orc.int_to_limbs(7))
    tw = zk.ntt.twiddle_table(log_out)
    out = zk.ScalarArray.zeros(1 << log_out)
    zk.ntt.coset_lde(out, to_dev(zk, coef), tw, zk.ntt.scalar_const(7), shoup=zk.ntt.shoup_table_of(tw))
    assert np.array_equal(out.numpy_u64(), orc.coset_ntt(coef, log_in, log_out, g))


def test_shoup_entries_reject_misaligned_table(zk):
    x = zk.ScalarArray.zeros(1 << 8)
    tw = zk.ntt.twiddle_table(8)
    sh = zk.ntt.shoup_table_of(tw)
    lib = zk.native.load("libntt.so")
    assert lib.zkp_ntt_ex_shoup(x.poly_ptr(), tw.values.data_ptr(), sh.data_ptr() + 4, 8, None, None, None) == 1
    assert lib.zkp_ntt_shoup_table(tw.values.data_ptr(), 0, sh.data_ptr(), None) == 1


@pytest.mark.parametrize("threads", [32, 64, 128, 256])
def test_ntt_register_pass_block_shapes(zk, orc, threads):
    """The tuner's NTT block shape (CTA size of the register passes) leaves results unchanged."""
    lib = zk.native.load("libntt.so")
    log_n = 17
    a = orc.gen_fr(130, 1 << log_n)
    try:
        assert lib.zkp_ntt_set_block(log_n, threads) == 0
        x = to_dev(zk, a)
        zk.ntt.ntt(x)
        assert np.array_equal(x.numpy_u64(), orc.ntt(a, log_n))
    finally:
        lib.zkp_ntt_set_block(log_n, 0)
        zk.tuner.apply_ntt_plans()
    assert lib.zkp_ntt_set_block(log_n, 48) == 1  # refused


@pytest.mark.parametrize("log_in,log_out", [(18, 20), (20, 21)])
def test_coset_elementwise_prep_sizes(zk, orc, log_in, log_out):
    """From 2^20 the coset shift and the zero-extension run as one elementwise pass before the
    transform.  Montgomery and Shoup twiddles, rotated source and destination views, and the
    in-place shift + scale form, each against the oracle."""
    n_in, n_out = 1 << log_in, 1 << log_out
    coef = orc.gen_fr(150 + log_in, n_in)
    seven = orc.to_mont(orc.int_to_limbs(7))
    tw = zk.ntt.twiddle_table(log_out)
    sh = zk.ntt.shoup_table_of(tw)
    expect = orc.coset_ntt(coef, log_in, log_out, seven)
    out = zk.ScalarArray.zeros(n_out)
    zk.ntt.coset_lde(out, to_dev(zk, coef), tw, zk.ntt.scalar_const(7))
    assert np.array_equal(out.numpy_u64(), expect)
    # rotated source (element i of the view is coef[(i - 5) mod n_in]) into a rotated destination
    src = zk.ScalarArray(to_dev(zk, coef).values, length=n_in, rotate=5)
    dst_base = zk.ScalarArray.zeros(n_out)
    dst = zk.ScalarArray(dst_base.values, length=n_out, rotate=9)
    zk.ntt.coset_lde(dst, src, tw, zk.ntt.scalar_const(7), shoup=sh)
    logical = orc.poly_ptr_view(coef, n_in, rotate=5)
    expect_rot = orc.coset_ntt(logical, log_in, log_out, seven)
    assert np.array_equal(orc.poly_ptr_view(dst_base.numpy_u64(), n_out, rotate=9), expect_rot)
    # in place: x <- 3 * NTT(5^i x_i) at the output size
    a = orc.gen_fr(160 + log_out, n_out)
    x = to_dev(zk, a)
    zk.ntt.ntt_ex(x, tw, shift=zk.ntt.scalar_const(5), scale=zk.ntt.scalar_const(3), shoup=sh)
    three = orc.to_mont(orc.int_to_limbs(3))
    want = orc.coset_ntt(a, log_out, log_out, orc.to_mont(orc.int_to_limbs(5)))
    assert np.array_equal(x.numpy_u64(), orc.vec_mul(want, np.tile(three, (n_out, 1))))
