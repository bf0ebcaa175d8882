"""The arithmetic of the NTT's twiddle product (Fr::mul_shoup in csrc/field.cuh), restated over
Python integers limb by limb: Shoup's product by a fixed factor w with ws = floor(w 2^256 / r),
where the quotient estimate keeps only the partial products of a * ws that land in 32-bit
columns 7 and up.  These checks pin the bounds the device code relies on: the estimate is the
true quotient or one less, the remainder a * w - q r is below 3r (so it fits 256 bits and one
conditional subtraction of 2r brings it below 2r), and ws can be formed from the Montgomery
form w R mod r as (w R) * (-r^-1) mod 2^256."""
import random

R_MOD = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
TWO256 = 1 << 256
MASK = (1 << 32) - 1


def limbs(x):
    return [(x >> (32 * i)) & MASK for i in range(8)]


def quotient_estimate(a, ws):
    """floor(S' / 2^256), S' = the low halves of a_i * ws_j with i + j >= 7 and the high halves
    with i + j >= 6, each at its column."""
    s = 0
    for i, ai in enumerate(limbs(a)):
        for j, wj in enumerate(limbs(ws)):
            prod = ai * wj
            if i + j >= 7:
                s += (prod & MASK) << (32 * (i + j))
            if i + j >= 6:
                s += (prod >> 32) << (32 * (i + j + 1))
    return s >> 256


def shoup(a, w):
    ws = (w << 256) // R_MOD
    q = quotient_estimate(a, ws)
    q_true = (a * ws) >> 256
    assert q_true - 1 <= q <= q_true
    r = (a * w + q * (TWO256 - R_MOD)) % TWO256  # the device's form: low halves only
    assert r == a * w - q * R_MOD and 0 <= r < 3 * R_MOD
    if r >= 2 * R_MOD:
        r -= 2 * R_MOD
    assert r % R_MOD == a * w % R_MOD
    return r


def test_quotient_estimate_bounds():
    rng = random.Random(5)
    edge_a = [0, 1, R_MOD - 1, R_MOD, 2 * R_MOD - 1, 2 * R_MOD, 3 * R_MOD, TWO256 - 1]
    edge_w = [0, 1, 2, R_MOD - 1, R_MOD // 2]
    for a in edge_a + [rng.randrange(TWO256) for _ in range(1500)]:
        for w in edge_w + [rng.randrange(R_MOD)]:
            shoup(a, w)
    # all-ones limbs make the dropped columns as large as they get
    for _ in range(500):
        shoup(TWO256 - 1 - rng.randrange(1 << 64), R_MOD - 1 - rng.randrange(1 << 64))


def test_ws_from_montgomery_form():
    minv = (-pow(R_MOD, -1, TWO256)) % TWO256
    assert minv & MASK == 4026531839  # the CIOS constant -r^-1 mod 2^32 is its low limb
    rng = random.Random(6)
    for w in [0, 1, R_MOD - 1] + [rng.randrange(R_MOD) for _ in range(500)]:
        w_mont = w * TWO256 % R_MOD
        assert w_mont * minv % TWO256 == (w << 256) // R_MOD


def test_montgomery_operand_gives_montgomery_result():
    """a = x R (Montgomery) times the plain w gives x w R, the Montgomery form of x * w."""
    rng = random.Random(7)
    for _ in range(200):
        x, w = rng.randrange(R_MOD), rng.randrange(R_MOD)
        a = x * TWO256 % R_MOD
        assert shoup(a, w) % R_MOD == x * w * TWO256 % R_MOD
