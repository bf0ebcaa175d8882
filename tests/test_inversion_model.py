"""The modular inversion of the device code (inv_binary in csrc/curve.cuh), restated over Python
integers step for step: T. Pornin's binary extended GCD with batched steps (IACR ePrint
2020/972, algorithm 2, k - 1 = 30).  Each of 17 outer iterations takes 30 steps on 62-bit
approximations of a and b (low 30 bits under the top 32 bits at the common length
n = max(len a, len b, 62)), collects them in signed factors, applies them to the full a, b
(exact division by 2^30) and to the coefficients u, v (one Montgomery step by 2^32 each), and
the result is v * 2^34.  These checks pin what the device code relies on: every row of factors
has |f| + |g| <= 2^30 (so the factors fit an int32 and u f + v g < m 2^30 fits 9 limbs), the
Montgomery step lands below 2m (one conditional subtraction), a and b stay below 2^255, and after
the fixed 510 steps a = 0, b = 1 and the result is the inverse, for both BN254 moduli."""
import random

FR = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
FQ = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
R = 1 << 256
STEPS, OUTER = 30, 17


def inv_model(y: int, m: int) -> int:
    a, b, u, v = y, m, 1, 0
    mprime = (-pow(m, -1, 1 << 32)) % (1 << 32)
    for _ in range(OUTER):
        n = max(a.bit_length(), b.bit_length(), 62)
        ab = ((a >> (n - 32)) << STEPS) | (a & ((1 << STEPS) - 1))
        bb = ((b >> (n - 32)) << STEPS) | (b & ((1 << STEPS) - 1))
        f0, g0, f1, g1 = 1, 0, 0, 1
        for _ in range(STEPS):
            if ab & 1:
                if ab < bb:
                    ab, bb, f0, g0, f1, g1 = bb, ab, f1, g1, f0, g0
                ab, f0, g0 = (ab - bb) >> 1, f0 - f1, g0 - g1
            else:
                ab >>= 1
            f1, g1 = 2 * f1, 2 * g1
        assert abs(f0) + abs(g0) <= 1 << STEPS and abs(f1) + abs(g1) <= 1 << STEPS
        na, nb = a * f0 + b * g0, a * f1 + b * g1
        assert na % (1 << STEPS) == 0 and nb % (1 << STEPS) == 0
        na, nb = na >> STEPS, nb >> STEPS
        if na < 0:
            na, f0, g0 = -na, -f0, -g0
        if nb < 0:
            nb, f1, g1 = -nb, -f1, -g1
        assert na < 1 << 255 and nb < 1 << 255

        def coef(f, g):
            x = (u if f >= 0 else m - u) * abs(f) + (v if g >= 0 else m - v) * abs(g)
            assert x < m << STEPS
            k = (x * mprime) % (1 << 32)
            r, rem = divmod(x + k * m, 1 << 32)
            assert rem == 0 and r < 2 * m
            return r - m if r >= m else r

        a, b, u, v = na, nb, coef(f0, g0), coef(f1, g1)
    assert a == 0 and b == 1
    return v * pow(2, 32 * OUTER - STEPS * OUTER, m) % m


def test_final_constants_match_field_cuh():
    """invk in field.cuh: 2^34 R^3 mod m turns v into the Montgomery form of the inverse."""
    want = {FR: [0xdd8b6d21, 0x352ff640, 0x331ce10a, 0x011e8bd1, 0x55d392c2, 0x438150ae, 0x73335b20, 0x21fe9388],
            FQ: [0x13bd45e1, 0x31d6a0d9, 0x382c59a2, 0x45fbf2bc, 0x1ab31dfb, 0x5b5fa369, 0xb36fd339, 0x24811383]}
    for m, limbs in want.items():
        k = pow(2, 32 * OUTER - STEPS * OUTER, m) * pow(R, 3, m) % m
        assert [(k >> (32 * i)) & 0xffffffff for i in range(8)] == limbs
    assert 32 * OUTER - STEPS * OUTER == 34 and STEPS * OUTER >= 2 * 254 - 1


def test_inverse_edge_and_seeded_values():
    rng = random.Random(7)
    for m in (FR, FQ):
        edge = [1, 2, 3, m - 1, m - 2, (m - 1) // 2, (m + 1) // 2, 1 << 253, (1 << 254) % m, R % m, R * R % m,
                (1 << 32) - 1, (1 << 62) - 1, (1 << 62) + 1, m - (1 << 200)]
        for y in edge + [rng.randrange(1, m) for _ in range(3000)]:
            assert inv_model(y, m) == pow(y, -1, m), hex(y)
