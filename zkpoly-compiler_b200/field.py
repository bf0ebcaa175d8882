"""Host-side BN254 constants and conversions (Python integers), used to prepare scalar
arguments (roots of unity, n^-1, coset shifts) the same way the reference's compiler does
(compiler/src/utils.rs:51-77) and to move values between integers and 8 x u32 limb arrays.
Device arithmetic never happens here."""
from __future__ import annotations

import numpy as np

FR_MODULUS = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
FQ_MODULUS = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
R = 1 << 256
TWO_ADICITY = 28
GENERATOR = 7  # multiplicative generator of Fr^*, also the coset shift of the extended domain


def to_mont(x: int, m: int = FR_MODULUS) -> int:
    return x % m * R % m


def from_mont(x: int, m: int = FR_MODULUS) -> int:
    return x * pow(R, -1, m) % m


def root_of_unity(log_n: int, inverse: bool = False) -> int:
    """omega_k = (7^((r-1)/2^28))^(2^(28-k)), canonical integer (compiler/src/utils.rs:51-77)."""
    root = pow(GENERATOR, (FR_MODULUS - 1) >> TWO_ADICITY, FR_MODULUS)
    w = pow(root, 1 << (TWO_ADICITY - log_n), FR_MODULUS)
    return pow(w, -1, FR_MODULUS) if inverse else w


def int_to_words(x: int, words: int = 8) -> np.ndarray:
    return np.array([(x >> (32 * i)) & 0xFFFFFFFF for i in range(words)], dtype=np.uint32)


def words_to_int(w) -> int:
    return sum(int(v) << (32 * i) for i, v in enumerate(np.asarray(w, dtype=np.uint32).ravel()))


def mont_words(x: int, m: int = FR_MODULUS) -> np.ndarray:
    """Montgomery-form limbs of the integer x."""
    return int_to_words(to_mont(x, m))


def ints_to_mont_array(values, m: int = FR_MODULUS) -> np.ndarray:
    return np.stack([mont_words(v, m) for v in values]) if len(values) else np.zeros((0, 8), np.uint32)
