"""ctypes wrapper around the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates the reference's CPU algorithms for the BN254 hot path (see oracle.h for
the reference files each part follows).  Only tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this module; the product path never does.

Arrays are numpy ``uint64`` with shape ``(n, 4)`` (field elements, little-endian limbs),
``(n, 8)`` (affine points: x limbs then y limbs) or ``(n, 16)`` (XYZZ points).  Byte for byte
this is the reference's 8 x u32 layout.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

FR, FQ = 0, 1
_u64p = ctypes.POINTER(ctypes.c_uint64)


def build(force: bool = False) -> str:
    """Compile oracle/liboracle.so with the committed Makefile (gcc)."""
    if force or not os.path.exists(_LIB_PATH) or _stale():
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


def _stale() -> bool:
    so = os.path.getmtime(_LIB_PATH)
    for f in os.listdir(_HERE):
        if f.endswith((".c", ".h")) and os.path.getmtime(os.path.join(_HERE, f)) > so:
            return True
    return False


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.or_get_threads.restype = ctypes.c_int
        _lib.or_g1_on_curve.restype = ctypes.c_int
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_u64p)


def zeros(n: int, words: int = 4) -> np.ndarray:
    return np.zeros((n, words), dtype=np.uint64)


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))


def threads() -> int:
    return int(lib().or_get_threads())


# ---------------------------------------------------------------- conversions
def int_to_limbs(x: int, words: int = 4) -> np.ndarray:
    return np.array([(x >> (64 * i)) & ((1 << 64) - 1) for i in range(words)], dtype=np.uint64)


def limbs_to_int(a) -> int:
    return sum(int(v) << (64 * i) for i, v in enumerate(np.asarray(a, dtype=np.uint64).ravel()))


def field_consts(f: int = FR):
    m, r1, r2 = zeros(1), zeros(1), zeros(1)
    minv = ctypes.c_uint64()
    lib().or_field_consts(f, _p(m), _p(r1), _p(r2), ctypes.byref(minv))
    return limbs_to_int(m), limbs_to_int(r1), limbs_to_int(r2), minv.value


# ---------------------------------------------------------------- field ops (single)
def _bin(fn, f, a, b):
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(1, 4)
    b = np.ascontiguousarray(b, dtype=np.uint64).reshape(1, 4)
    r = zeros(1)
    fn(f, _p(r), _p(a), _p(b))
    return r[0]


def mul(a, b, f=FR):
    return _bin(lib().or_mul, f, a, b)


def add(a, b, f=FR):
    return _bin(lib().or_add, f, a, b)


def sub(a, b, f=FR):
    return _bin(lib().or_sub, f, a, b)


def _un(fn, f, a):
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(1, 4)
    r = zeros(1)
    fn(f, _p(r), _p(a))
    return r[0]


def neg(a, f=FR):
    return _un(lib().or_neg, f, a)


def to_mont(a, f=FR):
    return _un(lib().or_to_mont, f, a)


def from_mont(a, f=FR):
    return _un(lib().or_from_mont, f, a)


def inv(a, f=FR):
    return _un(lib().or_inv, f, a)


def one(f=FR):
    r = zeros(1)
    lib().or_one(f, _p(r))
    return r[0]


def pow_(a, e: int, f=FR):
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(1, 4)
    el = int_to_limbs(e, 4).reshape(1, 4)
    r = zeros(1)
    lib().or_pow(f, _p(r), _p(a), _p(el), 4)
    return r[0]


def bn_mul(a, b):
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(1, 4)
    b = np.ascontiguousarray(b, dtype=np.uint64).reshape(1, 4)
    r = zeros(1, 8)
    lib().or_bn_mul(_p(r), _p(a), _p(b))
    return r[0]


def bn_slr(a, k: int):
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(1, 4)
    r = zeros(1)
    lib().or_bn_slr(_p(r), _p(a), ctypes.c_uint(k))
    return r[0]


def vec_mul(a, b):
    r = zeros(len(a))
    lib().or_vec_mul(_p(r), _p(a), _p(b), ctypes.c_size_t(len(a)))
    return r


def vec_add(a, b):
    r = zeros(len(a))
    lib().or_vec_add(_p(r), _p(a), _p(b), ctypes.c_size_t(len(a)))
    return r


def vec_sub(a, b):
    r = zeros(len(a))
    lib().or_vec_sub(_p(r), _p(a), _p(b), ctypes.c_size_t(len(a)))
    return r


# ---------------------------------------------------------------- generator / roots
def gen_fr(seed: int, n: int, start: int = 0) -> np.ndarray:
    out = zeros(n)
    lib().or_gen_fr(ctypes.c_uint64(seed), ctypes.c_uint64(start), ctypes.c_size_t(n), _p(out))
    return out


def root_of_unity(log_n: int, inverse: bool = False) -> np.ndarray:
    r = zeros(1)
    lib().or_root_of_unity(ctypes.c_uint(log_n), ctypes.c_int(int(inverse)), _p(r))
    return r[0]


def twiddles(omega, count: int) -> np.ndarray:
    w = np.ascontiguousarray(omega, dtype=np.uint64).reshape(1, 4)
    out = zeros(count)
    lib().or_twiddles(_p(w), ctypes.c_size_t(count), _p(out))
    return out


# ---------------------------------------------------------------- NTT family
def best_fft(a: np.ndarray, omega, log_n: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64).copy()
    w = np.ascontiguousarray(omega, dtype=np.uint64).reshape(1, 4)
    lib().or_best_fft(_p(a), _p(w), ctypes.c_uint(log_n))
    return a


def ntt(a: np.ndarray, log_n: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64).copy()
    lib().or_ntt(_p(a), ctypes.c_uint(log_n))
    return a


def intt(a: np.ndarray, log_n: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64).copy()
    lib().or_intt(_p(a), ctypes.c_uint(log_n))
    return a


def distribute_powers(a: np.ndarray, powers: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64).copy()
    powers = np.ascontiguousarray(powers, dtype=np.uint64)
    lib().or_distribute_powers(_p(a), ctypes.c_size_t(len(a)), _p(powers), ctypes.c_size_t(len(powers)))
    return a


def coset_ntt(coef: np.ndarray, log_in: int, log_out: int, g) -> np.ndarray:
    coef = np.ascontiguousarray(coef, dtype=np.uint64)
    g = np.ascontiguousarray(g, dtype=np.uint64).reshape(1, 4)
    out = zeros(1 << log_out)
    lib().or_coset_ntt(_p(out), _p(coef), ctypes.c_uint(log_in), ctypes.c_uint(log_out), _p(g))
    return out


def naive_dft(a: np.ndarray, omega) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    w = np.ascontiguousarray(omega, dtype=np.uint64).reshape(1, 4)
    out = zeros(len(a))
    lib().or_naive_dft(_p(out), _p(a), ctypes.c_size_t(len(a)), _p(w))
    return out


# ---------------------------------------------------------------- poly
def eval_poly(poly: np.ndarray, x) -> np.ndarray:
    poly = np.ascontiguousarray(poly, dtype=np.uint64)
    x = np.ascontiguousarray(x, dtype=np.uint64).reshape(1, 4)
    r = zeros(1)
    lib().or_eval(_p(r), _p(poly), ctypes.c_size_t(len(poly)), _p(x))
    return r[0]


def batch_invert(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64).copy()
    lib().or_batch_invert(_p(a), ctypes.c_size_t(len(a)))
    return a


def poly_ptr_view(base: np.ndarray, length: int, rotate: int = 0, offset: int = 0, whole_len: int = 0):
    base = np.ascontiguousarray(base, dtype=np.uint64)
    out = zeros(length)
    lib().or_poly_ptr_gather(_p(out), _p(base), ctypes.c_size_t(length), ctypes.c_size_t(rotate),
                             ctypes.c_size_t(offset), ctypes.c_size_t(whole_len))
    return out


# ---------------------------------------------------------------- G1
def g1_generator() -> np.ndarray:
    g = zeros(1, 8)
    lib().or_g1_generator(_p(g))
    return g[0]


def g1_on_curve(p) -> bool:
    p = np.ascontiguousarray(p, dtype=np.uint64).reshape(1, 8)
    return bool(lib().or_g1_on_curve(_p(p)))


def g1_affine_add(p, q) -> np.ndarray:
    p = np.ascontiguousarray(p, dtype=np.uint64).reshape(1, 8)
    q = np.ascontiguousarray(q, dtype=np.uint64).reshape(1, 8)
    r = zeros(1, 8)
    lib().or_g1_affine_add(_p(r), _p(p), _p(q))
    return r[0]


def g1_scalar_mul_affine(p, k: int) -> np.ndarray:
    p = np.ascontiguousarray(p, dtype=np.uint64).reshape(1, 8)
    kl = int_to_limbs(k, 4).reshape(1, 4)
    x = zeros(1, 16)
    lib().or_g1_scalar_mul(_p(x), _p(p), _p(kl))
    r = zeros(1, 8)
    lib().or_g1_to_affine(_p(r), _p(x))
    return r[0]


def g1_to_xyzz(p) -> np.ndarray:
    p = np.ascontiguousarray(p, dtype=np.uint64).reshape(1, 8)
    r = zeros(1, 16)
    lib().or_g1_to_xyzz(_p(r), _p(p))
    return r[0]


def g1_xyzz_to_affine(p) -> np.ndarray:
    p = np.ascontiguousarray(p, dtype=np.uint64).reshape(1, 16)
    r = zeros(1, 8)
    lib().or_g1_to_affine(_p(r), _p(p))
    return r[0]


def gen_points(seed: int, n: int, start: int = 0) -> np.ndarray:
    out = zeros(n, 8)
    lib().or_gen_points(ctypes.c_uint64(seed), ctypes.c_uint64(start), ctypes.c_size_t(n), _p(out))
    return out


def best_multiexp(scalars: np.ndarray, bases: np.ndarray) -> np.ndarray:
    scalars = np.ascontiguousarray(scalars, dtype=np.uint64)
    bases = np.ascontiguousarray(bases, dtype=np.uint64)
    r = zeros(1, 8)
    lib().or_best_multiexp(_p(r), _p(scalars), _p(bases), ctypes.c_size_t(len(scalars)))
    return r[0]


def naive_msm(scalars: np.ndarray, bases: np.ndarray) -> np.ndarray:
    scalars = np.ascontiguousarray(scalars, dtype=np.uint64)
    bases = np.ascontiguousarray(bases, dtype=np.uint64)
    r = zeros(1, 8)
    lib().or_naive_msm(_p(r), _p(scalars), _p(bases), ctypes.c_size_t(len(scalars)))
    return r[0]


def permute(inp: np.ndarray, table: np.ndarray, usable: int):
    """Lookup permutation (restates the expected output of core/tests/poly.rs:569-700, the
    contract of core/src/poly/src/permute.cuh:74-222).  Over the first `usable` rows: the input
    sorted ascending by canonical value; for the table, the first row of each run of equal input
    values holds that value (one occurrence removed from the table multiset), the other rows the
    remaining table values, ascending.  Montgomery (n, 4) uint64 in and out."""
    a_vals = sorted(limbs_to_int(from_mont(r)) for r in inp[:usable])
    left = {}
    for r in table[:usable]:
        v = limbs_to_int(from_mont(r))
        left[v] = left.get(v, 0) + 1
    out_t = [None] * usable
    repeated = []
    for i, v in enumerate(a_vals):
        if i == 0 or v != a_vals[i - 1]:
            assert left.get(v, 0) > 0, "input value missing from the table"
            left[v] -= 1
            out_t[i] = v
        else:
            repeated.append(i)
    rest = sorted(v for v, c in left.items() for _ in range(c))
    assert len(rest) == len(repeated)
    for i, v in zip(repeated, rest):
        out_t[i] = v
    pi = np.stack([to_mont(int_to_limbs(v)).reshape(4) for v in a_vals])
    pt = np.stack([to_mont(int_to_limbs(v)).reshape(4) for v in out_t])
    return pi, pt
