"""Poly operators: host-side mirror of the reference's Rust wrappers (core/src/poly.rs:37-784).

Binary ops take mut=[res], vars=[a, b, stream]; PolyEval mut=[temp, res], vars=[poly, x,
stream]; KateDivision mut=[temp, res], vars=[poly, b, stream]; PolyScan / PolyInvert
mut=[temp, target]; ScalarInv / ScalarPow mut=[scalar].  Temp buffers are sized with the same
null-pointer query the reference uses and allocated as torch uint8 device tensors.
"""
from __future__ import annotations

import ctypes

import torch

from .native import check, load
from .scalar import ScalarArray, require_cuda, stream_handle

LIB = "libpoly.so"


def _lib():
    require_cuda()
    return load(LIB)


def _query(fn, *args) -> int:
    size = ctypes.c_ulong(0)
    check(fn(None, ctypes.byref(size), *args), fn.__name__ + "(size query)")
    return size.value


def _temp(nbytes: int, device) -> torch.Tensor:
    return torch.empty(max(nbytes, 1), dtype=torch.uint8, device=device)


def poly_add(r: ScalarArray, a: ScalarArray, b: ScalarArray, stream=None):
    check(_lib().poly_add(r.poly_ptr(), a.poly_ptr(), b.poly_ptr(), stream_handle(stream)), "poly_add")


def poly_sub(r: ScalarArray, a: ScalarArray, b: ScalarArray, stream=None):
    check(_lib().poly_sub(r.poly_ptr(), a.poly_ptr(), b.poly_ptr(), stream_handle(stream)), "poly_sub")


def poly_mul(r: ScalarArray, a: ScalarArray, b: ScalarArray, stream=None):
    check(_lib().poly_mul(r.poly_ptr(), a.poly_ptr(), b.poly_ptr(), stream_handle(stream)), "poly_mul")


def poly_square(r: ScalarArray, a: ScalarArray, stream=None):
    check(_lib().zkp_poly_square(r.poly_ptr(), a.poly_ptr(), stream_handle(stream)), "zkp_poly_square")


def poly_one_lagrange(t: ScalarArray, stream=None):
    check(_lib().poly_one_lagrange(t.poly_ptr(), stream_handle(stream)), "poly_one_lagrange")


def poly_one_coef(t: ScalarArray, stream=None):
    check(_lib().poly_one_coef(t.poly_ptr(), stream_handle(stream)), "poly_one_coef")


def poly_zero(t: ScalarArray, stream=None):
    check(_lib().poly_zero(t.poly_ptr(), stream_handle(stream)), "poly_zero")


def _null_ptr(n):
    from .native import PolyPtr
    return PolyPtr(None, n, 0, 0, n)


def poly_eval(poly: ScalarArray, x: torch.Tensor, res: torch.Tensor, temp: torch.Tensor | None = None,
              stream=None):
    """res (8 int32, device) = sum poly[i] x^i with x a device scalar (8 int32)."""
    lib = _lib()
    need = _query(lib.poly_eval, _null_ptr(poly.len), None, None, None)
    temp = temp if temp is not None else _temp(need, poly.values.device)
    size = ctypes.c_ulong(temp.numel())
    check(lib.poly_eval(temp.data_ptr(), ctypes.byref(size), poly.poly_ptr(), res.data_ptr(), x.data_ptr(),
                        stream_handle(stream)), "poly_eval")


def kate_division(p: ScalarArray, b: torch.Tensor, q: ScalarArray, stream=None):
    lib = _lib()
    log_p = p.len.bit_length() - 1
    need = _query(lib.kate_division, log_p, _null_ptr(p.len), None, _null_ptr(p.len), None)
    temp = _temp(need, p.values.device)
    size = ctypes.c_ulong(temp.numel())
    check(lib.kate_division(temp.data_ptr(), ctypes.byref(size), log_p, p.poly_ptr(), b.data_ptr(), q.poly_ptr(),
                            stream_handle(stream)), "kate_division")


def scan_mul(t: ScalarArray, stream=None):
    lib = _lib()
    need = _query(lib.scan_mul, _null_ptr(t.len), None)
    temp = _temp(need, t.values.device)
    size = ctypes.c_ulong(temp.numel())
    check(lib.scan_mul(temp.data_ptr(), ctypes.byref(size), t.poly_ptr(), stream_handle(stream)), "scan_mul")


def batched_invert(t: ScalarArray, stream=None):
    lib = _lib()
    need = _query(lib.batched_invert, _null_ptr(t.len), None)
    temp = _temp(need, t.values.device)
    size = ctypes.c_ulong(temp.numel())
    check(lib.batched_invert(temp.data_ptr(), ctypes.byref(size), t.poly_ptr(), stream_handle(stream)),
          "batched_invert")


def permute(inp: ScalarArray, table: ScalarArray, usable: int, res_input: ScalarArray, res_table: ScalarArray,
            stream=None):
    """Lookup permutation of the first `usable` rows (core/src/poly.rs PolyPermute, reference
    permute.cuh:74-222): res_input = sorted input, res_table = the matching table arrangement."""
    lib = _lib()
    size = ctypes.c_ulong(0)
    check(lib.permute(None, ctypes.byref(size), usable, inp.poly_ptr(), table.poly_ptr(), res_input.poly_ptr(),
                      res_table.poly_ptr(), stream_handle(stream)), "permute(size query)")
    temp = _temp(size.value, inp.values.device)
    check(lib.permute(temp.data_ptr(), ctypes.byref(size), usable, inp.poly_ptr(), table.poly_ptr(),
                      res_input.poly_ptr(), res_table.poly_ptr(), stream_handle(stream)), "permute")


def inv_scalar(x: torch.Tensor, stream=None):
    check(_lib().inv_scalar(x.data_ptr(), stream_handle(stream)), "inv_scalar")


def scalar_pow(x: torch.Tensor, exp: int, stream=None):
    check(_lib().scalar_pow(x.data_ptr(), exp, stream_handle(stream)), "scalar_pow")


# ------------------------------------------------------------------ RegisteredFunction mirrors
class _Binary:
    def __init__(self, fn, name):
        self._fn, self.name = fn, name

    def get_fn(self):
        def f(mut_var, var):
            assert len(mut_var) == 1 and len(var) == 3
            self._fn(mut_var[0], var[0], var[1], var[2])
        return f


PolyAdd = lambda: _Binary(poly_add, "poly_add")  # noqa: E731  core/src/poly.rs:37-80
PolySub = lambda: _Binary(poly_sub, "poly_sub")  # noqa: E731
PolyMul = lambda: _Binary(poly_mul, "poly_mul")  # noqa: E731


class PolyEval:
    """core/src/poly.rs:94-130 / :632"""

    def get_fn(self):
        def f(mut_var, var):
            temp, res = mut_var
            poly, x, stream = var
            poly_eval(poly, x, res, temp, stream)
        return f


class PolyInvert:
    def get_fn(self):
        def f(mut_var, var):
            batched_invert(mut_var[-1], var[-1] if var else None)
        return f
