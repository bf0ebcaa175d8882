"""The fused polynomial pipeline of a prover round on the device (all B200 kernels):

  a, b, c (Lagrange, 2^k)  --INTT (n^-1 fused)-->  coefficients
  coefficients --coset LDE (zero-extend, shift g^i, NTT at 2^(k+e), fused)--> coset evaluations
  q = (a*b - c - z*z(wX)) * Z_H^-1   (one fused kernel)

This is what the reference's compiler emits for such a program: intt_mending's n^-1
(compiler/src/transit/type2/intt_mending.rs:11-70), Extend + distribute_powers + NTT for the
coset (compiler/src/ast/poly_coef.rs:252-255, core/src/ntt/src/distribute_powers.cuh:5-21),
and a fused arithmetic kernel (compiler/src/transit/type2/kernel_fusion.rs:390-563).
Z_H(X) = X^(2^k) - 1 takes 2^e distinct values on the coset g*<w_(k+e)>, so its inverse is a
periodic input of 2^e elements.
"""
from __future__ import annotations

import numpy as np
import torch

from . import field, fused, ntt
from .scalar import ScalarArray

SHIFT = field.GENERATOR


def zh_inv_values(k: int, ext: int, shift: int = SHIFT) -> list[int]:
    """1 / (shift^(2^k) * w_(k+ext)^(j*2^k) - 1) for j < 2^ext (canonical integers)."""
    m = field.FR_MODULUS
    w = field.root_of_unity(k + ext)
    gk = pow(shift, 1 << k, m)
    return [pow((gk * pow(w, j << k, m) - 1) % m, -1, m) for j in range(1 << ext)]


def zh_inv_device(k: int, ext: int, device="cuda") -> ScalarArray:
    vals = np.stack([field.mont_words(v) for v in zh_inv_values(k, ext)])
    return ScalarArray.from_numpy(vals, device)


def rotated(z: ScalarArray, ext: int) -> ScalarArray:
    """z(wX) on the extended coset: element i is z[(i + 2^ext) mod N]."""
    v = ScalarArray(z.values, z.len)
    v.rotate(-(1 << ext))
    return v


class QuotientPipeline:
    def __init__(self, k: int, ext: int = 3, device="cuda"):
        self.k, self.ext = k, ext
        self.N = 1 << (k + ext)
        self.kernel = fused.quotient_kernel()
        self.zh = zh_inv_device(k, ext, device)
        self.ext_bufs = [ScalarArray.alloc(self.N, device) for _ in range(3)]
        self.out = ScalarArray.alloc(self.N, device)

    def run(self, a: ScalarArray, b: ScalarArray, c: ScalarArray, z: ScalarArray, stream=None) -> ScalarArray:
        """a, b, c are overwritten with their coefficients; returns the quotient buffer."""
        for src, dst in zip((a, b, c), self.ext_bufs):
            ntt.intt(src, stream)
            ntt.coset_ntt(dst, src, SHIFT, stream)
        ea, eb, ec = self.ext_bufs
        self.kernel([self.out], [ea, eb, ec, z, rotated(z, self.ext), self.zh], stream)
        return self.out
