"""Writes tests/golden/prover_k10/: the served prover program of size 2^10 as a compiled-program
artifact in the reference's serde forms (a version_<size>.json chunk, constants-manifest.json,
constants.bin), for the program tests.

The program text comes from the package (program.prover_artifact); its constants - the inverse
and forward root tables, n^-1, the coset powers 7^i, 1/Z_H on the 4x coset and the bases
k_i * G (seed 2) - are computed here by the CPU oracle, so the fixture does not depend on the
device code it tests.  Run from the repository root:  python tests/golden/make_prover_artifact.py
"""
import importlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402

K, EXT = 10, 2
OUT = os.path.join(ROOT, "tests", "golden", f"prover_k{K}")


def u32(a: np.ndarray, words: int = 8) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint64).view(np.uint32).reshape(-1, words)


def constants(k: int, ext: int) -> dict:
    n, N = 1 << k, 1 << (k + ext)
    g = orc.to_mont(orc.int_to_limbs(7))
    w = orc.root_of_unity(k + ext)
    gn = orc.pow_(g, n)
    zh = orc.batch_invert(np.stack([orc.sub(orc.mul(gn, orc.pow_(w, j * n)), orc.one()) for j in range(1 << ext)]))
    return {"inv_twiddle": u32(orc.twiddles(orc.root_of_unity(k, inverse=True), n // 2)),
            "fwd_twiddle": u32(orc.twiddles(w, N // 2)),
            "n_inv": u32(orc.inv(orc.to_mont(orc.int_to_limbs(n)))[None, :]),
            "coset_powers": u32(orc.twiddles(g, n)),
            "zh_inv": u32(zh),
            "bases": u32(orc.gen_points(2, n), 16)}


def main():
    orc.build()
    program = importlib.import_module("zkpoly-compiler_b200.program")
    parts = program.prover_artifact(K, constants(K, EXT), ext=EXT)
    print(program.dump_artifact(OUT, *parts))


if __name__ == "__main__":
    main()
