"""Shared pytest setup: the ``gpu`` marker, import paths and small helpers."""
import importlib
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def load_package():
    """Import the zkpoly-compiler_b200 package (its directory name is not an identifier)."""
    mod = importlib.import_module("zkpoly-compiler_b200")
    sys.modules.setdefault("zkpoly_b200", mod)
    return mod


@pytest.fixture(scope="session")
def zk():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "reference_vectors.json")) as f:
        return json.load(f)


def u32_to_u64(v):
    a = np.asarray(v, dtype=np.uint64)
    return (a[0::2] | (a[1::2] << np.uint64(32))).astype(np.uint64)


def u32_to_int(v):
    return sum(int(x) << (32 * i) for i, x in enumerate(v))


def lookup_case(zk, n, usable, seed):
    """A lookup instance shaped like the reference's permute test (core/tests/poly.rs:569-625):
    table values uniform below 2n, inputs drawn from the distinct values of the table's usable
    rows; returned as Montgomery device arrays (converted on the device by multiplying the
    canonical values by R^2)."""
    import torch
    rng = np.random.default_rng(seed)
    table = rng.integers(0, 2 * n, n, dtype=np.uint64)
    distinct = np.unique(table[:usable])
    inp = distinct[rng.integers(0, len(distinct), n)]
    # raw words of R^2 mod r (the Montgomery form of R): multiplying by it maps x to x * R
    r2 = np.array(zk.field.mont_words((1 << 256) % zk.field.FR_MODULUS), dtype=np.uint32)
    out = []
    for vals in (inp, table):
        limbs = np.zeros((n, 8), dtype=np.uint32)
        limbs[:, 0] = vals.astype(np.uint32)
        arr = zk.ScalarArray.from_numpy(limbs)
        powers = zk.ScalarArray.from_numpy(r2.reshape(1, 8))
        zk.ntt.distribute_powers(arr, powers)
        out.append(arr)
    torch.cuda.synchronize()
    return out
