"""The allocation-free MSM entry point (zkp_msm_device_noalloc).

It exists for callers that cannot allocate device memory - a plugin whose host application only
hands it input and output buffers, or a loop that must not call cudaMalloc because that
synchronises the device.  Its workspace is a fixed array inside libmsm.so.  This file is
collected last so a failure here cannot hide the other tests; it passes alone in a fresh process
and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _call_noalloc(lib, pts, scalars, n, res, window=0):
    return lib.zkp_msm_device_noalloc(pts.data_ptr(), 1, scalars.data_ptr(), n, window, res.data_ptr(),
                                      torch.cuda.current_stream().cuda_stream)


def _call_workspace(lib, pts, scalars, n, res, window=0):
    size = lib.zkp_msm_workspace_size(n, window, 1)
    ws = torch.empty(size, dtype=torch.uint8, device="cuda")
    rc = lib.zkp_msm_device(ws.data_ptr(), size, pts.data_ptr(), 1, scalars.data_ptr(), n, window, res.data_ptr(),
                            torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return rc


def test_noalloc_matches_workspace_entry_two_calls(zk):
    lib = zk.native.load("libmsm.so")
    n = 1 << 14
    pts = zk.gen.points(2, n)
    for call, seed in enumerate((901, 902)):  # two calls in a row reuse the same fixed scratch
        scalars = zk.gen.fr(seed, n)
        got = torch.full((16,), -1, dtype=torch.int32, device="cuda")
        ref = torch.zeros(16, dtype=torch.int32, device="cuda")
        assert _call_noalloc(lib, pts, scalars, n, got) == 0, call
        torch.cuda.synchronize()
        assert _call_workspace(lib, pts, scalars, n, ref) == 0
        # exact integer arithmetic: the tolerance is zero
        assert torch.equal(got, ref), call


def test_noalloc_largest_fitting_size_and_refusal(zk):
    # the fixed array holds the layout without affine pairing rounds (the entry never runs
    # them), so the size queries below are made under that setting
    zk.msm.set_affine_rounds(0)
    try:
        _largest_fitting_size_and_refusal(zk)
    finally:
        zk.msm.set_affine_rounds(-1)


def _largest_fitting_size_and_refusal(zk):
    lib = zk.native.load("libmsm.so")
    cap = lib.zkp_msm_noalloc_capacity()
    assert cap == 64 << 20
    n = 1 << 15  # the largest power of two that fits with the default window
    assert lib.zkp_msm_workspace_size(n, 0, 1) <= cap < lib.zkp_msm_workspace_size(2 * n, 0, 1)
    pts = zk.gen.points(3, n)
    scalars = zk.gen.fr(903, n)
    got = torch.zeros(16, dtype=torch.int32, device="cuda")
    ref = torch.ones(16, dtype=torch.int32, device="cuda")
    assert _call_noalloc(lib, pts, scalars, n, got) == 0
    torch.cuda.synchronize()
    assert _call_workspace(lib, pts, scalars, n, ref) == 0
    assert torch.equal(got, ref)
    # a problem whose workspace exceeds the fixed array is refused before any device work
    # (the inputs are full size, so nothing could be read out of bounds either way)
    big = 1 << 20
    assert lib.zkp_msm_workspace_size(big, 0, 1) > cap
    big_pts = zk.gen.points(4, big)
    big_scalars = zk.gen.fr(904, big)
    untouched = torch.full((16,), 7, dtype=torch.int32, device="cuda")
    assert _call_noalloc(lib, big_pts, big_scalars, big, untouched) == 1  # cudaErrorInvalidValue
    torch.cuda.synchronize()
    assert int(untouched[0]) == 7
