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


def test_noalloc_largest_fitting_size_and_refusal(zk, orc):
    # the fixed array holds the layout without affine pairing rounds (the entry never runs
    # them), so the size queries below are made under that setting
    zk.msm.set_affine_rounds(0)
    try:
        _largest_fitting_size_and_refusal(zk, orc)
    finally:
        zk.msm.set_affine_rounds(-1)


def _largest_fitting_size_and_refusal(zk, orc):
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
    # and against the CPU oracle (halo2 best_multiexp) on the same seeded inputs
    expect = orc.best_multiexp(orc.gen_fr(903, n), orc.gen_points(3, n))
    assert np.array_equal(got.cpu().numpy().view(np.uint64), expect)
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


def test_noalloc_precomputed_tables_and_window(zk, orc):
    """Precomputed tables and an explicit window change the workspace layout (windows per
    table, buckets, segments).  Window 16 over 2^12 points needs about 103 MiB with one table
    (refused) and about 28 MiB with four (fits)."""
    lib = zk.native.load("libmsm.so")
    n, window = 1 << 12, 16
    zk.msm.set_affine_rounds(0)
    try:
        cap = lib.zkp_msm_noalloc_capacity()
        assert lib.zkp_msm_workspace_size(n, window, 4) <= cap < lib.zkp_msm_workspace_size(n, window, 1)
        p = orc.gen_points(905, n)
        bases = zk.msm.ResidentBases(p, window=window, n_tables=4)  # tables by zkp_msm_precompute_device
        stream = torch.cuda.current_stream().cuda_stream
        for call, seed in enumerate((906, 907)):
            s = orc.gen_fr(seed, n)
            dev_s = torch.from_numpy(s.view(np.int32).reshape(n, 8).copy()).cuda()
            got = torch.full((16,), -1, dtype=torch.int32, device="cuda")
            assert lib.zkp_msm_device_noalloc(bases.tables.data_ptr(), 4, dev_s.data_ptr(), n, window,
                                              got.data_ptr(), stream) == 0, call
            size = lib.zkp_msm_workspace_size(n, window, 4)
            ws = torch.empty(size, dtype=torch.uint8, device="cuda")
            ref = torch.zeros(16, dtype=torch.int32, device="cuda")
            assert lib.zkp_msm_device(ws.data_ptr(), size, bases.tables.data_ptr(), 4, dev_s.data_ptr(), n,
                                      window, ref.data_ptr(), stream) == 0
            torch.cuda.synchronize()
            assert torch.equal(got, ref), call
            assert np.array_equal(got.cpu().numpy().view(np.uint64), orc.best_multiexp(s, p)), call
        # the same problem over the first table alone no longer fits: refused, output untouched
        untouched = torch.full((16,), 7, dtype=torch.int32, device="cuda")
        assert lib.zkp_msm_device_noalloc(bases.tables.data_ptr(), 1, dev_s.data_ptr(), n, window,
                                          untouched.data_ptr(), stream) == 1  # cudaErrorInvalidValue
        torch.cuda.synchronize()
        assert int(untouched[0]) == 7
    finally:
        zk.msm.set_affine_rounds(-1)


def _driver():
    cu = ctypes.CDLL("libcuda.so.1")
    for name in ("cuInit", "cuDeviceGet", "cuCtxCreate_v2", "cuCtxPopCurrent_v2", "cuCtxDestroy_v2",
                 "cuMemAlloc_v2", "cuMemFree_v2", "cuMemcpyHtoD_v2", "cuMemcpyDtoH_v2", "cuCtxSynchronize"):
        getattr(cu, name).restype = ctypes.c_int
    cu.cuMemcpyHtoD_v2.argtypes = [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_size_t]
    cu.cuMemcpyDtoH_v2.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_size_t]
    cu.cuMemFree_v2.argtypes = [ctypes.c_uint64]
    return cu


def test_noalloc_in_a_context_the_host_created(zk, orc):
    """A host application may run the plugin under its own driver-API context instead of the
    runtime's primary context.  The array's address differs between contexts, so the entry
    looks it up per context: a call made in a second context on the same GPU uses that
    context's copy and gives the same result as one made in the primary context."""
    lib = zk.native.load("libmsm.so")
    n = 1 << 12
    s, p = orc.gen_fr(908, n), orc.gen_points(909, n)
    expect = orc.best_multiexp(s, p)
    # the primary context (torch's) first, so both contexts hold a cached entry afterwards
    got = torch.zeros(16, dtype=torch.int32, device="cuda")
    dev_p = torch.from_numpy(p.view(np.int32).reshape(n, 16).copy()).cuda()
    dev_s = torch.from_numpy(s.view(np.int32).reshape(n, 8).copy()).cuda()
    assert _call_noalloc(lib, dev_p, dev_s, n, got) == 0
    torch.cuda.synchronize()
    assert np.array_equal(got.cpu().numpy().view(np.uint64), expect)

    cu = _driver()
    assert cu.cuInit(0) == 0
    dev = ctypes.c_int()
    assert cu.cuDeviceGet(ctypes.byref(dev), torch.cuda.current_device()) == 0
    ctx = ctypes.c_void_p()
    if cu.cuCtxCreate_v2(ctypes.byref(ctx), 0, dev) != 0:
        pytest.skip("this GPU does not allow a second context in the process")
    bufs = []
    try:
        h_p = np.ascontiguousarray(p.view(np.uint32))
        h_s = np.ascontiguousarray(s.view(np.uint32))
        out = np.full(16, 0xFFFFFFFF, dtype=np.uint32)
        for nbytes in (h_p.nbytes, h_s.nbytes, out.nbytes):
            d = ctypes.c_uint64()
            assert cu.cuMemAlloc_v2(ctypes.byref(d), ctypes.c_size_t(nbytes)) == 0
            bufs.append(d.value)
        assert cu.cuMemcpyHtoD_v2(bufs[0], h_p.ctypes.data, h_p.nbytes) == 0
        assert cu.cuMemcpyHtoD_v2(bufs[1], h_s.ctypes.data, h_s.nbytes) == 0
        for call in range(2):
            # the null stream of the context current on this thread: the host's own context
            assert lib.zkp_msm_device_noalloc(bufs[0], 1, bufs[1], n, 0, bufs[2], None) == 0, call
            assert cu.cuCtxSynchronize() == 0
            assert cu.cuMemcpyDtoH_v2(out.ctypes.data, bufs[2], out.nbytes) == 0
            assert np.array_equal(out.view(np.uint64), expect), call
    finally:
        for d in bufs:
            cu.cuMemFree_v2(d)
        popped = ctypes.c_void_p()
        cu.cuCtxPopCurrent_v2(ctypes.byref(popped))
        cu.cuCtxDestroy_v2(ctx)
    # the primary context's cached entry still serves torch's stream
    again = torch.zeros(16, dtype=torch.int32, device="cuda")
    assert _call_noalloc(lib, dev_p, dev_s, n, again) == 0
    torch.cuda.synchronize()
    assert torch.equal(again, got)
