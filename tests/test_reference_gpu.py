"""The reference's own CUDA kernels, built from its sources into oracle/_ref (oracle/build_ref.py),
run next to this repository's kernels on the same inputs: NTT (ssip_ntt), MSM (msm, two of the
reference's library configurations) and the poly library (permute, poly_eval, batched_invert,
kate_division, scan_mul) must agree bit for bit.  Skipped when oracle/_ref was not
built (no reference checkout where the libraries were built).

With ZKP_REF_TIMING=1 the tests also time both sides (CUDA events for the NTT, host clock for
the synchronous host-buffer MSM ABI) and print one JSON line per comparison."""
import ctypes
import json
import os
import time

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

REF_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")
TIMING = os.environ.get("ZKP_REF_TIMING") == "1"


def _ref_lib(name):
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not built (reference checkout absent at build time)")
    return ctypes.CDLL(path)


def _ref_ntt(zk):
    lib = _ref_lib("libref_ntt.so")
    lib.ssip_ntt.restype = ctypes.c_int
    lib.ssip_ntt.argtypes = [zk.native.PolyPtr, ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p, ctypes.c_uint,
                             ctypes.c_uint]
    return lib


def _ref_msm(name):
    lib = _ref_lib(name)
    lib.msm.restype = ctypes.c_int
    lib.msm.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_uint, ctypes.c_uint,
                        ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint,
                        ctypes.c_void_p, ctypes.c_void_p]
    lib.msm_precompute.restype = ctypes.c_int
    lib.msm_precompute.argtypes = [ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_uint]
    return lib


def _call_msm(lib, n, tables, scalars, parts, stages):
    """One call of the reference-ABI msm with host tables and host scalar batches (the runtime's
    call, core/src/msm.rs:302-369); returns the affine results and the host-clock seconds."""
    cards = (ctypes.c_uint * 1)(0)
    sizes = (ctypes.c_ulong * 1)()
    assert lib.msm(None, sizes, n, 1, parts, stages, stages, 1, cards, None, 0, None, None) == 0
    buf = torch.empty(int(sizes[0]), dtype=torch.uint8, device="cuda")
    bufs = (ctypes.c_void_p * 1)(buf.data_ptr())
    h_points = (ctypes.c_void_p * len(tables))(*[t.ctypes.data for t in tables])
    h_scal = (ctypes.c_void_p * len(scalars))(*[s.ctypes.data for s in scalars])
    results = [np.zeros(16, dtype=np.uint32) for _ in scalars]
    h_res = (ctypes.c_void_p * len(results))(*[r.ctypes.data for r in results])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = lib.msm(bufs, None, n, 1, parts, stages, stages, 1, cards, h_points, len(scalars), h_scal, h_res)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    assert rc == 0
    return results, dt


def _pinned_u32(t: torch.Tensor) -> np.ndarray:
    return t.cpu().pin_memory().numpy().view(np.uint32)


@pytest.mark.parametrize("log_n", [4, 10, 13, 16, 20, 24])
def test_reference_ssip_ntt_matches(zk, log_n):
    ref = _ref_ntt(zk)
    n = 1 << log_n
    data = zk.gen.fr(300 + log_n, n)
    tw = zk.ntt.twiddle_table(log_n)
    x_ref, x, x_sh = (zk.ScalarArray(data.clone()) for _ in range(3))
    stream = torch.cuda.current_stream().cuda_stream
    assert ref.ssip_ntt(x_ref.poly_ptr(), tw.values.data_ptr(), log_n, stream, 8, 8) == 0
    zk.ntt.ssip_ntt(x, tw)
    zk.ntt.ntt(x_sh)  # the library's own transform (Shoup twiddle table)
    torch.cuda.synchronize()
    assert torch.equal(x_ref.values, x.values)
    assert torch.equal(x_ref.values, x_sh.values)
    if TIMING and log_n >= 20:
        def t(fn, reps=5):
            fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps
        ms_ref = t(lambda: ref.ssip_ntt(x_ref.poly_ptr(), tw.values.data_ptr(), log_n, stream, 8, 8))
        ms = t(lambda: zk.ntt.ssip_ntt(x, tw))
        ms_sh = t(lambda: zk.ntt.ntt(x_sh))
        print(json.dumps({"compare": "ssip_ntt", "log_n": log_n, "reference_ms": ms_ref, "this_ms": ms,
                          "speedup": ms_ref / ms, "this_shoup_ms": ms_sh, "speedup_shoup": ms_ref / ms_sh}))


@pytest.mark.parametrize("log_n", [4, 12, 17, 22])
def test_reference_recompute_ntt_matches(zk, log_n):
    """recompute_ntt (roots rebuilt from omegas and the pq table) and gen_pq_omegas against the
    reference's own (recompute_ntt.cuh:362-438, precompute.cuh:89-113) on the same input; then
    distribute_powers (distribute_powers.cuh:5-21) with a short powers array."""
    ref = _ref_lib("libref_ntt.so")
    ref.recompute_ntt.restype = ctypes.c_int
    ref.recompute_ntt.argtypes = [zk.native.PolyPtr, ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p, ctypes.c_uint,
                                  ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint]
    ref.gen_pq_omegas.restype = None
    ref.gen_pq_omegas.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, ctypes.c_void_p]
    ref.distribute_powers.restype = ctypes.c_int
    ref.distribute_powers.argtypes = [zk.native.PolyPtr, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_void_p]
    n = 1 << log_n
    w = np.ascontiguousarray(zk.field.mont_words(zk.field.root_of_unity(log_n)), dtype=np.uint32).copy()
    pq_len = zk.ntt.get_pq_len(log_n)
    pq_deg = int(np.log2(pq_len)) + 1
    pq, omegas = zk.ntt.gen_pq_omegas(pq_len, n, w)
    pq_ref, om_ref = np.zeros_like(pq), np.zeros_like(omegas)
    ref.gen_pq_omegas(pq_ref.ctypes.data, om_ref.ctypes.data, pq_deg, n, w.ctypes.data)
    assert np.array_equal(pq, pq_ref) and np.array_equal(omegas, om_ref)
    data = zk.gen.fr(350 + log_n, n)
    x_ref, x = zk.ScalarArray(data.clone()), zk.ScalarArray(data.clone())
    pq_d, om_d = zk.ScalarArray.from_numpy(pq), zk.ScalarArray.from_numpy(omegas)
    st = torch.cuda.current_stream().cuda_stream
    assert ref.recompute_ntt(x_ref.poly_ptr(), pq_d.values.data_ptr(), pq_deg, om_d.values.data_ptr(), log_n, st,
                             8, 8) == 0
    zk.ntt.recompute_ntt(x, pq_d, om_d)
    torch.cuda.synchronize()
    assert torch.equal(x_ref.values, x.values)
    powers = zk.ScalarArray(zk.gen.fr(360, 7))
    assert ref.distribute_powers(x_ref.poly_ptr(), powers.values.data_ptr(), 7, st) == 0
    zk.ntt.distribute_powers(x, powers)
    torch.cuda.synchronize()
    assert torch.equal(x_ref.values, x.values)


@pytest.mark.parametrize("log_n", [10, 16])
def test_reference_msm_one_table_matches(zk, log_n):
    """The runtime's default library (window 16, 16 target windows: one table)."""
    ref = _ref_msm("libref_msm_16_16.so")
    n = 1 << log_n
    pts = _pinned_u32(zk.gen.points(2, n))
    scal = [_pinned_u32(zk.gen.fr(400 + i, n)) for i in range(2)]
    got, _ = _call_msm(ref, n, [pts], scal, parts=1, stages=1)
    ours = zk.msm.msm_host_batches(scal, [pts])
    for a, b in zip(got, ours):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("log_n", [16, 20, 22])
def test_reference_msm_precomputed_matches(zk, log_n):
    """The reference cost model's configuration for 2^22 points (window 17, 8 target windows:
    two point tables built by the reference's msm_precompute, 16 parts, two stages)."""
    ref = _ref_msm("libref_msm_17_8.so")
    n = 1 << log_n
    pts_dev = zk.gen.points(2, n)
    tables = [_pinned_u32(pts_dev), np.zeros((n, 16), dtype=np.uint32)]
    h_tab = (ctypes.c_void_p * 2)(*[t.ctypes.data for t in tables])
    assert ref.msm_precompute(n, h_tab, 1) == 0
    scal_dev = zk.gen.fr(500, n)
    scal = [_pinned_u32(scal_dev)]
    parts = 16 if n >= (1 << 16) else 1
    got, dt_ref = _call_msm(ref, n, tables, scal, parts=parts, stages=2 if parts > 1 else 1)
    ours = zk.msm.msm_host_batches(scal, [tables[0]])
    assert np.array_equal(got[0], ours[0])
    if TIMING:
        # best of 3 for both sides; this repository's side twice: the same host-buffer ABI (one
        # table) and the device-resident form with the tuned precomputed tables
        dt_ref = min(dt_ref, *[_call_msm(ref, n, tables, scal, parts, 2)[1] for _ in range(2)])
        dt = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            zk.msm.msm_host_batches(scal, [tables[0]])
            torch.cuda.synchronize()
            dt.append(time.perf_counter() - t0)
        c, nt = zk.tuner.msm_resident_config(n)
        rb = zk.msm.ResidentBases(pts_dev, window=c, n_tables=nt)
        ws = rb.workspace()
        res = torch.zeros(16, dtype=torch.int32, device="cuda")
        rb.msm(scal_dev, res, ws)
        torch.cuda.synchronize()
        assert np.array_equal(res.cpu().numpy().view(np.uint32), got[0])
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            rb.msm(scal_dev, res, ws)
        e1.record()
        torch.cuda.synchronize()
        print(json.dumps({"compare": "msm host-buffer ABI", "log_n": log_n, "reference_s17_t8_ms": dt_ref * 1e3,
                          "this_abi_ms": min(dt) * 1e3, "this_resident_ms": e0.elapsed_time(e1) / 5,
                          "resident_config": [c, nt]}))


def test_reference_permute_matches(zk):
    """permute at 2^20 rows (24 + 1 blinding rows unused, as in the reference's test) against the
    reference's own CUB-based permute."""
    from conftest import lookup_case
    ref = _ref_lib("libref_poly.so")
    ref.permute.restype = ctypes.c_int
    ref.permute.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_ulong), ctypes.c_ulong, zk.native.PolyPtr,
                            zk.native.PolyPtr, zk.native.PolyPtr, zk.native.PolyPtr, ctypes.c_void_p]
    n = 1 << 20
    usable = n - 25
    inp, table = lookup_case(zk, n, usable, 5)
    outs = [zk.ScalarArray.alloc(usable) for _ in range(4)]
    size = ctypes.c_ulong(0)
    st = torch.cuda.current_stream().cuda_stream
    assert ref.permute(None, ctypes.byref(size), usable, inp.poly_ptr(), table.poly_ptr(), outs[0].poly_ptr(),
                       outs[1].poly_ptr(), st) == 0
    tmp = torch.empty(size.value, dtype=torch.uint8, device="cuda")
    run_ref = lambda: ref.permute(tmp.data_ptr(), ctypes.byref(size), usable, inp.poly_ptr(), table.poly_ptr(),
                                  outs[0].poly_ptr(), outs[1].poly_ptr(), st)
    assert run_ref() == 0
    zk.poly.permute(inp, table, usable, outs[2], outs[3])
    torch.cuda.synchronize()
    assert torch.equal(outs[0].values, outs[2].values)
    assert torch.equal(outs[1].values, outs[3].values)
    if TIMING:
        def t(fn, reps=5):
            fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps
        ms_ref = t(run_ref)
        ms = t(lambda: zk.poly.permute(inp, table, usable, outs[2], outs[3]))
        print(json.dumps({"compare": "permute", "rows": usable, "reference_ms": ms_ref, "this_ms": ms,
                          "speedup": ms_ref / ms}))


def _ref_poly(zk):
    lib = _ref_lib("libref_poly.so")
    P, V, UL = zk.native.PolyPtr, ctypes.c_void_p, ctypes.POINTER(ctypes.c_ulong)
    for name, args in (("poly_eval", [V, UL, P, V, V, V]), ("batched_invert", [V, UL, P, V]),
                       ("kate_division", [V, UL, ctypes.c_uint, P, V, P, V]), ("scan_mul", [V, UL, P, V])):
        getattr(lib, name).restype = ctypes.c_int
        getattr(lib, name).argtypes = args
    return lib


def _temp_for(fn, *args):
    size = ctypes.c_ulong(0)
    assert fn(None, ctypes.byref(size), *args) == 0
    return torch.empty(max(size.value, 1), dtype=torch.uint8, device="cuda"), size


def _event_ms(fn, reps=5):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


@pytest.mark.parametrize("log_n", [10, 20, 22])
def test_reference_poly_library_matches(zk, log_n):
    """poly_eval, batched_invert (with zeros), kate_division and scan_mul against the reference's
    own kernels on the same inputs; timed side by side at 2^22 with ZKP_REF_TIMING=1."""
    ref = _ref_poly(zk)
    n = 1 << log_n
    st = torch.cuda.current_stream().cuda_stream
    p = zk.ScalarArray(zk.gen.fr(800 + log_n, n))
    x = zk.gen.fr(801, 1)
    # poly_eval
    res_ref = torch.zeros(8, dtype=torch.int32, device="cuda")
    res = torch.zeros(8, dtype=torch.int32, device="cuda")
    tmp, size = _temp_for(ref.poly_eval, p.poly_ptr(), None, None, None)
    assert ref.poly_eval(tmp.data_ptr(), ctypes.byref(size), p.poly_ptr(), res_ref.data_ptr(), x.data_ptr(), st) == 0
    zk.poly.poly_eval(p, x, res)
    torch.cuda.synchronize()
    assert torch.equal(res_ref, res)
    # batched_invert, every 7th element zero
    v = p.values.clone()
    v[::7] = 0
    a_ref, a = zk.ScalarArray(v.clone()), zk.ScalarArray(v.clone())
    tmp, size = _temp_for(ref.batched_invert, a_ref.poly_ptr(), None)
    assert ref.batched_invert(tmp.data_ptr(), ctypes.byref(size), a_ref.poly_ptr(), st) == 0
    zk.poly.batched_invert(a)
    torch.cuda.synchronize()
    assert torch.equal(a_ref.values, a.values)
    # kate_division: q = p / (X - b), length n
    q_ref, q = zk.ScalarArray.zeros(n), zk.ScalarArray.zeros(n)
    tmp, size = _temp_for(ref.kate_division, log_n, p.poly_ptr(), None, q_ref.poly_ptr(), None)
    assert ref.kate_division(tmp.data_ptr(), ctypes.byref(size), log_n, p.poly_ptr(), x.data_ptr(),
                             q_ref.poly_ptr(), st) == 0
    zk.poly.kate_division(p, x, q)
    torch.cuda.synchronize()
    assert torch.equal(q_ref.values, q.values)
    # scan_mul (inclusive product scan in place)
    s_ref, s_ = zk.ScalarArray(p.values.clone()), zk.ScalarArray(p.values.clone())
    tmp, size = _temp_for(ref.scan_mul, s_ref.poly_ptr(), None)
    assert ref.scan_mul(tmp.data_ptr(), ctypes.byref(size), s_ref.poly_ptr(), st) == 0
    zk.poly.scan_mul(s_)
    torch.cuda.synchronize()
    assert torch.equal(s_ref.values, s_.values)
    if TIMING and log_n == 22:
        t_eval, z_eval = _temp_for(ref.poly_eval, p.poly_ptr(), None, None, None)
        t_inv, z_inv = _temp_for(ref.batched_invert, a_ref.poly_ptr(), None)
        t_kate, z_kate = _temp_for(ref.kate_division, log_n, p.poly_ptr(), None, q_ref.poly_ptr(), None)
        t_scan, z_scan = _temp_for(ref.scan_mul, s_ref.poly_ptr(), None)
        cases = [
            ("poly_eval", lambda: ref.poly_eval(t_eval.data_ptr(), ctypes.byref(z_eval), p.poly_ptr(),
                                                res_ref.data_ptr(), x.data_ptr(), st),
             lambda: zk.poly.poly_eval(p, x, res)),
            ("batched_invert", lambda: ref.batched_invert(t_inv.data_ptr(), ctypes.byref(z_inv), a_ref.poly_ptr(), st),
             lambda: zk.poly.batched_invert(a)),
            ("kate_division", lambda: ref.kate_division(t_kate.data_ptr(), ctypes.byref(z_kate), log_n, p.poly_ptr(),
                                                        x.data_ptr(), q_ref.poly_ptr(), st),
             lambda: zk.poly.kate_division(p, x, q)),
            ("scan_mul", lambda: ref.scan_mul(t_scan.data_ptr(), ctypes.byref(z_scan), s_ref.poly_ptr(), st),
             lambda: zk.poly.scan_mul(s_)),
        ]
        for name, run_ref, run in cases:
            ms_ref, ms = _event_ms(run_ref), _event_ms(run)
            print(json.dumps({"compare": name, "log_n": log_n, "reference_ms": ms_ref, "this_ms": ms,
                              "speedup": ms_ref / ms}))


def test_reference_batched_workload_per_call(zk):
    """Config 4's workload (seed 3: 64 NTTs 2^10..2^20 of mixed kinds, 16 MSMs 2^12..2^22)
    through the reference's own kernels one call at a time - ssip_ntt, with distribute_powers
    for the inverse's n^-1 and the coset's g^i (the compiler's composition), and the
    reference-ABI msm with host arrays from libref_msm_17_8 (its cost model's 2^22
    configuration, two tables built by msm_precompute per size) - must give this repository's
    batched results; with ZKP_REF_TIMING=1 both sides are timed."""
    ref_ntt = _ref_ntt(zk)
    ref_ntt.distribute_powers.restype = ctypes.c_int
    ref_ntt.distribute_powers.argtypes = [zk.native.PolyPtr, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_void_p]
    ref_msm = _ref_msm("libref_msm_17_8.so")
    w = zk.batched.MixedWorkload(seed=3)
    w.build_batched()
    w.reset_inputs()
    w.run_batched()
    torch.cuda.synchronize()
    ntt_ours, msm_ours = w.snapshot()
    st = torch.cuda.current_stream().cuda_stream
    # reference-side set-up (untimed): twiddles, inverse scales, coset powers, point tables
    tw = {(L, inv): zk.ntt.twiddle_table(L, inv) for L in set(w.ntt_logs) for inv in (False, True)}
    ninv = {L: zk.ntt.n_inv(L) for L in set(w.ntt_logs)}
    coset = {}
    for L, kind in zip(w.ntt_logs, w.ntt_kinds):
        if kind == "coset" and L not in coset:
            p = zk.ntt.scalar_const(7).repeat(1 << L, 1)
            p[0] = zk.ntt.scalar_const(1)[0]
            pa = zk.ScalarArray(p)
            zk.poly.scan_mul(pa)  # g^i
            coset[L] = pa
    tables = {}
    for L in set(w.msm_logs):
        n = 1 << L
        t = [_pinned_u32(w.bases[:n]), np.zeros((n, 16), dtype=np.uint32)]
        h_tab = (ctypes.c_void_p * 2)(*[a.ctypes.data for a in t])
        assert ref_msm.msm_precompute(n, h_tab, 1) == 0
        tables[L] = t
    h_scal = [_pinned_u32(s) for s in w.scalars]
    bufs = [zk.ScalarArray(t.clone()) for t in w.ntt_init]
    torch.cuda.synchronize()

    def run_reference():
        for x, t0, L, kind in zip(bufs, w.ntt_init, w.ntt_logs, w.ntt_kinds):
            x.values.copy_(t0)
            if kind == "coset":
                assert ref_ntt.distribute_powers(x.poly_ptr(), coset[L].values.data_ptr(), 1 << L, st) == 0
            assert ref_ntt.ssip_ntt(x.poly_ptr(), tw[(L, kind == "intt")].values.data_ptr(), L, st, 8, 8) == 0
            if kind == "intt":
                assert ref_ntt.distribute_powers(x.poly_ptr(), ninv[L].data_ptr(), 1, st) == 0
        out = []
        for hs, L in zip(h_scal, w.msm_logs):
            n = 1 << L
            parts = 16 if n >= (1 << 16) else 1
            res, _ = _call_msm(ref_msm, n, tables[L], [hs], parts=parts, stages=2 if parts > 1 else 1)
            out.append(res[0])
        torch.cuda.synchronize()
        return out

    msm_ref = run_reference()
    for a, b in zip(bufs, ntt_ours):
        assert torch.equal(a.values, b)
    for a, b in zip(msm_ref, msm_ours):
        assert np.array_equal(a, b.cpu().numpy().view(np.uint32))
    if TIMING:
        ref_ms = float("inf")
        for _ in range(3):  # best of three: the reference's msm allocates and frees per call
            t0 = time.perf_counter()
            run_reference()
            ref_ms = min(ref_ms, (time.perf_counter() - t0) * 1e3)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            w.run_batched()
        e1.record()
        torch.cuda.synchronize()
        batched_ms = e0.elapsed_time(e1) / 3
        print(json.dumps({"compare": "config-4 workload", "reference_per_call_ms": ref_ms,
                          "this_batched_ms": batched_ms, "speedup": ref_ms / batched_ms}))
