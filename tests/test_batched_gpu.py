"""Batched form (uneven NTTs and MSMs in one captured graph) equals the per-call path."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_mixed_workload_batched_equals_plain(zk, orc):
    w = zk.batched.MixedWorkload(seed=3, n_ntt=20, ntt_lo=1, ntt_hi=15, n_msm=9, msm_lo=8, msm_hi=14)
    w.reset_inputs()
    w.run_plain()
    torch.cuda.synchronize()
    plain_ntt, plain_msm = w.snapshot()
    w.reset_inputs()
    for r in w.results:
        r.zero_()
    w.run_batched()
    torch.cuda.synchronize()
    bat_ntt, bat_msm = w.snapshot()
    for a, b in zip(plain_ntt, bat_ntt):
        assert torch.equal(a, b)
    for a, b in zip(plain_msm, bat_msm):
        assert torch.equal(a, b)
    # spot-check against the oracle: one NTT of each kind and two MSMs
    g = orc.to_mont(orc.int_to_limbs(7))
    seen = set()
    for i, (L, kind) in enumerate(zip(w.ntt_logs, w.ntt_kinds)):
        if kind in seen:
            continue
        seen.add(kind)
        a = w.ntt_init[i].cpu().numpy().view(np.uint64).reshape(-1, 4)
        exp = {"ntt": lambda: orc.ntt(a, L), "intt": lambda: orc.intt(a, L),
               "coset": lambda: orc.coset_ntt(a, L, L, g)}[kind]()
        assert np.array_equal(bat_ntt[i].cpu().numpy().view(np.uint64).reshape(-1, 4), exp), (L, kind)
    pts = orc.gen_points(2, 1 << max(w.msm_logs))
    for i in (0, len(w.msm_logs) - 1):
        n = 1 << w.msm_logs[i]
        s = w.scalars[i].cpu().numpy().view(np.uint64).reshape(-1, 4)
        assert np.array_equal(bat_msm[i].cpu().numpy().view(np.uint64), orc.best_multiexp(s, pts[:n]))
    # the per-call path through the reference ABI (host arrays for the MSMs) agrees as well
    w.reset_inputs()
    ref_msm = w.run_plain_ref_abi()
    torch.cuda.synchronize()
    ref_ntt, _ = w.snapshot()
    assert all(torch.equal(a, b) for a, b in zip(plain_ntt, ref_ntt))
    for a, b in zip(ref_msm, plain_msm):
        assert np.array_equal(a, b.cpu().numpy().view(np.uint32))
    # the per-call path over the batch's own resident tables and Shoup twiddle tables agrees
    w.reset_inputs()
    for r in w.results:
        r.zero_()
    w.run_plain_same_tables()
    torch.cuda.synchronize()
    same_ntt, same_msm = w.snapshot()
    assert all(torch.equal(a, b) for a, b in zip(plain_ntt, same_ntt))
    assert all(torch.equal(a, b) for a, b in zip(plain_msm, same_msm))
    # replay again: same results
    w.reset_inputs()
    w.run_batched()
    torch.cuda.synchronize()
    again_ntt, again_msm = w.snapshot()
    assert all(torch.equal(a, b) for a, b in zip(bat_ntt, again_ntt))
    assert all(torch.equal(a, b) for a, b in zip(bat_msm, again_msm))
