"""The exact configurations bench.py times, checked bit for bit against the CPU oracle.

The benchmark's MSM is one 2^22-point MSM over resident bases with the tuned (window, tables)
pair and the library's pairing rounds; its NTT is the 2^24 forward transform with the Shoup
twiddle table (zkp_ntt_ex_shoup), and its e2e leg is ssip_ntt on the Montgomery root table.
Each is run here as the benchmark runs it and compared with halo2's best_multiexp / best_fft as
restated by the oracle, on the same seeded inputs (scalars seed 1, points k_i*G with k_i from
seed 2, NTT input seed 0).  One served request at the largest size of the serving workload
(k = 22) is checked against the oracle's restatement of the whole program.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

MSM_LOG, NTT_LOG = 22, 24


@pytest.fixture(scope="module")
def msm_inputs(orc):
    n = 1 << MSM_LOG
    s, p = orc.gen_fr(1, n), orc.gen_points(2, n)
    return s, p, orc.best_multiexp(s, p)


@pytest.fixture(scope="module")
def ntt_inputs(orc):
    a = orc.gen_fr(0, 1 << NTT_LOG)
    return a, orc.best_fft(a, orc.root_of_unity(NTT_LOG), NTT_LOG)


def _bench_msm_configs(zk):
    """The (window, tables) pair bench.py uses (the tuner's resident pair for 2^22), and the
    pair the shipped B200 tuning names, c = 20 with 13 tables (one table per window)."""
    return sorted({tuple(zk.tuner.msm_resident_config(1 << MSM_LOG)), (20, 13)})


def test_msm_2_22_resident_bench_config(zk, orc, msm_inputs):
    s, p, expect = msm_inputs
    n = 1 << MSM_LOG
    scalars = zk.gen.fr(1, n)
    points = zk.gen.points(2, n)
    for window, n_tables in _bench_msm_configs(zk):
        rounds = zk.msm.rounds_for(n, window, n_tables)
        assert rounds >= 1  # the benchmarked call runs the affine pairing rounds
        bases = zk.msm.ResidentBases(points, window=window, n_tables=n_tables)
        ws = bases.workspace()
        res = torch.full((16,), -1, dtype=torch.int32, device="cuda")
        for rep in range(2):  # the benchmark reuses the workspace step after step
            bases.msm(scalars, res, ws)
            torch.cuda.synchronize()
            got = res.cpu().numpy().view(np.uint64)
            assert np.array_equal(got, expect), (window, n_tables, rounds, rep)
        del bases, ws
        torch.cuda.empty_cache()


def test_msm_2_22_three_rounds_explicit(zk, orc, msm_inputs):
    """c = 20, 13 tables with exactly three pairing rounds (the benchmark's count at 2^22)."""
    s, p, expect = msm_inputs
    n = 1 << MSM_LOG
    zk.msm.set_affine_rounds(3)
    try:
        bases = zk.msm.ResidentBases(zk.gen.points(2, n), window=20, n_tables=13)
        assert zk.msm.rounds_for(n, 20, 13) == 3
        res = torch.zeros(16, dtype=torch.int32, device="cuda")
        bases.msm(zk.gen.fr(1, n), res, bases.workspace())
        torch.cuda.synchronize()
        assert np.array_equal(res.cpu().numpy().view(np.uint64), expect)
    finally:
        zk.msm.set_affine_rounds(-1)
    torch.cuda.empty_cache()


def test_ntt_2_24_shoup_matches_best_fft(zk, orc, ntt_inputs):
    """The benchmark's timed transform: zkp_ntt_ex_shoup at 2^24, every element."""
    a, expect = ntt_inputs
    x = zk.ScalarArray(zk.gen.fr(0, 1 << NTT_LOG))
    zk.ntt.ntt_ex(x, zk.ntt.twiddle_table(NTT_LOG), shoup=zk.ntt.shoup_table(NTT_LOG))
    torch.cuda.synchronize()
    assert np.array_equal(x.numpy_u64(), expect)


def test_ssip_ntt_2_24_matches_best_fft(zk, orc, ntt_inputs):
    """The reference-ABI transform the e2e leg times (Montgomery root table only)."""
    a, expect = ntt_inputs
    x = zk.ScalarArray.from_numpy(a)
    zk.ntt.ssip_ntt(x, zk.ntt.twiddle_table(NTT_LOG))
    torch.cuda.synchronize()
    assert np.array_equal(x.numpy_u64(), expect)


def test_served_request_k22_matches_oracle(zk, orc):
    """One request of the serving workload's largest size through the served form."""
    from test_serving_gpu import expected
    k, seed = 22, 7
    # the bench's served form: resident table sets with the tuned (window, tables) per size
    sets = zk.serving.resident_sets(zk.gen.points(2, 1 << k), k, k)
    srv = zk.serving.Server(sets, hbm_bytes=24 << 30, max_inflight=2, ext_log=2, min_k=k, max_k=k)
    try:
        res = srv.wait(srv.submit(k, seed))
        assert res.status == 0
        assert np.array_equal(zk.serving.result_words(res), expected(orc, k, seed))
    finally:
        srv.close()
    del sets
    torch.cuda.empty_cache()
