"""MSM on the GPU, bit-exact (canonical affine) against the oracle's halo2 best_multiexp."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 2, 7, 100, 1000, 4096])
def test_msm_reference_abi_small(zk, orc, n):
    s = orc.gen_fr(100 + n, n)
    p = orc.gen_points(200 + n, n)
    assert np.array_equal(zk.msm.msm_host(s, p), orc.best_multiexp(s, p))


def test_msm_edge_cases(zk, orc):
    n = 3000
    s = orc.gen_fr(31, n)
    p = orc.gen_points(32, n)
    s[0:50] = 0                                  # zero scalars
    p[50:60] = 0                                 # identity bases
    p[60:70] = p[70:80]                          # repeated bases -> doubling inside a bucket
    s[60:70] = s[70:80]
    s[80] = orc.neg(s[81])                       # cancelling pair
    p[80] = p[81]
    s[90] = orc.to_mont(orc.int_to_limbs(1))     # scalar 1
    s[91] = orc.neg(orc.to_mont(orc.int_to_limbs(1)))  # r - 1
    assert np.array_equal(zk.msm.msm_host(s, p), orc.best_multiexp(s, p))


def test_msm_all_equal_scalars_one_bucket(zk, orc):
    """Every digit lands in the same bucket of each window: runs cross many chunks."""
    n = 1 << 14
    s = np.repeat(orc.gen_fr(41, 1), n, axis=0)
    p = orc.gen_points(42, n)
    assert np.array_equal(zk.msm.msm_host(s, p), orc.best_multiexp(s, p))


def test_msm_zero_result_and_all_zero(zk, orc):
    n = 64
    p = orc.gen_points(43, n)
    s = np.zeros((n, 4), dtype=np.uint64)
    assert np.array_equal(zk.msm.msm_host(s, p), np.zeros(8, dtype=np.uint64))
    s = orc.gen_fr(44, n)
    s[n // 2:] = np.stack([orc.neg(x) for x in s[: n // 2]])
    p[n // 2:] = p[: n // 2]
    assert np.array_equal(zk.msm.msm_host(s, p), np.zeros(8, dtype=np.uint64))


@pytest.mark.parametrize("window", [8, 11, 13, 16, 20])
def test_msm_device_windows(zk, orc, window):
    n = 5000
    s = orc.gen_fr(50 + window, n)
    p = orc.gen_points(60 + window, n)
    bases = zk.msm.ResidentBases(p, window=window)
    res = torch.zeros(16, dtype=torch.int32, device="cuda")
    dev_s = torch.from_numpy(s.view(np.int32).reshape(n, 8).copy()).cuda()
    bases.msm(dev_s, res, bases.workspace())
    got = res.cpu().numpy().view(np.uint64)
    assert np.array_equal(got, orc.best_multiexp(s, p))


@pytest.mark.parametrize("window,n_tables", [(16, 2), (13, 4), (16, 16)])
def test_msm_precomputed_tables(zk, orc, window, n_tables):
    n = 3000
    s = orc.gen_fr(70 + n_tables, n)
    p = orc.gen_points(80 + n_tables, n)
    bases = zk.msm.ResidentBases(p, window=window, n_tables=n_tables)
    res = torch.zeros(16, dtype=torch.int32, device="cuda")
    ws = bases.workspace()
    for trial in range(2):  # workspace reuse
        dev_s = torch.from_numpy(s.view(np.int32).reshape(n, 8).copy()).cuda()
        bases.msm(dev_s, res, ws)
        assert np.array_equal(res.cpu().numpy().view(np.uint64), orc.best_multiexp(s, p)), trial
        s = orc.gen_fr(90 + trial, n)


def test_msm_batches_share_points(zk, orc):
    n = 2000
    p = orc.gen_points(91, n)
    batches = [orc.gen_fr(92 + b, n) for b in range(4)]
    res = zk.msm.msm_host_batches([b.view(np.uint32).reshape(n, 8) for b in batches],
                                  [p.view(np.uint32).reshape(n, 16)])
    for b, r in zip(batches, res):
        assert np.array_equal(r.view(np.uint64), orc.best_multiexp(b, p))


def test_msm_size_query(zk):
    sizes = zk.msm.MSM().get_buffer_size(1 << 20)
    assert len(sizes) == 1 and sizes[0] > (1 << 20) * 96


def test_config2_msm_2_20(zk, orc):
    """n = 2^20, scalars seed 1, points k_i * G with k_i from seed 2."""
    n = 1 << 20
    s = orc.gen_fr(1, n)
    p = orc.gen_points(2, n)
    assert np.array_equal(zk.msm.msm_host(s, p), orc.best_multiexp(s, p))


def test_msm_2_22_metric_size(zk, orc):
    n = 1 << 22
    s = orc.gen_fr(1, n)
    p = orc.gen_points(2, n)
    assert np.array_equal(zk.msm.msm_host(s, p), orc.best_multiexp(s, p))


def test_msm_batch_uneven(zk, orc):
    """Batched form: MSMs of different sizes and windows (one with tables) in one launch set."""
    sizes = [1, 5, 300, 4096, 20000, 0, 777]
    windows = [0, 8, 11, 16, 13, 0, 20]
    N = max(sizes)
    base_pts = orc.gen_points(300, N)
    pts_dev = torch.from_numpy(base_pts.view(np.int32).reshape(N, 16).copy()).cuda()
    tasks, expect = [], []
    for i, (n, w) in enumerate(zip(sizes, windows)):
        s = orc.gen_fr(310 + i, max(n, 1))
        tasks.append({"points": pts_dev, "scalars": torch.from_numpy(s.view(np.int32).reshape(-1, 8).copy()).cuda(),
                      "n": n, "window": w, "result": torch.full((16,), 7, dtype=torch.int32, device="cuda")})
        expect.append(orc.best_multiexp(s[:n], base_pts[:n]) if n else np.zeros(8, dtype=np.uint64))
    # a task over precomputed tables
    bt = zk.msm.ResidentBases(base_pts[:3000], window=16, n_tables=4)
    s = orc.gen_fr(320, 3000)
    tasks.append({"points": bt.tables, "n_tables": 4, "window": 16, "n": 3000,
                  "scalars": torch.from_numpy(s.view(np.int32).reshape(-1, 8).copy()).cuda(),
                  "result": torch.zeros(16, dtype=torch.int32, device="cuda")})
    expect.append(orc.best_multiexp(s, base_pts[:3000]))
    batch = zk.msm.MsmBatch(tasks)
    batch.run()
    for t, e in zip(tasks, expect):
        assert np.array_equal(t["result"].cpu().numpy().view(np.uint64), e)
    # graph capture and replay
    for t in tasks:
        t["result"].zero_()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        batch.run(s)
    g.replay()
    torch.cuda.synchronize()
    for t, e in zip(tasks, expect):
        assert np.array_equal(t["result"].cpu().numpy().view(np.uint64), e)


def _device_msm(zk, s, p, window, n_tables=1):
    n = s.shape[0]
    bases = zk.msm.ResidentBases(p, window=window, n_tables=n_tables)
    res = torch.zeros(16, dtype=torch.int32, device="cuda")
    dev_s = torch.from_numpy(s.view(np.int32).reshape(n, 8).copy()).cuda()
    bases.msm(dev_s, res, bases.workspace())
    return res.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("rounds", [0, 1, 2, 3, 4])
def test_msm_affine_rounds(zk, orc, rounds):
    """A fixed number of affine pairing rounds on buckets that hold equal points (doubling
    pairs), opposite points (pairs summing to the identity), identity bases and zero scalars."""
    n = 4096
    s = orc.gen_fr(500, n)
    p = orc.gen_points(501, n)
    s[0:300] = s[300]                              # one digit per window for 301 records
    p[0:200] = p[300]                              # equal points in one bucket
    p[200:300] = p[300]
    p[200:300, 4:8] = orc.neg(p[300, 4:8], orc.FQ)  # and their negatives
    p[400:440] = 0                                 # identity bases
    s[440:500] = 0                                 # zero scalars
    expect = orc.best_multiexp(s, p)
    zk.msm.set_affine_rounds(rounds)
    try:
        for window, n_tables in ((8, 1), (13, 1), (11, 24)):
            assert np.array_equal(_device_msm(zk, s, p, window, n_tables), expect), (window, n_tables)
    finally:
        zk.msm.set_affine_rounds(-1)


@pytest.mark.parametrize("rounds", [2, 4])
def test_msm_affine_rounds_degenerate(zk, orc, rounds):
    """Every record of a window in one bucket: all doublings, then P + (-P) cancellations."""
    n = 1 << 12
    P = orc.gen_points(502, 1)[0]
    s = np.repeat(orc.gen_fr(503, 1), n, axis=0)
    p = np.repeat(P[None, :], n, axis=0)
    zk.msm.set_affine_rounds(rounds)
    try:
        assert np.array_equal(_device_msm(zk, s, p, 10), orc.best_multiexp(s, p))
        p[1::3, 4:8] = orc.neg(P[4:8], orc.FQ)        # a third of them negated
        assert np.array_equal(_device_msm(zk, s, p, 10), orc.best_multiexp(s, p))
        p[::2, 4:8] = orc.neg(P[4:8], orc.FQ)
        p[1::2] = P                                    # alternate P, -P: the sum is the identity
        assert np.array_equal(_device_msm(zk, s, p, 10), np.zeros(8, dtype=np.uint64))
    finally:
        zk.msm.set_affine_rounds(-1)


def test_msm_batch_affine_rounds(zk, orc):
    """The batched form with pairing rounds: tasks of different sizes and windows share the
    rounds' lists (bucket ids are global across tasks)."""
    sizes, windows = [3000, 1, 20000, 777, 5000], [8, 0, 16, 11, 20]
    N = max(sizes)
    base_pts = orc.gen_points(510, N)
    pts_dev = torch.from_numpy(base_pts.view(np.int32).reshape(N, 16).copy()).cuda()
    zk.msm.set_affine_rounds(3)
    try:
        tasks, expect = [], []
        for i, (n, w) in enumerate(zip(sizes, windows)):
            s = orc.gen_fr(520 + i, n)
            tasks.append({"points": pts_dev, "n": n, "window": w,
                          "scalars": torch.from_numpy(s.view(np.int32).reshape(-1, 8).copy()).cuda(),
                          "result": torch.zeros(16, dtype=torch.int32, device="cuda")})
            expect.append(orc.best_multiexp(s, base_pts[:n]))
        batch = zk.msm.MsmBatch(tasks)
        batch.run()
        for t, e in zip(tasks, expect):
            assert np.array_equal(t["result"].cpu().numpy().view(np.uint64), e)
    finally:
        zk.msm.set_affine_rounds(-1)


@pytest.mark.parametrize("rounds", [0, 3])
def test_msm_one_bucket_long_chains(zk, orc, rounds):
    """2^16 equal scalars over full tables: every window's digits land in one bucket, whose run
    spans many walk chunks (the fix-up's long-chain path), with and without pairing rounds."""
    n = 1 << 16
    s = np.repeat(orc.gen_fr(530, 1), n, axis=0)
    p = orc.gen_points(531, n)
    zk.msm.set_affine_rounds(rounds)
    try:
        assert np.array_equal(_device_msm(zk, s, p, 13, 20), orc.best_multiexp(s, p))
    finally:
        zk.msm.set_affine_rounds(-1)


def test_msm_affine_rounds_empty_lists(zk, orc):
    """Pairing rounds over empty and near-empty digit lists: all-zero scalars (no live entries)
    and a single non-zero scalar."""
    n = 4096
    p = orc.gen_points(540, n)
    s = np.zeros((n, 4), dtype=np.uint64)
    zk.msm.set_affine_rounds(3)
    try:
        assert np.array_equal(_device_msm(zk, s, p, 9), np.zeros(8, dtype=np.uint64))
        s[1234] = orc.gen_fr(541, 1)[0]
        assert np.array_equal(_device_msm(zk, s, p, 9), orc.best_multiexp(s, p))
    finally:
        zk.msm.set_affine_rounds(-1)


@pytest.mark.parametrize("bits", [1, 8, 16, 32, 64, 128])
def test_msm_narrow_scalars(zk, orc, bits):
    """Scalars of 1..128 bits, as the reference's coefficient generator makes them
    (core/tests/msm.rs:70-120: a 128-bit draw masked to the width, then from_u128): the high
    windows are empty and a few buckets of the low windows take most points (1-bit scalars put
    about half the points in one bucket), with and without pairing rounds and tables."""
    n = 4096
    rng = np.random.default_rng(600 + bits)
    mask = (1 << bits) - 1
    vals = [(int(lo) | (int(hi) << 64)) & mask for lo, hi in rng.integers(0, np.iinfo(np.uint64).max, (n, 2), dtype=np.uint64, endpoint=True)]
    s = np.stack([orc.to_mont(orc.int_to_limbs(v)) for v in vals])
    p = orc.gen_points(601, n)
    expect = orc.best_multiexp(s, p)
    for rounds in (0, 3):
        zk.msm.set_affine_rounds(rounds)
        try:
            for window, n_tables in ((8, 1), (16, 1), (12, 8)):
                assert np.array_equal(_device_msm(zk, s, p, window, n_tables), expect), (rounds, window, n_tables)
        finally:
            zk.msm.set_affine_rounds(-1)
    assert np.array_equal(zk.msm.msm_host(s, p), expect)


@pytest.mark.parametrize("threads", [64, 128, 256])
def test_msm_stage_block_shapes(zk, orc, threads):
    """The tuner's MSM block shapes (CTA sizes of the pairing rounds and the walk) leave the
    result unchanged."""
    lib = zk.native.load("libmsm.so")
    n = 1 << 15
    s, p = orc.gen_fr(120, n), orc.gen_points(121, n)
    zk.msm.set_affine_rounds(3)
    try:
        for st in range(3):
            assert lib.zkp_msm_set_block(st, threads) == 0
        bases = zk.msm.ResidentBases(p, window=13, n_tables=4)
        res = torch.zeros(16, dtype=torch.int32, device="cuda")
        bases.msm(torch.from_numpy(s.view(np.int32).reshape(n, 8).copy()).cuda(), res, bases.workspace())
        torch.cuda.synchronize()
        assert np.array_equal(res.cpu().numpy().view(np.uint64), orc.best_multiexp(s, p))
    finally:
        zk.msm.set_affine_rounds(-1)
        zk.tuner.apply_msm_blocks()
    assert lib.zkp_msm_set_block(3, 128) == 1 and lib.zkp_msm_set_block(0, 96) == 1  # refused
