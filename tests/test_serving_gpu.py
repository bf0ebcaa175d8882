"""Served form: continuous batching with HBM admission.  Each request's result is bit-identical
alone and in the mix, matches the oracle, and failures stay with their request."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

MIN_K, MAX_K = 10, 14


@pytest.fixture(scope="module")
def bases(zk):
    return zk.gen.points(2, 1 << MAX_K)


def server(zk, bases, inflight, hbm=4 << 30):
    return zk.serving.Server(bases, hbm_bytes=hbm, max_inflight=inflight, ext_log=2, min_k=MIN_K, max_k=MAX_K)


def expected(orc, k, seed, ext=2):
    n, N = 1 << k, 1 << (k + ext)
    a, b, c = (orc.intt(orc.gen_fr(seed * 8 + i, n), k) for i in range(3))
    z = orc.gen_fr(seed * 8 + 3, N)
    x = orc.gen_fr(seed * 8 + 4, 1)[0]
    g = orc.to_mont(orc.int_to_limbs(7))
    e = orc.coset_ntt(c, k, k + ext, g)
    # 1/Z_H on the coset: (g^n w^(j n) - 1)^-1
    w = orc.root_of_unity(k + ext)
    gn = orc.pow_(g, n)
    zh = orc.batch_invert(np.stack([orc.sub(orc.mul(gn, orc.pow_(w, j * n)), orc.one()) for j in range(1 << ext)]))
    zw = np.roll(z, -(1 << ext), axis=0)
    t = orc.vec_sub(orc.vec_sub(orc.vec_mul(e, e), e), orc.vec_mul(z, zw))
    q = orc.vec_mul(t, np.tile(zh, (N >> ext, 1)))
    pts = orc.gen_points(2, n)
    msms = [orc.best_multiexp(v, pts) for v in (a, b, c, q[:n])]
    evals = [orc.eval_poly(a, x), orc.eval_poly(b, x)]
    return np.concatenate([m.view(np.uint32) for m in msms] + [v.view(np.uint32) for v in evals])


def test_request_matches_oracle(zk, orc, bases):
    srv = server(zk, bases, 2)
    try:
        for k, seed in ((10, 1), (11, 2)):
            res = srv.wait(srv.submit(k, seed))
            assert res.status == 0
            assert np.array_equal(zk.serving.result_words(res), expected(orc, k, seed)), (k, seed)
    finally:
        srv.close()


def test_same_alone_and_in_the_mix(zk, bases):
    reqs = [(k, 100 + i) for i, k in enumerate([14, 10, 12, 13, 11, 14, 10, 12, 13, 11, 12, 14])]
    alone = {}
    srv = server(zk, bases, 1)
    try:
        for k, seed in reqs:
            r = srv.wait(srv.submit(k, seed))
            assert r.status == 0
            alone[seed] = zk.serving.result_words(r)
    finally:
        srv.close()
    srv = server(zk, bases, 6)
    try:
        tickets = [(seed, srv.submit(k, seed)) for k, seed in reqs]
        results = {seed: srv.wait(t) for seed, t in tickets}
        st = srv.stats()
    finally:
        srv.close()
    assert st["peak_inflight"] > 1  # the requests really overlapped
    for seed, r in results.items():
        assert r.status == 0
        assert np.array_equal(zk.serving.result_words(r), alone[seed]), seed


def test_failures_stay_with_their_request(zk, bases):
    srv = server(zk, bases, 4)
    try:
        good = [srv.submit(11, 7), srv.submit(12, 8)]
        bad_k = srv.submit(MAX_K + 3, 9)           # malformed: size outside the server's range
        alloc = srv.submit(11, 10, inject_fault=1)  # allocation refused
        launch = srv.submit(11, 11, inject_fault=2) # a launch returns an error
        good.append(srv.submit(13, 12))
        assert srv.wait(bad_k).status == -1
        assert srv.wait(alloc).status == -4
        assert srv.wait(launch).status == -3
        res = [srv.wait(t) for t in good]
        assert all(r.status == 0 for r in res)
    finally:
        srv.close()
    ref = server(zk, bases, 1)
    try:
        for (k, seed), r in zip(((11, 7), (12, 8), (13, 12)), res):
            assert np.array_equal(zk.serving.result_words(ref.wait(ref.submit(k, seed))),
                                  zk.serving.result_words(r))
    finally:
        ref.close()


def test_admission_by_hbm_footprint(zk, bases):
    probe = server(zk, bases, 1)
    fp13, fp14 = probe.footprint(13), probe.footprint(14)
    probe.close()
    # an arena that holds one k=14 request (or two k=13 ones) at a time
    srv = server(zk, bases, 8, hbm=fp14 + (1 << 20))
    try:
        biggest = srv.submit(MAX_K, 1)
        tickets = [srv.submit(13, 20 + i) for i in range(6)] + [srv.submit(14, 30)]
        res = [srv.wait(t) for t in tickets]
        st = srv.stats()
        assert all(r.status == 0 for r in res)
        assert st["peak_bytes"] <= st["arena_bytes"]
        assert srv.wait(biggest).status == 0  # fits exactly
    finally:
        srv.close()
    small = server(zk, bases, 2, hbm=fp13 + (1 << 20))
    try:
        assert small.wait(small.submit(14, 1)).status == -2  # larger than the whole arena
        assert small.wait(small.submit(13, 2)).status == 0
    finally:
        small.close()


def test_poisson_load_smoke(zk, bases):
    sched = zk.serving.poisson_schedule(24, rate=50.0, k_lo=MIN_K, k_hi=MAX_K, seed=5)
    srv = server(zk, bases, 8)
    try:
        results, summary = zk.serving.run_schedule(srv, sched)
    finally:
        srv.close()
    assert summary["ok"] == 24 and summary["p99_ms"] >= summary["p50_ms"] > 0


def test_per_call_path_matches_served(zk, bases):
    """The plain per-call path (reference-ABI MSM with host arrays) gives the served results."""
    prover = zk.serving.PerCallProver(bases, ext_log=2)
    srv = server(zk, bases, 4)
    try:
        reqs = [(10, 41), (13, 42), (14, 43)]
        tickets = [(k, seed, srv.submit(k, seed)) for k, seed in reqs]
        for k, seed, t in tickets:
            r = srv.wait(t)
            assert r.status == 0
            assert np.array_equal(prover.run(k, seed), zk.serving.result_words(r)), (k, seed)
    finally:
        srv.close()
    words, summary = zk.serving.run_schedule_per_call(prover, [(0.0, 10, 41), (0.01, 11, 44)])
    assert summary["ok"] == 2 and summary["p99_ms"] >= summary["p50_ms"] > 0


def test_per_size_table_sets(zk, bases):
    """A server with two resident table sets (different windows and table counts by size)
    returns the same results as one with a single untabled set."""
    sets = [(zk.msm.ResidentBases(bases[: 1 << 12], window=9, n_tables=29), 12),
            (zk.msm.ResidentBases(bases, window=10, n_tables=26), MAX_K)]
    a = zk.serving.Server(sets, hbm_bytes=4 << 30, max_inflight=3, ext_log=2, min_k=MIN_K, max_k=MAX_K)
    b = server(zk, bases, 1)
    try:
        reqs = [(10, 61), (12, 62), (13, 63), (14, 64)]
        ta = [a.submit(k, s) for k, s in reqs]
        tb = [b.submit(k, s) for k, s in reqs]
        for x, y in zip(ta, tb):
            ra, rb = a.wait(x), b.wait(y)
            assert ra.status == 0 and rb.status == 0
            assert np.array_equal(zk.serving.result_words(ra), zk.serving.result_words(rb))
    finally:
        a.close()
        b.close()


def test_admission_policy(zk, bases):
    """With the tail policy (large requests on high-priority streams, at most one of them in
    flight) every result is still the one the request gets alone, and no two large requests
    ever run at the same time."""
    reqs = [(k, 300 + i) for i, k in enumerate([14, 10, 13, 14, 11, 13, 12, 14, 10, 13])]
    ref = server(zk, bases, 1)
    try:
        alone = {seed: zk.serving.result_words(ref.wait(ref.submit(k, seed))) for k, seed in reqs}
    finally:
        ref.close()
    srv = server(zk, bases, 6)
    try:
        srv.set_policy(priority_k=13, large_k=13, max_large_inflight=1)
        tickets = [(k, seed, srv.submit(k, seed)) for k, seed in reqs]
        res = [(k, seed, srv.wait(t)) for k, seed, t in tickets]
        assert srv.stats()["peak_inflight"] > 1
    finally:
        srv.close()
    large = []
    for k, seed, r in res:
        assert r.status == 0
        assert np.array_equal(zk.serving.result_words(r), alone[seed]), (k, seed)
        if k >= 13:
            large.append((r.start_s, r.done_s))
    large.sort()
    for (s0, d0), (s1, d1) in zip(large, large[1:]):
        assert s1 >= d0  # admitted only after the previous large request completed
