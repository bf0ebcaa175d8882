"""Compiled programs through the served loop (zkp_serve_program_* in libzkp_runtime.so): the
prover program read from a reference-form artifact gives the built-in prover's results and the
oracle's, alone and mixed with other programs and built-in requests."""
import ctypes
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from test_serving_gpu import expected

pytestmark = pytest.mark.gpu

ART = os.path.join(GOLDEN, "prover_k10")


def _inputs(orc, k, seed, ext=2):
    n, N = 1 << k, 1 << (k + ext)
    return [orc.gen_fr(seed * 8 + i, n) for i in range(3)] + [orc.gen_fr(seed * 8 + 3, N),
                                                              orc.gen_fr(seed * 8 + 4, 1)]


def _words(leaves):
    return np.concatenate([np.asarray(x, dtype=np.uint32).reshape(-1) for x in leaves])


@pytest.fixture(scope="module")
def server(zk):
    srv = zk.serving.Server(zk.gen.points(2, 1 << 14), hbm_bytes=4 << 30, max_inflight=4, ext_log=2, min_k=10,
                            max_k=14)
    yield srv
    srv.close()


def test_golden_artifact_matches_builtin_and_oracle(zk, orc, server):
    prog = zk.program.CompiledProgram.load(server, ART, zk.program.prover_input_types(10),
                                           fused=zk.program.prover_fused_graphs())
    try:
        for seed in (3, 4):
            r, leaves = prog.wait(prog.submit(_inputs(orc, 10, seed)))
            assert r.status == 0
            assert [x.shape for x in leaves] == [(16,)] * 4 + [(8,)] * 2
            got = _words(leaves)
            builtin = server.wait(server.submit(10, seed))
            assert builtin.status == 0
            assert np.array_equal(got, zk.serving.result_words(builtin)), seed
            assert np.array_equal(got, expected(orc, 10, seed)), seed
            assert r.footprint == prog.device_bytes
    finally:
        prog.close()


def _program(zk, server, k, bases=None):
    pts = zk.gen.points(2, 1 << k)
    consts = zk.program.prover_constants(k, 2, pts)
    parts = zk.program.prover_artifact(k, consts)
    return zk.program.CompiledProgram.from_parts(server, parts[1], parts[3], zk.program.prover_input_types(k),
                                                 fused=zk.program.prover_fused_graphs(), bases=bases)


def test_programs_same_alone_and_in_the_mix(zk, orc, server):
    """Two program sizes (one whose MSMs use precomputed tables registered for its bases
    constant) and built-in requests, submitted together: every result equals the one the same
    request gets alone."""
    rb = zk.msm.ResidentBases(zk.gen.points(2, 1 << 13), window=13, n_tables=4)
    progs = {12: _program(zk, server, 12), 13: _program(zk, server, 13, bases={"bases": rb})}
    try:
        reqs = [("p", 12, 20), ("b", 11, 21), ("p", 13, 22), ("p", 12, 23), ("b", 14, 24), ("p", 13, 25)]
        inputs = {seed: _inputs(orc, k, seed) for kind, k, seed in reqs if kind == "p"}
        alone = {}
        for kind, k, seed in reqs:
            if kind == "p":
                r, leaves = progs[k].wait(progs[k].submit(inputs[seed]))
                assert r.status == 0
                alone[seed] = _words(leaves)
            else:
                r = server.wait(server.submit(k, seed))
                assert r.status == 0
                alone[seed] = zk.serving.result_words(r)
        tickets = []
        for kind, k, seed in reqs:
            tickets.append((kind, k, seed, progs[k].submit(inputs[seed]) if kind == "p" else server.submit(k, seed)))
        for kind, k, seed, t in tickets:
            if kind == "p":
                r, leaves = progs[k].wait(t)
                got = _words(leaves)
            else:
                r = server.wait(t)
                got = zk.serving.result_words(r)
            assert r.status == 0
            assert np.array_equal(got, alone[seed]), (kind, k, seed)
        # and the oracle for one request of each program size
        for k, seed in ((12, 20), (13, 22)):
            assert np.array_equal(alone[seed], expected(orc, k, seed)), k
        assert server.stats()["peak_inflight"] >= 2
    finally:
        for p in progs.values():
            p.close()


def test_malformed_program_refused(zk, server):
    """zkp_serve_program_create checks every view against the planned blocks."""
    ZkpProgOp, ZkpProgOut = zk.native.ZkpProgOp, zk.native.ZkpProgOut
    op = ZkpProgOp()
    op.kind, op.n_views = 2, 16        # ZERO of 1000 elements at offset 0 of a 4 KiB block
    op.imm[0] = 32
    op.v[0].space, op.v[0].len, op.v[0].whole_len = 1, 1000, 1000
    ops = (ZkpProgOp * 1)(op)
    outs = (ZkpProgOut * 1)()
    h = ctypes.c_void_p()
    rc = server.lib.zkp_serve_program_create(server.h, ops, 1, 4096, 256, outs, 0, None, 0, ctypes.byref(h))
    assert rc == 1  # cudaErrorInvalidValue
    op.v[0].len = op.v[0].whole_len = 128  # fits: accepted, and a request runs it
    ops = (ZkpProgOp * 1)(op)
    rc = server.lib.zkp_serve_program_create(server.h, ops, 1, 4096, 256, outs, 0, None, 0, ctypes.byref(h))
    assert rc == 0
    t = server.lib.zkp_serve_submit_program(server.h, h, None, 0, None, 0)
    assert server.wait(t).status == 0
    server.lib.zkp_serve_program_destroy(server.h, h)


def test_program_destroyed_with_requests_in_flight(zk, orc, server):
    """Destroying a program whose requests are still queued or running defers the release to
    the last of them: each still completes with its results."""
    prog = zk.program.CompiledProgram.load(server, ART, zk.program.prover_input_types(10),
                                           fused=zk.program.prover_fused_graphs())
    seeds = (31, 32, 33)
    tickets = [(seed, prog.submit(_inputs(orc, 10, seed))) for seed in seeds]
    server.lib.zkp_serve_program_destroy(server.h, prog.h)
    handle, prog.h = prog.h, None
    for seed, t in tickets:
        r, leaves = prog.wait(t)
        assert r.status == 0
        assert np.array_equal(_words(leaves), expected(orc, 10, seed)), seed
    del handle
