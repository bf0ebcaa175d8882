"""Generated fused kernels and the fused quotient pipeline on the GPU, bit-exact vs the oracle."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

M = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001


def dev(zk, a):
    return zk.ScalarArray.from_numpy(a)


def scal(zk, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int32).reshape(1, 8).copy()).cuda()


def zh_oracle(orc, k, ext):
    g = orc.to_mont(orc.int_to_limbs(7))
    gk = orc.pow_(g, 1 << k)
    w = orc.root_of_unity(k + ext)
    one = orc.one()
    vals = [orc.sub(orc.mul(gk, orc.pow_(w, j << k)), one) for j in range(1 << ext)]
    return orc.batch_invert(np.stack(vals))


def quotient_oracle(orc, ea, eb, ec, z, zh, ext):
    n = len(z)
    zw = np.roll(z, -(1 << ext), axis=0)
    t = orc.vec_sub(orc.vec_sub(orc.vec_mul(ea, eb), ec), orc.vec_mul(z, zw))
    zhf = np.tile(zh, (n // len(zh), 1))
    return orc.vec_mul(t, zhf)


@pytest.mark.parametrize("log_n", [3, 10, 16])
def test_quotient_kernel(zk, orc, log_n):
    n = 1 << log_n
    a, b, c, z = (orc.gen_fr(s, n) for s in (1, 2, 3, 4))
    zh = orc.gen_fr(5, 8)
    k = zk.fused.quotient_kernel()
    out = zk.ScalarArray.zeros(n)
    zd = dev(zk, z)
    k([out], [dev(zk, a), dev(zk, b), dev(zk, c), zd, zk.pipeline.rotated(zd, 3), dev(zk, zh)])
    assert np.array_equal(out.numpy_u64(), quotient_oracle(orc, a, b, c, z, zh, 3))


def test_generic_graph_features(zk, orc):
    """scalar inputs, neg, pow, Ss ops, a scalar output, Sp on Coef vs Lagrange."""
    n = 1000
    a = orc.gen_fr(6, n)
    s = orc.gen_fr(7, 1)[0]
    t = orc.gen_fr(8, 1)[0]
    for coef in (False, True):
        g = zk.fused.FusedGraph([
            ("input", "a", "poly", "var", 0),
            ("input", "s", "scalar", "var", 1),
            ("input", "t", "scalar", "var", 2),
            ("mul", "st", "s", "t"),
            ("sp_add", "x", "st", "a"),
            ("sp_subby", "y", "s", "x"),
            ("neg", "ny", "y"),
            ("pow", "p", "ny", 5),
            ("output", 0, "p"),
            ("output", 1, "st"),
        ], coef=coef)
        kern = zk.fused.FusedKernel(zk.fused.FusedOp(g))
        out = zk.ScalarArray.zeros(n)
        sout = torch.zeros((1, 8), dtype=torch.int32, device="cuda")
        kern([out, sout], [dev(zk, a), scal(zk, s), scal(zk, t)])
        st = orc.mul(s, t)
        exp = []
        for i in range(n):
            if coef and i != 0:
                x = a[i]
                y = x
            else:
                x = orc.add(st, a[i])
                y = orc.sub(x, s)
            exp.append(orc.pow_(orc.neg(y), 5))
        assert np.array_equal(out.numpy_u64(), np.stack(exp)), coef
        assert np.array_equal(sout.cpu().numpy().view(np.uint64)[0], st)


def test_fused_rotated_and_sliced_inputs(zk, orc):
    n = 256
    a = orc.gen_fr(9, n)
    big = orc.gen_fr(10, 2 * n)
    g = zk.fused.FusedGraph([("input", "a", "poly", "var", 0), ("input", "b", "poly", "var", 1),
                             ("mul", "r", "a", "b"), ("output", 0, "r")])
    kern = zk.fused.FusedKernel(zk.fused.FusedOp(g))
    xa = dev(zk, a)
    xa.rotate(17)
    xb = dev(zk, big).set_slice_raw(2 * n - 3, n)
    out = zk.ScalarArray.zeros(n)
    kern([out], [xa, xb])
    va = orc.poly_ptr_view(a, n, rotate=17)
    vb = orc.poly_ptr_view(big, n, offset=2 * n - 3, whole_len=2 * n)
    assert np.array_equal(out.numpy_u64(), orc.vec_mul(va, vb))


@pytest.mark.parametrize("k", [10, 14])
def test_quotient_pipeline_small(zk, orc, k):
    ext = 3
    n, N = 1 << k, 1 << (k + ext)
    a, b, c = (orc.gen_fr(s, n) for s in (11, 12, 13))
    z = orc.gen_fr(14, N)
    pipe = zk.pipeline.QuotientPipeline(k, ext)
    q = pipe.run(dev(zk, a), dev(zk, b), dev(zk, c), dev(zk, z))
    g = orc.to_mont(orc.int_to_limbs(7))
    ea, eb, ec = (orc.coset_ntt(orc.intt(x, k), k, k + ext, g) for x in (a, b, c))
    zh = zh_oracle(orc, k, ext)
    assert np.array_equal(zh.view(np.uint32).reshape(-1, 8), pipe.zh.numpy_u32())
    assert np.array_equal(q.numpy_u64(), quotient_oracle(orc, ea, eb, ec, z, zh, ext))


def test_quotient_pipeline_config3_full(zk, orc):
    """k = 22, 8x extension (2^25), coset shift 7, bit-exact end to end."""
    k, ext = 22, 3
    n, N = 1 << k, 1 << (k + ext)
    a, b, c = (orc.gen_fr(s, n) for s in (21, 22, 23))
    z = orc.gen_fr(24, N)
    pipe = zk.pipeline.QuotientPipeline(k, ext)
    q = pipe.run(dev(zk, a), dev(zk, b), dev(zk, c), dev(zk, z))
    got = q.numpy_u64()
    g = orc.to_mont(orc.int_to_limbs(7))
    ea, eb, ec = (orc.coset_ntt(orc.intt(x, k), k, k + ext, g) for x in (a, b, c))
    assert np.array_equal(got, quotient_oracle(orc, ea, eb, ec, z, zh_oracle(orc, k, ext), ext))


def _host(a):
    """(n, 4) uint64 limbs -> pinned (n, 8) int32 CPU tensor"""
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int32).reshape(-1, 8).copy()).pin_memory()


@pytest.mark.parametrize("parts", [4, 8, 16])
def test_pipelined_fused_kernel(zk, orc, parts):
    """The pipelined form (host polynomials streamed in chunks, fused_kernels.rs:198-516) gives
    the one-shot kernel's results: a quotient-shaped graph with a periodic 1/Z_H input and an
    in-out mutable polynomial (out = (a*b - c - z*zw) * zh + out)."""
    n = 1 << 12
    g = zk.fused.FusedGraph([
        ("input", "a", "poly", "var", 0),
        ("input", "b", "poly", "var", 1),
        ("input", "c", "poly", "var", 2),
        ("input", "z", "poly", "var", 3),
        ("input", "zw", "poly", "var", 4),
        ("input", "zh", "periodic", "var", 5),
        ("input", "acc", "poly", "mut", 0),
        ("mul", "ab", "a", "b"),
        ("sub", "t0", "ab", "c"),
        ("mul", "zz", "z", "zw"),
        ("sub", "t1", "t0", "zz"),
        ("mul", "q", "t1", "zh"),
        ("add", "r", "q", "acc"),
        ("output", 0, "r"),
    ])
    a, b, c, z, zw, acc = (orc.gen_fr(700 + i, n) for i in range(6))
    zh = orc.gen_fr(706, 8)
    t = orc.vec_sub(orc.vec_sub(orc.vec_mul(a, b), c), orc.vec_mul(z, zw))
    expect = orc.vec_add(orc.vec_mul(t, np.tile(zh, (n // 8, 1))), acc)
    op = zk.fused.FusedOp(g, "zkp_test_pipelined_q")
    host_out = _host(acc)
    zk.fused.PipelinedFusedKernel(op, parts)([host_out], [_host(x) for x in (a, b, c, z, zw, zh)], n)
    assert np.array_equal(host_out.numpy().view(np.uint64).reshape(n, 4), expect)
    # the one-shot kernel on device copies agrees
    out = dev(zk, acc)
    zk.fused.FusedKernel(op)([out], [dev(zk, x) for x in (a, b, c, z, zw, zh)])
    assert np.array_equal(out.numpy_u64(), expect)


def test_pipelined_fused_kernel_write_only_output(zk, orc):
    """A mutable polynomial the kernel only writes is not copied in: stale host contents of
    the output do not matter."""
    n = 1 << 11
    g = zk.fused.FusedGraph([("input", "a", "poly", "var", 0), ("input", "b", "poly", "var", 1),
                             ("mul", "p", "a", "b"), ("sub", "d", "p", "a"), ("output", 0, "d")])
    a, b = orc.gen_fr(720, n), orc.gen_fr(721, n)
    out = _host(orc.gen_fr(722, n))  # stale contents
    zk.fused.PipelinedFusedKernel(zk.fused.FusedOp(g, "zkp_test_pipelined_wo"), 8)([out], [_host(a), _host(b)], n)
    assert np.array_equal(out.numpy().view(np.uint64).reshape(n, 4), orc.vec_sub(orc.vec_mul(a, b), a))


def test_pipelined_fused_kernel_rejects_bad_split(zk, orc):
    n = 1000
    g = zk.fused.FusedGraph([("input", "a", "poly", "var", 0), ("input", "b", "poly", "var", 1),
                             ("add", "s", "a", "b"), ("output", 0, "s")])
    k = zk.fused.PipelinedFusedKernel(zk.fused.FusedOp(g, "zkp_test_pipelined_add"), 6)  # 6 does not divide 1000
    a = orc.gen_fr(710, n)
    with pytest.raises(ValueError):
        k([_host(a)], [_host(a), _host(a)], n)
    with pytest.raises(ValueError):
        zk.fused.PipelinedFusedKernel(zk.fused.FusedOp(g, "zkp_test_pipelined_add"), 3)


def test_fixed_factor_products(zk, orc):
    """Products with a scalar or periodic operand (either side) take Shoup's product from
    per-CTA pairs; a periodic input above the shared-memory cap falls back to the Montgomery
    product.  Results are identical to the oracle's."""
    n = 4096
    a = orc.gen_fr(20, n)
    s = orc.gen_fr(21, 1)[0]
    p8 = orc.gen_fr(22, 8)
    p128 = orc.gen_fr(23, 128)
    g = zk.fused.FusedGraph([
        ("input", "a", "poly", "var", 0),
        ("input", "s", "scalar", "var", 1),
        ("input", "p", "periodic", "var", 2),
        ("input", "q", "periodic", "var", 3),
        ("mul", "as_", "a", "s"),
        ("mul", "sa", "s", "a"),
        ("mul", "ap", "a", "p"),
        ("mul", "pa", "p", "a"),
        ("mul", "aq", "a", "q"),
        ("add", "u", "as_", "s"),        # s also read as a plain value
        ("mul", "v", "u", "pa"),
        ("sub", "w", "ap", "p"),         # p also read as a plain value
        ("output", 0, "sa"),
        ("output", 1, "v"),
        ("output", 2, "w"),
        ("output", 3, "aq"),
    ])
    kern = zk.fused.FusedKernel(zk.fused.FusedOp(g))
    outs = [zk.ScalarArray.zeros(n) for _ in range(4)]
    kern(outs, [dev(zk, a), scal(zk, s), dev(zk, p8), dev(zk, p128)])
    pf = np.tile(p8, (n // 8, 1))
    qf = np.tile(p128, (n // 128, 1))
    sv = np.tile(s, (n, 1))
    as_ = orc.vec_mul(a, sv)
    pa = orc.vec_mul(pf, a)
    exp = [orc.vec_mul(sv, a), orc.vec_mul(orc.vec_add(as_, sv), pa), orc.vec_sub(orc.vec_mul(a, pf), pf),
           orc.vec_mul(a, qf)]
    for o, e in zip(outs, exp):
        assert np.array_equal(o.numpy_u64(), e)


def _arith_graph(repr_):
    import json
    from conftest import GOLDEN
    with open(os.path.join(GOLDEN, "arith_graph_coef.json")) as f:
        g = json.load(f)
    g["poly_repr"] = repr_
    return g


@pytest.mark.parametrize("repr_", ["Coef", "Lagrange"])
def test_kernel_from_reference_arith_graph(zk, orc, repr_):
    """A fused kernel generated from a serialised ArithGraph (the reference fusion pass's output):
    Pp / Ss / Sp ops, neg, pow, an in-place input and a scalar output, against the oracle; on a
    Coef graph the Sp add / sub / sub-by apply at index 0 only (kernel_gen.rs:501-545)."""
    n = 1000
    graph = zk.fused.FusedGraph.from_arith_graph(_arith_graph(repr_))
    kern = zk.fused.FusedKernel(zk.fused.FusedOp(graph))
    a, b, acc = (orc.gen_fr(s, n) for s in (71, 72, 73))
    s_, t = orc.gen_fr(74, 1)[0], orc.gen_fr(75, 1)[0]
    dev_acc = dev(zk, acc)
    scal = torch.zeros((1, 8), dtype=torch.int32, device="cuda")
    out2 = zk.ScalarArray.zeros(n)
    kern([dev_acc, scal, out2], [dev(zk, a), dev(zk, b), zk.ScalarArray.from_numpy(s_[None, :]).values,
                                 zk.ScalarArray.from_numpy(t[None, :]).values])
    torch.cuda.synchronize()
    S, T = np.tile(s_, (n, 1)), np.tile(t, (n, 1))
    coef = repr_ == "Coef"
    ab = orc.vec_mul(a, b)
    v6 = ab.copy()
    v6[: 1 if coef else n] = orc.vec_add(S, ab)[: 1 if coef else n]
    st = orc.mul(s_, t)
    v8 = v6.copy()
    v8[: 1 if coef else n] = orc.vec_sub(v6, np.tile(st, (n, 1)))[: 1 if coef else n]
    v9 = orc.vec_sub(np.zeros_like(v8), v8)
    v10 = orc.vec_mul(orc.vec_mul(a, a), a)
    v12 = orc.vec_add(orc.vec_sub(v9, v10), acc)
    v13 = orc.vec_sub(np.zeros_like(b), b)
    v13[: 1 if coef else n] = orc.vec_sub(T, b)[: 1 if coef else n]
    v15 = orc.vec_add(v12, orc.vec_mul(T, v13))
    assert np.array_equal(dev_acc.numpy_u64(), v15)
    assert np.array_equal(scal.cpu().numpy().view(np.uint64).reshape(4), orc.sub(s_, t))
    assert np.array_equal(out2.numpy_u64(), v9)
