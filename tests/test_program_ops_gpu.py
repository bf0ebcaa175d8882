"""Each instruction and kernel type the served loop lowers, in small hand-built chunks (the
reference's serde forms), against the oracle: view arithmetic and transfers across wrapping
views, GetScalarFromArray, and the poly / NTT kernels with their argument orders from
emit_func.rs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GPU = {"GPU": {"device_id": 0}}
M = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
R = 1 << 256


class ChunkBuilder:
    """Instruction list, function table and Offset plan of a small chunk."""

    def __init__(self):
        self.ins, self.f_table, self.n, self.off = [], [], 0, 0
        self.stream = self._new()
        self._emit({"Allocate": {"device": GPU, "typ": "Stream", "id": self.stream,
                                 "alloc_method": {"Dynamic": 0}}})

    def _new(self):
        self.n += 1
        return self.n - 1

    def _emit(self, node):
        self.ins.append({"node": node, "track": "MemoryManagement", "stream": None})

    def gpu(self, typ, nbytes):
        v = self._new()
        self._emit({"Allocate": {"device": GPU, "typ": typ, "id": v, "alloc_method": {"Offset": [self.off, nbytes]}}})
        self.off += (nbytes + 255) // 256 * 256
        return v

    def poly(self, n):
        return self.gpu({"ScalarArray": {"len": n, "meta": None}}, n * 32)

    def scalar(self):
        return self.gpu("Scalar", 32)

    def buffer(self):
        return self.gpu({"GpuBuffer": [0, None]}, 0)

    def cpu(self, typ):
        v = self._new()
        self._emit({"Allocate": {"device": "CPU", "typ": typ, "id": v, "alloc_method": {"Dynamic": 0}}})
        return v

    def input(self, entry):
        v = self._new()
        self._emit({"LoadInput": {"src": entry, "dst": v}})
        return v

    def node(self, kind, **fields):
        dst = self._new()
        self._emit({kind: dict(fields, dst=dst)})
        return dst

    def transfer(self, src, dst, to_cpu=False, from_cpu=False):
        self._emit({"Transfer": {"src_device": "CPU" if from_cpu else GPU, "dst_device": "CPU" if to_cpu else GPU,
                                 "stream": self.stream, "src_id": src, "dst_id": dst}})

    def call(self, kernel_type, arg_mut, arg):
        if kernel_type not in self.f_table:
            self.f_table.append(kernel_type)
        self._emit({"FuncCall": {"func_id": self.f_table.index(kernel_type), "arg_mut": arg_mut, "arg": arg}})

    def to_host(self, v, typ):
        h = self.cpu(typ)
        self.transfer(v, h, to_cpu=True)
        return h

    def chunk(self, returned):
        out = self.node("AssembleTuple", vars=returned)
        self._emit({"Return": out})
        return {"instructions": self.ins, "f_table": [self.f_table, None], "event_table": [[], None],
                "n_variables": self.n, "n_threads": 1, "lbss": []}


def sa(n):
    return {"ScalarArray": {"len": n, "meta": None}}


def ints(orc, a):
    return [orc.limbs_to_int(x) * pow(R, -1, M) % M for x in np.asarray(a, dtype=np.uint64).reshape(-1, 4)]


@pytest.fixture(scope="module")
def server(zk):
    srv = zk.serving.Server(zk.gen.points(2, 1 << 10), hbm_bytes=1 << 30, max_inflight=2, ext_log=2, min_k=10,
                            max_k=10)
    yield srv
    srv.close()


def _run(zk, server, chunk, input_types, inputs):
    prog = zk.program.CompiledProgram(server, chunk, [], input_types)
    try:
        r, leaves = prog.wait(prog.submit(inputs))
        assert r.status == 0
        return [np.ascontiguousarray(x).view(np.uint64).reshape(-1, 4) for x in leaves]
    finally:
        prog.close()


def test_views_transfers_and_scalar_extraction(zk, orc, server):
    """Rotation, Slice of a rotated array (a view that wraps), Transfers in both directions
    between views of different offsets, GetScalarFromArray (runtime.rs:480-505)."""
    n = 8
    a = orc.gen_fr(41, n)
    c = ChunkBuilder()
    x_in = c.input(0)
    x = c.poly(n)
    c.transfer(x_in, x, from_cpu=True)
    xr = c.node("Rotation", src=x, shift=3)           # element i = a[(i - 3) mod 8]
    y = c.poly(n)
    c.transfer(xr, y)                                  # y holds the rotated order
    ys = c.node("Slice", src=y, start=2, end=8)
    out1 = c.to_host(ys, sa(6))
    xs = c.node("Slice", src=xr, start=1, end=7)       # wraps the end of the array
    out2 = c.to_host(xs, sa(6))
    s = c.scalar()
    c._emit({"GetScalarFromArray": {"src": xr, "dst": s, "idx": 5, "stream": c.stream}})
    out3 = c.to_host(s, "Scalar")
    got = _run(zk, server, c.chunk([out1, out2, out3]), [sa(n)], [a])
    rot = np.stack([a[(i - 3) % n] for i in range(n)])
    assert np.array_equal(got[0], rot[2:8])
    assert np.array_equal(got[1], rot[1:7])
    assert np.array_equal(got[2], rot[5:6])


def test_poly_kernels(zk, orc, server):
    """PolyAdd / PolySub, ScanMul (target[0] = x0, target[1..] = p[..n-1], then the product
    scan: poly.rs:428-468), KateDivision, BatchedInvert, EvaluatePoly, NewZero / NewOneLagrange
    / NewOneCoef, ScalarInvert and ScalarPow, with their emit_func.rs argument orders."""
    n = 1024
    p, q = orc.gen_fr(42, n), orc.gen_fr(43, n)
    xv = orc.gen_fr(44, 1)
    c = ChunkBuilder()
    P, Q, X = c.poly(n), c.poly(n), c.scalar()
    for e, v in enumerate((P, Q, X)):
        c.transfer(c.input(e), v, from_cpu=True)
    st = c.stream
    add, sub = c.poly(n), c.poly(n)
    c.call("PolyAdd", [add], [P, Q, st])
    c.call("PolySub", [sub], [P, Q, st])
    scan = c.poly(n)
    c.call("ScanMul", [c.buffer(), scan], [P, X, st])
    kate = c.poly(n)
    c.call("KateDivision", [c.buffer(), kate], [P, X, st])
    inv = c.poly(n)
    c.transfer(Q, inv)
    c.call("BatchedInvert", [c.buffer(), inv], [st])
    ev = c.scalar()
    c.call("EvaluatePoly", [c.buffer(), ev], [P, X, st])
    zero, one_l, one_c = c.poly(4), c.poly(4), c.poly(4)
    c.call("NewZero", [zero], [st])
    c.call("NewOneLagrange", [one_l], [st])
    c.call("NewOneCoef", [one_c], [st])
    xi, xp = c.scalar(), c.scalar()
    c.transfer(X, xi)
    c.transfer(X, xp)
    c.call("ScalarInvert", [xi], [st])
    c.call({"ScalarPow": 5}, [xp], [st])
    outs = [c.to_host(v, sa(n)) for v in (add, sub, scan, kate, inv)]
    outs.append(c.to_host(ev, "Scalar"))
    outs += [c.to_host(v, sa(4)) for v in (zero, one_l, one_c)]
    outs += [c.to_host(v, "Scalar") for v in (xi, xp)]
    got = _run(zk, server, c.chunk(outs), [sa(n), sa(n), "Scalar"], [p, q, xv])
    assert np.array_equal(got[0], orc.vec_add(p, q))
    assert np.array_equal(got[1], orc.vec_sub(p, q))
    pi, x = ints(orc, p), ints(orc, xv)[0]
    acc, expect = x, [x]
    for v in pi[:-1]:
        acc = acc * v % M
        expect.append(acc)
    assert ints(orc, got[2]) == expect
    kexp = [0] * n
    for i in range(n - 2, -1, -1):
        kexp[i] = (pi[i + 1] + x * kexp[i + 1]) % M
    assert ints(orc, got[3]) == kexp
    assert np.array_equal(got[4], orc.batch_invert(q))
    assert np.array_equal(got[5][0], orc.eval_poly(p, xv[0]))
    one = orc.one()
    assert not got[6].any()
    assert np.array_equal(got[7], np.tile(one, (4, 1)))
    assert np.array_equal(got[8][0], one) and not got[8][1:].any()
    assert np.array_equal(got[9][0], orc.inv(xv[0]))
    assert np.array_equal(got[10][0], orc.pow_(xv[0], 5))


def test_ntt_kernels(zk, orc, server):
    """NttPrcompute on a twiddle table input, NttRecompute with the (pq, omegas) pair of
    gen_pq_omegas (pq_deg from the pq length, ntt.rs:265), DistributePowers with a short powers
    array; every result against the oracle."""
    log_n = 10
    n = 1 << log_n
    a = orc.gen_fr(45, n)
    w = np.ascontiguousarray(zk.field.mont_words(zk.field.root_of_unity(log_n)), dtype=np.uint32)
    tw = zk.ntt.ssip_precompute(n // 2, w)
    pq_len = zk.ntt.get_pq_len(log_n)
    pq, om = zk.ntt.gen_pq_omegas(pq_len, n, w.copy())
    powers = orc.gen_fr(46, 3)
    c = ChunkBuilder()
    A1, A2, A3 = c.poly(n), c.poly(n), c.poly(n)
    TW, PQ, OM, PW = c.poly(n // 2), c.poly(len(pq)), c.poly(len(om)), c.poly(3)
    for e, v in enumerate((TW, PQ, OM, PW)):
        c.transfer(c.input(e), v, from_cpu=True)
    a_in = c.input(4)
    for v in (A1, A2, A3):
        c.transfer(a_in, v, from_cpu=True)
    st = c.stream
    c.call("NttPrcompute", [A1], [TW, st])
    c.call("NttRecompute", [A2], [PQ, OM, st])
    c.call("DistributePowers", [A3], [PW, st])
    outs = [c.to_host(v, sa(n)) for v in (A1, A2, A3)]
    types = [sa(n // 2), sa(len(pq)), sa(len(om)), sa(3), sa(n)]
    got = _run(zk, server, c.chunk(outs), types,
               [tw.view(np.uint64), pq.view(np.uint64), om.view(np.uint64), powers, a])
    expect = orc.ntt(a, log_n)
    assert np.array_equal(got[0], expect)
    assert np.array_equal(got[1], expect)
    assert np.array_equal(got[2], orc.distribute_powers(a, powers))
