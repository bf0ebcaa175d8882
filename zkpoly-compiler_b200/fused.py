"""Fused elementwise kernels: host-side mirror of the reference's FusedOp code generator
(core/src/fused_kernels/kernel_gen.rs:47-617) and FusedKernel runtime wrapper
(core/src/fused_kernels.rs:76-196).

A FusedGraph is the reference's ArithGraph restated as a topologically ordered node list:
  ("input",  name, kind, side, index)   kind in {"poly", "scalar", "periodic"};
                                        side "var" (ConstPolyPtr) or "mut" (PolyPtr)
  (op, name, lhs, rhs)                  op in {"add", "sub", "mul"}: Pp / Ss / Sp products
  ("sp_add"|"sp_sub"|"sp_subby", name, scalar, poly)   scalar-poly add/sub; on a Coef graph
                                        they touch index 0 of the first chunk only
                                        (kernel_gen.rs:501-545)
  ("neg", name, x) / ("pow", name, x, exponent)
  ("output", mut_index, src)
"periodic" is an addition: input element i is read at i mod len (the 8 distinct values of
1/Z_H on an 8x coset are such an input).  Division and inversion are not fused, as in the
reference (batched_invert handles them).

The generated CUDA exports `cudaError_t <name>(ConstPolyPtr const* vars, PolyPtr const*
mut_vars, unsigned long long len, bool is_first, void* local_buffer, cudaStream_t)` - the
signature the reference's runtime calls (kernel_gen.rs:286-307) - and is compiled for sm_100a
into lib<name>.so.  Register allocation is left to ptxas; the local (spill) buffer argument is
accepted and unused, so get_temp_buffer_size() is 0.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess
from dataclasses import dataclass, field

import torch

from .native import PolyPtr, check
from .scalar import ScalarArray, require_cuda, stream_handle

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
FUSED_DIR = os.path.join(HERE, "lib", "fused")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

_BIN = {"add": "Fr::add", "sub": "Fr::sub", "mul": "Fr::mul"}


@dataclass
class FusedGraph:
    nodes: list
    coef: bool = False          # poly_repr == Coef (kernel_gen.rs:501-545)
    num_vars: int = field(init=False, default=0)
    num_mut_vars: int = field(init=False, default=0)

    def __post_init__(self):
        nv = nm = 0
        for n in self.nodes:
            if n[0] == "input":
                if n[3] == "var":
                    nv = max(nv, n[4] + 1)
                else:
                    nm = max(nm, n[4] + 1)
            elif n[0] == "output":
                nm = max(nm, n[1] + 1)
        self.num_vars, self.num_mut_vars = nv, nm

    def key(self) -> str:
        return hashlib.sha1(repr((self.nodes, self.coef)).encode()).hexdigest()[:16]

    @staticmethod
    def from_arith_graph(g: dict) -> "FusedGraph":
        """The node list of a serialised ArithGraph, the fusion pass's output that the
        reference's generator consumes (common/src/arith.rs:323-330; kernel_gen.rs:47-121).

        serde forms: ``{"outputs": [ids], "inputs": [ids], "g": [[vertex, ...], null],
        "poly_repr": "Coef" | "Lagrange", "poly_degree": n | null}`` with a vertex
        ``{"op": {"Input": {"outer_id", "typ": "Scalar" | "ScalarArray", "mutability": "Const" |
        "Mut"}}}``, ``{"op": {"Arith": {"Bin": [{"Pp" | "Ss" | "Sp": op}, lhs, rhs]}}}``,
        ``{"op": {"Arith": {"Unr": [{"P" | "S": "Neg" | {"Pow": e}}, x]}}}`` or ``{"op":
        {"Output": {"outer_id", "typ", "store_node", "in_node"}}}``.  Argument order follows
        ArithGraph::gen_var_lists (arith.rs:429-455): mut_vars are the outputs in order; vars
        are the inputs in order except in-place ones (a Mut input that is some output's
        in_node, arith.rs:411-427), which are read from that output's mut_vars slot
        (kernel_gen.rs:53-79).  An Sp op's lhs is the scalar and rhs the polynomial; on a Coef
        graph Sp add / sub / sub-by touch index 0 only (kernel_gen.rs:501-545).  Division,
        inversion and scalar powers are not fused (the reference rejects them as well)."""
        verts = g["g"][0] if isinstance(g["g"], list) and len(g["g"]) == 2 and g["g"][1] is None else g["g"]
        ops = [v["op"] if isinstance(v, dict) and "op" in v else v for v in verts]
        kind_of = {}
        for i, op in enumerate(ops):
            if op == "Todo" or not isinstance(op, dict) or len(op) != 1:
                raise ValueError(f"vertex {i}: unsupported operation {op!r:.80}")
            kind_of[i] = next(iter(op))
        inplace = {}
        for m, oid in enumerate(g["outputs"]):
            out = ops[oid].get("Output")
            if out is None:
                raise ValueError(f"output {oid} is not an Output vertex")
            src = out.get("in_node")
            if src is not None and ops[src]["Input"]["mutability"] == "Mut":
                inplace[src] = m
        var_index = {}
        for iid in g["inputs"]:
            if "Input" not in ops[iid]:
                raise ValueError(f"input {iid} is not an Input vertex")
            if iid not in inplace:
                var_index[iid] = len(var_index)

        def deps(i):
            op = ops[i]
            if "Arith" in op:
                a = op["Arith"]
                return a["Bin"][1:] if "Bin" in a else [a["Unr"][1]]
            if "Output" in op:
                return [op["Output"]["store_node"]]
            return []
        order, state = [], {}

        def visit(i):
            if state.get(i) == 2:
                return
            if state.get(i) == 1:
                raise ValueError("the arithmetic graph has a cycle")
            state[i] = 1
            for d in deps(i):
                visit(int(d))
            state[i] = 2
            order.append(i)
        for i in list(g["inputs"]) + list(g["outputs"]):
            visit(int(i))
        nodes = []
        bin_names = {"Add": "add", "Sub": "sub", "Mul": "mul"}
        for i in order:
            op, name = ops[i], f"v{i}"
            if "Input" in op:
                kind = "scalar" if op["Input"]["typ"] == "Scalar" else "poly"
                side, idx = ("mut", inplace[i]) if i in inplace else ("var", var_index[i])
                nodes.append(("input", name, kind, side, idx))
            elif "Output" in op:
                m = list(g["outputs"]).index(i)
                nodes.append(("output", m, f"v{op['Output']['store_node']}"))
            elif "Bin" in op["Arith"]:
                (cls, bop), lhs, rhs = next(iter(op["Arith"]["Bin"][0].items())), *op["Arith"]["Bin"][1:]
                if cls in ("Pp", "Ss"):
                    if bop not in bin_names:
                        raise ValueError(f"vertex {i}: {cls} {bop} is not fused (batched inversion handles it)")
                    nodes.append((bin_names[bop], name, f"v{lhs}", f"v{rhs}"))
                else:
                    sp = {"Add": "sp_add", "Sub": "sp_sub", "SubBy": "sp_subby", "Mul": "mul"}.get(bop)
                    if sp is None:
                        raise ValueError(f"vertex {i}: Sp {bop} is not fused (batched inversion handles it)")
                    nodes.append((sp, name, f"v{lhs}", f"v{rhs}"))
            else:
                (cls, uop), x = next(iter(op["Arith"]["Unr"][0].items())), op["Arith"]["Unr"][1]
                if uop == "Neg":
                    nodes.append(("neg", name, f"v{x}"))
                elif isinstance(uop, dict) and "Pow" in uop and cls == "P":
                    nodes.append(("pow", name, f"v{x}", int(uop["Pow"])))
                else:
                    raise ValueError(f"vertex {i}: {cls} {uop!r} is not fused")
        return FusedGraph(nodes, coef=g.get("poly_repr") == "Coef")


class FusedOp:
    """Generates and builds one fused kernel (kernel_gen.rs FusedOp::new / gen)."""

    def __init__(self, graph: FusedGraph, name: str | None = None):
        self.graph = graph
        self.name = name or f"fused_arith_{graph.key()}"

    def get_temp_buffer_size(self) -> int:
        return 0

    def _shoup_factors(self) -> dict:
        """mul node name -> (factor input, other operand) for products with exactly one operand
        that is a scalar or periodic input: those use Shoup's product by a fixed factor."""
        inputs = {n[1]: n[2] for n in self.graph.nodes if n[0] == "input"}
        fixed = {k for k, kind in inputs.items() if kind in ("scalar", "periodic")}
        out = {}
        for n in self.graph.nodes:
            if n[0] == "mul":
                _, name, lhs, rhs = n
                if (rhs in fixed) != (lhs in fixed):
                    out[name] = (rhs, lhs) if rhs in fixed else (lhs, rhs)
        return out

    def gen_source(self) -> str:
        g = self.graph
        kinds = {}
        pre, setup, body = [], [], []
        shoup = self._shoup_factors()
        factors = {f for f, _ in shoup.values()}
        # inputs read as plain values somewhere (not only as a Shoup factor)
        plain_uses = set()
        for n in g.nodes:
            if n[0] == "output":
                plain_uses.add(n[2])
            elif n[0] != "input" and not (n[0] == "mul" and n[1] in shoup):
                plain_uses.update(x for x in n[2:] if isinstance(x, str))
            elif n[0] == "mul":
                plain_uses.add(shoup[n[1]][1])
        where = {}
        for n in g.nodes:
            op = n[0]
            if op == "input":
                _, name, kind, side, idx = n
                arr = "sv" if side == "var" else "smv"
                where[name] = f"{arr}[{idx}]"
                kinds[name] = kind
                if kind == "scalar":
                    if name in plain_uses:
                        pre.append(f"    const Fr {name} = Fr::load({arr}[{idx}].base);")
                    if name in factors:
                        setup.append(f"    __shared__ __align__(16) u32 shs_{name}[16];")
                        setup.append(f"    if (threadIdx.x == 0) fused::shoup_pairs({arr}[{idx}], 1, shs_{name});")
                elif kind == "periodic":
                    body.append(f"        const u64 {name}_k = fused::periodic_index({arr}[{idx}], idx);")
                    if name in plain_uses:
                        body.append(f"        const Fr {name} = Fr::load({arr}[{idx}].at({name}_k));")
                    if name in factors:
                        setup.append(f"    __shared__ __align__(16) u32 shp_{name}[fused::SHOUP_PERIOD_MAX * 16];")
                        setup.append(f"    const bool {name}_fx = {arr}[{idx}].len <= fused::SHOUP_PERIOD_MAX;")
                        setup.append(f"    if ({name}_fx) fused::shoup_pairs({arr}[{idx}], {arr}[{idx}].len, shp_{name});")
                else:
                    body.append(f"        const Fr {name} = Fr::load({arr}[{idx}].at(idx));")
            elif op == "mul" and n[1] in shoup:
                _, name, lhs, rhs = n
                f, o = shoup[name]
                if kinds[f] == "scalar":
                    body.append(f"        const Fr {name} = Fr::mul_shoup({o}, Fr::load(shs_{f}), "
                                f"Fr::load(shs_{f} + 8));")
                else:
                    body.append(f"        const Fr {name} = {f}_fx ? Fr::mul_shoup({o}, Fr::load(shp_{f} + {f}_k * 16), "
                                f"Fr::load(shp_{f} + {f}_k * 16 + 8)) : Fr::mul({o}, Fr::load({where[f]}.at({f}_k)));")
                kinds[name] = "scalar" if kinds[lhs] == kinds[rhs] == "scalar" else "poly"
            elif op in _BIN:
                _, name, lhs, rhs = n
                body.append(f"        const Fr {name} = {_BIN[op]}({lhs}, {rhs});")
                kinds[name] = "scalar" if kinds[lhs] == kinds[rhs] == "scalar" else "poly"
            elif op in ("sp_add", "sp_sub", "sp_subby"):
                _, name, s, p = n
                full = {"sp_add": f"Fr::add({s}, {p})", "sp_sub": f"Fr::sub({s}, {p})",
                        "sp_subby": f"Fr::sub({p}, {s})"}[op]
                if g.coef:
                    rest = {"sp_add": p, "sp_sub": f"Fr::neg({p})", "sp_subby": p}[op]
                    body.append(f"        const Fr {name} = (idx == 0 && is_first) ? {full} : {rest};")
                else:
                    body.append(f"        const Fr {name} = {full};")
                kinds[name] = "poly"
            elif op == "neg":
                _, name, x = n
                body.append(f"        const Fr {name} = Fr::neg({x});")
                kinds[name] = kinds[x]
            elif op == "pow":
                _, name, x, e = n
                body.append(f"        const Fr {name} = Fr::pow_u64({x}, {int(e)}ull);")
                kinds[name] = kinds[x]
            elif op == "output":
                _, idx, src = n
                if kinds.get(src) == "scalar":
                    body.append(f"        if (idx == 0) {src}.canonical().store(smv[{idx}].base);")
                else:
                    body.append(f"        {src}.canonical().store(smv[{idx}].at(idx));")
            else:
                raise ValueError(f"unsupported fused op {op}")
        nv, nm = max(g.num_vars, 1), max(g.num_mut_vars, 1)
        inc = os.path.join(CSRC, "fused_rt.cuh")
        return f"""// generated by zkpoly-compiler_b200/fused.py for graph {g.key()}
#include "{inc}"
using namespace zk;

__global__ void __launch_bounds__(256) {self.name}_kernel(const ConstPolyPtr *vars, const PolyPtr *mut_vars,
                                                        unsigned long long len, bool is_first) {{
    __shared__ View sv[{nv}];
    __shared__ View smv[{nm}];
    if (threadIdx.x < {g.num_vars}) sv[threadIdx.x] = fused::device_view(vars[threadIdx.x]);
    if (threadIdx.x < {g.num_mut_vars}) smv[threadIdx.x] = fused::device_view(mut_vars[threadIdx.x]);
    __syncthreads();
{chr(10).join(setup)}
{"    __syncthreads();" if setup else ""}
{chr(10).join(pre)}
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 idx = (u64)blockIdx.x * blockDim.x + threadIdx.x; idx < len; idx += stride) {{
{chr(10).join(body)}
    }}
}}

extern "C" cudaError_t {self.name}(ConstPolyPtr const *vars, PolyPtr const *mut_vars, unsigned long long len,
                                   bool is_first, void *local_buffer, cudaStream_t stream) {{
    (void)local_buffer;
    if (len == 0) return cudaSuccess;
    if (vars == nullptr && {g.num_vars} > 0) return cudaErrorInvalidValue;
    if (mut_vars == nullptr) return cudaErrorInvalidValue;
    {self.name}_kernel<<<fused::fused_grid(len, 256), 256, 0, stream>>>(vars, mut_vars, len, is_first);
    return cudaGetLastError();
}}
"""

    def lib_path(self) -> str:
        return os.path.join(FUSED_DIR, f"lib{self.name}.so")

    def gen(self, target_dir: str = FUSED_DIR) -> str:
        os.makedirs(target_dir, exist_ok=True)
        src = os.path.join(target_dir, f"{self.name}.cu")
        text = self.gen_source()
        if not os.path.exists(src) or open(src).read() != text:
            with open(src, "w") as f:
                f.write(text)
        return src

    def build(self, force: bool = False) -> str:
        src = self.gen()
        out = self.lib_path()
        deps = [src, os.path.join(CSRC, "fused_rt.cuh"), os.path.join(CSRC, "field.cuh"),
                os.path.join(CSRC, "common.cuh")]
        if force or not os.path.exists(out) or any(os.path.getmtime(d) > os.path.getmtime(out) for d in deps):
            cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
                   "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-shared", "-o", out + ".tmp", src]
            res = subprocess.run(cmd, capture_output=True, text=True)
            if res.returncode != 0:
                raise RuntimeError(f"nvcc failed for fused kernel {self.name}:\n{res.stderr}")
            os.replace(out + ".tmp", out)
        return out


_loaded: dict[str, ctypes.CDLL] = {}


class FusedKernel:
    """core/src/fused_kernels.rs:76-196: loads the built kernel and calls it with the PolyPtr
    arrays copied into a device argument buffer."""

    def __init__(self, op: FusedOp):
        require_cuda()
        self.op = op
        path = op.build()
        if path not in _loaded:
            _loaded[path] = ctypes.CDLL(path)
        fn = getattr(_loaded[path], op.name)
        fn.restype = ctypes.c_int
        fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_bool, ctypes.c_void_p,
                       ctypes.c_void_p]
        self.fn = fn
        g = op.graph
        self.arg_buffer = torch.empty(max(g.num_vars + g.num_mut_vars, 1) * ctypes.sizeof(PolyPtr),
                                      dtype=torch.uint8, device="cuda")

    def __call__(self, mut_vars: list, vars_: list, stream=None, is_first: bool = True):
        """mut_vars / vars_: ScalarArray (polys) or (1, 8) int32 device tensors (scalars).
        The element count is the length of the polynomial arguments (fused_kernels.rs:110-160)."""
        g = self.op.graph
        length = 0
        ptrs = []
        for v in list(vars_) + list(mut_vars):
            if isinstance(v, ScalarArray):
                ptrs.append(v.poly_ptr())
            else:
                ptrs.append(PolyPtr(v.data_ptr(), 1, 0, 0, 1))
        periodic = {n[4] for n in g.nodes if n[0] == "input" and n[2] == "periodic" and n[3] == "var"}
        for i, v in enumerate(list(vars_) + list(mut_vars)):
            if isinstance(v, ScalarArray) and not (i < len(vars_) and i in periodic):
                if length in (0, 1):
                    length = v.len
                else:
                    assert length == v.len, "fused kernel operands differ in length"
        length = max(length, 1)
        arr = (PolyPtr * len(ptrs))(*ptrs)
        host = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8)
        self.arg_buffer[: host.numel()].copy_(host, non_blocking=False)
        base = self.arg_buffer.data_ptr()
        check(self.fn(base, base + len(vars_) * ctypes.sizeof(PolyPtr), length, is_first, None,
                      stream_handle(stream)), self.op.name)


class PipelinedFusedKernel:
    """core/src/fused_kernels.rs:198-516: the same fused kernel over HOST polynomials, streamed
    through the device in `divide_parts` chunks (> 3, dividing the length) with the copies of
    consecutive chunks overlapping the kernel (libzkp_pipeline.so, include/zkp_pipeline.h).
    For operands that do not fit device memory; results are identical to the one-shot kernel."""

    def __init__(self, op: FusedOp, divide_parts: int = 4):
        from .native import load
        if divide_parts <= 3:
            raise ValueError("divide_parts must be > 3 (fused_kernels.rs:201)")
        self.kernel = FusedKernel(op)
        self.divide_parts = divide_parts
        self.lib = load("libzkp_pipeline.so")
        self.workspace = None

    @staticmethod
    def _arg(t: torch.Tensor, stream_len: int, write_only: bool = False):
        from .native import ZkpPipelineArg
        if t.device.type != "cpu" or not t.is_contiguous() or t.dtype != torch.int32 or t.shape[-1] != 8:
            raise ValueError("host arguments are contiguous (n, 8) int32 CPU tensors (pinned for overlap)")
        rows = t.shape[0]
        return ZkpPipelineArg(t.data_ptr(), 0 if rows == stream_len else rows, int(write_only))

    def __call__(self, mut_vars: list, vars_: list, length: int) -> None:
        """mut_vars / vars_: (rows, 8) int32 CPU tensors - polynomials of `length` rows, or
        scalars / periodic inputs (fewer rows, copied once).  Blocks until the outputs are in
        host memory."""
        from .native import ZkpPipelineArg, check
        g = self.kernel.op.graph
        if len(vars_) != g.num_vars or len(mut_vars) != g.num_mut_vars:
            raise ValueError("argument count differs from the graph's")
        read_mut = {n[4] for n in g.nodes if n[0] == "input" and n[3] == "mut"}
        va = (ZkpPipelineArg * max(len(vars_), 1))(*[self._arg(t, length) for t in vars_])
        ma = (ZkpPipelineArg * max(len(mut_vars), 1))(*[self._arg(t, length, i not in read_mut)
                                                          for i, t in enumerate(mut_vars)])
        need = int(self.lib.zkp_fused_pipelined_workspace(va, len(vars_), ma, len(mut_vars), length,
                                                          self.divide_parts))
        if need == 0:
            raise ValueError("invalid pipelined arguments (length % divide_parts, periodic lengths)")
        if self.workspace is None or self.workspace.numel() < need:
            self.workspace = torch.empty(need, dtype=torch.uint8, device="cuda")
        fn = ctypes.cast(self.kernel.fn, ctypes.c_void_p).value
        check(self.lib.zkp_fused_pipelined(fn, va, len(vars_), ma, len(mut_vars), length, self.divide_parts,
                                           self.workspace.data_ptr(), self.workspace.numel(), None),
              "zkp_fused_pipelined")


# ------------------------------------------------------------------ graphs used by the path
def quotient_graph() -> FusedGraph:
    """(a*b - c - z*z(wX)) * zh_inv[i mod 8] on the 8x extended coset: the quotient numerator
    of the fused-pipeline workload divided by the vanishing polynomial."""
    return FusedGraph([
        ("input", "a", "poly", "var", 0),
        ("input", "b", "poly", "var", 1),
        ("input", "c", "poly", "var", 2),
        ("input", "z", "poly", "var", 3),
        ("input", "zw", "poly", "var", 4),
        ("input", "zh", "periodic", "var", 5),
        ("mul", "ab", "a", "b"),
        ("sub", "t0", "ab", "c"),
        ("mul", "zz", "z", "zw"),
        ("sub", "t1", "t0", "zz"),
        ("mul", "q", "t1", "zh"),
        ("output", 0, "q"),
    ])


def quotient_kernel() -> FusedKernel:
    return FusedKernel(FusedOp(quotient_graph(), "zkp_quotient_z8"))


def build_path_kernels() -> list[str]:
    """Builds the fused kernels the hot path uses (called by the package build): the quotient
    kernel of the built-in served program and the two kernels its compiled-artifact form
    names (program.prover_fused_graphs)."""
    from .program import prover_fused_graphs
    out = [FusedOp(quotient_graph(), "zkp_quotient_z8").build()]
    out += [FusedOp(g, name).build() for name, g in prover_fused_graphs().items()]
    return out
