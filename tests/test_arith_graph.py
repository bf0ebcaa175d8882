"""Reading the reference fusion pass's ArithGraph (serde JSON) into the generator's node list,
on the CPU: argument order, in-place inputs, Coef flag, and the operations the reference does
not fuse."""
import copy
import json
import os

import pytest

from conftest import GOLDEN


def _graph():
    with open(os.path.join(GOLDEN, "arith_graph_coef.json")) as f:
        return json.load(f)


def test_arith_graph_to_nodes(zk):
    g = zk.fused.FusedGraph.from_arith_graph(_graph())
    assert g.coef and (g.num_vars, g.num_mut_vars) == (4, 3)
    inputs = [n for n in g.nodes if n[0] == "input"]
    # vars in input order without the in-place input; the in-place one reads mut_vars[0], the
    # slot of the output whose in_node it is (arith.rs:411-455, kernel_gen.rs:53-79)
    assert inputs == [("input", "v0", "poly", "var", 0), ("input", "v1", "poly", "var", 1),
                      ("input", "v2", "scalar", "var", 2), ("input", "v3", "scalar", "var", 3),
                      ("input", "v4", "poly", "mut", 0)]
    assert [n for n in g.nodes if n[0] == "output"] == [("output", 0, "v15"), ("output", 1, "v16"),
                                                        ("output", 2, "v9")]
    ops = {n[1]: n for n in g.nodes if n[0] not in ("input", "output")}
    assert ops["v6"] == ("sp_add", "v6", "v2", "v5") and ops["v8"] == ("sp_subby", "v8", "v7", "v6")
    assert ops["v13"] == ("sp_sub", "v13", "v3", "v1") and ops["v10"] == ("pow", "v10", "v0", 3)
    # topological: every operand is defined before its use
    seen = set()
    for n in g.nodes:
        if n[0] == "input":
            seen.add(n[1])
            continue
        for x in n[2:]:
            if isinstance(x, str):
                assert x in seen, n
        if n[0] != "output":
            seen.add(n[1])
    lag = _graph()
    lag["poly_repr"] = "Lagrange"
    assert not zk.fused.FusedGraph.from_arith_graph(lag).coef
    # the generated source compiles for sm_100a
    assert os.path.exists(zk.fused.FusedOp(g, "arith_graph_test").build())


@pytest.mark.parametrize("vertex,match", [
    (5, {"op": {"Arith": {"Bin": [{"Pp": "Div"}, 0, 1]}}}, ),
    (10, {"op": {"Arith": {"Unr": [{"P": "Inv"}, 0]}}}, ),
    (16, {"op": {"Arith": {"Unr": [{"S": {"Pow": 2}}, 2]}}}, ),
    (14, {"op": {"Arith": {"Bin": [{"Sp": "DivBy"}, 3, 13]}}}, ),
    (7, {"op": "Todo"}, ),
])
def test_unfused_operations_refused(zk, vertex, match):
    g = copy.deepcopy(_graph())
    g["g"][0][vertex] = match
    with pytest.raises(ValueError):
        zk.fused.FusedGraph.from_arith_graph(g)
