"""GPUE's equation grammar: the library's C++ parser against the oracle's
restatement (oracle/ast_oracle.py), node for node, and GPUE's own
dynamic_test known answer (src/unit_test.cu:396-466).  CPU only."""
import ctypes as C
import math

import numpy as np
import pytest

import ast_oracle
import oracle

DOUBLES = {"omega": 0.7, "omegaX": 1.25, "omegaY": 0.8, "mass": 2.0, "xMax": 10.0,
           "fudge": 0.0, "rad": 10.0, "omegaR": 7071.0}

CORPUS = [
    "(((3*x)+7)+(5-7)+cos(0)*1)+pow(120,2)",
    "a-b-c".replace("a", "x").replace("b", "y").replace("c", "z"),
    "x-y+z",
    "2*x-3",
    "x/y*z",
    "x^2",
    "pow(x,3)+pow(y,2)",
    "exp(-x)".replace("-x", "0-x"),
    "sqrt(x*x+y*y)",
    "cos(omega*t)*x",
    "0.5*mass*((omegaX*x)*(omegaX*x)+(omegaY*y)*(omegaY*y))",
    "rad*omegaR*x*y*z",
    "((x))",
    "(x+1)*(y-2)",
    "sin(x)*cos(y)+tan(z)",
    "jn(0,x)+yn(1,y)",
    "1.5+2.25*x",
    "[x+y]*2",
    "x*y*omega*omegaX*30000",
    "((3*x)+(y-(2*z)))/(1+t)",
]


def lib():
    import gpue_b200
    L = gpue_b200.lib()
    L.gpue_ast_parse.argtypes = [C.c_char_p, C.POINTER(C.c_char_p), C.POINTER(C.c_double),
                                 C.c_int32, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]
    L.gpue_ast_parse.restype = C.c_int
    return L


def product_nodes(expr, doubles=DOUBLES):
    L = lib()
    names = (C.c_char_p * len(doubles))(*[k.encode() for k in doubles])
    vals = (C.c_double * len(doubles))(*doubles.values())
    cnt = C.c_int32()
    st = L.gpue_ast_parse(expr.encode(), names, vals, len(doubles), None, 0, C.byref(cnt))
    if st != 0:
        return st, None
    buf = (oracle.Node * cnt.value)()
    st = L.gpue_ast_parse(expr.encode(), names, vals, len(doubles), C.cast(buf, C.c_void_p),
                          cnt.value, C.byref(cnt))
    return st, [(n.val, n.is_dynamic, n.var, n.left, n.right, n.op_num) for n in buf]


def test_node_layout_is_32_bytes():
    assert C.sizeof(oracle.Node) == 32


@pytest.mark.parametrize("expr", CORPUS)
def test_parser_matches_restatement(expr):
    st, nodes = product_nodes(expr)
    assert st == 0
    ref = ast_oracle.tree_to_array(ast_oracle.parse_eqn(expr, DOUBLES, {}))
    assert len(nodes) == len(ref)
    for a, b in zip(nodes, ref):
        assert a[0] == b[0] and tuple(a[1:]) == tuple(int(v) for v in b[1:])


def test_dynamic_test_known_answer():
    """find_field of the expression at x = i must equal the formula exactly."""
    st, nodes = product_nodes(CORPUS[0])
    arr = oracle.nodes_array(nodes)
    for i in range(64):
        v = oracle.lib().orc_ast_eval(arr, float(i), 0.0, 0.0, 0.0)
        assert v == (((3 * i) + 7) + (5 - 7) + math.cos(0) * 1) + math.pow(120, 2)


def test_first_minus_split_quirk():
    """GPUE splits at the first '-', so a-b-c means a-(b-c)."""
    st, nodes = product_nodes("x-y-z")
    arr = oracle.nodes_array(nodes)
    assert oracle.lib().orc_ast_eval(arr, 10.0, 4.0, 1.0, 0.0) == 10.0 - (4.0 - 1.0)


def test_malformed_expressions_fail():
    for bad in ("x+", "unknown_name*2", ")x(", ""):
        st, _ = product_nodes(bad)
        assert st == 5, bad


def test_param_file_restatement_appends_gauge_energy_to_V():
    text = "Ax = 0-y*omega\nAy = x*omega\nAz = 0\nV = 0.5*(x*x+y*y)\nK = 1"
    asts, order, flags = ast_oracle.parse_param_text(text, DOUBLES)
    assert order == ["Ax", "Ay", "Az", "V", "K"]
    v = ast_oracle.tree_to_array(asts["V"])
    # V = 0.5*(x*x+y*y) + 0.5*mass*(Ax*Ax+Ay*Ay+Az*Az) at (x, y) = (2, 3)
    val = ast_oracle.evaluate(v, 2.0, 3.0, 0.0, 0.0)
    ax, ay = -3.0 * 0.7, 2.0 * 0.7
    assert val == pytest.approx(0.5 * 13 + 0.5 * 2.0 * (ax * ax + ay * ay), rel=1e-15)
    assert "V" in flags  # it names earlier expressions, so GPUE marks it time dependent
