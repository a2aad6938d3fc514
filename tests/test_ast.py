"""GPUE's equation grammar: the library's C++ parser and the oracle's
restatement (oracle/ast_oracle.py) against GPUE's own parser, node for node
(tests/golden/ast_gpue.json: parse_eqn, find_element_num and tree_to_array of
src/dynamic.cu:162-530, run host-only by the harness's mode=ast on the corpus,
on parameter texts and on GPUE's example parameter files), and GPUE's own
dynamic_test known answer (src/unit_test.cu:396-466).  CPU only."""
import ctypes as C
import json
import math
import os

import numpy as np
import pytest

import ast_oracle
import cases
import oracle

DOUBLES = cases.AST_DOUBLES
CORPUS = cases.AST_CORPUS
GPUE_AST = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                       "ast_gpue.json")))


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


def same_nodes(got, gpue_nodes):
    """Node for node: value bit for bit, flags, links; op_num where GPUE sets it
    (tree_to_array copies an unset op_num for leaves, written as 0)."""
    assert len(got) == len(gpue_nodes)
    for a, b in zip(got, gpue_nodes):
        a = list(a)
        assert a[0] == b[0] and [int(v) for v in a[1:5]] == b[1:5], (a, b)
        if b[3] >= 0:
            assert int(a[5]) == b[5], (a, b)


def product_file_entries(text, doubles=DOUBLES):
    L = lib()
    names = (C.c_char_p * len(doubles))(*[k.encode() for k in doubles])
    vals = (C.c_double * len(doubles))(*doubles.values())
    cnt, nent, tf = C.c_int32(), C.c_int32(), C.c_int32()
    st = L.gpue_ast_parse_file(text.encode(), names, vals, len(doubles), 0, None, 0, None,
                               None, 0, C.byref(cnt), C.byref(nent))
    if st != 0:
        return st, None
    out = []
    for i in range(nent.value):
        name = C.create_string_buffer(64)
        st = L.gpue_ast_parse_file(text.encode(), names, vals, len(doubles), i, name, 64,
                                   C.byref(tf), None, 0, C.byref(cnt), C.byref(nent))
        assert st == 0
        buf = (oracle.Node * cnt.value)()
        st = L.gpue_ast_parse_file(text.encode(), names, vals, len(doubles), i, name, 64,
                                   C.byref(tf), C.cast(buf, C.c_void_p), cnt.value,
                                   C.byref(cnt), C.byref(nent))
        assert st == 0
        out.append((name.value.decode(), tf.value,
                    [(n.val, n.is_dynamic, n.var, n.left, n.right, n.op_num) for n in buf]))
    return 0, out


def test_fixture_covers_the_corpus():
    assert [c["expr"] for c in GPUE_AST["corpus"]] == CORPUS
    assert GPUE_AST["doubles"] == DOUBLES


@pytest.mark.parametrize("k", range(len(CORPUS)))
def test_parser_matches_gpue(k):
    ref = GPUE_AST["corpus"][k]
    st, nodes = product_nodes(ref["expr"])
    assert st == 0
    same_nodes(nodes, ref["nodes"])
    same_nodes(ast_oracle.tree_to_array(ast_oracle.parse_eqn(ref["expr"], DOUBLES, {})),
               ref["nodes"])
    # GPUE's "<name>_time" flag, through a one-entry parameter text
    st, entries = product_file_entries("V = " + ref["expr"])
    assert st == 0 and len(entries) == 1
    assert entries[0][1] == ref["time"]
    same_nodes(entries[0][2], ref["nodes"])


@pytest.mark.parametrize("k", range(len(GPUE_AST["param_files"])),
                         ids=[p["name"] for p in GPUE_AST["param_files"]])
def test_param_file_matches_gpue(k):
    pf = GPUE_AST["param_files"][k]
    st, entries = product_file_entries(pf["text"])
    assert st == 0
    assert [e[0] for e in entries] == [e["name"] for e in pf["entries"]]
    asts, order, flags = ast_oracle.parse_param_text(pf["text"], DOUBLES)
    assert order == [e["name"] for e in pf["entries"]]
    for (name, tflag, nodes), ref in zip(entries, pf["entries"]):
        assert tflag == ref["time"], name
        same_nodes(nodes, ref["nodes"])
        same_nodes(ast_oracle.tree_to_array(asts[name]), ref["nodes"])
        assert (name in flags) == bool(ref["time"]), name


@pytest.mark.parametrize("k", range(len(cases.AST_REJECTED)))
def test_rejects_what_gpue_rejects(k):
    ref = GPUE_AST["rejected"][k]
    assert ref["exit_code"] != 0  # GPUE printed its message and exited
    st, _ = product_nodes(ref["expr"])
    assert st == 5
