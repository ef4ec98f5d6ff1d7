"""The expression language: engine compiler vs the oracle's restatement (no GPU).

The engine parses AdditionalCompute strings in C++ and compiles them to a register-stack
bytecode (pygranite_b200/csrc/expr.cpp).  The oracle restates the reference grammar
(source/granite/TrajectoryIntegrator.cpp:10-26) in Python and walks the reference's flat
pre-order AST (TrajectoryIntegrator.hpp:539-627).  Both are evaluated on the host through
glibc's float functions here, so values must agree bit for bit, and both must accept and
reject the same strings with the reference's messages.
"""
import ctypes

import numpy as np
import pytest

from oracle import expr_oracle as eo
from oracle import oracle as orc
from pygranite_b200 import capi

VOLS = ["T", "hum", "_q1"]
CONS = ["k", "rho"]


def oracle_eval(code, ref, dim=3, cm=3):
    arr = eo.compile_expression(code, VOLS, CONS, dim, cm)
    nodes = (orc._Node * len(arr))(*[orc._Node(int(r["type"]), float(r["value"]), int(r["left"]), int(r["right"]))
                                     for r in arr])
    lib = orc.lib()
    lib.oracle_interpret_f32.restype = ctypes.c_float
    lib.oracle_interpret_f32.argtypes = [ctypes.POINTER(orc._Node), ctypes.c_int64,
                                         ctypes.POINTER(ctypes.c_float), ctypes.c_int64]
    r = np.ascontiguousarray(ref, np.float32)
    return lib.oracle_interpret_f32(nodes, len(arr), r.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 0)


def engine_eval(code, ref, dim=3, cm=3):
    return capi.evaluate_expression(code, ref, VOLS, CONS, dim, cm)


def random_expr(rng, depth=0):
    leaves = ["x", "y", "z", "cv", "u", "v", "w", "T", "hum", "_q1", "k", "rho"]
    r = rng.random()
    if depth > 4 or r < 0.3:
        c = rng.random()
        if c < 0.6:
            return rng.choice(leaves)
        if c < 0.8:
            return str(int(rng.integers(-9, 10)))
        return f"{rng.integers(-9, 10)}.{rng.integers(0, 1000):03d}"
    if r < 0.75:
        op = rng.choice(["+", "-", "*", "/"])
        sp = rng.choice(["", " ", "  ", "\t"])
        a, b = random_expr(rng, depth + 1), random_expr(rng, depth + 1)
        if b.startswith("-") and op in "+-":
            b = f"({b})" if rng.random() < 0.5 else b
        return f"{a}{sp}{op}{sp}{b}"
    if r < 0.85:
        return f"({random_expr(rng, depth + 1)})"
    fn = rng.choice(["sqrt", "exp", "ln", "sin", "cos", "tan", "asin", "acos", "atan", "atan2"])
    if fn == "atan2":
        return f"atan2({random_expr(rng, depth + 1)}, {random_expr(rng, depth + 1)})"
    return f"{fn}({random_expr(rng, depth + 1)})"


def same(a, b):
    return (a == b) or (np.isnan(a) and np.isnan(b))


def test_random_expressions_agree_bitwise():
    rng = np.random.default_rng(123)
    checked = 0
    for _ in range(1500):
        code = random_expr(rng)
        ref = (rng.standard_normal(19) * 3).astype(np.float32)
        try:
            o = oracle_eval(code, ref)
        except eo.ExprError as ex:
            with pytest.raises(capi.GraniteError) as ei:
                engine_eval(code, ref)
            assert str(ei.value).split("|")[1].split()[0] == str(ex).split("|")[1].split()[0], (code, ex, ei.value)
            continue
        e = engine_eval(code, ref)
        assert same(np.float32(o), np.float32(e)), (code, o, e)
        checked += 1
    assert checked > 1000


@pytest.mark.parametrize("code,value", [
    ("sqrt(u*u+v*v)*T", None), ("1-2-3", -4.0), ("2*3+4*5", 26.0), ("8/4/2", 1.0), ("x - -1", None),
    ("atan2(1, 1)*4", None), ("((((x))))", None), ("k*rho + _q1", None), ("2 -1", 1.0), (" 3.250 ", 3.25),
])
def test_known_expressions(code, value):
    ref = np.arange(1, 20, dtype=np.float32) / 7
    o, e = oracle_eval(code, ref), engine_eval(code, ref)
    assert same(np.float32(o), np.float32(e))
    if value is not None:
        assert np.isclose(e, value)


@pytest.mark.parametrize("code,msg", [
    ("f0 + 1", "Identifier 'f0' is no longer allowed"),
    ("c3", "Identifier 'c3' is no longer allowed"),
    ("velocity", "syntax error"),      # 'v' commits as a register (no word boundary, cpp:16)
    ("x1", "syntax error"),
    ("", "syntax error"),
    ("1.", "syntax error"),
    (".5", "syntax error"),
    ("-x", "syntax error"),
    ("sqrt(x", "syntax error"),
    ("x + pressure", "Invalid identifier 'pressure'."),
    ("sqrt", "Invalid identifier 'sqrt'."),
])
def test_rejections_match(code, msg):
    ref = np.zeros(19, np.float32)
    with pytest.raises(eo.ExprError, match=msg.replace("(", r"\(").replace(")", r"\)")):
        oracle_eval(code, ref)
    with pytest.raises(capi.GraniteError, match=msg.replace("(", r"\(").replace(")", r"\)")):
        engine_eval(code, ref)


def test_feature_checks_match_reference_order():
    ref = np.zeros(19, np.float32)
    cases = [("z + 1", 2, 3, "undefinded token 'z'"), ("w", 2, 3, "undefinded token 'w'"),
             ("cv", 3, 1, "undefinded token 'cv'"), ("z + w", 2, 3, "undefinded token 'z'")]
    for code, dim, cm, msg in cases:
        with pytest.raises(eo.ExprError, match=msg):
            eo.compile_expression(code, VOLS, CONS, dim, cm)
        with pytest.raises(capi.GraniteError, match=msg):
            capi.evaluate_expression(code, ref, VOLS, CONS, dim, cm)


def test_deep_expressions_use_bounded_stack():
    # a left-deep chain needs one stack slot; a right-deep chain is reordered, so both compile
    left = "x" + "+x" * 60
    right = "x+(" * 20 + "x" + ")" * 20
    ref = np.ones(19, np.float32)
    assert engine_eval(left, ref) == 61.0
    assert engine_eval(right, ref) == 21.0
    # a balanced tree of depth 9 needs 10 slots: rejected with a clear message
    t = "x"
    for _ in range(9):
        t = f"({t})*({t})"
    with pytest.raises(capi.GraniteError):
        engine_eval(t, ref)
