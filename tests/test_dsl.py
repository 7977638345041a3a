"""The DSL compiler against the reference's known bytecode (tests/testthat/test-dsl.R)."""
import numpy as np
import pytest

from gpumetropolis_b200.dsl import DSLError, compile_expr, gpum_model, rhs


def test_golden_bytecode(golden):
    for case in golden["dsl"]:
        prog = compile_expr(rhs(case["formula"]), case["params"], case["data"])
        if "code" in case:
            assert prog.code.tolist() == case["code"]
        if "consts" in case:
            assert prog.consts.tolist() == case["consts"]
        if "min_depth" in case:
            assert prog.depth >= case["min_depth"]


def test_unknown_symbols_and_functions_rejected(golden):
    for case in golden["dsl_errors"]:
        with pytest.raises(DSLError):
            gpum_model(case["formula"], case["params"], case["data"])


def test_r_precedence():
    # -2^2 is -(2^2); ^ is right associative; unary minus binds tighter than *
    p = compile_expr(rhs("~ -2^2"), ["mu"], [])
    assert p.code.tolist() == [0, 0, 0, 0, 11, 0, 7, 0]
    p = compile_expr(rhs("~ mu^2^3"), ["mu"], [])
    assert p.code.tolist() == [1, 0, 0, 0, 0, 1, 11, 0, 11, 0]
    p = compile_expr(rhs("~ -mu * 2"), ["mu"], [])
    assert p.code.tolist() == [1, 0, 7, 0, 0, 0, 5, 0]
    p = compile_expr(rhs("~ 2^-mu"), ["mu"], [])
    assert p.code.tolist() == [0, 0, 1, 0, 7, 0, 11, 0]
    p = compile_expr(rhs("~ a - b - c"), ["a", "b", "c"], [])
    assert p.code.tolist() == [1, 0, 1, 1, 4, 0, 1, 2, 4, 0]


def test_stack_limit_and_depth():
    deep = "~ " + "(mu + " * 31 + "mu" + ")" * 31
    assert compile_expr(rhs(deep), ["mu"], []).depth == 32
    too_deep = "~ " + "(mu + " * 32 + "mu" + ")" * 32
    with pytest.raises(DSLError):
        compile_expr(rhs(too_deep), ["mu"], [])


def test_model_validation():
    m = gpum_model("~ -((y - mu)^2) / 8", params="mu", data="y")
    assert m.n_params == 1 and m.n_cols == 1 and m.prior.n_instr == 0
    with pytest.raises(DSLError):
        gpum_model("-((y - mu)^2) / 8", params="mu", data="y")
    with pytest.raises(DSLError):
        gpum_model("~ mu", params=["mu", "mu"])
    with pytest.raises(DSLError):
        gpum_model("~ mu", params=[])
    with pytest.raises(DSLError):  # the prior may reference parameters only
        gpum_model("~ mu", params="mu", data="y", prior="~ y")
    with pytest.raises(DSLError):  # unary plus is not supported by the reference
        gpum_model("~ +mu", params="mu")


def test_lgamma_and_numbers():
    p = compile_expr(rhs("~ lgamma(y + 1) + 1e-3 * mu + .5"), ["mu"], ["y"])
    assert p.consts.tolist() == [1.0, 1e-3, 0.5]
    assert 12 in p.code[0::2].tolist()
    assert np.all(p.code[1::2][p.code[0::2] >= 3] == 0)
