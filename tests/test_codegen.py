"""The compiled engine's code generation without a GPU: every workload model
and every rewrite the generator applies (the fused softplus, the
product-minus-softplus fold, log of two weighted exponentials, hoisted
reciprocals, materialized data-only columns, the chain-lane value and
gradient bodies of wide models, the tensor-core value kernel of models with a
linear predictor) goes through bytecode -> CUDA C -> NVRTC and
yields an sm_100a cubin (gpum_b200_compile_check)."""
import pytest

from gpumetropolis_b200 import _native
from gpumetropolis_b200 import workloads as W
from gpumetropolis_b200.build import build
from gpumetropolis_b200.dsl import gpum_model


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build()


def _extra_models():
    return {
        "softplus": gpum_model("~ log(1 + exp(a * x))", "a", "x"),
        "logaddexp_const_weights": gpum_model(
            "~ log(0.3 * exp(-((y - m1)^2) / 2) + 0.7 * exp(-((y - m2)^2) / 2))",
            ["m1", "m2"], "y"),
        "reciprocal_and_materialized": gpum_model(
            "~ -((log(y) - mu - b * x^2)^2) / (2 * exp(2 * ls)) - ls - log(y) - lgamma(y + 1)",
            ["mu", "b", "ls"], ["y", "x"]),
        # the tensor-core value kernel: coefficients that are parameter-only
        # expressions, a column with two coefficients, a constant divisor and
        # an offset
        "linear_predictor_tensor_cores": gpum_model(
            "~ -((y - (m + b0^2 + exp(ls) * x1 - b2 * x2 + 2 * b3 * x3 + b4 * x4 / 3"
            " + b5 * (x5 + x6) + b6 * x5))^2) / 2",
            ["m", "b0", "ls", "b2", "b3", "b4", "b5", "b6"],
            ["x1", "x2", "x3", "x4", "x5", "x6", "y"]),
        "wide_with_data_ops": gpum_model(
            "~ -((y - (" + " + ".join(f"b{j} * x{j}^2" for j in range(1, 56)) + "))^2) / 2",
            [f"b{j}" for j in range(1, 56)], [f"x{j}" for j in range(1, 56)] + ["y"]),
    }


@pytest.mark.parametrize("name", sorted(W.ALL))
def test_workload_models_compile(name):
    m = W.make(name, n_obs=16).model
    size = _native.compile_check(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                                 m.n_params, m.n_cols)
    assert size > 0


@pytest.mark.parametrize("name", sorted(_extra_models()))
def test_rewrite_patterns_compile(name):
    m = _extra_models()[name]
    size = _native.compile_check(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                                 m.n_params, m.n_cols)
    assert size > 0
