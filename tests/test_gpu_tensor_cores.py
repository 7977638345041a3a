"""The compiled engine's tensor-core value kernel (gm_iter_value_tc) against
the f64 oracle and against the FP32 value kernel of the same session setup.

The kernel computes a model's linear predictor (sum of parameter-only
coefficients times data columns, plus a parameter-only offset) for 128
chains x a tile of observations as a TF32 tensor-core product with both
operands split into hi + lo (three products, FP32 accumulation), and the rest
of each term on the FP32 pipes.  Tolerances: the summed log-likelihood within
1e-6 relative of the f64 oracle, as for every other kernel; against the FP32
kernel, 1e-6 relative as well (both are FP32 evaluations of the same terms).
Non-finite parameters must give exactly the oracle's non-finite results
(the split products would turn inf * 0 into NaN; the kernel evaluates such
chains' predictor on the FP32 pipe), and a non-finite value in a product
column keeps the session on the FP32 kernel.
"""
import os

import numpy as np
import pytest

from gpumetropolis_b200 import workloads as W
from gpumetropolis_b200.dsl import gpum_model
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL_SUM = 1e-6


def _base(w):
    m = w.model
    base = np.zeros(m.n_params)
    if w.name in ("logistic", "poisson"):
        base[:] = w.truth["beta"]
    elif w.name == "student_t":
        base[:-1] = w.truth["beta"]
        base[-1] = np.log(1.5)
    return base


def _points(w, n, seed=0, scale=0.05):
    rng = np.random.default_rng(seed)
    return _base(w) + rng.normal(0, scale, (n, w.model.n_params))


def _session(gpu, m, data, n_obs, tensor_cores=True):
    old = os.environ.get("GPUM_B200_TENSOR_CORES")
    os.environ["GPUM_B200_TENSOR_CORES"] = "1" if tensor_cores else "0"
    try:
        s = gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                        m.n_params, data, m.n_cols, n_obs, engine=1)
        s.tensor_cores  # the compiled engine is built (and the data packed) here
    finally:
        if old is None:
            del os.environ["GPUM_B200_TENSOR_CORES"]
        else:
            os.environ["GPUM_B200_TENSOR_CORES"] = old
    return s


def _oracle(m, w_data, n_obs, pts):
    return O.loglik_batch(m.loglik.code, m.loglik.consts, m.n_params, w_data, m.n_cols, n_obs,
                          pts)


@pytest.mark.parametrize("name,n_obs,n_pts", [("logistic", 4099, 37), ("logistic", 1, 3),
                                               ("logistic", 255, 129), ("logistic", 257, 300),
                                               ("poisson", 3001, 131), ("student_t", 1031, 37),
                                               ("student_t", 129, 5)])
def test_matches_oracle_and_fp32_kernel(gpu, name, n_obs, n_pts):
    # ragged in every dimension: observations around the 256-observation
    # tile, points around the 128-chain block
    w = W.make(name, n_obs=n_obs)
    m = w.model
    pts = _points(w, n_pts)
    ref = _oracle(m, w.data, w.n_obs, pts)
    with _session(gpu, m, w.data, w.n_obs) as s:
        assert s.tensor_cores
        got = s.loglik_batch(pts)
    with _session(gpu, m, w.data, w.n_obs, tensor_cores=False) as s:
        assert not s.tensor_cores
        fp32 = s.loglik_batch(pts)
    assert (np.abs(got - ref) / np.abs(ref)).max() <= REL_SUM
    assert (np.abs(got - fp32) / np.abs(ref)).max() <= REL_SUM


def test_hoisted_coefficients_offset_and_constant_divisors(gpu):
    # coefficients that are parameter-only expressions (exp(ls), 2 * b3),
    # a column shared by two coefficients, a division by a constant, and an
    # offset (m + b0^2); the tail reads y
    lp = "m + b0^2 + exp(ls) * x1 - b2 * x2 + 2 * b3 * x3 + b4 * x4 / 3 + b5 * (x5 + x6) + b6 * x5"
    f = f"~ -((y - ({lp}))^2) / 2"
    params = ["m", "b0", "ls", "b2", "b3", "b4", "b5", "b6"]
    data_names = ["x1", "x2", "x3", "x4", "x5", "x6", "y"]
    m = gpum_model(f, params, data_names)
    rng = np.random.default_rng(5)
    n = 3000
    data = rng.normal(0, 1, (n, 7))
    data[:, 6] = data[:, :6] @ rng.normal(0, 0.5, 6) + rng.normal(0, 1, n)
    pts = rng.normal(0, 0.3, (41, len(params)))
    ref = _oracle(m, data, n, pts)
    with _session(gpu, m, data, n) as s:
        assert s.tensor_cores
        got = s.loglik_batch(pts)
    assert (np.abs(got - ref) / np.abs(ref)).max() <= REL_SUM


def test_nonfinite_parameters_follow_the_oracle(gpu):
    w = W.make("logistic", n_obs=1000)
    m = w.model
    pts = _points(w, 8, seed=3)
    pts[1, 3] = np.inf        # a coefficient: +-inf terms
    pts[2, 0] = -np.inf       # the offset
    pts[3, 5] = np.nan
    pts[4, 2] = np.inf
    pts[4, 7] = -np.inf       # +inf and -inf coefficients together
    ref = _oracle(m, w.data, w.n_obs, pts)
    with _session(gpu, m, w.data, w.n_obs) as s:
        assert s.tensor_cores
        got = s.loglik_batch(pts)
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    np.testing.assert_array_equal(np.isposinf(got), np.isposinf(ref))
    np.testing.assert_array_equal(np.isneginf(got), np.isneginf(ref))
    fin = np.isfinite(ref)
    assert fin.sum() >= 4
    assert (np.abs(got[fin] - ref[fin]) / np.abs(ref[fin])).max() <= REL_SUM


def test_nonfinite_data_column_keeps_the_fp32_kernel(gpu):
    w = W.make("logistic", n_obs=700)
    m = w.model
    data = w.data.copy()
    data[123, 4] = np.inf
    pts = _points(w, 6, seed=4)
    ref = _oracle(m, data, w.n_obs, pts)
    with _session(gpu, m, data, w.n_obs) as s:
        assert not s.tensor_cores
        got = s.loglik_batch(pts)
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    fin = np.isfinite(ref)
    if fin.any():
        assert (np.abs(got[fin] - ref[fin]) / np.abs(ref[fin])).max() <= REL_SUM


@pytest.mark.parametrize("mode", [0, 1, 2], ids=["rwm", "de", "cholesky"])
def test_sampler_steps_on_tensor_cores_follow_the_fp32_kernel(gpu, mode):
    # the same run (triple32 stream) with and without the tensor-core kernel:
    # identical accept rates for nearly every chain (a decision inside the
    # FP32 rounding of the data sum may differ), and then log posteriors
    # equal to 1e-6
    w = W.make("logistic", n_obs=3001)
    m = w.model
    C, npar = 160, m.n_params
    init = _points(w, C, seed=6, scale=0.02)
    sd = np.full((C, npar), 0.01)
    gamma = 2.38 / np.sqrt(2 * npar) if mode == 1 else 0.0
    L = np.tile(np.eye(npar) * 0.01, (C, 1, 1)) if mode == 2 else None
    out = []
    for tc in (True, False):
        with _session(gpu, m, w.data, w.n_obs, tensor_cores=tc) as s:
            assert s.tensor_cores == tc
            out.append(s.run(init, sd, np.ones(C), 60, 7, mode, gamma, 1e-4, proposal_l=L))
    (_, a1, l1), (_, a0, l0) = out
    same = a1 == a0
    assert same.mean() >= 0.95
    assert (np.abs(l1[same] - l0[same]) / np.abs(l0[same])).max() <= REL_SUM


@pytest.mark.parametrize("formula,params,data,uses", [
    # five data columns: below the predictor's minimum of six
    ("~ -((y - (a + b1 * x1 + b2 * x2 + b3 * x3 + b4 * x4))^2) / 2",
     ["a", "b1", "b2", "b3", "b4"], ["x1", "x2", "x3", "x4", "y"], False),
    # a per-observation product inside the predictor is also read outside it
    ("~ -((y - (b1 * x1 + b2 * x2 + b3 * x3 + b4 * x4 + b5 * x5 + b6 * x6))^2) / 2"
     " - (b1 * x1)^2", ["b1", "b2", "b3", "b4", "b5", "b6"],
     ["x1", "x2", "x3", "x4", "x5", "x6", "y"], False),
    # no affine predictor at all
    ("~ -((y - mu)^2) / (2 * exp(2 * ls)) - ls", ["mu", "ls"], ["y"], False),
    # six columns: eligible
    ("~ -((y - (b1 * x1 + b2 * x2 + b3 * x3 + b4 * x4 + b5 * x5))^2) / 2",
     ["b1", "b2", "b3", "b4", "b5"], ["x1", "x2", "x3", "x4", "x5", "y"], True),
])
def test_which_models_run_on_tensor_cores(gpu, formula, params, data, uses):
    # eligibility of the linear predictor, and the value either way against
    # the oracle
    m = gpum_model(formula, params, data)
    rng = np.random.default_rng(9)
    n = 1500
    d = rng.normal(0, 1, (n, len(data)))
    pts = rng.normal(0, 0.3, (9, len(params)))
    ref = _oracle(m, d, n, pts)
    with _session(gpu, m, d, n) as s:
        assert s.tensor_cores == uses
        got = s.loglik_batch(pts)
        # pointwise output keeps the FP32 kernel in every case
        pw = s.loglik_pointwise(pts[:2])
    assert (np.abs(got - ref) / np.abs(ref)).max() <= REL_SUM
    pref = O.loglik_pointwise(m.loglik.code, m.loglik.consts, m.n_params, d, m.n_cols, n, pts[:2])
    np.testing.assert_allclose(pw, pref, rtol=2e-5, atol=2e-5)
