"""The compiled engine: reverse-mode gradients and MALA against the oracle.

The gradient is the reverse-mode adjoint of the bytecode (cpu_native.rs:148-279
restated as generated straight-line code); tolerances: 2e-5 relative to the
gradient's norm (FP32 per-observation adjoints, FP32 per-thread sums, FP64
across threads).
"""
import math

import numpy as np
import pytest

from gpumetropolis_b200 import workloads as W
from gpumetropolis_b200.dsl import gpum_model
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_grad_golden_and_fd(gpu, golden):
    c = golden["gamma"]
    m = gpum_model(c["formula"], c["params"], c["data"])
    y = np.array(c["y"])
    g = gpu.grad_batch(m.loglik.code, m.loglik.consts, 2, y, 1, y.size, c["point"])
    np.testing.assert_allclose(g, c["grad"], rtol=1e-5, atol=1e-5)
    for case in golden["grad_fd"]:
        m = gpum_model(case["formula"], case["params"], case["data"])
        y = np.array(case["y"])
        g = gpu.grad_batch(m.loglik.code, m.loglik.consts, 2, y, 1, y.size, case["point"])
        np.testing.assert_allclose(g, case["grad"], rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("name,n_obs", [("logistic", 3001), ("poisson", 2049),
                                         ("mixture", 4001), ("student_t", 1003)])
def test_grad_batch_matches_oracle(gpu, name, n_obs):
    w = W.make(name, n_obs=n_obs)
    m = w.model
    rng = np.random.default_rng(0)
    base = np.zeros(m.n_params)
    if name in ("logistic", "poisson"):
        base[:] = w.truth["beta"]
    elif name == "student_t":
        base[:-1] = w.truth["beta"]
        base[-1] = math.log(1.5)
    else:
        base[:] = [math.log(0.3 / 0.7), -2.0, 3.0, 0.0, math.log(1.5)]
    pts = base + rng.normal(0, 0.1, (9, m.n_params))
    ref = O.grad_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols, w.n_obs,
                       pts).reshape(9, -1)
    got = gpu.grad_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols,
                         w.n_obs, pts).reshape(9, -1)
    err = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert err.max() < 2e-5, err


def test_grad_fd_check_f64_step_1e4(gpu):
    # Poisson regression gradient vs f64 central differences, step 1e-4
    w = W.make("poisson", n_obs=1500)
    m = w.model
    x = w.truth["beta"] + 0.05
    g = gpu.grad_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols, w.n_obs, x)
    fd = np.empty(m.n_params)
    for j in range(m.n_params):
        e = np.zeros(m.n_params)
        e[j] = 1e-4
        hi = O.loglik_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols,
                            w.n_obs, x + e)[0]
        lo = O.loglik_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols,
                            w.n_obs, x - e)[0]
        fd[j] = (hi - lo) / 2e-4
    assert np.linalg.norm(g - fd) / np.linalg.norm(fd) < 1e-4


def _args(w):
    m = w.model
    return (m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, m.n_params, w.data,
            m.n_cols, w.n_obs)


@pytest.mark.parametrize("with_L", [False, True])
def test_mala_trajectories_follow_the_oracle(gpu, with_L):
    w = W.make("poisson", n_obs=1000, p=6)
    m = w.model
    C, n_iter, seed = 16, 60, 4
    rng = np.random.default_rng(5)
    init = w.truth["beta"] + rng.normal(0, 0.03, (C, m.n_params))
    sd = np.full((C, m.n_params), 0.02)
    L = None
    if with_L:
        A = rng.normal(0, 1, (m.n_params, m.n_params))
        Lc = np.linalg.cholesky(A @ A.T / m.n_params + np.eye(m.n_params)) * 0.02
        L = np.broadcast_to(Lc, (C, m.n_params, m.n_params)).copy()
    temps = np.ones(C)
    d_g, a_g, l_g = gpu.run(*_args(w), init, sd, temps, n_iter, seed, 3, proposal_l=L)
    d_o, a_o, l_o = O.run(*_args(w), init, sd, temps, n_iter, seed, 3, proposal_l=L)
    same = a_g == a_o
    assert same.mean() >= 0.75, (a_g, a_o)
    assert 0.3 < a_g.mean() < 0.99
    dg = d_g.reshape((n_iter, C, m.n_params), order="F")
    do = d_o.reshape((n_iter, C, m.n_params), order="F")
    np.testing.assert_allclose(dg[:, same], do[:, same], rtol=1e-4, atol=1e-5)


def test_mala_and_rwm_on_compiled_engine_recover_gaussian(gpu):
    w = W.make("gaussian", n_obs=4000)
    m = w.model
    C, n_iter = 8, 4000
    init = np.linspace(3.0, 3.8, C).reshape(C, 1)
    sd = np.full((C, 1), 0.03)
    with gpu.Session(*_args(w), engine=1) as s:
        for mode in (0, 3):
            d, acc, _ = s.run(init, sd, np.ones(C), n_iter, 1, mode, rng=1)
            dr = d.reshape((n_iter, C), order="F")[n_iter // 2:]
            from gpumetropolis_b200.diagnostics import ess, rhat
            e = ess(dr, warmup=0)
            assert abs(dr.mean() - w.data.mean()) < 5 * dr.std() / math.sqrt(e)
            assert rhat(dr, warmup=0) < 1.01


def test_softplus_rewrite_is_accurate(gpu):
    # LOG(1 + EXP(z)) is evaluated as max(z, 0) + log1p(e^-|z|) in the value
    # kernels.  Per observation it is compared with an exact f64 softplus of
    # the same FP32 argument z = fl32(a * x): relative error of a few FP32
    # ulp wherever softplus(z) is a normal FP32 number (the naive f64 form of
    # the oracle rounds to 0 once e^z < 1e-16, so it is not the yardstick
    # here); the sums are still checked against the oracle.
    from gpumetropolis_b200.dsl import gpum_model
    m = gpum_model("~ log(1 + exp(a * x))", "a", "x")
    x = np.concatenate([np.linspace(-95, 95, 4001), np.linspace(-3, 3, 4001),
                        [0.0, 1e-30, -1e-30, 87.0, -87.0, 200.0, -200.0]])
    x = x.astype(np.float32).astype(np.float64)
    a = np.array([1.0, -0.5])
    with gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, 1,
                     x.reshape(-1, 1), 1, x.size, engine=1) as s:
        got = s.loglik_pointwise(a.reshape(-1, 1)).reshape(2, -1)
        tot = s.loglik_batch(a.reshape(-1, 1))
    z = (a[:, None].astype(np.float32) * x[None, :].astype(np.float32)).astype(np.float64)
    exact = np.logaddexp(0.0, z)
    assert np.all(np.isfinite(got))
    normal = exact > 1e-30
    rel = np.abs(got[normal] - exact[normal]) / exact[normal]
    assert rel.max() < 6e-7, rel.max()
    assert np.abs(got[~normal] - exact[~normal]).max() < 1e-30
    want = O.loglik_pointwise(m.loglik.code, m.loglik.consts, 1, x.reshape(-1, 1), 1, x.size,
                              a.reshape(-1, 1)).reshape(2, -1)
    np.testing.assert_allclose(tot, want.sum(axis=1), rtol=1e-6)


def test_materialized_data_columns(gpu):
    # log(y), x^2 and lgamma(y + 1) depend on the data only: the compiled
    # engine computes them once per session into three extra columns (y + 1 is
    # an intermediate, not a column) and loads them per observation; the
    # interpreter on the same session reads the original columns
    rng = np.random.default_rng(4)
    n = 3001
    y = rng.lognormal(0.5, 0.7, n)
    x = rng.normal(0.0, 1.0, n)
    m = gpum_model("~ -((log(y) - mu - b * x^2)^2) / (2 * exp(2 * ls)) - ls - log(y)"
                   " - lgamma(y + 1)", ["mu", "b", "ls"], ["y", "x"])
    data = np.column_stack([y, x])
    pts = np.array([0.5, 0.0, math.log(0.7)]) + rng.normal(0, 0.05, (40, 3))
    args = (m.loglik.code, m.loglik.consts, 3, data, 2, n)
    ref = O.loglik_batch(*args, pts)
    ref_pw = O.loglik_pointwise(*args, pts[:4])
    ref_g = O.grad_batch(*args, pts[:6]).reshape(6, -1)
    with gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, 3, data, 2,
                     n, engine=1) as s:
        got = s.loglik_batch(pts)
        pw = s.loglik_pointwise(pts[:4])
        g = s.grad_batch(pts[:6]).reshape(6, -1)
        s.set_engine(0)
        got_i = s.loglik_batch(pts)
        s.set_engine(1)
        again = s.loglik_batch(pts)
    np.testing.assert_allclose(got, ref, rtol=1e-6)
    np.testing.assert_allclose(pw, ref_pw, rtol=2e-5, atol=2e-5)
    err = np.linalg.norm(g - ref_g, axis=1) / np.linalg.norm(ref_g, axis=1)
    assert err.max() < 2e-5, err
    np.testing.assert_allclose(got_i, ref, rtol=1e-6)
    np.testing.assert_array_equal(again, got)


def test_log_sum_of_exponentials_rewrite(gpu):
    # log(c1 e^a + c2 e^b) with positive parameter-only weights is evaluated
    # as logaddexp(a + log c1, b + log c2): finite where FP32 e^a and e^b both
    # underflow (|y| far in the tails) and the oracle's f64 sum is finite
    from gpumetropolis_b200 import workloads as W
    w = W.make("mixture", n_obs=200)
    m = w.model
    y = np.concatenate([np.linspace(-40, 40, 801), w.data[:200, 0]])
    pts = np.array([[math.log(0.3 / 0.7), -2.0, 3.0, 0.0, math.log(1.5)],
                    [0.4, -1.0, 2.0, -0.3, 0.2]])
    args = (m.loglik.code, m.loglik.consts, m.n_params, y.reshape(-1, 1), 1, y.size)
    ref = O.loglik_pointwise(*args, pts).reshape(2, -1)
    with gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, m.n_params,
                     y.reshape(-1, 1), 1, y.size, engine=1) as s:
        got = s.loglik_pointwise(pts).reshape(2, -1)
        tot = s.loglik_batch(pts)
    assert np.all(np.isfinite(ref)) and np.all(np.isfinite(got))
    np.testing.assert_allclose(got, ref, rtol=2e-6, atol=1e-5)
    np.testing.assert_allclose(tot, ref.sum(axis=1), rtol=1e-6)


@pytest.mark.parametrize("n_pts", [300, 5])
def test_grad_batch_chain_lanes(gpu, n_pts):
    # the Student-t model (65 parameters) runs the chain-lane gradient body:
    # 300 points are two blocks of 256 chains, 5 points share one warp group
    # whose warps split the observation quads; 20,011 observations make many
    # tiles per CTA (per-tile FP64 flushes) and a ragged last quad
    w = W.make("student_t", n_obs=20011)
    m = w.model
    rng = np.random.default_rng(6)
    base = np.append(w.truth["beta"], math.log(1.5))
    pts = base + rng.normal(0, 0.02, (n_pts, m.n_params))
    ref = O.grad_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols, w.n_obs,
                       pts).reshape(n_pts, -1)
    got = gpu.grad_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols,
                         w.n_obs, pts).reshape(n_pts, -1)
    err = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert err.max() < 2e-5, err.max()


def test_wide_model_with_materialized_columns(gpu):
    # 50 parameters (the chain-lane value and gradient bodies) whose 50
    # data-only terms x_j^2 are materialized columns: values and gradients
    # against the oracle
    p = 50
    rng = np.random.default_rng(8)
    n = 2003
    X = rng.normal(0.0, 1.0, (n, p))
    beta = rng.normal(0.0, 0.1, p)
    y = (X ** 2) @ beta + rng.normal(0.0, 1.0, n)
    params = [f"b{j}" for j in range(1, p + 1)]
    xs = [f"x{j}" for j in range(1, p + 1)]
    m = gpum_model("~ -((y - (" + " + ".join(f"b{j} * x{j}^2" for j in range(1, p + 1))
                   + "))^2) / 2", params, xs + ["y"])
    data = np.column_stack([X, y])
    pts = beta + rng.normal(0.0, 0.02, (40, p))
    args = (m.loglik.code, m.loglik.consts, p, data, p + 1, n)
    ref = O.loglik_batch(*args, pts)
    ref_g = O.grad_batch(*args, pts).reshape(40, -1)
    got = gpu.loglik_batch(*args, pts)
    g = gpu.grad_batch(*args, pts).reshape(40, -1)
    np.testing.assert_allclose(got, ref, rtol=1e-6)
    err = np.linalg.norm(g - ref_g, axis=1) / np.linalg.norm(ref_g, axis=1)
    assert err.max() < 2e-5, err.max()


@pytest.mark.parametrize("name,n_obs", [("logistic", 3001), ("poisson", 2049),
                                         ("mixture", 4001), ("student_t", 1003)])
def test_interpreter_grad_batch_matches_oracle(gpu, name, n_obs):
    # the interpreter engine's gradient (a reverse sweep over each
    # observation's tape of the interpreted program) without NVRTC's code:
    # against the oracle, at the compiled engine's tolerance
    w = W.make(name, n_obs=n_obs)
    m = w.model
    rng = np.random.default_rng(1)
    base = np.zeros(m.n_params)
    if name in ("logistic", "poisson"):
        base[:] = w.truth["beta"]
    elif name == "student_t":
        base[:-1] = w.truth["beta"]
        base[-1] = math.log(1.5)
    else:
        base[:] = [math.log(0.3 / 0.7), -2.0, 3.0, 0.0, math.log(1.5)]
    pts = base + rng.normal(0, 0.1, (7, m.n_params))
    ref = O.grad_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols, w.n_obs,
                       pts).reshape(7, -1)
    with gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, m.n_params,
                     w.data, m.n_cols, w.n_obs, engine=0) as s:
        got = s.grad_batch(pts).reshape(7, -1)
    err = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert err.max() < 2e-5, err


@pytest.mark.parametrize("with_L", [False, True])
def test_mala_on_the_interpreter_engine_follows_the_oracle(gpu, with_L):
    # MALA with the interpreter engine's gradient and the interpreted prior's
    # tape gradient: the oracle's trajectories, as on the compiled engine
    w = W.make("poisson", n_obs=1000, p=6)
    m = w.model
    C, n_iter, seed = 16, 60, 4
    rng = np.random.default_rng(5)
    init = w.truth["beta"] + rng.normal(0, 0.03, (C, m.n_params))
    sd = np.full((C, m.n_params), 0.02)
    L = None
    if with_L:
        A = rng.normal(0, 1, (m.n_params, m.n_params))
        Lc = np.linalg.cholesky(A @ A.T / m.n_params + np.eye(m.n_params)) * 0.02
        L = np.broadcast_to(Lc, (C, m.n_params, m.n_params)).copy()
    temps = np.ones(C)
    with gpu.Session(*_args(w), engine=0) as s:
        d_g, a_g, l_g = s.run(init, sd, temps, n_iter, seed, 3, proposal_l=L)
    d_o, a_o, l_o = O.run(*_args(w), init, sd, temps, n_iter, seed, 3, proposal_l=L)
    same = a_g == a_o
    assert same.mean() >= 0.75, (a_g, a_o)
    assert 0.3 < a_g.mean() < 0.99
    dg = d_g.reshape((n_iter, C, m.n_params), order="F")
    do = d_o.reshape((n_iter, C, m.n_params), order="F")
    np.testing.assert_allclose(dg[:, same], do[:, same], rtol=1e-4, atol=1e-5)
