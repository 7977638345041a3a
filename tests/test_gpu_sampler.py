"""The fused B200 iteration kernel against the oracle sampler.

With the reference's triple32 stream the b200 chains see the same uniforms as
the CPU backend (cpu_native.rs:14-28, 561-562), so proposals agree to f64
rounding and accept decisions agree except where |log ratio - log u| is
inside the FP32 evaluation error of the data sum.
"""
import math

import numpy as np
import pytest

from gpumetropolis_b200 import workloads as W
from gpumetropolis_b200.diagnostics import ess, rhat
from gpumetropolis_b200.dsl import gpum_model
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TIE = 1e-4   # |log ratio - log u| below which FP32 evaluation may flip a decision


def _model_args(w):
    m = w.model
    return (m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, m.n_params,
            w.data, m.n_cols, w.n_obs)


def _logpost(w, pts):
    m = w.model
    pts = np.atleast_2d(pts)
    ll = O.loglik_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols, w.n_obs,
                        pts)
    pr = O.loglik_batch(m.prior.code, m.prior.consts, m.n_params, np.zeros(1), 1, 1, pts)
    return ll + pr


def _normals(seed, c, n, start=0):
    sm = O.seedmix(seed, c)
    z = []
    k = start
    for _ in range(n):
        u1 = O.uniform(sm, k + 1)
        u2 = O.uniform(sm, k + 2)
        k += 2
        z.append(math.sqrt(-2.0 * math.log(u1)) * math.cos(6.283185307179586 * u2))
    return np.array(z), k


@pytest.mark.parametrize("name,n_obs,C,step", [("logistic", 4096, 512, 0.01),
                                                ("student_t", 1031, 300, 0.006)])
def test_single_step_decisions_match(gpu, name, n_obs, C, step):
    # both models run the tensor-core value kernel (their linear predictors
    # as TF32 products): 512 and 300 chains are 4 and 3 (ragged) blocks of
    # 128 chains
    w = W.make(name, n_obs=n_obs)
    m = w.model
    seed = 11
    rng = np.random.default_rng(0)
    centre = w.truth["beta"] if name == "logistic" else np.append(w.truth["beta"], np.log(1.5))
    init = centre + rng.normal(0, 0.02 if name == "logistic" else 0.002, (C, m.n_params))
    sd = np.full((C, m.n_params), step)
    temps = np.where(np.arange(C) % 2 == 0, 1.0, 3.0)
    d_g, a_g, l_g = gpu.run(*_model_args(w), init, sd, temps, 1, seed, 0)
    d_o, a_o, l_o = O.run(*_model_args(w), init, sd, temps, 1, seed, 0)
    cur = _logpost(w, init)
    margins, agree = [], []
    for c in range(C):
        z, k = _normals(seed, c, m.n_params)
        prop = init[c] + sd[c] * z
        plp = _logpost(w, prop)[0]
        lu = math.log(O.uniform(O.seedmix(seed, c), k + 1))
        margins.append(abs((plp - cur[c]) / temps[c] - lu))
        agree.append(a_g[c] == a_o[c])
    margins, agree = np.array(margins), np.array(agree)
    assert np.all(agree[margins > TIE]), np.nonzero(~agree & (margins > TIE))
    assert 0.05 < a_g.mean() < 0.95
    # the recorded state is the proposal or the start, to f32
    dg = d_g.reshape((1, C, m.n_params), order="F")[0]
    do = d_o.reshape((1, C, m.n_params), order="F")[0]
    same = agree & (margins > TIE)
    np.testing.assert_allclose(dg[same], do[same], rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(l_g[same], l_o[same], rtol=1e-6)


@pytest.mark.parametrize("engine", [0, 1], ids=["interp", "compiled"])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_trajectories_follow_the_oracle(gpu, mode, engine):
    w = W.make("gaussian", n_obs=2000)
    C, n_iter, seed = 8, 300, 5
    rng = np.random.default_rng(1)
    init = (w.data.mean() + rng.normal(0, 0.1, C)).reshape(C, 1)
    sd = np.full((C, 1), 0.05)
    temps = np.array([1, 1, 1, 1, 1.5, 2, 4, 8.0])
    L = None
    if mode == 2:
        L = np.full((C, 1, 1), 0.05)
    kw = dict(gamma=0.9, de_noise=0.01, proposal_l=L)
    with gpu.Session(*_model_args(w), engine=engine) as s:
        d_g, a_g, l_g = s.run(init, sd, temps, n_iter, seed, mode, **kw)
    d_o, a_o, l_o = O.run(*_model_args(w), init, sd, temps, n_iter, seed, mode, **kw)
    np.testing.assert_array_equal(a_g, a_o)
    np.testing.assert_allclose(d_g, d_o, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(l_g, l_o, rtol=1e-6)


def test_cholesky_multivariate_trajectories(gpu):
    w = W.make("mixture", n_obs=3000)
    m = w.model
    C, n_iter, seed = 16, 100, 9
    rng = np.random.default_rng(2)
    base = np.array([np.log(0.3 / 0.7), -2.0, 3.0, 0.0, np.log(1.5)])
    init = base + rng.normal(0, 0.02, (C, 5))
    A = rng.normal(0, 1, (5, 5))
    Lc = np.linalg.cholesky(A @ A.T + 5 * np.eye(5)) * 0.004
    L = np.broadcast_to(Lc, (C, 5, 5)).copy()
    sd = np.full((C, 5), 0.01)
    d_g, a_g, l_g = gpu.run(*_model_args(w), init, sd, np.ones(C), n_iter, seed, 2,
                            proposal_l=L)
    d_o, a_o, l_o = O.run(*_model_args(w), init, sd, np.ones(C), n_iter, seed, 2, proposal_l=L)
    # chains that never met a near tie follow the oracle exactly
    same = a_g == a_o
    assert same.mean() >= 0.9
    dg = d_g.reshape((n_iter, C, 5), order="F")
    do = d_o.reshape((n_iter, C, 5), order="F")
    np.testing.assert_allclose(dg[:, same], do[:, same], rtol=1e-5, atol=1e-6)


def test_reproducible_from_the_seed(gpu):
    w = W.make("gaussian", n_obs=3000)
    C = 16
    init = np.linspace(0, 6, C).reshape(C, 1)
    args = (*_model_args(w), init, np.full((C, 1), 0.05), np.ones(C), 200)
    a = gpu.run(*args, 7, 0)[0]
    b = gpu.run(*args, 7, 0)[0]
    c = gpu.run(*args, 8, 0)[0]
    assert np.array_equal(a, b) and not np.array_equal(a, c)


@pytest.mark.parametrize("rng_kind", [0, 1])
def test_gaussian_posterior_recovered(gpu, rng_kind):
    # the Gaussian-mean configuration: y ~ N(3.4, 2^2), N = 20,000; closed form N(mean y, 4/N)
    w = W.make("gaussian")
    C, n_iter = 8, 3000
    init = np.linspace(2.5, 4.5, C).reshape(C, 1)
    sd = np.full((C, 1), 0.03)
    with gpu.Session(*_model_args(w)) as s:
        d, acc, last = s.run(init, sd, np.ones(C), n_iter, 1, 0, rng=rng_kind)
    dr = d.reshape((n_iter, C), order="F")[n_iter // 2:]
    post = w.truth
    e = ess(dr, warmup=0)
    mcse = dr.std() / math.sqrt(e)
    assert abs(dr.mean() - post["post_mean"]) < 5 * mcse
    assert abs(dr.std() - post["post_sd"]) < 0.1 * post["post_sd"]
    assert rhat(dr, warmup=0) < 1.01
    assert np.all((acc > 0.2) & (acc < 0.8))


def test_device_resident_stepping_matches_one_call(gpu):
    w = W.make("logistic", n_obs=3001)
    m = w.model
    C = 70
    init = w.truth["beta"] + np.random.default_rng(3).normal(0, 0.02, (C, m.n_params))
    sd = np.full((C, m.n_params), 0.004)
    with gpu.Session(*_model_args(w)) as s:
        d1, a1, l1 = s.run(init, sd, np.ones(C), 90, 4, 0)
        s.prepare(init, sd, np.ones(C), 90, 4, 0)
        s.advance(33)
        s.advance(40)   # crosses a graph replay boundary
        s.advance(17)
        d2, a2, l2, n = s.fetch()
    assert n == 90
    assert np.array_equal(d1, d2) and np.array_equal(a1, a2) and np.array_equal(l1, l2)


@pytest.mark.parametrize("engine", [0, 1], ids=["interp", "compiled"])
def test_de_sync_generations_follow_the_oracle(gpu, engine):
    # path B: every proposal reads the previous generation of the whole
    # population (cpu_native.rs:400-506), so one flipped decision would
    # change every later generation; with the triple32 stream the GPU
    # population follows the CPU restatement exactly
    w = W.make("gaussian", n_obs=2000)
    C, n_iter, seed = 8, 200, 13
    rng = np.random.default_rng(4)
    init = (w.data.mean() + rng.normal(0, 0.1, C)).reshape(C, 1)
    sd = np.full((C, 1), 0.05)
    with gpu.Session(*_model_args(w), engine=engine) as s:
        d_g, a_g, l_g = s.run_de_sync(init, sd, n_iter, seed, 0.8, 0.01)
    d_o, a_o, l_o = O.run_de_sync(*_model_args(w), init, sd, n_iter, seed, 0.8, 0.01)
    np.testing.assert_array_equal(a_g, a_o)
    np.testing.assert_allclose(d_g, d_o, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(l_g, l_o, rtol=1e-6)
    assert 0.05 < a_g.mean() < 0.95


def test_de_sync_one_shot_entry_matches_session(gpu):
    w = W.make("gaussian", n_obs=1500)
    m = w.model
    C, n_iter = 6, 50
    init = np.linspace(3.0, 3.8, C).reshape(C, 1)
    sd = np.full((C, 1), 0.05)
    d1, a1, l1 = gpu.run_de_sync(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                                 m.n_params, w.data, m.n_cols, w.n_obs, init, sd, n_iter, 3,
                                 0.7, 0.02)
    with gpu.Session(*_model_args(w)) as s:
        d2, a2, l2 = s.run_de_sync(init, sd, n_iter, 3, 0.7, 0.02)
        with pytest.raises(gpu.GpumError, match="at least 3 chains"):
            s.run_de_sync(init[:2], sd[:2], 10, 3, 0.7, 0.02)
    np.testing.assert_array_equal(d1, d2)
    np.testing.assert_array_equal(a1, a2)
