"""Power posteriors and thermodynamic-integration evidence on the B200.

The reference builds a "power model" per rung by appending PUSH_CONST beta;
MUL to the log-likelihood bytecode (R/bayes.R:266-277); the oracle runs that
model, the GPU runs the original model with a per-chain likelihood power."""
import math

import numpy as np
import pytest

from gpumetropolis_b200 import api
from gpumetropolis_b200 import workloads as W
from gpumetropolis_b200.dsl import gpum_model
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _power_program(prog, beta):
    code = np.concatenate([np.asarray(prog.code, np.uint32),
                           np.array([0, len(prog.consts), 5, 0], np.uint32)])
    consts = np.concatenate([np.asarray(prog.consts, np.float64), [beta]])
    return code, consts


def test_likelihood_power_follows_the_power_model(gpu):
    w = W.make("gaussian", n_obs=2000)
    m = gpum_model("~ -((y - mu)^2) / 8", "mu", "y", prior="~ -((mu - 3)^2) / 50")
    beta, C, n_iter, seed = 0.3, 8, 200, 6
    rng = np.random.default_rng(2)
    init = (w.data.mean() + rng.normal(0, 0.1, C)).reshape(C, 1)
    sd = np.full((C, 1), 0.08)
    with gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, 1, w.data,
                     1, w.n_obs) as s:
        s.set_likelihood_powers(np.full(C, beta))
        d_g, a_g, l_g = s.run(init, sd, np.ones(C), n_iter, seed, 0)
        with pytest.raises(gpu.GpumError, match="likelihood powers were set for 8"):
            s.run(init[:4], sd[:4], np.ones(4), 5, seed, 0)
        s.set_likelihood_powers(None)
        d_1, _, _ = s.run(init, sd, np.ones(C), n_iter, seed, 0)
    code, consts = _power_program(m.loglik, beta)
    d_o, a_o, l_o = O.run(code, consts, m.prior.code, m.prior.consts, 1, w.data, 1, w.n_obs,
                          init, sd, np.ones(C), n_iter, seed, 0)
    np.testing.assert_array_equal(a_g, a_o)
    np.testing.assert_allclose(d_g, d_o, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(l_g, l_o, rtol=1e-6)
    assert not np.array_equal(d_g, d_1)  # clearing the powers restores beta = 1


def _gauss_log_evidence(y, sigma, m0, s0):
    # log of the integral of exp(-sum (y - mu)^2 / (2 sigma^2)) N(mu; m0, s0^2) dmu
    n, ybar = y.size, y.mean()
    S = np.sum((y - ybar) ** 2)
    v = s0 ** 2 + sigma ** 2 / n
    return (-S / (2 * sigma ** 2) + 0.5 * math.log(2 * math.pi * sigma ** 2 / n)
            - 0.5 * math.log(2 * math.pi * v) - (ybar - m0) ** 2 / (2 * v))


def test_evidence_matches_the_closed_form():
    rng = np.random.default_rng(7)
    y = rng.normal(3.0, 2.0, 400)
    m = gpum_model("~ -((y - mu)^2) / 8", "mu", "y", prior="~ -((mu - 3)^2) / 50")
    ev = api.gpum_evidence(m, {"y": y}, n_rungs=24, n_iter=3000, n_chains=8, seed=3)
    want = _gauss_log_evidence(y, 2.0, 3.0, 5.0)
    assert ev.betas[0] == 0.0 and ev.betas[-1] == 1.0 and ev.expected_loglik.size == 25
    assert np.all(np.diff(ev.expected_loglik) >= -1.0)  # E_beta[log L] rises with beta
    assert abs(ev.log_evidence - want) < 0.25, (ev.log_evidence, want)


def test_bayes_factor_favours_the_prior_near_the_data():
    # test-bayes.R:84-98
    rng = np.random.default_rng(1)
    y = rng.normal(3.0, 2.0, 400)
    near = gpum_model("~ -((y - mu)^2) / 8", "mu", "y", prior="~ -((mu - 3)^2) / (2 * 25)")
    far = gpum_model("~ -((y - mu)^2) / 8", "mu", "y", prior="~ -((mu + 3)^2) / (2 * 25)")
    bf = api.gpum_bayes_factor(near, far, {"y": y}, n_rungs=8, n_iter=2000, n_chains=8, seed=1)
    assert bf.bf10 > 1 and math.isfinite(bf.log_bf10)
    # 8 rungs leave a trapezoidal bias of a few tenths of a nat; the sign of
    # the log Bayes factor is the closed form's
    want = (_gauss_log_evidence(y, 2.0, 3.0, 5.0) - _gauss_log_evidence(y, 2.0, -3.0, 5.0))
    assert want > 0 and bf.log_bf10 > 0
    assert bf.interpretation in ("barely worth mention", "substantial", "strong")
