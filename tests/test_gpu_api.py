"""gpu_metropolis end to end on the B200 backend, mirroring the reference's
integration tests (tests/testthat/test-api.R, test-pt.R, test-de.R,
test-mala.R, test-adaptive.R) with posterior checks against closed forms."""
import math

import numpy as np
import pytest

from gpumetropolis_b200 import workloads as W
from gpumetropolis_b200.api import gpu_metropolis
from gpumetropolis_b200.diagnostics import ess, rhat
from gpumetropolis_b200.dsl import gpum_model

pytestmark = pytest.mark.gpu


def _mcse(d):
    return d.std() / math.sqrt(ess(d, warmup=0))


def test_config1_adaptive_rwm_recovers_closed_form(gpu):
    # the Gaussian-mean configuration: y ~ N(3.4, 2^2), N = 20,000; rwm, 8 chains x 3,000
    # iterations, adaptive warmup, proposal_sd 0.5; posterior N(mean y, 4/N)
    w = W.make("gaussian")
    fit = gpu_metropolis(w.model, data={"y": w.data[:, 0]}, proposal_sd=0.5, n_iter=3000,
                         n_chains=8, seed=1)
    d = fit["mu"]
    assert d.shape == (1500, 8)
    assert fit.warmup == 1500 and fit.n_iter_total == 3000
    assert abs(d.mean() - w.truth["post_mean"]) < 5 * _mcse(d)
    assert abs(d.std() - w.truth["post_sd"]) < 0.15 * w.truth["post_sd"]
    assert rhat(d, warmup=0) < 1.01
    assert fit.adaptation is not None and fit.adaptation["batch_sizes"].sum() == 1500


def test_adaptation_rescues_a_bad_proposal(gpu):
    # test-adaptive.R:275-294
    rng = np.random.default_rng(42)
    y = rng.normal(5.0, 1.0, 500)
    m = gpum_model("~ -((y - mu)^2) / 2", "mu", "y")
    on = gpu_metropolis(m, {"y": y}, proposal_sd=1e-4, n_iter=2000, n_chains=4, warmup=1000,
                        adapt=True, seed=1)
    off = gpu_metropolis(m, {"y": y}, proposal_sd=1e-4, n_iter=2000, n_chains=4, warmup=1000,
                         adapt=False, seed=1)
    assert abs(on["mu"].mean() - y.mean()) < 0.1
    assert abs(off["mu"].mean() - y.mean()) > abs(on["mu"].mean() - y.mean())
    assert off.adaptation is None


def test_same_seed_same_draws(gpu):
    rng = np.random.default_rng(2)
    y = rng.normal(1.0, 2.0, 1000)
    m = gpum_model("~ -((y - mu)^2) / 8", "mu", "y")
    a = gpu_metropolis(m, {"y": y}, proposal_sd=0.1, n_iter=500, n_chains=2, seed=7)
    b = gpu_metropolis(m, {"y": y}, proposal_sd=0.1, n_iter=500, n_chains=2, seed=7)
    assert np.array_equal(a.draws, b.draws)


def test_pt_cold_chain_covers_both_modes(gpu):
    # test-pt.R:198-217: y ~ N(|mu|, 1); without swaps a chain keeps its mode
    rng = np.random.default_rng(1)
    y = rng.normal(3.0, 1.0, 400)
    m = gpum_model("~ log(exp(-((y - mu)^2) / 2) + exp(-((y + mu)^2) / 2))", "mu", "y")
    init = np.linspace(-6, 6, 8).reshape(8, 1)
    fit = gpu_metropolis(m, {"y": y}, init=init, proposal_sd=0.15, n_iter=4000, method="pt",
                         seed=1)
    cold = fit.draws[:, 0, 0]
    assert fit.extra["temperatures"][0] == 1.0
    assert np.any(cold > 1.5) and np.any(cold < -1.5)
    assert abs(cold[cold > 0].mean() - 3) < 0.4 and abs(cold[cold < 0].mean() + 3) < 0.4
    sh = fit.adaptation["swap_history"]
    assert sh.shape == (7, fit.adaptation["n_batches"])


def test_de_recovers_correlated_bivariate(gpu):
    # test-de.R:43-72
    rng = np.random.default_rng(1)
    rho = 0.9
    S = np.array([[1, rho], [rho, 1]])
    y = rng.standard_normal((500, 2)) @ np.linalg.cholesky(S).T + np.array([2.0, -1.0])
    Si = np.linalg.inv(S)
    f = (f"~ -0.5 * ({Si[0, 0]:.6f}*(y1-mu1)^2 + 2*{Si[0, 1]:.6f}*(y1-mu1)*(y2-mu2)"
         f" + {Si[1, 1]:.6f}*(y2-mu2)^2)")
    m = gpum_model(f, ["mu1", "mu2"], ["y1", "y2"])
    fit = gpu_metropolis(m, {"y1": y[:, 0], "y2": y[:, 1]}, n_iter=8000, n_chains=16,
                         method="de", seed=1)
    d1, d2 = fit["mu1"].ravel(), fit["mu2"].ravel()
    assert abs(d1.mean() - y[:, 0].mean()) < 0.02
    assert abs(d2.mean() - y[:, 1].mean()) < 0.02
    assert abs(np.corrcoef(d1, d2)[0, 1] - rho) < 0.05
    assert rhat(fit["mu1"], warmup=0) < 1.05


def test_de_sync_recovers_correlated_bivariate(gpu):
    # path B (R/api.R:464-497): per-generation population, trim-only warmup
    rng = np.random.default_rng(3)
    rho = 0.9
    S = np.array([[1, rho], [rho, 1]])
    y = rng.standard_normal((500, 2)) @ np.linalg.cholesky(S).T + np.array([2.0, -1.0])
    Si = np.linalg.inv(S)
    f = (f"~ -0.5 * ({Si[0, 0]:.6f}*(y1-mu1)^2 + 2*{Si[0, 1]:.6f}*(y1-mu1)*(y2-mu2)"
         f" + {Si[1, 1]:.6f}*(y2-mu2)^2)")
    m = gpum_model(f, ["mu1", "mu2"], ["y1", "y2"])
    fit = gpu_metropolis(m, {"y1": y[:, 0], "y2": y[:, 1]}, n_iter=8000, n_chains=16,
                         method="de", de_sync=True, seed=2)
    assert fit.extra["de_sync"] and fit.adaptation is None
    assert fit.draws.shape == (4000, 16, 2) and fit.warmup == 4000
    d1, d2 = fit["mu1"].ravel(), fit["mu2"].ravel()
    assert abs(d1.mean() - y[:, 0].mean()) < 0.02
    assert abs(d2.mean() - y[:, 1].mean()) < 0.02
    assert abs(np.corrcoef(d1, d2)[0, 1] - rho) < 0.05
    assert rhat(fit["mu1"], warmup=0) < 1.05


def test_mala_recovers_gaussian_at_its_target_rate(gpu):
    # test-mala.R:35-46 (runs on the GPU here; the reference refuses a GPU)
    rng = np.random.default_rng(1)
    y = rng.normal(2.5, 1.0, 400)
    m = gpum_model("~ -((y - mu)^2) / 2", "mu", "y")
    fit = gpu_metropolis(m, {"y": y}, n_iter=8000, n_chains=4, method="mala", seed=1)
    assert fit.method == "mala"
    assert abs(fit.draws.mean() - y.mean()) < 0.01
    assert abs(fit.draws.std() - 1 / math.sqrt(400)) < 0.15 / math.sqrt(400)
    assert np.all((fit.accept_rate > 0.45) & (fit.accept_rate < 0.70))


def test_nonfinite_start_and_proposals(gpu):
    # test-numerical.R:32-67
    m = gpum_model("~ log(mu) - mu + 0 * y", "mu", "y")
    fit = gpu_metropolis(m, {"y": [0.0]}, init=[[1.5]], proposal_sd=0.4, n_iter=3000, seed=1)
    d = fit.draws[:, 0, 0]
    assert np.all(np.isfinite(d)) and d.min() > 0 and abs(d.mean() - 2) < 0.4
    fit = gpu_metropolis(m, {"y": [0.0]}, init=[[-1.0]], proposal_sd=0.3, n_iter=500, seed=1)
    assert fit.draws.shape == (250, 1, 1)


def test_device_moments_match_the_draws(gpu):
    # the adaptive warmup reduces each batch on the device instead of copying
    # its draws; the moments equal those of the draws themselves
    from gpumetropolis_b200 import adaptive as AD
    from gpumetropolis_b200 import workloads as W
    w = W.make("logistic", n_obs=3000)
    m = w.model
    C, n = 40, 30
    rng = np.random.default_rng(2)
    init = w.truth["beta"] + rng.normal(0, 0.05, (C, m.n_params))
    sd = np.full((C, m.n_params), 0.02)
    with gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, m.n_params,
                     w.data, m.n_cols, w.n_obs) as s:
        s.prepare(init, sd, np.ones(C), n, 4, 0)
        s.advance(n)
        cm, c2, pm, p2 = s.draw_moments(0, n)
        last = s.state()
        d, _, _, _ = s.fetch()
    ref = AD.moments_of(d.reshape((n, C, m.n_params), order="F"))
    np.testing.assert_allclose(cm, ref.chain_mean, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(c2, ref.chain_m2, rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(pm, ref.pool_mean, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(p2, ref.pool_m2, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(last, ref.last, rtol=1e-6)  # draws are stored in f32


def test_device_exchanges_permute_equal_temperature_ladders(gpu):
    # all temperatures equal: delta = 0, so every attempted exchange happens;
    # with negligible moves the draws show the exact permutations (even pairs
    # at the first exchange, odd pairs at the second)
    w = W.make("gaussian", n_obs=500)
    m = w.model
    C, n_iter = 8, 12
    init = np.arange(1, C + 1, dtype=np.float64).reshape(C, 1)
    with gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, 1, w.data,
                     1, w.n_obs) as s:
        s.set_exchange(4, 5)        # two ladders of 4 chains
        d, _, _ = s.run(init, np.full((C, 1), 1e-12), np.ones(C), n_iter, 3, 0,
                        rng=gpu.RNG_PHILOX)
        att, ok, n_ex = s.exchange_stats()
    d = d.reshape((n_iter, C), order="F")
    np.testing.assert_allclose(d[4], init[:, 0], atol=1e-6)
    even = [1, 0, 3, 2, 5, 4, 7, 6]                 # pairs (0,1),(2,3) in each ladder
    np.testing.assert_allclose(d[5], d[4][even], atol=1e-6)
    odd = [0, 2, 1, 3, 4, 6, 5, 7]                  # pair (1,2) in each ladder
    np.testing.assert_allclose(d[10], d[9][odd], atol=1e-6)
    np.testing.assert_allclose(d[11], d[10], atol=1e-6)
    assert n_ex == 2
    np.testing.assert_array_equal(att, [1, 1, 1, 0, 1, 1, 1, 0])
    np.testing.assert_array_equal(ok, att)


def test_pt_with_device_exchanges_covers_both_modes(gpu):
    rng = np.random.default_rng(1)
    y = rng.normal(3.0, 1.0, 400)
    m = gpum_model("~ log(exp(-((y - mu)^2) / 2) + exp(-((y + mu)^2) / 2))", "mu", "y")
    init = np.tile(np.linspace(-6, 6, 8), 4).reshape(32, 1)
    fit = gpu_metropolis(m, {"y": y}, init=init, proposal_sd=0.15, n_iter=4000, method="pt",
                         seed=2, swap_on_device=True, ladder_len=8, swap_every=10)
    assert fit.extra["swap_on_device"] and fit.extra["exchanges"] == 199  # t = 10 .. 1990
    cold = fit.draws[:, ::8, 0].ravel()               # rung 0 of each ladder
    assert np.any(cold > 1.5) and np.any(cold < -1.5)
    assert abs(cold[cold > 0].mean() - 3) < 0.4 and abs(cold[cold < 0].mean() + 3) < 0.4
    r = fit.extra["exchange_rate"]
    assert np.nanmax(r) > 0.2 and np.nanmin(r) >= 0.0
