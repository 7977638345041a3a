"""Host-side logic without a GPU: the adaptive-warmup primitives
(tests/testthat/test-adaptive.R of the reference), the PT ladder and swap
draws (test-pt.R), diagnostics, and gpu_metropolis input validation."""
import numpy as np
import pytest

from gpumetropolis_b200 import adaptive as AD
from gpumetropolis_b200.api import GpumInputError, gpu_metropolis
from gpumetropolis_b200.diagnostics import ess, gaussian_mean_posterior, rhat
from gpumetropolis_b200.dsl import gpum_model


def test_welford_matches_cov():
    rng = np.random.default_rng(1)
    x = rng.standard_normal(500)
    st = AD.Welford.init(1, 1, 1.0)
    for v in x:  # row by row, as the reference's R loop does
        st.update(np.array([[[v]]]))
    assert np.allclose(st.mean[0, 0], x.mean()) and np.allclose(st.covariance()[0, 0, 0],
                                                                x.var(ddof=1))
    X = rng.standard_normal((300, 3))
    st = AD.Welford.init(1, 3, 1.0)
    st.update(X[:100, None, :]).update(X[100:, None, :])
    np.testing.assert_allclose(st.mean[0], X.mean(0), rtol=1e-12)
    np.testing.assert_allclose(st.covariance()[0], np.cov(X.T), rtol=1e-10)
    perm = rng.permutation(300)
    s2 = AD.Welford.init(1, 3, 1.0).update(X[perm][:, None, :])
    np.testing.assert_allclose(s2.covariance()[0], st.covariance()[0], rtol=1e-12)


def test_covariance_seed_before_two_samples():
    st = AD.Welford.init(1, 2, 0.5)
    np.testing.assert_array_equal(st.covariance()[0], np.diag([0.5, 0.5]))
    st.update(np.array([[[1.0, 2.0]]]))
    np.testing.assert_array_equal(st.covariance()[0], np.diag([0.5, 0.5]))


def test_robbins_monro_direction_and_decay():
    for d in (1, 2, 5):
        t = AD.target_accept(d)
        assert AD.robbins_monro_scale(1.0, t + 0.1, 1, d) > 1.0
        assert AD.robbins_monro_scale(1.0, t - 0.1, 1, d) < 1.0
    early = AD.robbins_monro_scale(1.0, 0.5, 1, 2) - 1.0
    late = AD.robbins_monro_scale(1.0, 0.5, 100, 2) - 1.0
    assert early > late > 0
    assert AD.target_accept(1) == 0.44 and AD.target_accept(9) == 0.234


def test_cholesky_reconstructs_and_regularises():
    rng = np.random.default_rng(4)
    A = rng.standard_normal((3, 3))
    S = A.T @ A + 0.1 * np.eye(3)
    L = AD.cholesky_reg(S, eps=1e-12)
    np.testing.assert_allclose(L @ L.T, S, rtol=1e-6)
    assert np.all(np.triu(L, 1) == 0)
    L2 = AD.cholesky_reg(np.ones((2, 2)), eps=1e-3)
    assert np.all(np.isfinite(L2)) and np.all(np.linalg.eigvalsh(L2 @ L2.T) > 0)


def test_pt_ladder_and_swap_draws():
    T = AD.pt_default_ladder(8, 10.0)
    assert T[0] == 1 and abs(T[-1] - 10) < 1e-12 and np.all(np.diff(T) > 0)
    r = T[1:] / T[:-1]
    assert np.max(np.abs(r - r[0])) < 1e-9
    u1 = AD.pt_swap_draws(1, 1, 5)
    assert np.array_equal(u1, AD.pt_swap_draws(1, 1, 5))
    assert not np.array_equal(u1, AD.pt_swap_draws(1, 2, 5))


def test_warmup_batches_with_a_fake_backend():
    """The orchestrator's batch plan and bookkeeping (R/adaptive.R:101-254)
    with a stand-in that returns random-walk draws: no GPU."""
    calls = []

    def call(init, sd, n_iter, seed, temps, mode, gamma, noise, L):
        calls.append((n_iter, seed, mode, L is not None))
        rng = np.random.default_rng(seed)
        d = init[None] + np.cumsum(rng.normal(0, 0.1, (n_iter,) + init.shape), axis=0)
        return d, np.full(init.shape[0], 0.3), np.zeros(init.shape[0])

    r = AD.am_orchestrate_warmup(call, 2, 4, np.zeros((4, 2)), np.full((4, 2), 0.1), 500, 7)
    assert sum(c[0] for c in calls) == 500 and r.warmup_used == 500
    assert r.n_batches == 10 and [c[1] for c in calls] == list(range(7, 17))
    assert calls[0][2] == 0 and calls[-1][2] == 2 and calls[-1][3]  # Cholesky after batch 1
    assert r.final_L.shape == (4, 2, 2) and r.seed_next == 17
    assert r.accept_history.shape == (4, 10)


def test_diagnostics():
    rng = np.random.default_rng(3)
    iid = rng.standard_normal((2000, 4))
    assert 0.8 * 4000 < ess(iid) <= 4000
    assert abs(rhat(iid) - 1.0) < 0.01
    ar = np.zeros((2000, 4))
    for t in range(1, 2000):
        ar[t] = 0.95 * ar[t - 1] + rng.standard_normal(4)
    assert ess(ar) < 0.2 * 4000
    p = gaussian_mean_posterior([1.0, 2.0, 3.0], 2.0)
    assert p["mean"] == 2.0 and abs(p["sd"] - 2 / np.sqrt(3)) < 1e-15


def test_gpu_metropolis_input_validation():
    m = gpum_model("~ -((y - mu)^2) / 8", "mu", "y")
    y = {"y": np.zeros(10)}
    with pytest.raises(GpumInputError):
        gpu_metropolis(m, {"z": [1, 2]})
    with pytest.raises(GpumInputError):
        gpu_metropolis(m, y, proposal_sd=-1)
    with pytest.raises(GpumInputError, match="n_chains"):
        gpu_metropolis(m, y, proposal_sd=np.full((3, 1), 0.1), n_chains=4)
    with pytest.raises(GpumInputError, match="positive and finite"):
        gpu_metropolis(m, y, proposal_sd=np.array([[0.1], [0.0], [0.2], [0.1]]), n_chains=4)
    with pytest.raises(GpumInputError, match="at least 4 chains"):
        gpu_metropolis(m, y, n_chains=3, method="de")
    with pytest.raises(GpumInputError, match="one value per chain"):
        gpu_metropolis(m, y, n_chains=4, method="pt", temperatures=[1, 2])
    with pytest.raises(GpumInputError, match="positive and finite"):
        gpu_metropolis(m, y, n_chains=4, method="pt", temperatures=[1, 2, -1, 3])
    with pytest.raises(GpumInputError, match="not available"):
        gpu_metropolis(m, y, backend="cuda")
    with pytest.raises(GpumInputError, match="warmup"):
        gpu_metropolis(m, y, n_iter=10, warmup=10)
    with pytest.raises(GpumInputError, match="ladder_len"):
        gpu_metropolis(m, y, n_chains=8, method="pt", swap_on_device=True, ladder_len=3)
    with pytest.raises(GpumInputError, match="ladder_len"):
        gpu_metropolis(m, y, n_chains=8, method="pt", swap_on_device=True, ladder_len=1)


def test_pooled_ess_on_ar1_and_stuck_chains():
    from gpumetropolis_b200.diagnostics import ess_pooled
    rng = np.random.default_rng(0)
    n, m = 3000, 32
    for phi in (0.0, 0.5, 0.9):
        x = np.zeros((n, m))
        e = rng.standard_normal((n, m))
        for t in range(1, n):
            x[t] = phi * x[t - 1] + e[t]
        want = (1 - phi) / (1 + phi)
        assert abs(ess_pooled(x) / (n * m) - want) < 0.12 * want + 0.01
    # chains that never move carry one value each, not n
    stuck = np.repeat(rng.standard_normal((1, m)), 400, axis=0)
    assert ess_pooled(stuck) < 2 * m


def test_evidence_needs_a_proper_prior():
    # test-bayes.R:77-82
    from gpumetropolis_b200.api import gpum_evidence
    flat = gpum_model("~ -((y - mu)^2) / 8", "mu", "y")
    with pytest.raises(GpumInputError, match="proper prior"):
        gpum_evidence(flat, {"y": np.zeros(10)})


def test_batch_moments_merge_like_the_row_updates():
    rng = np.random.default_rng(3)
    x = rng.normal(size=(40, 6, 3)) * np.array([1.0, 3.0, 0.2])
    wd = AD.WelfordDiag.init(6, 3, np.ones(3))
    wf = AD.Welford.init(1, 3, np.ones(3))
    for b in range(4):
        mo = AD.moments_of(x[10 * b:10 * (b + 1)])
        wd.merge(mo.n, mo.chain_mean, mo.chain_m2)
        wf.merge(mo.n * 6, mo.pool_mean[None], mo.pool_m2[None])
        assert np.array_equal(mo.last, x[10 * b + 9])
    np.testing.assert_allclose(wd.variances(), x.var(axis=0, ddof=1), rtol=1e-12)
    np.testing.assert_allclose(wf.covariance()[0], np.cov(x.reshape(-1, 3), rowvar=False),
                               rtol=1e-12)
    full = AD.Welford.init(6, 3, np.ones(3)).update(x)
    np.testing.assert_allclose(np.diagonal(full.covariance(), axis1=1, axis2=2),
                               wd.variances(), rtol=1e-12)
