"""Delayed acceptance on the B200: pair recording, the two-stage kernels
against the CPU restatement (oracle/da_oracle.py) with the very surrogate the
GPU uses, and the posterior of the API-level surrogate mode."""
import numpy as np
import pytest

from gpumetropolis_b200 import api
from gpumetropolis_b200 import workloads as W
from gpumetropolis_b200.diagnostics import rhat
from oracle import da_oracle
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _session(gpu, w):
    m = w.model
    return gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, m.n_params,
                       w.data, m.n_cols, w.n_obs)


def _trained(gpu, s, w, init, sd, n_iter=100, steps=600, hidden=128, batch=1024):
    """A surrogate trained on the pairs of one recorded exact run."""
    C = init.shape[0]
    s.record(n_iter * C)
    s.run(init, sd, np.ones(C), n_iter, 5, 0)
    theta, ll = s.recorded()
    s.record(0)
    net = gpu.Surrogate(w.model.n_params, hidden=hidden, batch=batch, seed=3)
    net.fit_normalizer(theta.astype(np.float64), ll)
    net.train(theta.astype(np.float64), ll, steps, lr=2e-3)
    return net


def test_recording_stores_every_exact_proposal(gpu):
    w = W.make("logistic", n_obs=3000)
    m = w.model
    C, n = 48, 12
    rng = np.random.default_rng(1)
    init = w.truth["beta"] + rng.normal(0, 0.05, (C, m.n_params))
    sd = np.full((C, m.n_params), 0.02)
    with _session(gpu, w) as s:
        s.record(10 * C * n)
        s.run(init, sd, np.ones(C), n, 7, 0)
        theta, ll = s.recorded()
        assert theta.shape == (n * C, m.n_params) and ll.shape == (n * C,)
        want = O.loglik_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols,
                              w.n_obs, theta.astype(np.float64))
        np.testing.assert_allclose(ll, want, rtol=1e-6)
        # a second run appends; the proposals of iteration 0 are slot 0..C-1
        s.run(init, sd, np.ones(C), n, 8, 0)
        theta2, ll2 = s.recorded()
        assert theta2.shape[0] == 2 * n * C
        np.testing.assert_array_equal(theta2[: n * C], theta)
        # capacity bounds the store
        s.record(C + 5)
        s.run(init, sd, np.ones(C), n, 9, 0)
        assert s.recorded()[0].shape[0] == C + 5
        s.record(0)
        assert s.recorded()[0].shape[0] == 0


@pytest.mark.parametrize("whiten", [True, False])
def test_surrogate_fit_on_device_matches_the_host_path(gpu, whiten):
    # The device path (split, moments, normaliser, training, held-out check)
    # against the same steps done from host copies of the pairs: every tenth
    # pair held out, the normaliser from numpy, train_stages on the rest.
    w = W.make("logistic", n_obs=3000, p=6)
    m = w.model
    d = m.n_params
    C, n = 64, 40
    rng = np.random.default_rng(4)
    init = w.truth["beta"] + rng.normal(0, 0.05, (C, d))
    sd = np.full((C, d), 0.02)
    stages = [(60, 2e-3), (30, 5e-4)]
    with _session(gpu, w) as s:
        s.record(n * C)
        s.run(init, sd, np.ones(C), n, 5, 0)
        theta, ll = s.recorded()
        net = gpu.Surrogate(d, hidden=128, batch=1024, seed=3)
        loss, info = s.train_surrogate(net, stages, holdout_every=10, whiten=whiten)
    idx = np.arange(theta.shape[0])
    tr, ho = idx % 10 != 0, idx % 10 == 0
    assert info["pairs"] == n * C
    assert info["train_pairs"] == tr.sum() and info["holdout_pairs"] == ho.sum()
    assert info["whitened"] == whiten
    assert loss.shape == (90,) and np.all(np.isfinite(loss))
    th64 = theta.astype(np.float64)
    ref = gpu.Surrogate(d, hidden=128, batch=1024, seed=3)
    ref.fit_normalizer(th64[tr], ll[tr], whiten=whiten)
    ref_loss = ref.train_stages(th64[tr], ll[tr], stages)
    pd, pr = net.predict(th64[ho]), ref.predict(th64[ho])
    # the normalisers agree to f64 rounding, so the two trainings follow each
    # other to within f32 noise
    scale = np.std(ll)
    assert np.max(np.abs(pd - pr)) <= 1e-3 * scale, np.max(np.abs(pd - pr)) / scale
    np.testing.assert_allclose(loss, ref_loss, rtol=1e-3, atol=1e-6)
    r = pd - ll[ho]
    assert info["holdout_resid_sd"] == pytest.approx(np.std(r), rel=1e-9)
    net.close()
    ref.close()


def test_surrogate_fit_on_device_refuses_bad_arguments(gpu):
    w = W.make("logistic", n_obs=500, p=3)
    m = w.model
    d = m.n_params
    with _session(gpu, w) as s:
        net = gpu.Surrogate(d + 1, hidden=128, batch=128, seed=1)
        with pytest.raises(gpu.GpumError, match="input width"):
            s.train_surrogate(net, [(5, 1e-3)])
        net.close()
        net = gpu.Surrogate(d, hidden=128, batch=128, seed=1)
        with pytest.raises(gpu.GpumError, match="fewer than two"):
            s.train_surrogate(net, [(5, 1e-3)])
        s.record(100)
        s.run(np.tile(w.truth["beta"], (4, 1)), np.full((4, d), 0.01), np.ones(4), 3, 1, 0)
        with pytest.raises(gpu.GpumError, match="holdout_every"):
            s.train_surrogate(net, [(5, 1e-3)], holdout_every=1)
        net.close()


@pytest.mark.parametrize("temps_kind", ["cold", "tempered"])
def test_two_stage_trajectories_match_oracle(gpu, temps_kind):
    w = W.make("logistic", n_obs=2048, p=4)
    m = w.model
    rng = np.random.default_rng(2)
    C, n_iter, seed = 12, 30, 21
    init = w.truth["beta"] + rng.normal(0, 0.05, (C, m.n_params))
    sd = np.full((C, m.n_params), 0.04)
    temps = np.ones(C) if temps_kind == "cold" else np.where(np.arange(C) % 3 == 0, 2.5, 1.0)
    with _session(gpu, w) as s:
        big = w.truth["beta"] + rng.normal(0, 0.05, (256, m.n_params))
        net = _trained(gpu, s, w, big, np.full((256, m.n_params), 0.04))
        try:
            d, acc, last, exact = s.run_da(net, init, sd, temps, n_iter, seed, 0)
            d = d.reshape((n_iter, C, m.n_params), order="F")
            od, oacc, oexact, tie_at = da_oracle.run_da(
                m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, m.n_params,
                w.data, m.n_cols, w.n_obs, init, sd, temps, n_iter, seed, net.predict)
        finally:
            net.close()
    clean = tie_at == n_iter
    assert clean.sum() >= C // 2
    for c in range(C):
        t = tie_at[c]
        np.testing.assert_allclose(d[:t, c], od[:t, c], rtol=2e-6, atol=1e-6)
    np.testing.assert_array_equal(exact[clean], oexact[clean])
    np.testing.assert_allclose(acc[clean], oacc[clean] / n_iter, atol=1e-6)
    # the surrogate screens: fewer exact evaluations than iterations
    assert exact.sum() < C * n_iter


def test_run_da_refuses_de_sync(gpu):
    w = W.make("gaussian", n_obs=500)
    C = 4
    with _session(gpu, w) as s:
        net = gpu.Surrogate(1, hidden=128, batch=128)
        try:
            with pytest.raises(gpu.GpumError, match="proposal mode"):
                s.run_da(net, np.zeros((C, 1)), np.full((C, 1), 0.1), np.ones(C), 10, 1, 4)
        finally:
            net.close()


@pytest.mark.parametrize("whiten", [False, True])
def test_surrogate_input_gradient_matches_cpu_oracle(gpu, whiten):
    # the drift of the Langevin proposal: d(surrogate)/d(theta) through the
    # network's backward pass and the input transform, against the numpy
    # restatement with the same BF16 roundings
    from oracle import mlp_oracle as MO
    rng = np.random.default_rng(7)
    d, H = 6, 256
    theta = rng.normal(0, 1, (4000, d)) @ rng.normal(0, 0.5, (d, d)) + 1.0
    ll = -0.5 * np.sum((theta - 1.0) ** 2, axis=1) * 50.0 - 1e3
    net = gpu.Surrogate(d, hidden=H, batch=1024, seed=2)
    try:
        net.fit_normalizer(theta, ll, whiten=whiten)
        net.train(theta, ll, 200, lr=2e-3)
        pts = theta[:300]
        val, grad = net.predict_grad(pts)
        # the fused inference kernel sums the head in another order
        np.testing.assert_allclose(val, net.predict(pts), rtol=1e-6)
        mu = theta.mean(axis=0)
        th = pts.astype(np.float32)
        if whiten:
            cov = np.cov(theta, rowvar=False)
            cov = cov + np.eye(d) * 1e-10 * float(np.mean(np.diag(cov)))
            T = np.linalg.inv(np.linalg.cholesky(cov)).astype(np.float32).astype(np.float64)
            X = MO.f32((th - mu.astype(np.float32)) @ T.T.astype(np.float32))
        else:
            inv = (1.0 / theta.std(axis=0)).astype(np.float32).astype(np.float64)
            T = np.diag(inv)
            X = MO.f32((th - mu.astype(np.float32)) * inv.astype(np.float32))
        _, dX = MO.input_grad(net.params(), d, H, X)
        ref = dX @ T * np.float32(np.std(ll))
        err = np.linalg.norm(grad - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert np.median(err) < 2e-3 and err.max() < 2e-2, (np.median(err), err.max())
    finally:
        net.close()


@pytest.mark.parametrize("with_L", [False, True])
def test_langevin_two_stage_trajectories_match_oracle(gpu, with_L):
    # delayed acceptance with the Langevin proposal driven by the surrogate
    # gradient: same draws, decisions and exact-evaluation counts as the
    # oracle (outside the tie band), with the very network the GPU uses
    w = W.make("logistic", n_obs=2048, p=4)
    m = w.model
    rng = np.random.default_rng(8)
    C, n_iter, seed = 12, 30, 41
    init = w.truth["beta"] + rng.normal(0, 0.05, (C, m.n_params))
    sd = np.full((C, m.n_params), 0.03)
    L = None
    if with_L:
        A = rng.normal(0, 1, (m.n_params, m.n_params))
        Lc = np.linalg.cholesky(A @ A.T / m.n_params + np.eye(m.n_params)) * 0.03
        L = np.broadcast_to(Lc, (C, m.n_params, m.n_params)).copy()
    temps = np.ones(C)
    with _session(gpu, w) as s:
        big = w.truth["beta"] + rng.normal(0, 0.05, (256, m.n_params))
        net = _trained(gpu, s, w, big, np.full((256, m.n_params), 0.04))
        try:
            d, acc, last, exact = s.run_da(net, init, sd, temps, n_iter, seed, 3, proposal_l=L)
            d = d.reshape((n_iter, C, m.n_params), order="F")
            od, oacc, oexact, tie_at = da_oracle.run_da(
                m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, m.n_params,
                w.data, m.n_cols, w.n_obs, init, sd, temps, n_iter, seed, net.predict_grad,
                proposal="mala", proposal_l=L)
        finally:
            net.close()
    clean = tie_at == n_iter
    assert clean.sum() >= C // 2
    for c in range(C):
        t = tie_at[c]
        np.testing.assert_allclose(d[:t, c], od[:t, c], rtol=1e-5, atol=1e-6)
    np.testing.assert_array_equal(exact[clean], oexact[clean])
    np.testing.assert_allclose(acc[clean], oacc[clean] / n_iter, atol=1e-6)
    assert 0 < exact.sum() < C * n_iter
    assert acc.mean() > 0.05


def test_surrogate_mode_mala_recovers_closed_form(gpu):
    w = W.make("gaussian", n_obs=20000)
    fit = api.gpu_metropolis(w.model, {"y": w.data[:, 0]}, init=np.full((128, 1), 3.0),
                             proposal_sd=0.02, n_iter=3000, warmup=1500, seed=4, method="mala",
                             surrogate={"hidden": 128, "batch": 2048, "steps": 800})
    info = fit.extra["surrogate"]
    assert info["used"], info
    assert 0.0 < info["exact_fraction"] < 1.0
    d = fit.draws[:, :, 0]
    n_eff = d.size / 20.0
    mcse = d.std() / np.sqrt(n_eff)
    assert abs(d.mean() - w.truth["post_mean"]) < 5 * mcse
    assert abs(d.std() - w.truth["post_sd"]) < 0.1 * w.truth["post_sd"]
    assert rhat(d, warmup=0) < 1.01


def test_surrogate_mode_recovers_closed_form(gpu):
    w = W.make("gaussian", n_obs=20000)
    fit = api.gpu_metropolis(w.model, {"y": w.data[:, 0]}, init=np.full((128, 1), 3.0),
                             proposal_sd=0.02, n_iter=3000, warmup=1500, seed=4,
                             surrogate={"hidden": 128, "batch": 2048, "steps": 800})
    info = fit.extra["surrogate"]
    assert info["used"], info
    assert 0.0 < info["exact_fraction"] < 0.9
    d = fit.draws[:, :, 0]
    n_eff = d.size / 20.0  # conservative: autocorrelation time <= 20 at this acceptance
    mcse = d.std() / np.sqrt(n_eff)
    assert abs(d.mean() - w.truth["post_mean"]) < 5 * mcse
    assert abs(d.std() - w.truth["post_sd"]) < 0.1 * w.truth["post_sd"]
    assert rhat(d, warmup=0) < 1.01


def test_surrogate_mode_pt(gpu):
    # y ~ N(|mu|, 1): two modes ~1500 nats apart, so chains start on both
    # sides and swaps carry states to the cold chain (as test-pt.R:198-217)
    rng = np.random.default_rng(5)
    y = rng.normal(3.0, 1.0, 400)
    from gpumetropolis_b200.dsl import gpum_model
    m = gpum_model("~ log(exp(-0.5 * (y - mu)^2) + exp(-0.5 * (y + mu)^2))", params="mu",
                   data="y")
    init = np.linspace(-6, 6, 8).reshape(8, 1)
    fit = api.gpu_metropolis(m, {"y": y}, init=init, proposal_sd=0.15,
                             n_iter=4000, warmup=2000, method="pt", seed=6,
                             surrogate={"hidden": 128, "batch": 1024, "steps": 600,
                                        "min_pairs": 512})
    assert fit.extra["surrogate"]["used"], fit.extra["surrogate"]
    cold = fit.draws[:, 0, 0]
    assert np.any(cold > 1.5) and np.any(cold < -1.5)
    assert abs(cold[cold > 0].mean() - 3) < 0.4 and abs(cold[cold < 0].mean() + 3) < 0.4


def test_two_stage_with_device_exchanges_matches_oracle(gpu):
    # three ladders of four tempered chains, an exchange after every third
    # iteration: same trajectories and exchange counts as the oracle, whose
    # exchange step also moves each state's cached surrogate value and prior
    w = W.make("logistic", n_obs=2048, p=4)
    m = w.model
    rng = np.random.default_rng(3)
    C, K, every, n_iter, seed = 12, 4, 3, 30, 33
    init = w.truth["beta"] + rng.normal(0, 0.05, (C, m.n_params))
    sd = np.full((C, m.n_params), 0.04)
    temps = np.tile([1.0, 1.3, 1.7, 2.2], C // K)
    with _session(gpu, w) as s:
        big = w.truth["beta"] + rng.normal(0, 0.05, (256, m.n_params))
        net = _trained(gpu, s, w, big, np.full((256, m.n_params), 0.04))
        try:
            s.set_exchange(K, every)
            d, acc, last, exact = s.run_da(net, init, sd, temps, n_iter, seed, 0)
            att, ok, n_ex = s.exchange_stats()
            s.set_exchange(0)
            d = d.reshape((n_iter, C, m.n_params), order="F")
            od, oacc, oexact, tie_at, (oatt, ook) = da_oracle.run_da(
                m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, m.n_params,
                w.data, m.n_cols, w.n_obs, init, sd, temps, n_iter, seed, net.predict,
                exchange=(K, every))
        finally:
            net.close()
    assert n_ex == (n_iter - 1) // every
    np.testing.assert_array_equal(att, np.tile([5, 4, 5, 0], C // K))  # 5 odd, 4 even exchanges
    np.testing.assert_array_equal(att, oatt)
    t_min = int(tie_at.min())  # exchanges spread a tie to other chains: compare before it
    assert t_min >= 9, t_min
    np.testing.assert_allclose(d[:t_min], od[:t_min], rtol=2e-6, atol=1e-6)
    if t_min == n_iter:
        np.testing.assert_array_equal(ok, ook)
        np.testing.assert_array_equal(exact, oexact)
    assert ook.sum() > 0


def test_surrogate_mode_pt_with_device_exchanges(gpu):
    # four ladders of eight rungs on the |mu| target, two-stage sampling with
    # the exchanges on the device
    rng = np.random.default_rng(5)
    y = rng.normal(3.0, 1.0, 400)
    from gpumetropolis_b200.dsl import gpum_model
    m = gpum_model("~ log(exp(-0.5 * (y - mu)^2) + exp(-0.5 * (y + mu)^2))", params="mu",
                   data="y")
    init = np.tile(np.linspace(-6, 6, 8), 4).reshape(32, 1)
    fit = api.gpu_metropolis(m, {"y": y}, init=init, proposal_sd=0.15, n_iter=4000,
                             warmup=2000, method="pt", seed=6, swap_on_device=True,
                             ladder_len=8, swap_every=10,
                             surrogate={"hidden": 128, "batch": 1024, "steps": 600,
                                        "min_pairs": 512})
    info = fit.extra["surrogate"]
    assert info["used"], info
    assert info["exact_fraction"] < 1.0
    assert fit.extra["exchanges"] == 199  # t = 10 .. 1990 of the sampling run
    cold = fit.draws[:, ::8, 0].ravel()
    assert np.any(cold > 1.5) and np.any(cold < -1.5)
    assert abs(cold[cold > 0].mean() - 3) < 0.4 and abs(cold[cold < 0].mean() + 3) < 0.4
    assert np.nanmax(fit.extra["exchange_rate"]) > 0.2


def test_trained_surrogate_gains_ess_per_exact_evaluation(gpu):
    # What the trained network gains over the method without it, counted
    # rather than timed: logistic regression (4096 observations, 5
    # parameters), 256 chains, adaptive exact warmup whose second half is
    # recorded, the surrogate trained on those pairs, then exact MH and
    # two-stage sampling of equal length from the same state.  The two-stage
    # run must reach at least twice the exact sampler's ESS per exact
    # log-likelihood evaluation, with the same posterior means within MCSE.
    from gpumetropolis_b200 import _native
    from gpumetropolis_b200 import adaptive as AD
    from gpumetropolis_b200.diagnostics import ess_pooled
    w = W.make("logistic", n_obs=4096, p=4)
    m = w.model
    npar, C, n_warm, n_samp, seed = m.n_params, 256, 800, 1500, 13
    cfg = dict(api.SURROGATE_DEFAULTS)
    cfg.update({"hidden": 128, "batch": 2048, "steps": 600, "min_pairs": 1024})
    call = api._Backend(m, w.data, w.n_obs, _native.RNG_PHILOX, cfg)
    try:
        call.record_at = n_warm // 2
        rng = np.random.default_rng(seed)
        init = w.truth["beta"] + rng.normal(0, 0.05, (C, npar))
        am = AD.am_orchestrate_warmup(call, npar, C, init, np.full((C, npar), 0.02), n_warm,
                                      seed)
        call.start_da()
        assert call.net is not None, call.info
        L = am.final_L
        mode = _native.MODE_CHOL if L is not None else _native.MODE_RWM
        d_ex, _, _ = call.session.run(am.final_init, am.final_proposal_sd, np.ones(C), n_samp,
                                      seed + 1, mode, 0.0, 0.0, L, rng=_native.RNG_PHILOX)
        d_ex = d_ex.reshape((n_samp, C, npar), order="F").astype(np.float64)
        e0 = call.exact_evals
        d_da, _, _ = call(am.final_init, am.final_proposal_sd, n_samp, seed + 2, None, mode,
                          0.0, 0.0, L)
        n_exact_da = call.exact_evals - e0
    finally:
        call.close()
    d_da = np.asarray(d_da, dtype=np.float64)
    e_ex = np.array([ess_pooled(d_ex[:, :, j]) for j in range(npar)])
    e_da = np.array([ess_pooled(d_da[:, :, j]) for j in range(npar)])
    per_eval_ex = e_ex / (n_samp * C)
    per_eval_da = e_da / max(n_exact_da, 1)
    assert np.all(per_eval_da >= 2.0 * per_eval_ex), per_eval_da / per_eval_ex
    mc = np.sqrt(d_ex.reshape(-1, npar).var(axis=0) / e_ex +
                 d_da.reshape(-1, npar).var(axis=0) / e_da)
    z = np.abs(d_ex.mean(axis=(0, 1)) - d_da.mean(axis=(0, 1))) / mc
    assert z.max() < 4.0, z
