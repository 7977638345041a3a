"""The CPU oracle pinned against the reference tests' known answers.

The oracle restates src/rust/src/cpu_native.rs; these tests are the pin
(tests/testthat/test-catalog.R, test-mala.R, test-kernel.R, test-api.R,
test-numerical.R, test-de.R of the reference).
"""
import numpy as np
import pytest

from gpumetropolis_b200.dsl import gpum_model
from gpumetropolis_b200 import workloads as W
from oracle import cjit
from oracle import oracle as O


def _ll(m, y, pts):
    y = np.asarray(y, float)
    return O.loglik_batch(m.loglik.code, m.loglik.consts, m.n_params, y, m.n_cols,
                          len(y) // max(m.n_cols, 1), pts)


def test_gamma_loglik_and_gradient(golden):
    c = golden["gamma"]
    m = gpum_model(c["formula"], c["params"], c["data"])
    y = np.array(c["y"])
    v = _ll(m, y, c["point"])[0]
    assert abs(v - c["loglik"]) <= c["loglik_tol"] * max(1.0, abs(c["loglik"]))
    g = O.grad_batch(m.loglik.code, m.loglik.consts, 2, y, 1, len(y), c["point"])
    np.testing.assert_allclose(g, c["grad"], rtol=c["grad_tol"], atol=c["grad_tol"])


def test_gradient_matches_analytic_and_fd(golden):
    for c in golden["grad_fd"]:
        m = gpum_model(c["formula"], c["params"], c["data"])
        y = np.array(c["y"])
        pt = np.array(c["point"])
        g = O.grad_batch(m.loglik.code, m.loglik.consts, 2, y, 1, len(y), pt)
        np.testing.assert_allclose(g, c["grad"], rtol=c["grad_tol"], atol=c["grad_tol"])
        h = 1e-6
        fd = []
        for j in range(2):
            e = np.zeros(2)
            e[j] = h
            fd.append((_ll(m, y, pt + e)[0] - _ll(m, y, pt - e)[0]) / (2 * h))
        np.testing.assert_allclose(g, fd, rtol=1e-6, atol=1e-6)


def test_phase0_closed_forms(golden):
    for c in golden["phase0"]:
        m = gpum_model(c["formula"], "mu", "y")
        np.testing.assert_allclose(_ll(m, c["y"], c["points"]), c["expect"], atol=1e-12)


def test_lgamma_digamma_against_scipy():
    import scipy.special as sp
    for x in [0.1, 0.5, 1.0, 2.5, 7.3, 40.0, 1e3]:
        assert abs(O.lgamma(x) - sp.gammaln(x)) <= 1e-13 * max(1.0, abs(sp.gammaln(x)))
        # the reference's series (shift past 6, terms to x^-6) is good to ~3e-9
        assert abs(O.digamma(x) - sp.digamma(x)) <= 1e-8 * max(1.0, abs(sp.digamma(x)))


def test_empty_program_and_unknown_opcode():
    y = np.array([1.0, 2.0])
    assert O.loglik_batch(np.zeros(0, np.uint32), [], 1, y, 1, 2, [0.3])[0] == 0.0
    # opcode 42 acts as POW (cpu_native.rs:103): 2^3 per observation
    code = np.array([0, 0, 0, 1, 42, 0], np.uint32)
    assert O.loglik_batch(code, [2.0, 3.0], 1, y, 1, 2, [0.0])[0] == 16.0


def test_jit_matches_interpreter_bitwise():
    w = W.make("logistic", n_obs=512)
    m = w.model
    pts = np.random.default_rng(0).normal(0, 0.3, (4, m.n_params))
    ref = O.loglik_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols,
                         w.n_obs, pts)
    fn = cjit.compile_loglik(m.loglik.code, m.loglik.consts)
    init = pts.copy()
    sd = np.full_like(init, 1e-3)
    d1, a1, l1 = O.run(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                       m.n_params, w.data, m.n_cols, w.n_obs, init, sd, np.ones(4), 20, 3, 0)
    d2, a2, l2 = O.run(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                       m.n_params, w.data, m.n_cols, w.n_obs, init, sd, np.ones(4), 20, 3, 0,
                       jit=fn)
    assert np.array_equal(d1, d2) and np.array_equal(l1, l2) and np.array_equal(a1, a2)
    assert np.all(np.isfinite(ref))


@pytest.mark.parametrize("name", ["logistic", "poisson", "mixture", "student_t"])
def test_full_size_checkers_agree_with_the_oracle(name):
    # The checkers used at the configurations' full sizes: the compiled
    # evaluator per point equals loglik_batch bitwise, its absolute-value
    # variant bounds |loglik|, and the blocked parallel gradient equals
    # grad_batch up to the f64 reordering of the sum.
    w = W.make(name, n_obs=3001)
    m = w.model
    pts = np.random.default_rng(1).normal(0, 0.2, (5, m.n_params))
    if name == "student_t":
        pts[:, -1] += np.log(1.5)
    ref = O.loglik_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols,
                         w.n_obs, pts)
    fn = cjit.compile_loglik(m.loglik.code, m.loglik.consts)
    got = O.jit_batch(fn, m.n_params, w.data, m.n_cols, w.n_obs, pts)
    assert np.array_equal(got, ref)
    fa = cjit.compile_loglik(m.loglik.code, m.loglik.consts, absolute=True)
    ab = O.jit_batch(fa, m.n_params, w.data, m.n_cols, w.n_obs, pts)
    assert np.all(ab >= np.abs(ref))
    gref = O.grad_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols, w.n_obs,
                        pts).reshape(5, -1)
    g, ga = O.grad_abs_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols,
                             w.n_obs, pts, block=257)
    np.testing.assert_allclose(g, gref, rtol=1e-12, atol=1e-12 * np.abs(ga).max())
    assert np.all(ga >= np.abs(g))


def _draws(d, n_iter, C, np_):
    return d.reshape((n_iter, C, np_), order="F")


def test_gaussian_posterior_recovery_cpu():
    # test-api.R:80-95: mean within 0.03 of mean(y), split R-hat < 1.05
    from gpumetropolis_b200.diagnostics import rhat
    w = W.make("gaussian", n_obs=5000)
    m = w.model
    init = np.linspace(-3, 8, 4)
    d, acc, last = O.run(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, 1,
                         w.data, 1, w.n_obs, init, np.full(4, 0.06), np.ones(4), 3000, 1, 0)
    dr = _draws(d, 3000, 4, 1)[1500:, :, 0]
    assert abs(dr.mean() - w.data.mean()) < 0.03
    assert rhat(dr, warmup=0) < 1.05


def test_reproducible_and_seed_sensitive():
    w = W.make("gaussian", n_obs=300)
    m = w.model
    args = (m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, 1, w.data, 1,
            w.n_obs, np.zeros(2), np.full(2, 0.1), np.ones(2), 200)
    a = O.run(*args, 7, 0)[0]
    b = O.run(*args, 7, 0)[0]
    c = O.run(*args, 8, 0)[0]
    assert np.array_equal(a, b) and not np.array_equal(a, c)


def test_nonfinite_proposals_rejected():
    # test-numerical.R:32-45: log(mu) with mu <= 0 proposals are rejected
    m = gpum_model("~ log(mu) - mu + 0 * y", "mu", "y")
    d, acc, last = O.run(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, 1,
                         np.zeros(1), 1, 1, [1.5], [0.4], [1.0], 3000, 1, 0)
    assert np.all(np.isfinite(d)) and d.min() > 0
    assert abs(d.mean() - 2.0) < 0.4
    # a -inf start accepts the first finite proposal (test-numerical.R:58-67)
    d, acc, last = O.run(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, 1,
                         np.zeros(1), 1, 1, [-1.0], [0.3], [1.0], 500, 1, 0)
    assert np.isfinite(last[0]) or acc[0] == 0


def test_de_and_de_sync_recover_correlated_target():
    # test-de.R:43-72 / :96-121, with a reduced iteration budget
    rng = np.random.default_rng(1)
    rho = 0.9
    Lc = np.linalg.cholesky(np.array([[1, rho], [rho, 1]]))
    y = rng.standard_normal((500, 2)) @ Lc.T + np.array([2.0, -1.0])
    Si = np.linalg.inv(np.array([[1, rho], [rho, 1]]))
    f = (f"~ -0.5 * ({Si[0, 0]:.6f}*(y1-mu1)^2 + 2*{Si[0, 1]:.6f}*(y1-mu1)*(y2-mu2)"
         f" + {Si[1, 1]:.6f}*(y2-mu2)^2)")
    m = gpum_model(f, ["mu1", "mu2"], ["y1", "y2"])
    C = 16
    init = rng.normal(0, 1, (C, 2)) + y.mean(0)
    sd = np.full((C, 2), 0.05)
    d, acc, _ = O.run_de_sync(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                              2, y, 2, 500, init, sd, 3000, 1, 2.38 / 2, 1e-3)
    dr = d.reshape((3000, C, 2), order="F")[1000:]
    assert abs(dr[..., 0].mean() - y[:, 0].mean()) < 0.02
    assert abs(np.corrcoef(dr[..., 0].ravel(), dr[..., 1].ravel())[0, 1] - rho) < 0.05


def test_philox_known_answers():
    # Philox4x32-10 known-answer vectors of the Random123 distribution
    # (counter, key -> output); the exchange uniforms of the delayed-
    # acceptance oracle come from this function.
    from oracle.da_oracle import philox4x32_10, u53
    cases = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
             ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF),
              (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
             ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
              (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for c, k, want in cases:
        assert philox4x32_10(c, *k) == want
    assert 0.0 < u53(0, 0) < 1e-15 and u53(0xFFFFFFFF, 0xFFFFFFFF) == 1.0


def test_da_oracle_exchanges_permute_equal_temperature_ladders():
    # with equal temperatures every attempted exchange is accepted: the
    # oracle's draws show the pairs (0,1),(2,3) swapped after the first
    # exchange and (1,2) after the second, in each ladder of four chains
    from oracle import da_oracle
    w = W.make("gaussian", n_obs=200)
    m = w.model
    C, K, every, n_iter = 8, 4, 3, 8
    init = np.arange(1, C + 1, dtype=np.float64).reshape(C, 1)

    def exact(th):
        return O.loglik_batch(m.loglik.code, m.loglik.consts, 1, w.data, 1, w.n_obs,
                              np.asarray(th, dtype=np.float64).reshape(-1, 1))

    d, _, _, _, (att, ok) = da_oracle.run_da(
        m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, 1, w.data, 1, w.n_obs,
        init, np.full((C, 1), 1e-12), np.ones(C), n_iter, 5, exact, exchange=(K, every))
    np.testing.assert_allclose(d[2, :, 0], init[:, 0], atol=1e-9)
    np.testing.assert_allclose(d[3, :, 0], d[2, [1, 0, 3, 2, 5, 4, 7, 6], 0], atol=1e-9)
    np.testing.assert_allclose(d[6, :, 0], d[5, [0, 2, 1, 3, 4, 6, 5, 7], 0], atol=1e-9)
    np.testing.assert_array_equal(att, [1, 1, 1, 0, 1, 1, 1, 0])
    np.testing.assert_array_equal(ok, att)
