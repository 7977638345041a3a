"""B200 log-density evaluation against the f64 oracle (through the C ABI).

Tolerances: the summed log-likelihood within 1e-6 relative of the f64
oracle (the per-observation bytecode runs in FP32; the sums are compensated
FP32 per thread and FP64 across threads); per-observation values within
2e-5 absolute + 2e-5 relative (one FP32 evaluation each).
"""
import numpy as np
import pytest

from gpumetropolis_b200 import workloads as W
from gpumetropolis_b200.dsl import gpum_model
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL_SUM = 1e-6


def _points(w, n, seed=0, scale=0.05):
    rng = np.random.default_rng(seed)
    m = w.model
    base = np.zeros(m.n_params)
    if w.name == "logistic" or w.name == "poisson":
        base[:] = w.truth["beta"]
    elif w.name == "student_t":
        base[:-1] = w.truth["beta"]
        base[-1] = np.log(1.5)
    elif w.name == "mixture":
        base[:] = [np.log(0.3 / 0.7), -2.0, 3.0, 0.0, np.log(1.5)]
    elif w.name == "gaussian":
        base[:] = 3.4
    return base + rng.normal(0, scale, (n, m.n_params))


@pytest.mark.parametrize("engine", [0, 1], ids=["interp", "compiled"])
@pytest.mark.parametrize("name,n_obs", [("gaussian", 5003), ("logistic", 4099),
                                         ("poisson", 3001), ("mixture", 6007),
                                         ("student_t", 1031)])
def test_loglik_batch_matches_oracle(gpu, name, n_obs, engine):
    w = W.make(name, n_obs=n_obs)
    m = w.model
    pts = _points(w, 37)
    ref = O.loglik_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols,
                         w.n_obs, pts)
    with gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                     m.n_params, w.data, m.n_cols, w.n_obs, engine=engine) as s:
        assert s.engine == engine
        got = s.loglik_batch(pts)
    rel = np.abs(got - ref) / np.abs(ref)
    assert rel.max() <= REL_SUM, (name, rel.max())


@pytest.mark.parametrize("engine", [0, 1], ids=["interp", "compiled"])
@pytest.mark.parametrize("name,n_obs", [("logistic", 777), ("mixture", 513),
                                         ("student_t", 300)])
def test_pointwise_matches_oracle(gpu, name, n_obs, engine):
    w = W.make(name, n_obs=n_obs)
    m = w.model
    pts = _points(w, 5, seed=1)
    ref = O.loglik_pointwise(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols,
                             w.n_obs, pts)
    with gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                     m.n_params, w.data, m.n_cols, w.n_obs, engine=engine) as s:
        got = s.loglik_pointwise(pts)
    np.testing.assert_allclose(got, ref, rtol=2e-5, atol=2e-5)


def test_many_points_and_chain_blocks(gpu):
    # 1000 points spread over several chain blocks, ragged in every dimension
    w = W.make("logistic", n_obs=2053)
    m = w.model
    pts = _points(w, 1000, seed=2)
    ref = O.loglik_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols,
                         w.n_obs, pts)
    got = gpu.loglik_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data, m.n_cols,
                           w.n_obs, pts)
    assert (np.abs(got - ref) / np.abs(ref)).max() <= REL_SUM


@pytest.mark.parametrize("depth", [3, 12, 24])
def test_interpreter_variants_by_depth(gpu, depth):
    """Through the one-shot ABI call (default engine) and the interpreter."""
    # right-nested sums push `depth` values: exercises the 8x8, 4x16, 2x32 variants
    f = "~ " + "(y * a + " * (depth - 1) + "b" + ")" * (depth - 1)
    m = gpum_model(f, ["a", "b"], "y")
    assert m.loglik.depth >= depth
    y = np.random.default_rng(3).normal(size=999)
    pts = np.array([[0.5, 1.5], [-0.25, 2.0], [1.0, -1.0]])
    ref = O.loglik_batch(m.loglik.code, m.loglik.consts, 2, y, 1, y.size, pts)
    got = gpu.loglik_batch(m.loglik.code, m.loglik.consts, 2, y, 1, y.size, pts)
    with gpu.Session(m.loglik.code, m.loglik.consts, [], [], 2, y, 1, y.size, engine=0) as s:
        got_i = s.loglik_batch(pts)
    # these sums cancel (terms of both signs): bound the error by the sum of
    # |per-observation values|, the condition of an FP32-per-observation sum
    pw = O.loglik_pointwise(m.loglik.code, m.loglik.consts, 2, y, 1, y.size, pts)
    scale = np.abs(pw.reshape(3, -1)).sum(axis=1)
    assert np.all(np.abs(got - ref) <= 1e-6 * scale)
    assert np.all(np.abs(got_i - ref) <= 1e-6 * scale)


# Programs that compute a subtree again (the interpreter evaluates it once and
# reuses the value): one repeated linear predictor at a shallow stack, two
# different repeated subtrees, three copies of one, a repeated subtree inside a
# repeated subtree, and a repeat at a stack deeper than the reuse limit.
_LP = "(a + b * x + c * z)"
_LQ = "(d * x + e * z + a)"
_REPEATS = [
    f"~ y * {_LP} - log(1 + exp({_LP}))",
    f"~ y * {_LP} - exp({_LQ}) + {_LQ} / (1 + {_LP}^2)",
    f"~ {_LP} * {_LP} - {_LP} / (2 + exp(-{_LP}))",
    f"~ exp(-({_LP} + {_LQ})^2 / 8) + log(1 + ({_LP} + {_LQ})^2) - {_LP}",
    "~ " + "(y * a + " * 9 + f"log(1 + exp({_LP})) - {_LP}" + ")" * 9,
]


@pytest.mark.parametrize("k", range(len(_REPEATS)))
def test_interpreter_reuses_repeated_subtrees(gpu, k):
    m = gpum_model(_REPEATS[k], ["a", "b", "c", "d", "e"], ["y", "x", "z"])
    rng = np.random.default_rng(10 + k)
    n = 1537
    data = np.column_stack([rng.uniform(0, 1, n) < 0.5, rng.normal(size=n),
                            rng.normal(size=n)]).astype(np.float64)
    pts = rng.normal(0, 0.3, (19, 5))
    ref = O.loglik_pointwise(m.loglik.code, m.loglik.consts, 5, data, 3, n, pts)
    with gpu.Session(m.loglik.code, m.loglik.consts, [], [], 5, data, 3, n, engine=0) as s:
        got = s.loglik_pointwise(pts)
        tot = s.loglik_batch(pts)
    np.testing.assert_allclose(got, ref, rtol=2e-5, atol=2e-5)
    pw = ref.reshape(pts.shape[0], -1)
    assert np.all(np.abs(tot - pw.sum(axis=1)) <= 1e-6 * np.abs(pw).sum(axis=1))


def test_every_opcode_and_edge_sizes(gpu, golden):
    c = golden["gamma"]
    m = gpum_model(c["formula"], c["params"], c["data"])
    y = np.array(c["y"])
    got = gpu.loglik_batch(m.loglik.code, m.loglik.consts, 2, y, 1, y.size, c["point"])
    assert abs(got[0] - c["loglik"]) <= 1e-6 * abs(c["loglik"])
    # sqrt, pow with a non-constant exponent, division by a parameter, neg
    m2 = gpum_model("~ -sqrt((y - a)^2 + 1) - log(1 + (y - a)^2 / b^2) + y^b / (1 + a^2)",
                    ["a", "b"], "y")
    yy = np.abs(np.random.default_rng(4).normal(2, 1, 257))
    pts = np.array([[3.5, 1.3], [0.2, 0.7]])
    ref = O.loglik_batch(m2.loglik.code, m2.loglik.consts, 2, yy, 1, yy.size, pts)
    got = gpu.loglik_batch(m2.loglik.code, m2.loglik.consts, 2, yy, 1, yy.size, pts)
    np.testing.assert_allclose(got, ref, rtol=1e-6)
    # a single observation; no observations; an empty program; unknown opcode = POW
    one = gpu.loglik_batch(m2.loglik.code, m2.loglik.consts, 2, yy[:1], 1, 1, pts)
    np.testing.assert_allclose(one, O.loglik_batch(m2.loglik.code, m2.loglik.consts, 2, yy[:1],
                                                   1, 1, pts), rtol=1e-6)
    zero = gpu.loglik_batch(m2.loglik.code, m2.loglik.consts, 2, np.zeros(0), 1, 0, pts)
    assert np.all(zero == 0.0)
    empty = gpu.loglik_batch(np.zeros(0, np.uint32), [], 2, yy, 1, yy.size, pts)
    assert np.all(empty == 0.0)
    code = np.array([0, 0, 0, 1, 42, 0], np.uint32)
    assert gpu.loglik_batch(code, [2.0, 3.0], 1, yy[:2], 1, 2, [0.0])[0] == 16.0


def test_nonfinite_terms_propagate_like_the_reference(gpu):
    m = gpum_model("~ log(mu - y)", "mu", "y")
    y = np.array([0.0, 1.0, 2.0, 3.0])
    got = gpu.loglik_batch(m.loglik.code, m.loglik.consts, 1, y, 1, 4, [[2.0], [5.0], [3.0]])
    ref = O.loglik_batch(m.loglik.code, m.loglik.consts, 1, y, 1, 4, [[2.0], [5.0], [3.0]])
    assert np.isnan(got[0]) == np.isnan(ref[0])      # log of a negative: NaN
    assert got[2] == -np.inf and ref[2] == -np.inf   # log(0): -inf
    assert abs(got[1] - ref[1]) <= 1e-6 * abs(ref[1])


def test_session_reuse_and_determinism(gpu):
    w = W.make("mixture", n_obs=20011)
    m = w.model
    pts = _points(w, 70, seed=5)
    with gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                     m.n_params, w.data, m.n_cols, w.n_obs) as s:
        a = s.loglik_batch(pts)
        b = s.loglik_batch(pts)
        c = s.loglik_batch(pts[:3])
    assert np.array_equal(a, b)        # fixed-order reductions: bitwise repeatable
    # another launch geometry partitions the observations differently, so
    # the FP32 blocks (about 1,250 here, each rounding ~1e-6 of a ~20-unit
    # partial) differ: ~4e-5 absolute on a ~2.7e4 total, ~1.5e-9 relative
    np.testing.assert_allclose(a[:3], c, rtol=5e-9)
