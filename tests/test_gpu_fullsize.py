"""Log-density and gradient parity at the configurations' full sizes.

The per-observation bytecode runs in FP32 on the GPU; the summed
log-likelihood must stay within 1e-6 relative of the f64 oracle (the
restatement of cpu_native.rs:339-360, loglik_batch) at the sizes the sampler
is benchmarked on, where the sums run over 2^20 .. 2^24 observations:

* logistic regression, N = 2^20, 17 parameters;
* Poisson regression, N = 2^21, 24 parameters (value and gradient);
* two-component Gaussian mixture, N = 2^22, 5 parameters;
* Student-t regression, N = 2^24, 65 parameters (value and gradient).

Bound for the value: |b200 - oracle| <= 1e-6 * sum_i |l_i(theta)|, the sum of
the per-observation terms' absolute values (the scale of an FP32 sum's
rounding error).  Every term of these four models is a log density below 0,
so the sum does not cancel and the bound is 1e-6 relative of the total; the
test asserts that too.

Bound for the gradient (cpu_native.rs:306-329, grad_batch): near the
posterior every component is a sum that cancels almost completely (it is 0
at the mode), so each component is held to 1e-5 * sum_i |dl_i/dtheta_j|: FP32
per-observation adjoints (a few roundings each) added in FP32 blocks and
FP64 across blocks.

The oracle runs the compiled f64 evaluator (bitwise the interpreter's value)
and the blocked parallel tape gradient on the host's cores.
"""
import math
import os

import numpy as np
import pytest

from gpumetropolis_b200 import workloads as W
from oracle import cjit
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL_SUM = 1e-6
REL_GRAD = 1e-5
N_POINTS = 16


def _centre(w):
    m = w.model
    base = np.zeros(m.n_params)
    if w.name in ("logistic", "poisson"):
        base[:] = w.truth["beta"]
    elif w.name == "student_t":
        base[:-1] = w.truth["beta"]
        base[-1] = math.log(1.5)
    else:
        base[:] = [math.log(0.3 / 0.7), -2.0, 3.0, 0.0, math.log(1.5)]
    return base


def _points(w, n, seed):
    # points a few posterior standard deviations (~1/sqrt(N)) around the
    # generating values, where the sampler spends its time
    scale = 4.0 / math.sqrt(w.n_obs)
    return _centre(w) + np.random.default_rng(seed).normal(0.0, scale, (n, w.model.n_params))


def _oracle_value(w, pts):
    m = w.model
    fn = cjit.compile_loglik(m.loglik.code, m.loglik.consts)
    fa = cjit.compile_loglik(m.loglik.code, m.loglik.consts, absolute=True)
    ref = O.jit_batch(fn, m.n_params, w.data, m.n_cols, w.n_obs, pts)
    scale = O.jit_batch(fa, m.n_params, w.data, m.n_cols, w.n_obs, pts)
    return ref, scale


@pytest.mark.parametrize("name", ["logistic", "poisson", "mixture", "student_t"])
def test_loglik_at_full_size(gpu, name):
    w = W.make(name)
    m = w.model
    pts = _points(w, N_POINTS, seed=3)
    ref, scale = _oracle_value(w, pts)
    assert np.all(np.isfinite(ref))
    with gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                     m.n_params, w.data, m.n_cols, w.n_obs) as s:
        engines = [s.engine]
        got = {s.engine: s.loglik_batch(pts)}
        if name != "student_t":  # the interpreter engine too (minutes at 2^24 x 65)
            s.set_engine(gpu.ENGINE_INTERP)
            got[gpu.ENGINE_INTERP] = s.loglik_batch(pts)
            engines.append(gpu.ENGINE_INTERP)
    for e in engines:
        err = np.abs(got[e] - ref)
        assert np.all(err <= REL_SUM * scale), (name, e, (err / scale).max())
        assert np.all(err <= REL_SUM * np.abs(ref)), (name, e, (err / np.abs(ref)).max())


@pytest.mark.parametrize("name,n_points", [("poisson", 8), ("student_t", 4)])
def test_grad_at_full_size(gpu, name, n_points):
    w = W.make(name)
    m = w.model
    pts = _points(w, n_points, seed=5)
    threads = len(os.sched_getaffinity(0))
    g_ref, g_abs = O.grad_abs_batch(m.loglik.code, m.loglik.consts, m.n_params, w.data,
                                    m.n_cols, w.n_obs, pts, block=1 << 14, n_threads=threads)
    with gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                     m.n_params, w.data, m.n_cols, w.n_obs) as s:
        got = s.grad_batch(pts).reshape(n_points, m.n_params)
    err = np.abs(got - g_ref)
    assert np.all(err <= REL_GRAD * g_abs), (name, (err / g_abs).max())
