"""Seeded synthetic workloads with the shapes of the five benchmark configs.

No dataset is involved: every config is synthetic (numpy ``PCG64``).  Models
are written as a user writes them in the DSL, so their bytecode is what the
reference would run.  ``n_obs`` can be reduced for parity tests; the full
sizes are the defaults.

* ``gaussian``  -- y ~ N(3.4, 2^2), N = 20,000, loglik -(y-mu)^2/8, flat prior
* ``logistic``  -- N = 2^20, 16 N(0,1) covariates + intercept, beta ~ N(0,.5^2),
                   y ~ Bernoulli(sigmoid(eta)), N(0,10^2) priors (17 params)
* ``poisson``   -- N = 2^21, 24 U(-1,1) covariates, beta ~ N(0,.2^2),
                   y ~ Poisson(exp(eta)), N(0,1) priors (24 params)
* ``mixture``   -- N = 2^22, y ~ .3 N(-2,1) + .7 N(3,1.5^2); params logit w,
                   mu1, mu2, log s1, log s2
* ``student_t`` -- N = 2^24, 64 N(0,1) covariates with AR(1) correlation .6,
                   residuals t(4) * 1.5; 65 params (beta, log sigma)
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, Optional

import numpy as np

from .dsl import GpumModel, gpum_model, linear_predictor


@dataclass
class Workload:
    name: str
    model: GpumModel
    data: np.ndarray          # row-major (n_obs, n_cols) float64
    truth: Dict[str, object]
    n_chains: int
    n_iter: int
    method: str

    @property
    def n_obs(self) -> int:
        return self.data.shape[0]


def _prior(params, sd):
    """Independent N(0, sd^2) prior, written ``~ -b0^2 / 200 - b1^2 / 200 ...``."""
    inv = 2.0 * sd * sd
    inv_s = str(int(inv)) if float(inv).is_integer() else repr(inv)
    return "~ -" + " - ".join(f"{p}^2 / {inv_s}" for p in params)


def gaussian(n_obs: int = 20_000, seed: int = 1) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    y = rng.normal(3.4, 2.0, n_obs)
    m = gpum_model("~ -((y - mu)^2) / 8", params="mu", data="y")
    truth = {"post_mean": float(y.mean()), "post_sd": float(2.0 / np.sqrt(n_obs))}
    return Workload("gaussian", m, y.reshape(-1, 1).astype(np.float64), truth, 8, 3000, "rwm")


def logistic(n_obs: int = 1 << 20, seed: int = 2, p: int = 16) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n_obs, p), dtype=np.float32)
    beta = rng.normal(0.0, 0.5, p + 1)
    eta = beta[0] + X.astype(np.float64) @ beta[1:]
    y = (rng.random(n_obs) < 1.0 / (1.0 + np.exp(-eta))).astype(np.float64)
    params = [f"b{j}" for j in range(p + 1)]
    xs = [f"x{j}" for j in range(1, p + 1)]
    lp = linear_predictor(params, [None] + xs)
    m = gpum_model(f"~ y * ({lp}) - log(1 + exp({lp}))", params=params, data=xs + ["y"],
                   prior=_prior(params, 10.0))
    data = np.concatenate([X.astype(np.float64), y[:, None]], axis=1)
    return Workload("logistic", m, data, {"beta": beta}, 1024, 5000, "rwm")


def poisson(n_obs: int = 1 << 21, seed: int = 3, p: int = 24) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.uniform(-1.0, 1.0, (n_obs, p)).astype(np.float32)
    beta = rng.normal(0.0, 0.2, p)
    eta = X.astype(np.float64) @ beta
    y = rng.poisson(np.exp(eta)).astype(np.float64)
    params = [f"b{j}" for j in range(1, p + 1)]
    xs = [f"x{j}" for j in range(1, p + 1)]
    lp = linear_predictor(params, xs)
    m = gpum_model(f"~ y * ({lp}) - exp({lp}) - lgamma(y + 1)", params=params,
                   data=xs + ["y"], prior=_prior(params, 1.0))
    data = np.concatenate([X.astype(np.float64), y[:, None]], axis=1)
    return Workload("poisson", m, data, {"beta": beta}, 4096, 4000, "mala")


def mixture(n_obs: int = 1 << 22, seed: int = 4) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    z = rng.random(n_obs) < 0.3
    y = np.where(z, rng.normal(-2.0, 1.0, n_obs), rng.normal(3.0, 1.5, n_obs))
    y = y.astype(np.float32).astype(np.float64)
    params = ["lw", "mu1", "mu2", "ls1", "ls2"]
    ll = ("~ log(exp(-((y - mu1)^2) / (2 * exp(2 * ls1)) - ls1) / (1 + exp(-lw))"
          " + exp(-((y - mu2)^2) / (2 * exp(2 * ls2)) - ls2) / (1 + exp(lw)))")
    prior = "~ -lw^2 / 8 - mu1^2 / 50 - mu2^2 / 50 - ls1^2 / 2 - ls2^2 / 2"
    m = gpum_model(ll, params=params, data="y", prior=prior)
    truth = {"w": 0.3, "mu1": -2.0, "mu2": 3.0, "s1": 1.0, "s2": 1.5}
    return Workload("mixture", m, y.reshape(-1, 1), truth, 16 * 512, 2000, "pt")


def student_t(n_obs: int = 1 << 24, seed: int = 5, p: int = 64) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    # Covariates generated column by column (contiguous rows of XT, so the
    # AR(1) recursion streams memory), then written into the row-major data.
    XT = np.empty((p, n_obs), np.float32)
    XT[0] = rng.standard_normal(n_obs, dtype=np.float32)
    for j in range(1, p):
        XT[j] = 0.6 * XT[j - 1] + 0.8 * rng.standard_normal(n_obs, dtype=np.float32)
    beta = rng.normal(0.0, 0.3, p)
    y = np.zeros(n_obs)
    for j in range(p):
        y += beta[j] * XT[j].astype(np.float64)
    y += 1.5 * rng.standard_t(4.0, n_obs)
    y = y.astype(np.float32).astype(np.float64)
    params = [f"b{j}" for j in range(1, p + 1)] + ["ls"]
    xs = [f"x{j}" for j in range(1, p + 1)]
    lp = linear_predictor(params[:-1], xs)
    ll = (f"~ lgamma(2.5) - lgamma(2) - 0.5 * log(4 * 3.141592653589793) - ls"
          f" - 2.5 * log(1 + ((y - ({lp})) / exp(ls))^2 / 4)")
    m = gpum_model(ll, params=params, data=xs + ["y"], prior=_prior(params, 10.0))
    data = np.empty((n_obs, p + 1))
    step = 1 << 16
    for r0 in range(0, n_obs, step):
        data[r0:r0 + step, :p] = XT[:, r0:r0 + step].T
    data[:, p] = y
    del XT
    return Workload("student_t", m, data, {"beta": beta, "sigma": 1.5}, 8192, 2000, "de")


ALL = {"gaussian": gaussian, "logistic": logistic, "poisson": poisson, "mixture": mixture,
       "student_t": student_t}


def make(name: str, n_obs: Optional[int] = None, **kw) -> Workload:
    f = ALL[name]
    return f(n_obs=n_obs, **kw) if n_obs is not None else f(**kw)
