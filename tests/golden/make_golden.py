"""Generate tests/golden/golden.json: the known answers the reference's own
tests pin, restated as numbers.

The reference (R + Rust) cannot be built or run here, so the fixtures are the
expected values written in its test files, plus the R builtins those tests
compare against recomputed with scipy/numpy:

* ``R/dsl.R`` bytecode for ``~ mu + 2`` and ``~ 2 * mu + 2``
  (tests/testthat/test-dsl.R:3-19);
* the gamma log-likelihood against R's ``dgamma`` and its gradient against the
  digamma closed form (tests/testthat/test-catalog.R:35-50), with
  ``scipy.stats.gamma.logpdf`` and ``scipy.special.digamma`` in place of R;
* the two reverse-mode gradient models checked against central differences
  (tests/testthat/test-mala.R:1-33), with the analytic gradients here;
* the Phase-0 Gaussian closed forms (tests/testthat/test-kernel.R:4-21).

Run: ``python tests/golden/make_golden.py`` (rewrites golden.json).
"""
from __future__ import annotations

import json
import os

import numpy as np
import scipy.special as sp
import scipy.stats as st

HERE = os.path.dirname(os.path.abspath(__file__))


def gamma_case():
    y = np.array([0.5, 1.2, 2.0, 3.5])
    a, b = 2.5, 1.3
    val = float(st.gamma.logpdf(y, a=a, scale=1.0 / b).sum())
    ga = len(y) * np.log(b) - len(y) * sp.digamma(a) + np.log(y).sum()
    gb = len(y) * a / b - y.sum()
    return {"formula": "~ a * log(b) - lgamma(a) + (a - 1) * log(y) - b * y",
            "params": ["a", "b"], "data": ["y"], "y": y.tolist(), "point": [a, b],
            "loglik": val, "loglik_tol": 1e-10, "grad": [float(ga), float(gb)],
            "grad_tol": 1e-6}


def gumbel_case():
    y = np.array([3.2, 4.1, 3.8, 4.5, 3.6, 4.0, 3.9])
    mu, lb = 3.9, -0.7
    s = np.exp(lb)
    z = (y - mu) / s
    # ll_i = -z - exp(-z) - lb ; dz/dmu = -1/s ; dz/dlb = -z
    d_mu = np.sum((1.0 - np.exp(-z)) / s)
    d_lb = np.sum(z - z * np.exp(-z) - 1.0)
    return {"formula": "~ -(y - mu) / exp(lb) - exp(-(y - mu) / exp(lb)) - lb",
            "params": ["mu", "lb"], "data": ["y"], "y": y.tolist(), "point": [mu, lb],
            "grad": [float(d_mu), float(d_lb)], "grad_tol": 1e-6}


def pow_case():
    y = np.array([3.2, 4.1, 3.8])
    a, b = 3.5, 1.3
    r = y - a
    q = np.sqrt(r ** 2 + 1.0)
    w = 1.0 + r ** 2 / b ** 2
    # ll_i = -sqrt(r^2 + 1) - log(1 + r^2 / b^2)
    d_a = np.sum(r / q + (2.0 * r / b ** 2) / w)
    d_b = np.sum((2.0 * r ** 2 / b ** 3) / w)
    return {"formula": "~ -sqrt((y - a)^2 + 1) - log(1 + (y - a)^2 / b^2)",
            "params": ["a", "b"], "data": ["y"], "y": y.tolist(), "point": [a, b],
            "grad": [float(d_a), float(d_b)], "grad_tol": 1e-6}


def main():
    golden = {
        "dsl": [
            {"formula": "~ mu + 2", "params": ["mu"], "data": [],
             "code": [1, 0, 0, 0, 3, 0], "consts": [2.0]},
            {"formula": "~ 2 * mu + 2", "params": ["mu"], "data": [], "consts": [2.0]},
            {"formula": "~ (y - mu) * (y - mu)", "params": ["mu"], "data": ["y"],
             "min_depth": 2},
        ],
        "dsl_errors": [
            {"formula": "~ foo + mu", "params": ["mu"], "data": ["y"]},
            {"formula": "~ cos(mu)", "params": ["mu"], "data": ["y"]},
            {"formula": "~ sin(mu)", "params": ["mu"], "data": ["y"]},
            {"formula": "~ y + z", "params": ["mu"], "data": ["y"]},
        ],
        "gamma": gamma_case(),
        "grad_fd": [gumbel_case(), pow_case()],
        "phase0": [
            # -0.5/sigma^2 * sum (d - mu)^2 at data (0,0,0): mu = 0,1,2 (test-kernel.R:4-13)
            {"formula": "~ -0.5 * (y - mu)^2", "y": [0.0, 0.0, 0.0], "points": [0.0, 1.0, 2.0],
             "expect": [0.0, -1.5, -6.0]},
            # sigma = 1 and 2 at candidate 2, data (0,0) (test-kernel.R:15-21)
            {"formula": "~ -0.5 * (y - mu)^2", "y": [0.0, 0.0], "points": [2.0],
             "expect": [-4.0]},
            {"formula": "~ -0.125 * (y - mu)^2", "y": [0.0, 0.0], "points": [2.0],
             "expect": [-1.0]},
        ],
    }
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
