"""CPU oracle of delayed-acceptance Metropolis -- TEST INFRASTRUCTURE ONLY.

Two-stage Metropolis-Hastings (Christen & Fox, "Markov chain Monte Carlo using
an approximation", JCGS 14(4), 2005) with a surrogate log-likelihood s() as
the first stage and the exact log-likelihood l() as the second:

  stage 1: accept y with prob. min(1, exp([s(y) + p(y) - s(x) - p(x)] / T))
  stage 2: accept with prob.   min(1, exp([l(y) - l(x) - (s(y) - s(x))] / T))

The single-stage rule it refines is the reference's tempered acceptance
(``src/rust/src/cpu_native.rs:792``); the proposal and the triple32 uniform
stream are the reference's random-walk ones (``cpu_native.rs:726-735``,
``:12-40``).  The stream order per chain is: the initial proposal's normals,
then per iteration the stage-1 uniform, the stage-2 uniform (only when stage 1
accepted), and the next proposal's normals.  The surrogate is a callable, so
the test can hand in the very network the GPU uses.  Used by tests only.
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O


def _prior(pcode, pconsts, theta):
    pcode = np.ascontiguousarray(pcode, dtype=np.uint32).reshape(-1)
    if pcode.size == 0:
        return 0.0
    pconsts = np.ascontiguousarray(pconsts, dtype=np.float64).reshape(-1)
    th = np.ascontiguousarray(theta, dtype=np.float64)
    return O.lib().gpo_eval(pcode, pcode.size // 2, pconsts if pconsts.size else np.zeros(1),
                            th, None)


class _Stream:
    def __init__(self, seed, chain):
        self.mix = O.seedmix(seed, chain)
        self.ctr = 0

    def next(self):
        self.ctr += 1
        return O.uniform(self.mix, self.ctr)

    def normal(self):
        u1 = self.next()
        u2 = self.next()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(6.283185307179586 * u2)


def run_da(code, consts, prior_code, prior_consts, n_params, data, n_cols, n_obs, init,
           proposal_sd, temperatures, n_iter, seed, surrogate, tie=1e-4):
    """Random-walk delayed acceptance for every chain.

    ``surrogate(theta (n x np)) -> (n,)``.  Returns ``(draws (n_iter, C, np),
    accepts (C,), exact_evals (C,), tie_at (C,))``; ``tie_at[c]`` is the first
    iteration whose decision lay within ``tie`` of its threshold (the chain's
    later draws are not comparable), or n_iter."""
    init = np.asarray(init, dtype=np.float64).reshape(-1, n_params)
    C = init.shape[0]
    sd = np.asarray(proposal_sd, dtype=np.float64).reshape(C, n_params)
    temps = np.asarray(temperatures, dtype=np.float64).reshape(C)

    def exact(th):
        return O.loglik_batch(code, consts, n_params, data, n_cols, n_obs,
                              np.asarray(th, dtype=np.float64).reshape(-1, n_params))

    x = init.copy()
    streams = [_Stream(seed, c) for c in range(C)]
    llx = exact(x)
    px = np.array([_prior(prior_code, prior_consts, x[c]) for c in range(C)])
    sx = np.asarray(surrogate(x), dtype=np.float64)
    draws = np.zeros((n_iter, C, n_params))
    accepts = np.zeros(C, dtype=np.int64)
    exact_n = np.zeros(C, dtype=np.int64)
    tie_at = np.full(C, n_iter, dtype=np.int64)

    def propose():
        y = np.empty_like(x)
        for c in range(C):
            for j in range(n_params):
                y[c, j] = x[c, j] + sd[c, j] * streams[c].normal()
        return y

    y = propose()
    for t in range(n_iter):
        sy = np.asarray(surrogate(y), dtype=np.float64)
        for c in range(C):
            py = _prior(prior_code, prior_consts, y[c])
            u1 = streams[c].next()
            a1 = ((sy[c] + py) - (sx[c] + px[c])) / temps[c]
            if abs(math.log(u1) - a1) < tie and tie_at[c] == n_iter:
                tie_at[c] = t
            if math.log(u1) < a1:
                exact_n[c] += 1
                lly = float(exact(y[c])[0])
                u2 = streams[c].next()
                a2 = ((lly - llx[c]) - (sy[c] - sx[c])) / temps[c]
                if abs(math.log(u2) - a2) < tie and tie_at[c] == n_iter:
                    tie_at[c] = t
                if math.log(u2) < a2:
                    x[c] = y[c]
                    llx[c], px[c], sx[c] = lly, py, sy[c]
                    accepts[c] += 1
        draws[t] = x
        if t + 1 < n_iter:
            y = propose()
    return draws, accepts, exact_n, tie_at
