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

With ``proposal="mala"`` the proposal is the reference's Langevin move
(``cpu_native.rs:617-703``: drift (1/2) f M g with M = L L' or diag sd^2, the
whitened drift capped at 2 sqrt(d), then y = mean + L z or mean + sd z) whose
gradient g is the surrogate log posterior's (the surrogate's gradient plus
the prior's, by the oracle's tape), and stage 1 carries q(x|y) / q(y|x)
(``cpu_native.rs:704-714``); the surrogate callable then returns (values,
gradients).  The stream starts with the np normals of the random-walk start
proposal that the device draws and discards before its first Langevin
proposal.

With ``exchange=(ladder_len, every)`` it adds the device replica exchange:
after every ``every``-th iteration the adjacent pairs of one parity within
each ladder of ``ladder_len`` consecutive chains (pairs 0-1, 2-3, ... at odd
exchange numbers, 1-2, 3-4, ... at even ones, as ``R/adaptive.R:362-387``)
swap states with probability min(1, exp((lp[i+1] - lp[i]) (1/T[i] -
1/T[i+1]))) on the exact log posteriors; the uniform is Philox4x32-10
(Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as easy as 1, 2,
3", SC 2011) keyed by (seed, exchange number, pair); both chains of an
exchanged pair draw a new proposal from their own streams.
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


_M32 = 0xFFFFFFFF


def philox4x32_10(c, k0, k1):
    """Philox4x32 with 10 rounds on the counter (c0, c1, c2, c3), key (k0, k1)."""
    c0, c1, c2, c3 = (x & _M32 for x in c)
    for _ in range(10):
        p0 = 0xD2511F53 * c0
        p1 = 0xCD9E8D57 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & _M32, p1 & _M32, ((p0 >> 32) ^ c3 ^ k1) & _M32, \
            p0 & _M32
        k0 = (k0 + 0x9E3779B9) & _M32
        k1 = (k1 + 0xBB67AE85) & _M32
    return c0, c1, c2, c3


def u53(a, b):
    """Uniform in (0, 1] from the top 53 bits of two 32-bit words (the top
    value rounds to 1 in f64, as on the device)."""
    m = ((a << 21) ^ (b >> 11)) & ((1 << 53) - 1)
    return (m + 0.5) / 9007199254740992.0


def exchange_uniform(seed, exchange, pair):
    r = philox4x32_10((pair, exchange, 0x50545357, 0), seed & _M32, 0x3C6EF372)
    return u53(r[0], r[1])


def _half_m_times(sd, L, g):
    """(1/2) f M g with the MALTA cap (``cpu_native.rs:617-651``)."""
    n = g.size
    dmax = 2.0 * math.sqrt(n)
    tmp = np.empty(n)
    if L is None:
        for j in range(n):
            tmp[j] = 0.5 * sd[j] * g[j]
    else:
        for j in range(n):
            acc = 0.0
            for k in range(j, n):
                acc += L[k, j] * g[k]
            tmp[j] = 0.5 * acc
    ss = 0.0
    for j in range(n):
        ss += tmp[j] * tmp[j]
    norm = math.sqrt(ss)
    f = dmax / norm if norm > dmax else 1.0
    out = np.empty(n)
    if L is None:
        for j in range(n):
            out[j] = f * sd[j] * tmp[j]
    else:
        for k in range(n):
            acc = 0.0
            for j in range(k + 1):
                acc += L[k, j] * tmp[j]
            out[k] = f * acc
    return out


def _log_q(sd, L, v, m):
    """-1/2 |Ls^-1 (v - m)|^2 (``cpu_native.rs:655-673``)."""
    n = v.size
    q = 0.0
    if L is None:
        for j in range(n):
            r = (v[j] - m[j]) / sd[j]
            q -= 0.5 * r * r
        return q
    tmp = np.empty(n)
    for k in range(n):
        acc = v[k] - m[k]
        for j in range(k):
            acc -= L[k, j] * tmp[j]
        tmp[k] = acc / L[k, k]
        q -= 0.5 * tmp[k] * tmp[k]
    return q


def _prior_grad(pcode, pconsts, n_params, theta):
    """Gradient of the prior at theta by the oracle's tape (a program that
    reads no data, evaluated once)."""
    pcode = np.ascontiguousarray(pcode, dtype=np.uint32).reshape(-1)
    if pcode.size == 0:
        return np.zeros(n_params)
    return O.grad_batch(pcode, pconsts, n_params, np.zeros(1), 0, 1,
                        np.asarray(theta, dtype=np.float64).reshape(1, n_params))


def run_da(code, consts, prior_code, prior_consts, n_params, data, n_cols, n_obs, init,
           proposal_sd, temperatures, n_iter, seed, surrogate, tie=1e-4, exchange=None,
           proposal="rwm", proposal_l=None):
    """Random-walk delayed acceptance for every chain.

    ``surrogate(theta (n x np)) -> (n,)``.  Returns ``(draws (n_iter, C, np),
    accepts (C,), exact_evals (C,), tie_at (C,))``; ``tie_at[c]`` is the first
    iteration whose decision lay within ``tie`` of its threshold (the chain's
    later draws are not comparable), or n_iter.  With ``exchange`` the tuple
    also holds ``(attempts (C,), accepted (C,))`` per pair (c, c + 1), and a
    tie in an exchange decision marks both chains of the pair."""
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
    mala = proposal == "mala"
    Ls = None
    if proposal_l is not None:
        Ls = np.asarray(proposal_l, dtype=np.float64).reshape(C, n_params, n_params)
    if mala:
        sx, gsx = surrogate(x)
        sx = np.asarray(sx, dtype=np.float64)
        gx = np.asarray(gsx, dtype=np.float64).reshape(C, n_params).copy()
        for c in range(C):
            gx[c] += _prior_grad(prior_code, prior_consts, n_params, x[c])
            for _ in range(2 * n_params):  # the discarded random-walk start proposal
                streams[c].next()
        mx = np.zeros_like(x)
    else:
        sx = np.asarray(surrogate(x), dtype=np.float64)
    draws = np.zeros((n_iter, C, n_params))
    accepts = np.zeros(C, dtype=np.int64)
    exact_n = np.zeros(C, dtype=np.int64)
    tie_at = np.full(C, n_iter, dtype=np.int64)

    def propose_one(c, y):
        if not mala:
            for j in range(n_params):
                y[c, j] = x[c, j] + sd[c, j] * streams[c].normal()
            return
        L = None if Ls is None else Ls[c]
        mx[c] = _half_m_times(sd[c], L, gx[c]) + x[c]
        z = np.array([streams[c].normal() for _ in range(n_params)])
        if L is None:
            y[c] = mx[c] + sd[c] * z
        else:
            for k in range(n_params):
                acc = mx[c, k]
                for j in range(k + 1):
                    acc += L[k, j] * z[j]
                y[c, k] = acc

    def propose():
        y = np.empty_like(x)
        for c in range(C):
            propose_one(c, y)
        return y

    att = np.zeros(C, dtype=np.int64)
    ok = np.zeros(C, dtype=np.int64)

    def exchange_step(t_done, y):
        K, every = exchange
        if t_done % every or t_done >= n_iter:
            return
        s = t_done // every
        for i in range(C - 1):
            if i % K == K - 1 or (i % K) % 2 != (s + 1) % 2:
                continue
            lpa, lpb = llx[i] + px[i], llx[i + 1] + px[i + 1]
            delta = (lpb - lpa) * (1.0 / temps[i] - 1.0 / temps[i + 1])
            lu = math.log(exchange_uniform(seed, s, i))
            att[i] += 1
            if abs(lu - delta) < tie:
                for c in (i, i + 1):
                    tie_at[c] = min(tie_at[c], t_done)
            if not (math.isfinite(delta) and lu < delta):
                continue
            ok[i] += 1
            for arr in (x, llx, px, sx) + ((gx,) if mala else ()):
                arr[[i, i + 1]] = arr[[i + 1, i]]
            for c in (i, i + 1):
                propose_one(c, y)

    y = propose()
    for t in range(n_iter):
        if mala:
            sy, gsy = surrogate(y)
            sy = np.asarray(sy, dtype=np.float64)
            gsy = np.asarray(gsy, dtype=np.float64).reshape(C, n_params)
        else:
            sy = np.asarray(surrogate(y), dtype=np.float64)
        for c in range(C):
            py = _prior(prior_code, prior_consts, y[c])
            lqd, finite = 0.0, True
            if mala:
                L = None if Ls is None else Ls[c]
                gy = gsy[c] + _prior_grad(prior_code, prior_consts, n_params, y[c])
                my = _half_m_times(sd[c], L, gy) + y[c]
                lqd = _log_q(sd[c], L, x[c], my) - _log_q(sd[c], L, y[c], mx[c])
                finite = math.isfinite(sy[c] + py)
            u1 = streams[c].next()
            a1 = ((sy[c] + py) - (sx[c] + px[c])) / temps[c] + lqd
            if abs(math.log(u1) - a1) < tie and tie_at[c] == n_iter:
                tie_at[c] = t
            if finite and math.log(u1) < a1:
                exact_n[c] += 1
                lly = float(exact(y[c])[0])
                u2 = streams[c].next()
                a2 = ((lly - llx[c]) - (sy[c] - sx[c])) / temps[c]
                if abs(math.log(u2) - a2) < tie and tie_at[c] == n_iter:
                    tie_at[c] = t
                if math.log(u2) < a2:
                    x[c] = y[c]
                    llx[c], px[c], sx[c] = lly, py, sy[c]
                    if mala:
                        gx[c] = gy
                    accepts[c] += 1
        draws[t] = x
        if t + 1 < n_iter:
            y = propose()
            if exchange is not None:
                exchange_step(t + 1, y)
    if exchange is not None:
        return draws, accepts, exact_n, tie_at, (att, ok)
    return draws, accepts, exact_n, tie_at
