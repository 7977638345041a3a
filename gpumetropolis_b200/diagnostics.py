"""Convergence and efficiency diagnostics (restating ``R/diagnostics.R``).

* :func:`ess` -- Geyer's initial positive sequence per chain, summed over
  chains (``R/diagnostics.R:36-59,96-99``), the package's own estimator;
* :func:`ess_pooled` -- multi-chain ESS from the chain-averaged
  autocovariance and the between-chain variance (Vehtari, Gelman, Simpson,
  Carpenter & Buerkner 2021, without rank normalisation), with Geyer's
  initial monotone sequence; robust where chains barely move, where the
  per-chain estimator counts a constant chain as fully independent.  Not in
  the reference; used to compare samplers' ESS per second;
* :func:`rhat` -- split R-hat (``R/diagnostics.R:127-159``);
* :func:`gaussian_mean_posterior` -- the closed form N(mean(y), sigma^2/n)
  (``R/diagnostics.R:246-257``).

Draw arrays are ``(n_iter, n_chains)`` as in the R functions.
"""
from __future__ import annotations

import numpy as np


def _acf(v: np.ndarray, lag_max: int) -> np.ndarray:
    """R's ``acf(demean=TRUE)``: autocovariance with divisor n, normalised."""
    n = v.size
    x = v - v.mean()
    m = 1 << int(np.ceil(np.log2(2 * n)))
    f = np.fft.rfft(x, m)
    acov = np.fft.irfft(f * np.conj(f), m)[: lag_max + 1] / n
    return acov / acov[0]


def ess_chain(v) -> float:
    """Effective sample size of one chain (``R/diagnostics.R:36-59``)."""
    v = np.asarray(v, dtype=np.float64)
    n = v.size
    if n < 8 or np.var(v) == 0:
        return float(n)
    lag_max = min(n - 1, 2000)
    rho = _acf(v, lag_max)[1:]
    m = rho.size // 2
    if m < 1:
        return float(n)
    pair = rho[0:2 * m:2] + rho[1:2 * m:2]
    neg = np.nonzero(pair <= 0)[0]
    last = neg[0] if neg.size else m
    if last < 1:
        return float(n)
    tau = 1.0 + 2.0 * pair[:last].sum()
    tau = max(tau, 1.0)
    return float(min(n / tau, n))


def ess(draws, warmup: int | None = None) -> float:
    """Summed per-chain ESS of an ``(n_iter, n_chains)`` array (``:96-99``)."""
    x = np.asarray(draws, dtype=np.float64)
    if x.ndim == 1:
        x = x[:, None]
        warmup = 0 if warmup is None else warmup
    n = x.shape[0]
    w = n // 2 if warmup is None else int(warmup)
    if w < 0 or w >= n:
        raise ValueError("`warmup` must be in [0, n_iter).")
    return float(sum(ess_chain(x[w:, c]) for c in range(x.shape[1])))


def acov_chain_mean(xc: np.ndarray) -> np.ndarray:
    """Autocovariance (divisor n) at lags 0..n-1 of each column of the
    centred ``(n, m)`` array, averaged over the m columns."""
    n = xc.shape[0]
    L = 1 << int(np.ceil(np.log2(2 * n)))
    f = np.fft.rfft(xc, L, axis=0)
    acov = np.fft.irfft(f * np.conj(f), L, axis=0)[:n] / n       # (n, m), divisor n
    return acov.mean(axis=1)


def ess_pooled(draws, acov_mean_fn=None) -> float:
    """Multi-chain ESS of an ``(n_iter, n_chains)`` array (all draws kept).
    ``acov_mean_fn`` replaces :func:`acov_chain_mean` (e.g. the same FFTs
    on a GPU for thousands of chains)."""
    x = np.asarray(draws, dtype=np.float64)
    if x.ndim == 1:
        x = x[:, None]
    n, m = x.shape
    if n < 4:
        return float(n * m)
    xc = x - x.mean(axis=0)
    acov_mean = (acov_mean_fn or acov_chain_mean)(xc)
    W = acov_mean[0] * n / (n - 1)
    B_over_n = x.mean(axis=0).var(ddof=1) if m > 1 else 0.0
    var_plus = W * (n - 1) / n + B_over_n
    if not var_plus > 0:
        return 0.0
    rho = 1.0 - (W - acov_mean) / var_plus
    rho[0] = 1.0
    k = (n - 1) // 2
    P = rho[0:2 * k:2] + rho[1:2 * k:2]
    # initial positive sequence, then made monotone
    pos = np.nonzero(P <= 0)[0]
    P = P[: pos[0]] if pos.size else P
    if P.size == 0:
        return float(n * m)
    P = np.minimum.accumulate(P)
    tau = max(-1.0 + 2.0 * P.sum(), 1.0 / np.log10(max(n * m, 10)))
    return float(n * m / tau)


def rhat(draws, warmup: int | None = None) -> float:
    """Split R-hat of an ``(n_iter, n_chains)`` array (``R/diagnostics.R:127-159``)."""
    x = np.asarray(draws, dtype=np.float64)
    if x.ndim != 2:
        raise ValueError("`draws` must be an (n_iter, n_chains) matrix.")
    n = x.shape[0]
    w = n // 2 if warmup is None else int(warmup)
    if w < 0 or w >= n:
        raise ValueError("`warmup` must be in [0, n_iter).")
    kept = x[w:]
    nk = kept.shape[0]
    half = nk // 2
    if half < 2:
        raise ValueError("need at least 4 post-warmup iterations per chain for split R-hat.")
    splits = np.concatenate([kept[:half], kept[nk - half:]], axis=1)
    means = splits.mean(axis=0)
    variances = splits.var(axis=0, ddof=1)
    between = half * means.var(ddof=1)
    within = variances.mean()
    if within <= 0:
        return float("nan")
    var_hat = ((half - 1) * within + between) / half
    return float(np.sqrt(var_hat / within))


def mcse(draws, warmup: int | None = None) -> float:
    """Monte Carlo standard error of the mean, sd / sqrt(ESS)."""
    x = np.asarray(draws, dtype=np.float64)
    n = x.shape[0]
    w = n // 2 if warmup is None else int(warmup)
    return float(x[w:].std(ddof=1) / np.sqrt(ess(x, warmup=w)))


def gaussian_mean_posterior(data, sigma: float):
    """Closed-form posterior of a Gaussian mean, flat prior (``:246-257``)."""
    d = np.asarray(data, dtype=np.float64).ravel()
    if d.size < 1 or not np.all(np.isfinite(d)):
        raise ValueError("`data` must be a non-empty numeric vector of finite values.")
    if not (np.isfinite(sigma) and sigma > 0):
        raise ValueError("`sigma` must be a single positive finite number.")
    return {"mean": float(d.mean()), "sd": float(sigma / np.sqrt(d.size))}
