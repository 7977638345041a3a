"""Host orchestration of batched runs: adaptive warmup, parallel tempering and
differential evolution (restating ``R/adaptive.R``).

Every batch is one call into the B200 session (model and data stay resident
on the GPU, unlike the reference, which re-uploads everything per batch,
``src/rust/src/chain_kernel.rs:391-413``).  Between batches the host updates
Welford moments, Robbins-Monro scales and Cholesky factors exactly as the
reference's R code does, vectorised over chains.

``call(init, sd, n_iter, seed, temperatures, proposal_mode, gamma, de_noise,
proposal_l)`` returns ``(draws (n_iter, C, np), accept_rate (C,),
last_log_post (C,))``.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

_LOW_D = [0.44, 0.35, 0.32, 0.30, 0.28, 0.27, 0.26, 0.25]


def target_accept(d: int) -> float:
    """Optimal RWM acceptance by dimension (``R/adaptive.R:69-72``)."""
    return _LOW_D[d - 1] if 1 <= d <= 8 else 0.234


def robbins_monro_scale(scale, accept_rate, batch_idx, d, target=None):
    """``log s += b^(-2/3) (acc - target)`` (``R/adaptive.R:78-85``)."""
    if target is None:
        target = target_accept(d)
    gamma = float(batch_idx) ** (-2.0 / 3.0)
    return np.exp(np.log(scale) + gamma * (np.asarray(accept_rate) - target))


def cholesky_reg(sigma, eps=1e-8):
    """Regularised lower Cholesky factor (``R/adaptive.R:548-558``)."""
    sigma = np.asarray(sigma, dtype=np.float64)
    d = sigma.shape[0]
    reg = eps * float(np.mean(np.diag(sigma)))
    if not np.isfinite(reg) or reg <= 0:
        reg = eps
    s = sigma + reg * np.eye(d)
    try:
        return np.linalg.cholesky(s)
    except np.linalg.LinAlgError:
        return np.diag(np.sqrt(np.maximum(np.diag(s), reg)))


@dataclass
class Welford:
    """Running mean / cross-product for a stack of chains (``R/adaptive.R:15-61``).

    ``mean`` is (C, d), ``m2`` (C, d, d); batches merge with Chan's pairwise
    update, equal in exact arithmetic to the row-by-row Welford update."""
    n: np.ndarray
    mean: np.ndarray
    m2: np.ndarray
    sigma: np.ndarray

    @classmethod
    def init(cls, n_chains: int, d: int, sigma_diag):
        sig = np.zeros((n_chains, d, d))
        sd = np.broadcast_to(np.asarray(sigma_diag, dtype=np.float64), (n_chains, d))
        idx = np.arange(d)
        sig[:, idx, idx] = sd
        return cls(np.zeros(n_chains, np.int64), np.zeros((n_chains, d)),
                   np.zeros((n_chains, d, d)), sig)

    def update(self, x):
        """Merge a batch ``x`` of shape (n_b, C, d)."""
        x = np.asarray(x, dtype=np.float64)
        nb = x.shape[0]
        if nb == 0:
            return self
        mb = x.mean(axis=0)
        dev = x - mb
        return self.merge(nb, mb, np.einsum("ncd,nce->cde", dev, dev))

    def merge(self, nb, mb, m2b):
        """Merge a batch given by its size, means (C, d) and cross-deviation
        sums (C, d, d) -- Chan, Golub & LeVeque's pairwise update."""
        if nb == 0:
            return self
        na = self.n.astype(np.float64)
        n = na + nb
        delta = np.asarray(mb, dtype=np.float64) - self.mean
        self.mean = self.mean + delta * (nb / n)[:, None]
        self.m2 = self.m2 + m2b + np.einsum("cd,ce->cde", delta, delta) * (na * nb / n)[:, None,
                                                                                         None]
        self.n = self.n + nb
        return self

    def covariance(self):
        cov = self.m2 / np.maximum(self.n - 1, 1)[:, None, None]
        return np.where((self.n < 2)[:, None, None], self.sigma, cov)


@dataclass
class WelfordDiag:
    """Per-chain running means and variances only: the per-chain adaptation
    uses nothing but the diagonal (``R/adaptive.R:150-160``).  ``m2`` is
    (C, d)."""
    n: np.ndarray
    mean: np.ndarray
    m2: np.ndarray
    sigma: np.ndarray

    @classmethod
    def init(cls, n_chains: int, d: int, sigma_diag):
        sd = np.broadcast_to(np.asarray(sigma_diag, dtype=np.float64), (n_chains, d)).copy()
        return cls(np.zeros(n_chains, np.int64), np.zeros((n_chains, d)),
                   np.zeros((n_chains, d)), sd)

    def update(self, x):
        x = np.asarray(x, dtype=np.float64)
        nb = x.shape[0]
        if nb == 0:
            return self
        mb = x.mean(axis=0)
        return self.merge(nb, mb, ((x - mb) ** 2).sum(axis=0))

    def merge(self, nb, mb, m2b):
        if nb == 0:
            return self
        na = self.n.astype(np.float64)
        n = na + nb
        delta = np.asarray(mb, dtype=np.float64) - self.mean
        self.mean = self.mean + delta * (nb / n)[:, None]
        self.m2 = self.m2 + m2b + delta * delta * (na * nb / n)[:, None]
        self.n = self.n + nb
        return self

    def variances(self):
        var = self.m2 / np.maximum(self.n - 1, 1)[:, None]
        return np.where((self.n < 2)[:, None], self.sigma, var)


@dataclass
class BatchMoments:
    """What the adaptation needs from a batch of draws (n, C, d)."""
    n: int
    chain_mean: np.ndarray   # (C, d)
    chain_m2: np.ndarray     # (C, d) sums of squared deviations
    pool_mean: np.ndarray    # (d,)
    pool_m2: np.ndarray      # (d, d) sums of cross deviations over n * C draws
    last: np.ndarray         # (C, d) the final states


def moments_of(draws) -> BatchMoments:
    """Host version of the device moment reduction (for backends that return
    draws)."""
    x = np.asarray(draws, dtype=np.float64)
    n = x.shape[0]
    cm = x.mean(axis=0)
    pool = x.reshape(-1, x.shape[2])
    pm = pool.mean(axis=0)
    dev = pool - pm
    return BatchMoments(n, cm, ((x - cm) ** 2).sum(axis=0), pm, dev.T @ dev, x[-1].copy())


def _run_batch(call, init, sd, n, seed, mode, L):
    """One warmup batch: device moments when the backend has them (no draws
    copied), else moments of the returned draws."""
    if hasattr(call, "run_moments"):
        return call.run_moments(init, sd, n, seed, None, mode, 0.0, 0.0, L)
    draws, acc, _ = call(init, sd, n, seed, None, mode, 0.0, 0.0, L)
    return moments_of(draws), acc


@dataclass
class WarmupResult:
    final_proposal_sd: np.ndarray
    final_init: np.ndarray
    final_scales: np.ndarray
    final_L: Optional[np.ndarray]
    n_batches: int
    batch_sizes: np.ndarray
    warmup_used: int
    accept_history: np.ndarray
    seed_next: int


def am_orchestrate_warmup(call: Callable, np_: int, n_chains: int, init_mat, proposal_sd,
                          warmup: int, seed: int, auto_stop=False, langevin=False):
    """Batched adaptive warmup (``R/adaptive.R:101-254``)."""
    if warmup <= 0:
        raise ValueError("warmup must be positive")
    n_batches = min(40, max(10, warmup // 50))
    n_batches = min(n_batches, warmup)
    k = warmup // n_batches
    sizes = np.full(n_batches, k, dtype=np.int64)
    sizes[-1] += warmup - n_batches * k
    C = n_chains
    states = WelfordDiag.init(C, np_, np.asarray(proposal_sd) ** 2)
    scale0 = 1.65 / np_ ** (1.0 / 6.0) if langevin else 2.38 / np.sqrt(np_)
    scales = np.full(C, scale0)
    cur_init = np.array(init_mat, dtype=np.float64, copy=True)
    cur_sd = np.array(proposal_sd, dtype=np.float64, copy=True)
    acc_hist = np.full((C, n_batches), np.nan)
    cur_L = None
    L_pool = None
    pool = Welford.init(1, np_, np.asarray(proposal_sd)[0] ** 2)
    target = 0.574 if langevin else target_accept(np_)
    reset_batch = n_batches // 2
    prev_scales = scales.copy()
    streak = 0
    batches_run = 0
    consumed = 0
    for b in range(1, n_batches + 1):
        use_L = np_ > 1 and cur_L is not None
        pm = 3 if langevin else (2 if use_L else 0)
        mo, acc = _run_batch(call, cur_init, cur_sd, int(sizes[b - 1]), seed + b - 1, pm,
                             cur_L if use_L else None)
        states.merge(mo.n, mo.chain_mean, mo.chain_m2)
        pool.merge(mo.n * C, mo.pool_mean[None], mo.pool_m2[None])
        bi = b - reset_batch if b > reset_batch else b
        scales = robbins_monro_scale(scales, acc, bi, np_, target)
        cur_init = mo.last
        diag_sd = np.sqrt(np.maximum(states.variances(), 1e-12))
        cur_sd = scales[:, None] * diag_sd
        acc_hist[:, b - 1] = acc
        if b == reset_batch:
            diag_now = np.maximum(np.diag(pool.covariance()[0]), 1e-12)
            pool = Welford.init(1, np_, diag_now)
            states = WelfordDiag.init(C, np_, diag_now)
            scales = np.full(C, scale0)
        if np_ > 1:
            if pool.n[0] >= 2:
                L_pool = cholesky_reg(pool.covariance()[0])
            if L_pool is not None:
                cur_L = scales[:, None, None] * L_pool[None]
        batches_run = b
        consumed += int(sizes[b - 1])
        if auto_stop and b >= max(10, reset_batch + 5):
            drift = float(np.max(np.abs(scales / prev_scales - 1.0)))
            if np.mean(np.abs(acc - target)) < 0.05 and drift < 0.03:
                streak += 1
            else:
                streak = 0
            if streak >= 2:
                break
        prev_scales = scales.copy()
    return WarmupResult(cur_sd, cur_init, scales, cur_L if np_ > 1 else None, batches_run,
                        sizes[:batches_run], consumed, acc_hist[:, :batches_run],
                        seed + batches_run)


def pt_default_ladder(n_chains: int, t_max: float = 10.0):
    """Geometric ladder from 1 to t_max (``R/adaptive.R:261-265``)."""
    if n_chains <= 1:
        return np.ones(n_chains)
    beta = t_max ** (1.0 / (n_chains - 1))
    return beta ** np.arange(n_chains)


def pt_swap_draws(seed, batch, n_draws):
    """Swap uniforms reproducible from (seed, batch) (``R/adaptive.R:530-546``).
    The reference seeds R's Mersenne twister with the same mix; R's stream is not
    reproducible outside R, so a PCG64 stream is seeded with the mix instead."""
    if n_draws <= 0:
        return np.zeros(0)
    mix = int((float(seed) + float(batch) * 2654435761.0) % 2 ** 31)
    return np.random.Generator(np.random.PCG64(mix)).random(n_draws)


def _batches(total, every):
    n = max(1, total // every)
    sizes = np.full(n, every, dtype=np.int64)
    rem = total - n * every
    if rem > 0:
        sizes[-1] += rem
    return sizes


@dataclass
class BatchedResult:
    draws: np.ndarray
    accept_rate: np.ndarray
    final_proposal_sd: np.ndarray
    final_init: np.ndarray
    n_batches: int
    batch_sizes: np.ndarray
    warmup_batches: int
    warmup_used: int
    accept_history: np.ndarray
    seed_next: int
    final_scales: Optional[np.ndarray] = None
    swap_history: Optional[np.ndarray] = None
    disp_history: Optional[np.ndarray] = None
    extra: dict = field(default_factory=dict)


def pt_orchestrate(call, np_, n_chains, init_mat, proposal_sd, temperatures, n_iter, warmup,
                   swap_every, adapt, seed):
    """Parallel tempering with adjacent swaps between batches
    (``R/adaptive.R:272-413``)."""
    temps = np.asarray(temperatures, dtype=np.float64)
    if temps.size != n_chains:
        raise ValueError("`temperatures` must have one value per chain.")
    if swap_every < 1:
        raise ValueError("`swap_every` must be a positive integer.")
    sizes = _batches(n_iter, int(swap_every))
    nb = sizes.size
    wb = max(0, min(nb, warmup // swap_every))
    wused = int(sizes[:wb].sum()) if wb > 0 else 0
    C = n_chains
    states = WelfordDiag.init(C, np_, np.asarray(proposal_sd) ** 2)
    scales = np.ones(C)
    cur_init = np.array(init_mat, dtype=np.float64, copy=True)
    cur_sd = np.array(proposal_sd, dtype=np.float64, copy=True)
    samp = max(1, n_iter - wused)
    kept = np.full((samp, C, np_), np.nan)
    acc_sum = np.zeros(C)
    iters = 0
    filled = 0
    pairs = C - 1 if C >= 2 else 0
    swap_hist = np.full((pairs, nb), np.nan)
    acc_hist = np.full((C, nb), np.nan)
    acc = np.zeros(C)
    for b in range(1, nb + 1):
        bs = int(sizes[b - 1])
        draws, acc, last = call(cur_init, cur_sd, bs, seed + b - 1, temps, 0, 0.0, 0.0, None)
        lp = np.array(last, dtype=np.float64)
        acc_hist[:, b - 1] = acc
        in_warm = b <= wb
        if not in_warm:
            kept[filled:filled + bs] = draws
            acc_sum += bs * acc
            iters += bs
            filled += bs
        if in_warm and adapt:
            states.update(draws)
            scales = robbins_monro_scale(scales, acc, b, np_)
            cur_sd = scales[:, None] * np.sqrt(np.maximum(states.variances(), 1e-12))
        cur_init = draws[-1].copy()
        if pairs > 0:
            order = (np.arange(1, pairs + 1, 2) if b % 2 == 1
                     else np.arange(min(2, pairs), pairs + 1, 2))
            u = pt_swap_draws(seed, b, order.size)
            att = np.zeros(pairs, np.int64)
            okc = np.zeros(pairs, np.int64)
            for k, i1 in enumerate(order):
                i = i1 - 1
                delta = (lp[i + 1] - lp[i]) * (1.0 / temps[i] - 1.0 / temps[i + 1])
                att[i] += 1
                if np.isfinite(delta) and np.log(u[k]) < delta:
                    cur_init[[i, i + 1]] = cur_init[[i + 1, i]]
                    lp[[i, i + 1]] = lp[[i + 1, i]]
                    okc[i] += 1
            with np.errstate(invalid="ignore", divide="ignore"):
                swap_hist[:, b - 1] = np.where(att > 0, okc / np.maximum(att, 1), np.nan)
    rate = acc_sum / iters if iters > 0 else acc
    return BatchedResult(kept[:filled], rate, cur_sd, cur_init, nb, sizes, wb, wused, acc_hist,
                         seed + nb, final_scales=scales, swap_history=swap_hist)


def de_orchestrate(call, np_, n_chains, init_mat, proposal_sd, gamma, de_noise, n_iter, warmup,
                   de_every, adapt, seed):
    """DE-MC path A: the pool is the batch-start snapshot (``R/adaptive.R:427-524``)."""
    if de_every < 1:
        raise ValueError("`de_every` must be a positive integer.")
    sizes = _batches(n_iter, int(de_every))
    nb = sizes.size
    wb = max(0, min(nb, warmup // de_every))
    wused = int(sizes[:wb].sum()) if wb > 0 else 0
    C = n_chains
    states = WelfordDiag.init(C, np_, np.asarray(proposal_sd) ** 2)
    cur_init = np.array(init_mat, dtype=np.float64, copy=True)
    cur_sd = np.array(proposal_sd, dtype=np.float64, copy=True)
    samp = max(1, n_iter - wused)
    kept = np.full((samp, C, np_), np.nan)
    acc_sum = np.zeros(C)
    iters = 0
    filled = 0
    acc_hist = np.full((C, nb), np.nan)
    disp = np.full((np_, nb), np.nan)
    acc = np.zeros(C)
    for b in range(1, nb + 1):
        bs = int(sizes[b - 1])
        draws, acc, _ = call(cur_init, cur_sd, bs, seed + b - 1, None, 1, gamma, de_noise, None)
        acc_hist[:, b - 1] = acc
        in_warm = b <= wb
        if not in_warm:
            kept[filled:filled + bs] = draws
            acc_sum += bs * acc
            iters += bs
            filled += bs
        if in_warm and adapt:
            states.update(draws)
            cur_sd = np.sqrt(np.maximum(states.variances(), 1e-12))
        cur_init = draws[-1].copy()
        disp[:, b - 1] = cur_init.std(axis=0, ddof=1) if C > 1 else np.nan
    rate = acc_sum / iters if iters > 0 else acc
    return BatchedResult(kept[:filled], rate, cur_sd, cur_init, nb, sizes, wb, wused, acc_hist,
                         seed + nb, disp_history=disp)
