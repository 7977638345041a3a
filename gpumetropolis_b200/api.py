"""User-facing sampler: ``gpu_metropolis(model, data, ..., backend="b200")``.

Restates the reference's ``gpu_metropolis`` (``R/api.R:247-599``) over the B200
session: input validation and flattening (``R/api.R:281-346``), method routing
(rwm with adaptive warmup, pt, de, mala) and the fit object.  The compute
backend is always the B200 library; ``backend`` accepts ``"b200"`` (and
``"auto"``, which resolves to it) -- the reference's ``"cpu"``/``"cuda"``/
``"vulkan"`` backends live in the reference package, not here.

Differences forced by leaving R: when ``init`` is omitted the starting values
are standard normals from a PCG64 stream seeded with ``seed`` (the reference
draws them with R's ``rnorm`` after ``set.seed(seed)``, ``R/api.R:302-307``),
and PT swap uniforms use PCG64 seeded with the reference's mix
(``R/adaptive.R:537-539``).

``surrogate=True`` (or a dict of options) adds delayed acceptance, which the
reference does not have: the exact proposals of the second half of warmup are
recorded on the device, an MLP surrogate of the log-likelihood is trained on
them on the tensor cores, and the sampling phase runs two-stage
Metropolis-Hastings (surrogate screen, exact correction), which leaves the
target posterior unchanged while evaluating only the screened proposals
exactly.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _native
from . import adaptive as AD
from .dsl import GpumModel


class GpumInputError(ValueError):
    """Invalid argument to gpu_metropolis (the reference raises an R error)."""


@dataclass
class GpumFit:
    draws: np.ndarray              # (n_iter_kept, n_chains, n_params)
    accept_rate: np.ndarray
    model: GpumModel
    n_iter: int
    n_iter_total: int
    warmup: int
    n_chains: int
    n_params: int
    backend: str
    seed: int
    method: str
    adaptation: Optional[dict] = None
    extra: dict = field(default_factory=dict)

    def __getitem__(self, name):
        return self.draws[:, :, self.model.params.index(name)]

    def __repr__(self):
        lines = ["<gpum_fit>",
                 f"  parameters  : {', '.join(self.model.params)}",
                 f"  method      : {self.method}",
                 f"  backend     : {self.backend}",
                 f"  chains      : {self.n_chains}",
                 f"  iterations  : {self.n_iter} per chain ({self.n_iter_total} raw, "
                 f"{self.warmup} {'adaptive' if self.adaptation else 'trim'} warmup discarded)",
                 f"  accept_rate : {self.accept_rate.min():.3f} to {self.accept_rate.max():.3f}"]
        for j, p in enumerate(self.model.params):
            post = self.draws[:, 0, j] if self.method == "pt" else self.draws[:, :, j]
            lines.append(f"  {p:<11} : posterior mean {post.mean():.4f} (sd {post.std(ddof=1):.4f})")
        return "\n".join(lines)


def _data_matrix(model: GpumModel, data):
    if model.n_cols == 0:
        return np.zeros((0, 0)), 0
    if data is None:
        raise GpumInputError("missing data columns: " + ", ".join(model.data))
    if isinstance(data, np.ndarray):
        mat = np.asarray(data, dtype=np.float64)
        if mat.ndim == 1:
            mat = mat[:, None]
        if mat.shape[1] != model.n_cols:
            raise GpumInputError(f"data must have {model.n_cols} columns")
        return np.ascontiguousarray(mat), mat.shape[0]
    missing = [c for c in model.data if c not in data]
    if missing:
        raise GpumInputError("missing data columns: " + ", ".join(missing))
    cols = [np.asarray(data[c], dtype=np.float64).ravel() for c in model.data]
    n = cols[0].size
    if any(c.size != n for c in cols):
        raise GpumInputError("data columns must have equal length")
    return np.ascontiguousarray(np.stack(cols, axis=1)), n


# hidden: network width (128, 256 or 512); batch: training batch (a multiple of 128); steps/lr:
# Adam steps at lr, then steps at lr/3 and lr/10; step_scale multiplies the
# adapted random-walk proposal in the two-stage phase (screening makes
# rejections cheap, so longer steps pay: Sherlock, Thiery & Golightly 2021);
# whiten: inputs whitened by the pairs' covariance.
SURROGATE_DEFAULTS = {"hidden": 128, "batch": 4096, "steps": 800, "lr": 3e-3,
                      "max_pairs": 1 << 20, "min_pairs": 2048, "seed": 1,
                      "step_scale": 1.6, "whiten": True}


class _Backend:
    """One data-resident session serving every batch of a run (the
    ``rust_call`` closure of ``R/api.R:379-393``).

    With a surrogate configuration it also drives delayed acceptance:
    recording starts once `record_at` iterations have run, the surrogate is
    trained when `da_at` iterations have run (or on ``start_da()``), and
    from then on batches run two-stage steps."""

    def __init__(self, model: GpumModel, data_mat, n_obs, rng_kind, surrogate=None):
        m = model
        self.np = m.n_params
        self.rng = rng_kind
        self.session = _native.Session(m.loglik.code, m.loglik.consts, m.prior.code,
                                       m.prior.consts, m.n_params, data_mat, m.n_cols, n_obs)
        self.cfg = surrogate
        self.consumed = 0
        self.record_at = None
        self.da_at = None
        self.recording = False
        self.net = None
        self.info = {}
        self.exact_evals = 0
        self.da_iters = 0

    def _maybe_record(self, C, n_iter):
        if self.cfg is None or self.net is not None or self.recording or self.record_at is None:
            return
        if self.consumed >= self.record_at:
            self.session.record(int(self.cfg["max_pairs"]))
            self.recording = True

    def start_da(self):
        """Train the surrogate on the recorded pairs; later batches use it."""
        if self.cfg is None or self.net is not None:
            return
        if not self.recording:
            self.info = {"used": False, "reason": "no exact pairs were recorded"}
            return
        n_rec = self.session.recorded_count()
        if n_rec < int(self.cfg["min_pairs"]):
            self.session.record(0)
            self.recording = False
            self.info = {"used": False, "reason": f"only {n_rec} recorded pairs"}
            return
        # The pairs stay on the device: split (every tenth held out), moments
        # for the normaliser, training and the held-out check in one call.
        net = _native.Surrogate(self.np, hidden=int(self.cfg["hidden"]),
                                batch=int(self.cfg["batch"]), seed=int(self.cfg["seed"]))
        steps, lr = int(self.cfg["steps"]), float(self.cfg["lr"])
        try:
            loss, fit = self.session.train_surrogate(
                net, [(steps, lr), (steps, lr / 3.0), (steps, lr / 10.0)], holdout_every=10,
                whiten=bool(self.cfg["whiten"]))
        except _native.GpumError as e:
            net.close()
            self.session.record(0)
            self.recording = False
            self.info = {"used": False, "reason": str(e)}
            return
        self.session.record(0)
        self.recording = False
        self.net = net
        self.info = {"used": True, "pairs": fit["train_pairs"] + fit["holdout_pairs"],
                     "final_loss": float(np.mean(loss[-50:])),
                     "holdout_resid_sd": fit["holdout_resid_sd"]}

    def __call__(self, init, sd, n_iter, seed, temperatures=None, proposal_mode=0, gamma=0.0,
                 de_noise=0.0, proposal_l=None, out_draws=None):
        init = np.asarray(init, dtype=np.float64)
        C = init.shape[0]
        temps = np.ones(C) if temperatures is None else np.asarray(temperatures, np.float64)
        if self.da_at is not None and self.consumed >= self.da_at:
            self.start_da()
        self._maybe_record(C, n_iter)
        if self.net is not None:
            k = float(self.cfg["step_scale"])
            if proposal_mode in (_native.MODE_RWM, _native.MODE_CHOL) and k != 1.0:
                sd = np.asarray(sd, dtype=np.float64) * k
                if proposal_l is not None:
                    proposal_l = np.asarray(proposal_l, dtype=np.float64) * k
            d, acc, last, exact = self.session.run_da(
                self.net, init, sd, temps, int(n_iter), int(seed) & 0xFFFFFFFF, proposal_mode,
                gamma, de_noise, proposal_l, rng=self.rng, out_draws=out_draws)
            self.exact_evals += int(exact.sum())
            self.da_iters += int(n_iter) * C
        else:
            d, acc, last = self.session.run(init, sd, temps, int(n_iter),
                                            int(seed) & 0xFFFFFFFF, proposal_mode, gamma,
                                            de_noise, proposal_l, rng=self.rng,
                                            out_draws=out_draws)
        self.consumed += int(n_iter)
        return d.reshape((int(n_iter), C, self.np), order="F"), acc.astype(np.float64), last

    def run_moments(self, init, sd, n_iter, seed, temperatures=None, proposal_mode=0,
                    gamma=0.0, de_noise=0.0, proposal_l=None):
        """A warmup batch that returns the moments of its draws (computed on
        the device) instead of the draws: (BatchMoments, accept rates)."""
        init = np.asarray(init, dtype=np.float64)
        C = init.shape[0]
        temps = np.ones(C) if temperatures is None else np.asarray(temperatures, np.float64)
        if self.cfg is not None and self.da_at is not None and self.consumed >= self.da_at:
            self.start_da()
        self._maybe_record(C, n_iter)
        s = self.session
        s.prepare(init, sd, temps, int(n_iter), int(seed) & 0xFFFFFFFF, proposal_mode, gamma,
                  de_noise, proposal_l, rng=self.rng)
        s.advance(int(n_iter))
        cm, c2, pm, p2 = s.draw_moments(0, int(n_iter))
        last = s.state()
        _, acc, _, _ = s.fetch(want_draws=False)
        self.consumed += int(n_iter)
        return AD.BatchMoments(int(n_iter), cm, c2, pm, p2, last), acc.astype(np.float64)

    def da_summary(self):
        out = dict(self.info)
        if self.da_iters:
            out["exact_fraction"] = self.exact_evals / self.da_iters
        return out

    def close(self):
        if self.net is not None:
            self.net.close()
        self.session.close()


def gpu_metropolis(model: GpumModel, data=None, init=None, proposal_sd=0.1, n_iter=2000,
                   n_chains=4, warmup=None, adapt=True, method="rwm", temperatures=None,
                   swap_every=None, gamma=None, de_noise=1e-3, de_every=None, de_sync=False,
                   seed=1, backend="b200", rng="triple32", surrogate=None, swap_on_device=False,
                   ladder_len=None) -> GpumFit:
    """Run the batched Metropolis sampler on the B200 backend (``R/api.R:247-599``).

    ``surrogate``: None/False (exact Metropolis, the reference's behaviour),
    True, or a dict overriding ``SURROGATE_DEFAULTS`` -- delayed acceptance
    in the sampling phase (rwm, pt, de, mala; needs warmup > 0).  With mala
    the two-stage phase proposes Langevin moves whose drift is the
    surrogate's log-posterior gradient, so it evaluates no exact gradient.

    ``swap_on_device`` (pt): exchanges run on the GPU after every
    ``swap_every`` iterations inside one run instead of between host batches;
    the chains form ladders of ``ladder_len`` consecutive chains (default: one
    ladder of all chains, as the reference), temperatures repeating per
    ladder."""
    if not isinstance(model, GpumModel):
        raise GpumInputError("`model` must be a gpum_model from gpum_model().")
    if backend not in ("b200", "auto"):
        raise GpumInputError(f"backend '{backend}' is not available in this build. "
                             "Available: b200")
    if method not in ("rwm", "pt", "de", "mala"):
        raise GpumInputError("`method` must be one of rwm, pt, de, mala")
    rng_kind = {"triple32": _native.RNG_TRIPLE32, "philox": _native.RNG_PHILOX}[rng]
    data_mat, n_obs = _data_matrix(model, data)
    npar = model.n_params
    if init is None:
        n_chains = int(n_chains)
        g = np.random.Generator(np.random.PCG64(int(seed)))
        init_mat = g.standard_normal((n_chains, npar))
    else:
        init_mat = np.asarray(init, dtype=np.float64)
        if init_mat.ndim == 1:
            init_mat = init_mat.reshape(-1, 1) if npar == 1 else init_mat.reshape(1, -1)
        if init_mat.shape[1] != npar:
            raise GpumInputError(f"`init` must have one column per parameter ({npar}).")
        n_chains = init_mat.shape[0]
    n_iter = int(n_iter)
    warmup_auto = isinstance(warmup, str) and warmup == "auto"
    if warmup is None or warmup_auto:
        warmup = n_iter // 2
    warmup = int(warmup)
    if warmup < 0 or warmup >= n_iter:
        raise GpumInputError("`warmup` must be a non-negative integer strictly less than "
                             "`n_iter`.")
    psd = np.asarray(proposal_sd, dtype=np.float64)
    if psd.ndim == 2:
        if psd.shape != (n_chains, npar):
            raise GpumInputError(f"`proposal_sd` matrix must be `n_chains` by `n_params` "
                                 f"({n_chains} by {npar}).")
        sd_mat = psd.copy()
    else:
        sd_mat = np.tile(np.resize(psd.ravel(), npar), (n_chains, 1))
    if not np.all(np.isfinite(sd_mat)) or np.any(sd_mat <= 0):
        raise GpumInputError("`proposal_sd` must be positive and finite.")

    C = n_chains
    temps = None
    if method == "pt":
        ladder_len = C if ladder_len is None else int(ladder_len)
        if swap_on_device and (ladder_len < 2 or C % ladder_len != 0):
            raise GpumInputError("`ladder_len` must be at least 2 and divide `n_chains`.")
        if temperatures is None:
            temps = (np.tile(AD.pt_default_ladder(ladder_len), C // ladder_len)
                     if swap_on_device else AD.pt_default_ladder(C))
        else:
            temps = np.asarray(temperatures, dtype=np.float64).ravel()
            if temps.size != C:
                raise GpumInputError("`temperatures` must have one value per chain.")
            if not np.all(np.isfinite(temps)) or np.any(temps <= 0):
                raise GpumInputError("`temperatures` must be positive and finite.")
        if swap_every is None:
            swap_every = max(C, 10)
    if method == "de":
        if C < 4:
            raise GpumInputError('`method = "de"` needs at least 4 chains; the proposal draws '
                                 "a distinct pair of other chains for each difference vector. "
                                 "Increase `n_chains`.")
        gamma = 2.38 / np.sqrt(2 * npar) if gamma is None else float(gamma)
        if not np.isfinite(gamma) or gamma <= 0:
            raise GpumInputError("`gamma` must be positive and finite.")
        de_noise = float(de_noise)
        if not np.isfinite(de_noise) or de_noise < 0:
            raise GpumInputError("`de_noise` must be non-negative and finite.")
        if de_every is None:
            de_every = max(C, 10)
        if de_sync and surrogate is not None and surrogate is not False:
            raise GpumInputError("`surrogate` is not available with `de_sync = TRUE`.")

    scfg = None
    if surrogate is not None and surrogate is not False:
        if warmup <= 0:
            raise GpumInputError("`surrogate` needs warmup > 0: its training pairs come from "
                                 "the warmup's exact evaluations.")
        scfg = dict(SURROGATE_DEFAULTS)
        if isinstance(surrogate, dict):
            unknown = set(surrogate) - set(scfg)
            if unknown:
                raise GpumInputError("unknown surrogate option(s): " + ", ".join(sorted(unknown)))
            scfg.update(surrogate)
        elif surrogate is not True:
            raise GpumInputError("`surrogate` must be None, True or a dict of options.")

    call = _Backend(model, data_mat, n_obs, rng_kind, scfg)
    if method == "pt" and swap_on_device:
        if scfg is not None:  # exact pairs from the second half of warmup
            call.record_at = warmup // 2
            call.da_at = warmup
        try:
            fit = _pt_device(model, call, npar, n_chains, init_mat, sd_mat, temps, n_iter,
                             warmup, int(swap_every), ladder_len, bool(adapt), int(seed),
                             backend)
            if scfg is not None:
                fit.extra["surrogate"] = call.da_summary()
            return fit
        finally:
            call.close()
    if method == "de" and de_sync:
        # Path B (R/api.R:464-497): per-generation DE over the whole run,
        # trim-only warmup, proposal_sd the fixed jitter base.
        try:
            d, acc, _ = call.session.run_de_sync(init_mat, sd_mat, n_iter, int(seed), gamma,
                                                 de_noise, rng=rng_kind)
        finally:
            call.close()
        draws = d.reshape((n_iter, n_chains, npar), order="F")
        return GpumFit(draws[warmup:], acc.astype(np.float64), model, n_iter - warmup, n_iter,
                       warmup, n_chains, npar, backend, int(seed), "de", None,
                       {"gamma": gamma, "de_noise": de_noise, "de_sync": True})
    if scfg is not None:
        every = {"pt": swap_every, "de": de_every}.get(method)
        w_eff = warmup if every is None else max(0, min(-(-n_iter // every), warmup // every)) * every
        call.record_at = w_eff // 2
        call.da_at = w_eff if method != "rwm" else None
    try:
        fit = _route(model, call, method, npar, n_chains, init_mat, sd_mat, n_iter, warmup,
                     warmup_auto, adapt, temps, swap_every, gamma, de_noise, de_every,
                     int(seed), backend)
        if scfg is not None:
            fit.extra["surrogate"] = call.da_summary()
        return fit
    finally:
        call.close()


def _pt_device(model, call, npar, C, init_mat, sd_mat, temps, n_iter, warmup, swap_every,
               ladder_len, adapt, seed, backend):
    """Parallel tempering with the exchanges on the device: adaptive warmup
    batches (per-chain Robbins-Monro scales and variances as in the host
    orchestration, R/adaptive.R:330-355, from device moments) with exchanges
    inside each batch, then one sampling run with an exchange every
    ``swap_every`` iterations (two-stage when the backend has a surrogate
    schedule: trained on the warmup's exact pairs, exchanges on the exact
    log posteriors)."""
    s = call.session
    s.set_exchange(ladder_len, swap_every)
    cur, sd = np.array(init_mat, dtype=np.float64), np.array(sd_mat, dtype=np.float64)
    scales = np.ones(C)
    sizes = np.zeros(0, np.int64)
    if warmup > 0:
        nb = min(40, max(10, warmup // 50), warmup) if adapt else 1
        sizes = np.full(nb, warmup // nb, dtype=np.int64)
        sizes[-1] += warmup - sizes.sum()
        states = AD.WelfordDiag.init(C, npar, sd ** 2)
        for b, n in enumerate(sizes, start=1):
            mo, acc = call.run_moments(cur, sd, int(n), seed + b - 1, temps, 0)
            cur = mo.last
            if adapt:
                states.merge(mo.n, mo.chain_mean, mo.chain_m2)
                scales = AD.robbins_monro_scale(scales, acc, b, npar)
                sd = scales[:, None] * np.sqrt(np.maximum(states.variances(), 1e-12))
    samp = n_iter - warmup
    d, acc, _ = call(cur, sd, samp, seed + sizes.size, temps, 0)
    att, ok, n_ex = s.exchange_stats()
    s.set_exchange(0)
    with np.errstate(invalid="ignore", divide="ignore"):
        rate = np.where(att > 0, ok / np.maximum(att, 1), np.nan)
    return GpumFit(d, acc, model, samp, n_iter, warmup, C, npar, backend, seed, "pt",
                   {"final_proposal_sd": sd, "final_scales": scales,
                    "n_batches": int(sizes.size), "batch_sizes": sizes} if adapt else None,
                   {"temperatures": temps, "swap_every": swap_every, "ladder_len": ladder_len,
                    "swap_on_device": True, "exchanges": n_ex,
                    "exchange_rate": rate[: C - 1]})


def _route(model, call, method, npar, C, init_mat, sd_mat, n_iter, warmup, warmup_auto, adapt,
           temps, swap_every, gamma, de_noise, de_every, seed, backend):
    if method == "pt":
        r = AD.pt_orchestrate(call, npar, C, init_mat, sd_mat, temps, n_iter, warmup,
                              int(swap_every), bool(adapt), seed)
        return GpumFit(r.draws, r.accept_rate, model, r.draws.shape[0],
                       r.warmup_used + r.draws.shape[0], r.warmup_used, C, npar, backend, seed,
                       "pt", {"final_proposal_sd": r.final_proposal_sd,
                              "final_scales": r.final_scales, "n_batches": r.n_batches,
                              "batch_sizes": r.batch_sizes, "accept_history": r.accept_history,
                              "swap_history": r.swap_history},
                       {"temperatures": temps, "swap_every": int(swap_every)})
    if method == "de":
        g, dn = gamma, de_noise
        r = AD.de_orchestrate(call, npar, C, init_mat, sd_mat, g, dn, n_iter, warmup,
                              int(de_every), bool(adapt), seed)
        return GpumFit(r.draws, r.accept_rate, model, r.draws.shape[0],
                       r.warmup_used + r.draws.shape[0], r.warmup_used, C, npar, backend, seed,
                       "de", {"final_proposal_sd": r.final_proposal_sd,
                              "n_batches": r.n_batches, "batch_sizes": r.batch_sizes,
                              "accept_history": r.accept_history,
                              "disp_history": r.disp_history},
                       {"gamma": g, "de_noise": dn, "de_every": int(de_every)})
    langevin = method == "mala"
    if adapt and warmup > 0:
        am = AD.am_orchestrate_warmup(call, npar, C, init_mat, sd_mat, warmup, seed,
                                      auto_stop=warmup_auto, langevin=langevin)
        call.start_da()
        samp = max(1, n_iter - am.warmup_used)
        use_L = npar > 1 and am.final_L is not None
        draws, acc, _ = call(am.final_init, am.final_proposal_sd, samp, am.seed_next, None,
                             3 if langevin else (2 if use_L else 0), 0.0, 0.0,
                             am.final_L if use_L else None)
        return GpumFit(draws, acc, model, samp, am.warmup_used + samp, am.warmup_used, C, npar,
                       backend, seed, method,
                       {"final_proposal_sd": am.final_proposal_sd,
                        "final_scales": am.final_scales, "n_batches": am.n_batches,
                        "batch_sizes": am.batch_sizes, "accept_history": am.accept_history})
    if call.cfg is not None:
        # Delayed acceptance without adaptation: exact warmup in two halves
        # (the second recorded), then two-stage sampling from its last state.
        h1 = warmup // 2
        cur = init_mat
        if h1 > 0:
            d1, _, _ = call(cur, sd_mat, h1, seed, None, 0)
            cur = d1[-1]
        d2, _, _ = call(cur, sd_mat, warmup - h1, seed + 1, None, 0)
        call.start_da()
        draws, acc, _ = call(d2[-1], sd_mat, n_iter - warmup, seed + 2, None, 0)
        return GpumFit(draws, acc, model, n_iter - warmup, n_iter, warmup, C, npar, backend,
                       seed, method)
    draws, acc, _ = call(init_mat, sd_mat, n_iter, seed, None, 3 if langevin else 0)
    kept = draws[warmup:] if warmup > 0 else draws
    return GpumFit(kept, acc, model, n_iter - warmup, n_iter, warmup, C, npar, backend, seed,
                   method)


# ------------------------------------------------------------ evidence (TI)
@dataclass
class GpumEvidence:
    log_evidence: float
    betas: np.ndarray
    expected_loglik: np.ndarray
    n_rungs: int
    power: float
    accept_rate: np.ndarray = field(default_factory=lambda: np.zeros(0))

    def __repr__(self):
        return (f"<gpum_evidence>\n  log marginal likelihood {self.log_evidence:.3f}\n"
                f"  thermodynamic integration over {self.n_rungs} rungs (power {self.power:g})")


@dataclass
class GpumBayesFactor:
    bf10: float
    log_bf10: float
    log_evidence1: float
    log_evidence0: float
    interpretation: str


def gpum_evidence(model: GpumModel, data=None, n_rungs=24, power=5, n_iter=4000, n_chains=8,
                  warmup=None, seed=1, backend="b200", max_points_per_rung=20000,
                  rng="triple32") -> GpumEvidence:
    """Log marginal likelihood by thermodynamic integration (``R/bayes.R:279-338``).

    Power posteriors ``p_beta ∝ p(y|θ)^beta p(θ)`` on the grid
    ``beta = (k / n_rungs)^power``; the log evidence is the trapezoidal
    integral over beta of E_beta[log p(y|θ)] (Gelman & Meng 1998; Friel &
    Pettitt 2008).  The reference samples the rungs one after another with a
    "power model" each; here every rung is a group of ``n_chains`` chains of
    one batched run on the device (per-chain likelihood powers), with
    adaptive random-walk proposals fitted per chain (a DE pool or a pooled
    covariance would mix rungs whose targets differ).  E_beta[log p(y|θ)] is
    the mean of ``loglik_batch`` over each rung's kept draws."""
    if not isinstance(model, GpumModel):
        raise GpumInputError("`model` must be a gpum_model from gpum_model().")
    if backend not in ("b200", "auto"):
        raise GpumInputError(f"backend '{backend}' is not available in this build. "
                             "Available: b200")
    if model.prior.code.size == 0:
        raise GpumInputError("Evidence requires a proper prior; this model has none. The "
                             "marginal likelihood is undefined for a flat or absent prior.")
    n_rungs, n_chains, n_iter = int(n_rungs), int(n_chains), int(n_iter)
    if n_rungs < 1 or n_chains < 1:
        raise GpumInputError("`n_rungs` and `n_chains` must be positive.")
    warmup = n_iter // 2 if warmup is None else int(warmup)
    if warmup < 1 or warmup >= n_iter:
        raise GpumInputError("`warmup` must be in [1, n_iter).")
    rng_kind = {"triple32": _native.RNG_TRIPLE32, "philox": _native.RNG_PHILOX}[rng]
    data_mat, n_obs = _data_matrix(model, data)
    npar = model.n_params
    betas = (np.arange(n_rungs + 1) / n_rungs) ** float(power)
    C = (n_rungs + 1) * n_chains
    beta_c = np.repeat(betas, n_chains)              # chain r*n_chains + k is on rung r
    g = np.random.Generator(np.random.PCG64(int(seed)))
    init = g.standard_normal((C, npar))
    call = _Backend(model, data_mat, n_obs, rng_kind)
    try:
        s = call.session
        s.set_likelihood_powers(beta_c)
        ones = np.ones(C)
        # Warmup: batches of diagonal RWM, per-chain Welford covariance and
        # Robbins-Monro scale (R/adaptive.R:101-254 without the pooled
        # covariance), statistics restarted at the half.
        n_batches = min(40, max(10, warmup // 50), warmup)
        sizes = np.full(n_batches, warmup // n_batches)
        sizes[-1] += warmup - sizes.sum()
        states = AD.Welford.init(C, npar, np.full(npar, 0.01))
        scale0 = 2.38 / np.sqrt(npar)
        scales = np.full(C, scale0)
        sd = np.full((C, npar), 0.1)
        target = AD.target_accept(npar)
        cur = init
        for b in range(1, n_batches + 1):
            d, acc, _ = s.run(cur, sd, ones, int(sizes[b - 1]), int(seed) + b - 1, 0, rng=rng_kind)
            d = d.reshape((int(sizes[b - 1]), C, npar), order="F")
            states.update(d)
            bi = b - n_batches // 2 if b > n_batches // 2 else b
            scales = AD.robbins_monro_scale(scales, acc, bi, npar, target)
            cur = d[-1].copy()
            if b == n_batches // 2:
                diag = np.maximum(np.diagonal(states.covariance(), axis1=1, axis2=2), 1e-12)
                states = AD.Welford.init(C, npar, diag.mean(axis=0))
            cov = states.covariance()
            sd = scales[:, None] * np.sqrt(np.maximum(np.diagonal(cov, axis1=1, axis2=2), 1e-12))
        # Sampling with per-chain Cholesky factors of the warmup covariance.
        samp = n_iter - warmup
        if npar > 1:
            cov = states.covariance()
            L = np.stack([scales[c] * AD.cholesky_reg(cov[c]) for c in range(C)])
            d, acc, _ = s.run(cur, sd, ones, samp, int(seed) + n_batches, 2, proposal_l=L,
                              rng=rng_kind)
        else:
            d, acc, _ = s.run(cur, sd, ones, samp, int(seed) + n_batches, 0, rng=rng_kind)
        d = d.reshape((samp, C, npar), order="F")
        s.set_likelihood_powers(None)
        expected = np.empty(n_rungs + 1)
        for r in range(n_rungs + 1):
            pts = d[:, r * n_chains:(r + 1) * n_chains, :].reshape(-1, npar)
            if pts.shape[0] > max_points_per_rung:
                pts = pts[np.linspace(0, pts.shape[0] - 1, max_points_per_rung).astype(int)]
            expected[r] = float(np.mean(s.loglik_batch(pts)))
    finally:
        call.close()
    log_ev = float(np.sum(0.5 * (expected[1:] + expected[:-1]) * np.diff(betas)))
    return GpumEvidence(log_ev, betas, expected, n_rungs, float(power), acc.astype(np.float64))


def _jeffreys(b: float) -> str:
    if b < 1:
        return f"favours model0 ({_jeffreys(1 / b)} reversed)"
    if b < 3:
        return "barely worth mention"
    if b < 10:
        return "substantial"
    if b < 30:
        return "strong"
    if b < 100:
        return "very strong"
    return "decisive"


def gpum_bayes_factor(model1: GpumModel, model0: GpumModel, data=None,
                      **kw) -> GpumBayesFactor:
    """B_10 = p(y | model1) / p(y | model0) by thermodynamic integration
    (``R/bayes.R:374-393``); keyword arguments go to :func:`gpum_evidence`."""
    e1 = gpum_evidence(model1, data, **kw)
    e0 = gpum_evidence(model0, data, **kw)
    log_bf = e1.log_evidence - e0.log_evidence
    bf = float(np.exp(log_bf))
    return GpumBayesFactor(bf, log_bf, e1.log_evidence, e0.log_evidence, _jeffreys(bf))
