#!/usr/bin/env python
"""Throughput of the B200 sampler hot path on the logistic-regression workload.

Workload (the config the headline metric is quoted on that fits one GPU):
logistic regression, N = 2^20 observations, 16 N(0,1) covariates plus an
intercept (17 parameters, 17 data columns), N(0, 10^2) priors, 1,024 chains,
plain exact random-walk Metropolis with FP32 per-observation bytecode and
compensated sums.  One *step* is one Metropolis iteration of all 1,024 chains
over all N observations (1.07e9 chain-observation evaluations plus the
accept/propose step).

* ``value``: chain-obs/s with the data and chain state resident in HBM,
  device-timed with CUDA events around each step on the session's stream;
  L2 is flushed (256 MiB write) before every timed step because the data
  (71 MB in f32) fits in the 126 MB L2.
* ``e2e``: the same metric through the reference-facing C ABI
  (``gpum_b200_run``) with host buffers: data upload + layout conversion,
  K iterations, draws copied back, wall-clock.
* ``roofline``: the iteration kernel against the pipe that bounds it.  With
  the model's linear predictor on the tensor cores (gm_iter_value_tc) that is
  the special-function (XU) pipe: two MUFU operations (ex2, rcp) per
  chain-observation in the softplus; the tensor-core, FP32-equivalent and HBM
  views of the same launch are sub-objects.
* ``cpu_baseline``: the oracle port of the reference CPU backend (bytecode ->
  C -> gcc JIT, OpenMP over chains) on this host, a bounded sample.
* ``delayed_acceptance``: the ESS/s half of the metric on the same workload --
  adaptive warmup (exact, its second half recorded as training pairs), the
  surrogate trained on the GPU, then the same number of sampling iterations
  with plain exact MH and with surrogate delayed acceptance from the same
  start (5,000 iterations each, the configuration's length); multi-chain ESS
  per parameter (min and mean over the 17) per second of sampling, also
  with the surrogate's training time added to the two-stage run, and the
  posterior means' agreement in MCSE units.
* ``logp_rel_err``: the log posterior the sampler holds for 32 chains'
  final states against the f64 oracle at the same states (untimed).
* ``configs``: the Poisson (MALA), mixture (512 PT ladders with device
  exchanges), Student-t (DE) and Student-t (MALA) configurations at full
  size: ms per iteration, chain-obs/s, FP32 and MUFU fractions, and each
  one's ``logp_rel_err``.
* ``pt_da``: exact vs surrogate delayed-acceptance ESS/s for PT on the
  mixture configuration, with and without the training time.

``--impl reference`` times that CPU implementation alone as the reference arm.
``--configs`` prints only the configuration timings, one JSON line each
(``--configs-obs-shift`` shrinks them for profiler captures); ``--pt-da``
prints only the PT + delayed-acceptance leg.
Multi-GPU (torchrun): one independent replica per GPU (the chains shard with
no collective), weak scaling, max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("ESS/s on 1 B200, surrogate-DA vs plain exact MH at <=1e-6 rel logp err; "
          "chain-obs/s")
UNIT = "chain-obs/s"
FLOP_PER_CHAIN_OBS = 34.0   # the logistic term's 17-term linear predictor (FMA = 2)
MUFU_PER_CHAIN_OBS = 2.0    # ex2 and rcp of the softplus
TC_COLS = 17                # product columns of the tensor-core kernel (16 + ones)
PACKED_ROW_BYTES = (2 * 24 + 1) * 4  # hi | lo (17 columns padded to 24) | y, f32
ROW_BYTES = 17 * 4          # one f32 observation row


def _args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--n-obs", type=int, default=1 << 20)
    p.add_argument("--chains", type=int, default=1024)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-interp", action="store_true")
    p.add_argument("--engine", type=int, default=2, help="0 interpreter, 1 compiled, 2 auto")
    p.add_argument("--no-da", action="store_true")
    p.add_argument("--no-logp", action="store_true")
    p.add_argument("--no-configs", action="store_true",
                   help="leave the Poisson / mixture / Student-t timings out of the line")
    p.add_argument("--no-pt-da", action="store_true",
                   help="leave the mixture PT + delayed-acceptance leg out of the line")
    p.add_argument("--da-warmup", type=int, default=1000)
    p.add_argument("--da-step-scale", type=float, default=None,
                   help="two-stage proposal scale (default: the library's)")
    p.add_argument("--da-train-steps", type=int, default=None,
                   help="surrogate steps per learning-rate stage (default: the library's)")
    p.add_argument("--da-iters", type=int, default=5000,
                   help="sampling iterations of each delayed-acceptance leg (the logistic "
                        "configuration's 5,000)")
    p.add_argument("--configs", action="store_true",
                   help="instead of the headline line: time the Poisson (MALA), mixture (PT "
                        "ladders) and Student-t (DE) configurations at full size, one JSON "
                        "line each")
    p.add_argument("--pt-da", action="store_true",
                   help="instead of the headline line: exact vs surrogate delayed-acceptance "
                        "ESS/s on the mixture configuration (512 ladders of 16 temperatures, "
                        "device exchanges), one JSON line")
    p.add_argument("--pt-da-warmup", type=int, default=300)
    p.add_argument("--c5-da", action="store_true",
                   help="instead of the headline line: exact vs delayed-acceptance ESS/s for "
                        "DE and the Langevin move on the Student-t configuration at full size "
                        "with the 65-512-512-1 surrogate (minutes), one JSON line")
    p.add_argument("--profile-da", action="store_true",
                   help="profiler target: a short warmup, surrogate training inside the "
                        "NVTX range 'training' and 48 two-stage iterations inside "
                        "'da_sampling' (logistic configuration)")
    p.add_argument("--c5-warmup", type=int, default=128)
    p.add_argument("--c5-iters", type=int, default=40)
    p.add_argument("--pt-da-iters", type=int, default=400)
    p.add_argument("--configs-obs-shift", type=int, default=0,
                   help="with --configs: divide each configuration's observation count by "
                        "2^S (small cases for profiler captures)")
    p.add_argument("--configs-only", default="poisson,mixture,student_t,student_t_mala",
                   help="with --configs: comma-separated configurations to run "
                        "(student_t_mala: the Student-t configuration with MALA)")
    return p.parse_args()


def _pow2(n):
    """n as 2^k when it is a power of two (the configurations' sizes)."""
    return f"2^{n.bit_length() - 1}" if n > 0 and n & (n - 1) == 0 else str(n)


def _workload(n_obs):
    from gpumetropolis_b200 import workloads as W
    return W.make("logistic", n_obs=n_obs)


def _init(w, C, seed=0):
    rng = np.random.default_rng(seed)
    m = w.model
    init = w.truth["beta"] + rng.normal(0, 0.01, (C, m.n_params))
    sd = np.full((C, m.n_params), 0.0015)
    return init, sd, np.ones(C)


def _cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_sample(w, seconds, chains_cap):
    """Time the oracle port (JIT'd data term, OpenMP over chains) on a bounded
    sample of the workload: all N observations, one iteration of a number of
    chains sized to about `seconds` of work.  Every (chain, observation)
    evaluation counts, the start-state evaluation included."""
    from oracle import cjit
    from oracle import oracle as O
    m = w.model
    cores = _cpu_cores()
    fn = cjit.compile_loglik(m.loglik.code, m.loglik.consts)

    def once(C, n_iter):
        init, sd, temps = _init(w, C, seed=1)
        t = time.perf_counter()
        O.run(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, m.n_params,
              w.data, m.n_cols, w.n_obs, init, sd, temps, n_iter, 1, 0, jit=fn,
              n_threads=cores)
        return time.perf_counter() - t, C * (n_iter + 1) * w.n_obs

    dt, work = once(cores, 0)
    rate = work / dt
    C = int(max(cores, min(chains_cap, round(rate * seconds / (2 * w.n_obs)))))
    C = max(cores, (C // cores) * cores)
    dt, work = once(C, 1)
    return {"value": work / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{C} chains x 1 iteration (+ start evaluation) x {w.n_obs} obs, "
                      f"{work:.3g} chain-obs in {dt:.1f} s; oracle port of cpu_native::run "
                      "with the bytecode->C gcc JIT, OpenMP over chains"}


class Clocks:
    """nvidia-smi sampled every 100 ms; the summary keeps the samples whose
    timestamps fall inside the marked (timed) window."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.t0 = self.t1 = None

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        import datetime
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                ts = None
            self.rows.append((ts, f[1:]))

    def summary(self):
        rows = getattr(self, "rows", [])
        window = "timed region"
        if self.t0 is not None and self.t1 is not None:
            inside = [r for ts, r in rows if ts is not None and self.t0 - 0.05 <= ts <= self.t1 + 0.05]
        else:
            inside = []
        if not inside:
            inside = [r for _, r in rows]
            window = "whole sampler lifetime (no sample fell inside the timed region)"
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in inside if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in inside if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in inside for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(inside), "window": window}


def _pinned_f32(n):
    """A float32 host array of n values in pinned (page-locked, pre-faulted)
    memory: the draws of a timed sampling call land there, so the timing holds
    no first-touch page faults."""
    import torch
    return torch.empty(max(n, 1), dtype=torch.float32, pin_memory=True).numpy()


def _acov_mean_gpu(xc):
    """diagnostics.acov_chain_mean with the FFTs on the GPU (torch, f64):
    thousands of chains x thousands of iterations per parameter."""
    import torch
    n = xc.shape[0]
    L = 1 << int(np.ceil(np.log2(2 * n)))
    t = torch.from_numpy(np.ascontiguousarray(xc)).cuda()
    f = torch.fft.rfft(t, L, dim=0)
    acov = torch.fft.irfft(f * f.conj(), L, dim=0)[:n] / n
    out = acov.mean(dim=1).cpu().numpy()
    del t, f, acov
    return out


def _ess_all(d):
    """Multi-chain ESS per parameter of an (n_iter, C, np) array."""
    from gpumetropolis_b200.diagnostics import ess_pooled
    return np.array([ess_pooled(d[:, :, j], acov_mean_fn=_acov_mean_gpu)
                     for j in range(d.shape[2])])


def _oracle_logpost(w, states):
    """The oracle's log posterior at each state: the data term through the
    compiled f64 evaluator (bitwise the interpreter oracle's value) plus the
    f64 prior, on all host cores."""
    from oracle import cjit
    from oracle import oracle as O
    m = w.model
    fn = cjit.compile_loglik(m.loglik.code, m.loglik.consts)
    n = states.shape[0]
    _, _, last = O.run(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                       m.n_params, w.data, m.n_cols, w.n_obs, states, np.ones_like(states),
                       np.ones(n), 0, 1, 0, jit=fn, n_threads=_cpu_cores())
    return last


def logp_check(sess, w, n=32):
    """Largest relative error, over the first `n` chains of the session's
    last run, of the log posterior the sampler holds for its current state
    (FP32 per-observation terms, FP64 sums, the value its accept decisions
    used) against the f64 oracle at the same state.  Outside any timed
    region."""
    states = sess.state()[:n]
    _, _, cur, _ = sess.fetch(want_draws=False)
    ref = _oracle_logpost(w, states)
    return float(np.max(np.abs(cur[:n] - ref) / np.abs(ref)))


def da_measure(w, C, n_warm, n_samp, seed=11, step_scale=None, train_steps=None):
    """Exact MH vs surrogate delayed acceptance, ESS per second of sampling.

    Runs through the production driver (gpumetropolis_b200.api._Backend): the
    same pair recording, training and two-stage runs as
    gpu_metropolis(surrogate=True)."""
    from gpumetropolis_b200 import _native, api
    from gpumetropolis_b200 import adaptive as AD
    from gpumetropolis_b200.diagnostics import ess_pooled
    m = w.model
    npar = m.n_params
    cfg = dict(api.SURROGATE_DEFAULTS)
    if step_scale:
        cfg["step_scale"] = float(step_scale)
    if train_steps:
        cfg["steps"] = int(train_steps)
    call = api._Backend(m, w.data, w.n_obs, _native.RNG_PHILOX, cfg)
    try:
        call.record_at = n_warm // 2
        rng = np.random.default_rng(seed)
        init = w.truth["beta"] + rng.normal(0, 0.05, (C, npar))
        sd0 = np.full((C, npar), 0.01)
        t = time.perf_counter()
        am = AD.am_orchestrate_warmup(call, npar, C, init, sd0, n_warm, seed)
        t_warm = time.perf_counter() - t
        t = time.perf_counter()
        call.start_da()
        t_train = time.perf_counter() - t
        if call.net is None:
            return {"used": False, "reason": call.info.get("reason")}
        L = am.final_L
        mode = _native.MODE_CHOL if L is not None else _native.MODE_RWM
        ones = np.ones(C)

        def timed(f):
            call.session.sync()
            t0 = time.perf_counter()
            r = f()
            return r, time.perf_counter() - t0

        buf_ex, buf_da = _pinned_f32(n_samp * C * npar), _pinned_f32(n_samp * C * npar)
        (d_ex, acc_ex, _), t_ex = timed(lambda: call.session.run(
            am.final_init, am.final_proposal_sd, ones, n_samp, seed + 1, mode, 0.0, 0.0, L,
            rng=_native.RNG_PHILOX, out_draws=buf_ex))
        e0 = call.exact_evals
        (d_da, acc_da, _), t_da = timed(lambda: call(
            am.final_init, am.final_proposal_sd, n_samp, seed + 2, None, mode, 0.0, 0.0, L,
            out_draws=buf_da))
        exact_frac = (call.exact_evals - e0) / (n_samp * C)
        d_ex = d_ex.reshape((n_samp, C, npar), order="F")
        d_da = np.asarray(d_da)
        e_ex, e_da = _ess_all(d_ex), _ess_all(d_da)
        sd_ex = np.array([d_ex[:, :, j].std(dtype=np.float64) for j in range(npar)])
        sd_da = np.array([d_da[:, :, j].std(dtype=np.float64) for j in range(npar)])
        mu_ex = np.array([d_ex[:, :, j].mean(dtype=np.float64) for j in range(npar)])
        mu_da = np.array([d_da[:, :, j].mean(dtype=np.float64) for j in range(npar)])
        mc_ex, mc_da = sd_ex / np.sqrt(e_ex), sd_da / np.sqrt(e_da)
        z = np.abs(mu_ex - mu_da) / np.sqrt(mc_ex**2 + mc_da**2)
        r_ex, r_da = e_ex.min() / t_ex, e_da.min() / t_da
        r_da_t = e_da.min() / (t_da + t_train)
        return {
            "used": True, "n_chains": C, "warmup_iters": n_warm, "sampling_iters": n_samp,
            "proposal": "cholesky rwm (adapted)" if L is not None else "diagonal rwm",
            "step_scale": cfg["step_scale"], "warmup_s": round(t_warm, 3),
            "train_s": round(t_train, 3), "surrogate": call.da_summary(),
            "exact": {"seconds": round(t_ex, 4), "accept": float(np.mean(acc_ex)),
                      "ess_min": float(e_ex.min()), "ess_mean": float(e_ex.mean()),
                      "ess_per_s_min": r_ex, "ess_per_s_mean": float(e_ex.mean() / t_ex)},
            "da": {"seconds": round(t_da, 4), "accept": float(np.mean(acc_da)),
                   "exact_fraction": exact_frac,
                   "stage2_accept": float(np.mean(acc_da)) / max(exact_frac, 1e-12),
                   "ess_min": float(e_da.min()), "ess_mean": float(e_da.mean()),
                   "ess_per_s_min": r_da, "ess_per_s_mean": float(e_da.mean() / t_da)},
            "gain_ess_per_s_min": r_da / r_ex,
            "gain_ess_per_s_mean": float((e_da.mean() / t_da) / (e_ex.mean() / t_ex)),
            "gain_ess_per_s_min_with_training": r_da_t / r_ex,
            "gain_ess_per_s_mean_with_training":
                float((e_da.mean() / (t_da + t_train)) / (e_ex.mean() / t_ex)),
            "gain_ess_per_exact_eval_min": float((e_da.min() / max(exact_frac, 1e-12))
                                                 / e_ex.min()),
            "posterior_mean_max_z": float(z.max()),
            "ess": "multi-chain (chain-averaged autocovariance + between-chain variance, "
                   "Geyer initial monotone sequence) per parameter over all chains",
            "with_training": "two-stage seconds + surrogate training seconds (train_s) "
                             "against the exact sampler's seconds; warmup is common to both",
            "draws_buffers": "pinned host memory allocated before the timed calls",
            "timing": "wall seconds of each blocking sampling call (draws copied back in both, "
                      "into pinned buffers allocated before the calls)",
        }
    finally:
        call.close()


def _traffic_per_launch(profile):
    """dram read+write bytes of one iteration launch from a committed ncu
    summary under profiles/ (its line `dram_bytes_per_launch: X`)."""
    path = os.path.join(ROOT, "profiles", profile)
    try:
        for line in open(path):
            cell = line.strip().strip("|").strip()
            if cell.startswith("dram_bytes_per_launch:"):
                return float(cell.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def run_b200(a):
    import torch
    import torch.distributed as dist

    from gpumetropolis_b200 import replicas as R
    rank, world, local = R.rank_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    from gpumetropolis_b200 import _native
    from gpumetropolis_b200.build import build
    build()
    if not _native.available():
        raise SystemExit("gpum_b200: no usable sm_100 device")

    w = _workload(a.n_obs)
    m = w.model
    C, N = a.chains, w.n_obs
    init, sd, temps = _init(w, C, seed=rank)
    K, Wm = a.steps, max(3, a.warmup)

    sess = _native.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                           m.n_params, w.data, m.n_cols, w.n_obs, engine=a.engine)
    engine = {0: "interpreter", 1: "compiled"}[sess.engine]
    tensor_cores = sess.tensor_cores
    sess.prepare(init, sd, temps, Wm + K, R.replica_seed(1, rank), 0, rng=_native.RNG_PHILOX)
    sess.advance(Wm)
    sess.sync()
    stream = torch.cuda.ExternalStream(sess.stream, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = sess.launches
    with Clocks(local) as clk:
        time.sleep(0.5)  # let the sampler start before the timed region
        clk.mark_start()
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            for k in range(K):
                flush.zero_()
                starts[k].record(stream)
                sess.advance(1)
                ends[k].record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        clk.mark_end()
    launches = sess.launches - l0
    step_ms = np.array([s.elapsed_time(e) for s, e in zip(starts, ends)])
    dev_ms = float(step_ms.sum())
    if world > 1:
        dev_ms = R.max_over_ranks(dev_ms, device=dev)
        dist.barrier()
    _, acc, _, _ = sess.fetch(want_draws=False)
    value = R.whole_job_rate(K * C * N, world, dev_ms / 1e3)
    ms_step = dev_ms / K

    clocks = clk.summary()
    mhz = clocks["sm_mhz"] or 1965.0
    n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
    fp32_peak = n_sm * 128 * 2 * mhz * 1e6 / 1e12
    fp32_achieved = C * N * FLOP_PER_CHAIN_OBS / (ms_step / 1e3) / 1e12
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    hbm_src = "measured" if "hbm_gbs" in peaks else "fallback"
    secs = ms_step / 1e3
    if tensor_cores:
        # gm_iter_value_tc: the linear predictor on the tensor cores, the
        # softplus tail on the FP32 and special-function pipes
        mufu_peak = n_sm * 16 * mhz * 1e6 / 1e12
        mufu = C * N * MUFU_PER_CHAIN_OBS / secs / 1e12
        bf16 = float(peaks.get("bf16_tflops", 1590.0))
        tf32_peak = bf16 / 2.0
        tf32 = C * N * 3 * 2 * TC_COLS / secs / 1e12
        packed = N * PACKED_ROW_BYTES
        roofline = {
            "bound": "xu", "kernel": "gm_iter_value_tc",
            "achieved": round(mufu, 4), "peak": round(mufu_peak, 4),
            "unit": "Tops/s (MUFU ex2 + rcp)", "frac": round(mufu / mufu_peak, 4),
            "traffic": _traffic_per_launch("gm_iter_value_tc_logistic_n2e20_c1024.md"),
            "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one launch of "
                              "this kernel on this workload from the committed ncu capture "
                              "(profiles/gm_iter_value_tc_logistic_n2e20_c1024.md), not "
                              "measured by this run",
            "peak_source": f"nominal {n_sm} SMs x 16 SFU lanes x {mhz:.0f} MHz (median SM "
                           "clock sampled in the timed region; MEASURED_PEAKS.json has no "
                           "SFU figure)",
            "work_per_launch": f"{C} chains x {N} obs x {MUFU_PER_CHAIN_OBS:.0f} MUFU "
                               f"(+ {3 * 2 * TC_COLS} TF32 flop on the tensor cores)",
            "tensor": {"achieved_tflops": round(tf32, 2), "peak_tflops": round(tf32_peak, 1),
                       "frac": round(tf32 / tf32_peak, 4),
                       "work": f"3 split products x {TC_COLS} columns x 2 flop per "
                               "chain-observation",
                       "peak_source": "half the measured dense bf16 burst of "
                                      "MEASURED_PEAKS.json (TF32 runs at half the bf16 rate)"},
            "fp32_equiv": {"achieved_tflops": round(fp32_achieved, 3),
                           "peak_tflops": round(fp32_peak, 3),
                           "frac": round(fp32_achieved / fp32_peak, 4),
                           "work": f"{FLOP_PER_CHAIN_OBS:.0f} flop per chain-observation (the "
                                   "linear predictor), against the FP32 pipes it no longer "
                                   "runs on"},
            "hbm": {"achieved_gbs": round(packed / secs / 1e9, 2), "peak_gbs": hbm_peak,
                    "peak_source": hbm_src, "frac": round(packed / secs / 1e9 / hbm_peak, 5),
                    "bytes_per_launch": packed},
        }
    else:
        roofline = {
            "bound": "fp32", "kernel": "gm_iter_value",
            "achieved": round(fp32_achieved, 3), "peak": round(fp32_peak, 3),
            "unit": "TFLOP/s", "frac": round(fp32_achieved / fp32_peak, 4),
            "traffic": _traffic_per_launch("gm_iter_value_logistic_n2e20_c1024.md"),
            "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one launch of "
                              "this kernel on this workload from the committed ncu capture "
                              "(profiles/gm_iter_value_logistic_n2e20_c1024.md), not "
                              "measured by this run",
            "peak_source": f"nominal {n_sm} SMs x 128 FP32 lanes x 2 flop x {mhz:.0f} MHz "
                           "(median SM clock sampled in the timed region; "
                           "MEASURED_PEAKS.json has no FP32 figure)",
            "work_per_launch": f"{C} chains x {N} obs x {FLOP_PER_CHAIN_OBS:.0f} flop "
                               f"(+{MUFU_PER_CHAIN_OBS:.0f} MUFU)",
            "hbm": {"achieved_gbs": round(N * ROW_BYTES / secs / 1e9, 2),
                    "peak_gbs": hbm_peak, "peak_source": hbm_src,
                    "frac": round(N * ROW_BYTES / secs / 1e9 / hbm_peak, 5),
                    "bytes_per_launch": N * ROW_BYTES},
        }

    # The interpreter engine on the same workload (a few steps, same timing).
    interp = None
    if rank == 0 and not a.no_interp:
        si = _native.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                             m.n_params, w.data, m.n_cols, w.n_obs, engine=_native.ENGINE_INTERP)
        Ki = max(3, min(K, 10))
        si.prepare(init, sd, temps, 3 + Ki, 1 + rank, 0, rng=_native.RNG_PHILOX)
        si.advance(3)
        si.sync()
        st_i = torch.cuda.ExternalStream(si.stream, device=dev)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(Ki)]
        with torch.cuda.stream(st_i):
            for s0, s1 in ev:
                flush.zero_()
                s0.record(st_i)
                si.advance(1)
                s1.record(st_i)
        torch.cuda.synchronize()
        ms_i = float(np.mean([s0.elapsed_time(s1) for s0, s1 in ev]))
        si.close()
        interp = {"value": C * N / (ms_i / 1e3), "unit": UNIT, "ms_per_step": ms_i,
                  "steps": Ki,
                  "fp32_frac": round(C * N * FLOP_PER_CHAIN_OBS / (ms_i / 1e3) / 1e12
                                     / fp32_peak, 4)}

    e2e = None
    if rank == 0 and not a.no_e2e:
        init2, sd2, temps2 = _init(w, C, seed=7)
        # inputs and draws in pinned host memory, filled once before the timed calls
        data_h = torch.empty(w.data.shape, dtype=torch.float64, pin_memory=True).numpy()
        data_h[...] = w.data
        draws_h = _pinned_f32(K * C * m.n_params)

        def e2e_call(n_iter, seed):
            t = time.perf_counter()
            _native.run(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                        m.n_params, data_h, m.n_cols, w.n_obs, init2, sd2, temps2, n_iter,
                        seed, 0, out_draws=draws_h)
            return time.perf_counter() - t

        e2e_call(3, 2)  # untimed: first-call library and module set-up
        dt = float(np.median([e2e_call(K, 3 + i) for i in range(3)]))
        h2d = (w.data.nbytes + init2.nbytes + sd2.nbytes + temps2.nbytes
               + m.loglik.code.nbytes + m.loglik.consts.nbytes + m.prior.code.nbytes
               + m.prior.consts.nbytes)
        d2h = K * C * m.n_params * 4 + C * 4 + C * 8
        e2e = {"value": K * C * N / dt, "unit": UNIT, "h2d_bytes_per_step": h2d / K,
               "d2h_bytes_per_step": d2h / K,
               "note": "gpum_b200_run: one call of K iterations from pinned host buffers "
                       "(data upload + f64->f32 column layout + K iterations + draws back), "
                       "wall clock, median of 3 calls after one untimed call"}

    # the precision clause of the metric, outside every timed region and after
    # the e2e leg (the oracle's threads occupy every host core): the log
    # posterior of 32 chains' final states against the f64 oracle
    logp_err = logp_check(sess, w, n=32) if rank == 0 and not a.no_logp else None
    sess.close()

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu = cpu_sample(w, a.cpu_seconds, C)

    da = None
    if rank == 0 and world == 1 and not a.no_da:
        da = da_measure(w, C, a.da_warmup, a.da_iters, step_scale=a.da_step_scale,
                        train_steps=a.da_train_steps)

    configs = None
    if rank == 0 and world == 1 and not a.no_configs:
        configs = configs_measure(a.configs_only.split(","), a.configs_obs_shift, n_warm=1,
                                  n_timed=3)

    pt_da = None
    if rank == 0 and world == 1 and not a.no_pt_da:
        pt_da = pt_da_measure(a.pt_da_warmup, a.pt_da_iters)

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": Wm, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"logistic regression: N={_pow2(N)} obs, 16 N(0,1) covariates + "
                               "intercept, 17 params, 1024 chains, exact RWM, "
                               + ("linear predictor as split-TF32 tensor-core products, the "
                                  "rest of each term FP32" if tensor_cores
                                  else "FP32 bytecode")
                               + ", f64 sums/totals/accept",
                   "n_obs": N, "n_chains": C, "n_params": m.n_params,
                   "bytecode_instructions": m.loglik.n_instr,
                   "l2": "flushed (256 MiB write) before every timed step",
                   "rng": "philox", "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
        "engine": engine, "tensor_cores": tensor_cores, "interpreter_engine": interp,
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "delayed_acceptance": da, "logp_rel_err": logp_err,
        "logp_rel_err_note": "max over 32 chains of |sampler's log posterior of its final state "
                             "- f64 oracle| / |oracle|",
        "configs": configs, "pt_da": pt_da,
        "clocks": clocks, "wall_s_timed_region": wall,
        "accept_rate_mean": float(np.mean(acc)),
    }
    print(json.dumps(line), flush=True)


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = _workload(a.n_obs)
    m = w.model
    from oracle import cjit
    from oracle import oracle as O
    cores = _cpu_cores()
    fn = cjit.compile_loglik(m.loglik.code, m.loglik.consts)
    K, Wm = a.steps, max(3, a.warmup)
    # size each step to about min(2 s, 150 s / (K + W)) of work
    budget = min(2.0, 150.0 / (K + Wm))
    init, sd, temps = _init(w, cores, seed=1)
    t = time.perf_counter()
    O.run(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, m.n_params, w.data,
          m.n_cols, w.n_obs, init, sd, temps, 0, 1, 0, jit=fn, n_threads=cores)
    rate = cores * w.n_obs / (time.perf_counter() - t)
    C = max(cores, int(rate * budget / (2 * w.n_obs)) // cores * cores)
    init, sd, temps = _init(w, C, seed=1)
    times = []
    for k in range(Wm + K):
        t = time.perf_counter()
        O.run(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, m.n_params,
              w.data, m.n_cols, w.n_obs, init, sd, temps, 1, 1 + k, 0, jit=fn,
              n_threads=cores)
        if k >= Wm:
            times.append(time.perf_counter() - t)
    work = 2 * C * w.n_obs
    value = K * work / sum(times)
    sample = (f"{C} chains x 1 iteration (+ start evaluation) x {w.n_obs} obs per step; "
              "oracle port of cpu_native::run (reference Rust/R unbuildable here) with the "
              "bytecode->C gcc JIT, OpenMP over chains")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
        "steps": K, "warmup": Wm, "ms_per_step": 1e3 * sum(times) / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"logistic regression: N={_pow2(w.n_obs)} obs, 17 params; bounded chain "
                               "sample per step", "n_obs": w.n_obs,
                   "n_chains_per_step": C},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# Essential work per chain-observation of each configuration's iteration
# (FP32 flops, FMA = 2, after common subexpressions and parameter-only values
# are hoisted; MUFU = exp/log/ex2/rcp-class operations), as the model is
# written: the units behind each configuration's roofline fractions.
CONFIG_WORK = {
    "poisson": {"flop": 98.0, "mufu": 1.0,
                "what": "forward 50 flop + 1 exp, adjoint of 24 parameters 48 flop (MALA)"},
    "mixture": {"flop": 20.0, "mufu": 5.0,
                "what": "two Gaussian kernels, their weights and the log (RWM)"},
    "student_t": {"flop": 133.0, "mufu": 1.0,
                  "what": "64-term linear predictor, scaled residual, log (DE); on the "
                          "tensor-core kernel the 130 flop of the predictor run as TF32 MMAs, "
                          "so fp32_frac is an FP32-equivalent rate and can exceed 1"},
    "student_t_mala": {"flop": 263.0, "mufu": 1.0,
                       "what": "forward 133 flop + adjoint of 65 parameters 130 flop (MALA)"},
}
MUFU_PER_SM_CLK = 16  # SFU lanes per SM per clock


def configs_measure(configs, obs_shift=0, n_warm=2, n_timed=6, logp_points=16):
    """Timing of the other configurations at full size: per configuration one
    session, `n_warm` untimed iterations, then `n_timed` single-iteration
    advances, each after an L2 flush and bracketed by CUDA events on the
    session's stream; then (untimed) the log posterior the sampler holds for
    `logp_points` chains against the f64 oracle.  Returns one dict per
    configuration."""
    import torch

    from gpumetropolis_b200 import _native
    from gpumetropolis_b200 import workloads as W
    dev = torch.device("cuda", 0)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
    import inspect
    out = []
    for label in configs:
        name = label.replace("_mala", "")
        full = inspect.signature(W.ALL[name]).parameters["n_obs"].default
        t_gen = time.perf_counter()
        w = W.make(name, n_obs=max(1024, full >> max(obs_shift, 0)))
        t_gen = time.perf_counter() - t_gen
        m = w.model
        C, N, npar = w.n_chains, w.n_obs, m.n_params
        rng = np.random.default_rng(7)
        temps = np.ones(C)
        gamma, ladder = 0.0, 0
        if name == "poisson":
            mode, centre, jitter, step = _native.MODE_MALA, w.truth["beta"], 0.01, 2e-4
            method = "mala (value + adjoint kernel gm_iter_grad, chain-lane body)"
        elif name == "mixture":
            mode, jitter, step = _native.MODE_RWM, 0.01, 5e-4
            centre = np.array([math.log(0.3 / 0.7), -2.0, 3.0, 0.0, math.log(1.5)])
            ladder = 16
            temps = np.tile(np.geomspace(1.0, 64.0, ladder), C // ladder)
            method = "rwm, 512 ladders of 16 geometric temperatures 1..64, device exchanges every 10"
        elif label == "student_t_mala":
            mode, jitter, step = _native.MODE_MALA, 0.01, 1e-4
            centre = np.concatenate([w.truth["beta"], [math.log(1.5)]])
            method = "mala (value + adjoint kernel gm_iter_grad, chain-lane body)"
        else:
            mode, jitter, step = _native.MODE_DE, 0.01, 1e-4
            centre = np.concatenate([w.truth["beta"], [math.log(1.5)]])
            gamma = 2.38 / math.sqrt(2 * npar)
            method = "de"
        init = centre + rng.normal(0.0, jitter, (C, npar))
        sd = np.full((C, npar), step)
        sess = _native.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts,
                               npar, w.data, m.n_cols, N)
        tc = mode != _native.MODE_MALA and sess.tensor_cores
        if mode != _native.MODE_MALA:
            method += (" (tensor-core value kernel gm_iter_value_tc: the linear predictor as "
                       "TF32 MMAs, the rest of the term on the FP32 pipes)" if tc
                       else " (value kernel gm_iter_value)")
        try:
            if ladder:
                sess.set_exchange(ladder, 10)
            sess.prepare(init, sd, temps, n_warm + n_timed, 3, mode, gamma, 1e-3,
                         rng=_native.RNG_PHILOX)
            sess.advance(n_warm)
            sess.sync()
            stream = torch.cuda.ExternalStream(sess.stream, device=dev)
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(n_timed)]
            torch.cuda.synchronize()
            with Clocks(0) as clk:
                clk.mark_start()
                with torch.cuda.stream(stream):
                    for s0, s1 in ev:
                        flush.zero_()
                        s0.record(stream)
                        sess.advance(1)
                        s1.record(stream)
                torch.cuda.synchronize()
                clk.mark_end()
            ms = float(np.mean([s0.elapsed_time(s1) for s0, s1 in ev]))
            _, acc, last, _ = sess.fetch(want_draws=False)
            logp = logp_check(sess, w, n=logp_points)
        finally:
            sess.close()
        clocks = clk.summary()
        mhz = clocks["sm_mhz"] or 1965.0
        wk = CONFIG_WORK[label]
        rate = C * N / (ms / 1e3)
        fp32_peak = n_sm * 128 * 2 * mhz * 1e6
        mufu_peak = n_sm * MUFU_PER_SM_CLK * mhz * 1e6
        out.append({
            "config": label, "n_chains": C, "n_obs": N, "n_params": npar, "method": method,
            "ms_per_iter": round(ms, 3), "chain_obs_per_s": rate,
            "tensor_cores": tc,
            "fp32_frac": round(rate * wk["flop"] / fp32_peak, 4),
            "mufu_frac": round(rate * wk["mufu"] / mufu_peak, 4),
            "work_per_chain_obs": f"{wk['flop']:.0f} flop + {wk['mufu']:.0f} MUFU: {wk['what']}",
            "logp_rel_err": logp, "logp_points": logp_points,
            "all_finite": bool(np.all(np.isfinite(last))),
            "sm_mhz": clocks["sm_mhz"], "clock_reasons": clocks["reasons"],
            "data_gen_s": round(t_gen, 1),
            "timing": f"{n_timed} single-iteration advances after {n_warm} warm-up, L2 "
                      "flushed before each, CUDA events on the session stream"})
        del w
    return out


def run_configs(a):
    from gpumetropolis_b200 import _native
    from gpumetropolis_b200.build import build
    build()
    if not _native.available():
        raise SystemExit("gpum_b200: no usable sm_100 device")
    for r in configs_measure(a.configs_only.split(","), a.configs_obs_shift):
        print(json.dumps(r), flush=True)


def pt_da_measure(n_warm, n_samp, K=16, every=10, seed=21):
    """Mixture configuration, PT + surrogate delayed acceptance: 8192 chains
    as 512 ladders of K geometric temperatures 1..64 with device exchanges
    every `every` iterations; adaptive warmup (per-chain Robbins-Monro scales
    and variances from device moments) whose second half records the exact
    pairs (at most 2^18) for the 5-256-256-1 surrogate; then, from the same
    state, exact sampling and two-stage sampling of equal length, timed by
    the wall clock around each blocking run (draws copied back in both).
    ESS: multi-chain over the 512 temperature-1 chains, per parameter."""
    from gpumetropolis_b200 import _native, api
    from gpumetropolis_b200 import adaptive as AD
    from gpumetropolis_b200 import workloads as W
    w = W.make("mixture")
    m = w.model
    C, npar = w.n_chains, m.n_params
    temps = np.tile(np.geomspace(1.0, 64.0, K), C // K)
    cfg = dict(api.SURROGATE_DEFAULTS)
    cfg.update({"max_pairs": 1 << 18, "hidden": 256})  # the configuration's 5-256-256-1
    call = api._Backend(m, w.data, w.n_obs, _native.RNG_PHILOX, cfg)
    try:
        s = call.session
        s.set_exchange(K, every)
        rng = np.random.default_rng(seed)
        centre = np.array([math.log(0.3 / 0.7), -2.0, 3.0, 0.0, math.log(1.5)])
        cur = centre + rng.normal(0.0, 0.01, (C, npar))
        sd = np.full((C, npar), 1e-3) * np.sqrt(temps)[:, None]
        call.record_at = n_warm // 2
        nb = min(40, max(10, n_warm // 50), n_warm)
        sizes = np.full(nb, n_warm // nb, dtype=np.int64)
        sizes[-1] += n_warm - sizes.sum()
        states = AD.WelfordDiag.init(C, npar, sd ** 2)
        scales = np.ones(C)
        t = time.perf_counter()
        for b, n in enumerate(sizes, start=1):
            mo, acc = call.run_moments(cur, sd, int(n), seed + b, temps, 0)
            cur = mo.last
            states.merge(mo.n, mo.chain_mean, mo.chain_m2)
            scales = AD.robbins_monro_scale(scales, acc, b, npar)
            sd = scales[:, None] * np.sqrt(np.maximum(states.variances(), 1e-12))
        t_warm = time.perf_counter() - t
        t = time.perf_counter()
        call.start_da()
        t_train = time.perf_counter() - t
        if call.net is None:
            return {"used": False, "reason": call.info.get("reason")}

        def timed(f):
            s.sync()
            t0 = time.perf_counter()
            r = f()
            return r, time.perf_counter() - t0

        buf_ex, buf_da = _pinned_f32(n_samp * C * npar), _pinned_f32(n_samp * C * npar)
        (d_ex, acc_ex, _), t_ex = timed(lambda: s.run(cur, sd, temps, n_samp, seed + 100, 0,
                                                      rng=_native.RNG_PHILOX, out_draws=buf_ex))
        att, ok_ex, _ = s.exchange_stats()
        e0 = call.exact_evals
        (d_da, acc_da, _), t_da = timed(lambda: call(cur, sd, n_samp, seed + 200, temps, 0,
                                                     out_draws=buf_da))
        _, ok_da, _ = s.exchange_stats()
        exact_frac = (call.exact_evals - e0) / (n_samp * C)
        d_ex = d_ex.reshape((n_samp, C, npar), order="F").astype(np.float64)[:, ::K, :]
        d_da = np.asarray(d_da, dtype=np.float64)[:, ::K, :]
        e_ex, e_da = _ess_all(d_ex), _ess_all(d_da)
        mc_ex = d_ex.reshape(-1, npar).std(axis=0) / np.sqrt(e_ex)
        mc_da = d_da.reshape(-1, npar).std(axis=0) / np.sqrt(e_da)
        z = np.abs(d_ex.mean(axis=(0, 1)) - d_da.mean(axis=(0, 1))) / np.sqrt(mc_ex**2 + mc_da**2)
        r_ex, r_da = e_ex.min() / t_ex, e_da.min() / t_da
        with np.errstate(invalid="ignore", divide="ignore"):
            x_ex = float(np.nansum(ok_ex) / max(np.sum(att), 1))
            x_da = float(np.nansum(ok_da) / max(np.sum(att), 1))
        r_da_t = e_da.min() / (t_da + t_train)
        return {
            "used": True,
            "config": "mixture N=2^22, 8192 chains = 512 ladders x 16 geometric temperatures "
                      "1..64, device exchanges every %d iterations, surrogate 5-%d-%d-1 on "
                      "<= 2^18 warmup pairs" % (every, cfg["hidden"], cfg["hidden"]),
            "warmup_iters": n_warm, "sampling_iters": n_samp, "warmup_s": round(t_warm, 3),
            "train_s": round(t_train, 3), "surrogate": call.da_summary(),
            "exact": {"seconds": round(t_ex, 3), "accept_cold": float(np.mean(acc_ex[::K])),
                      "exchange_rate": x_ex, "ess_min": float(e_ex.min()),
                      "ess_mean": float(e_ex.mean()), "ess_per_s_min": r_ex},
            "da": {"seconds": round(t_da, 3), "accept_cold": float(np.mean(acc_da[::K])),
                   "exchange_rate": x_da, "exact_fraction": exact_frac,
                   "ess_min": float(e_da.min()), "ess_mean": float(e_da.mean()),
                   "ess_per_s_min": r_da},
            "gain_ess_per_s_min": r_da / r_ex,
            "gain_ess_per_s_mean": float((e_da.mean() / t_da) / (e_ex.mean() / t_ex)),
            "gain_ess_per_s_min_with_training": r_da_t / r_ex,
            "gain_ess_per_s_mean_with_training":
                float((e_da.mean() / (t_da + t_train)) / (e_ex.mean() / t_ex)),
            "posterior_mean_max_z": float(z.max()),
            "ess": "multi-chain over the 512 temperature-1 chains, per parameter"}
    finally:
        call.close()


def run_pt_da(a):
    import torch

    from gpumetropolis_b200 import _native
    from gpumetropolis_b200.build import build
    build()
    if not _native.available():
        raise SystemExit("gpum_b200: no usable sm_100 device")
    torch.cuda.set_device(0)
    print(json.dumps({"pt_da": pt_da_measure(a.pt_da_warmup, a.pt_da_iters)}), flush=True)


def c5_da_measure(n_warm, n_samp, seed=31, modes=("de", "mala")):
    """Student-t regression at full size (N = 2^24, 65 parameters, 8192
    chains) with the 65-512-512-1 surrogate: adaptive exact warmup (random
    walk with the pooled Cholesky factor) whose draws' proposals are all
    recorded (n_warm x 8192 pairs, 2^20 at n_warm = 128), the surrogate
    trained on them, then for each method exact and two-stage sampling of
    equal length from the warmup's last state: DE (snapshot differences,
    gamma 2.38 / sqrt(2 d)) and the Langevin move (exact MALA with the
    adjoint kernel against delayed acceptance whose drift is the surrogate's
    gradient).  Seconds are wall seconds of each blocking call (draws back);
    ESS multi-chain per parameter."""
    from gpumetropolis_b200 import _native, api
    from gpumetropolis_b200 import adaptive as AD
    from gpumetropolis_b200 import workloads as W
    t = time.perf_counter()
    w = W.make("student_t")
    t_gen = time.perf_counter() - t
    m = w.model
    C, npar = w.n_chains, m.n_params
    cfg = dict(api.SURROGATE_DEFAULTS)
    cfg.update({"hidden": 512, "max_pairs": 1 << 20})
    call = api._Backend(m, w.data, w.n_obs, _native.RNG_PHILOX, cfg)
    out = {"config": "student-t regression N=2^24, 65 params, 8192 chains; surrogate 65-512-512-1",
           "data_gen_s": round(t_gen, 1), "warmup_iters": n_warm, "sampling_iters": n_samp}
    try:
        call.record_at = 0
        rng = np.random.default_rng(seed)
        centre = np.concatenate([w.truth["beta"], [math.log(1.5)]])
        init = centre + rng.normal(0.0, 1e-3, (C, npar))
        t = time.perf_counter()
        am = AD.am_orchestrate_warmup(call, npar, C, init, np.full((C, npar), 2e-4), n_warm,
                                      seed)
        out["warmup_s"] = round(time.perf_counter() - t, 2)
        t = time.perf_counter()
        call.start_da()
        out["train_s"] = round(time.perf_counter() - t, 3)
        out["surrogate"] = call.da_summary()
        if call.net is None:
            return out
        x0, sd0, L0 = am.final_init, am.final_proposal_sd, am.final_L
        ones = np.ones(C)
        s = call.session
        buf = _pinned_f32(n_samp * C * npar)

        def timed(f):
            s.sync()
            t0 = time.perf_counter()
            r = f()
            return r, time.perf_counter() - t0

        for meth in modes:
            if meth == "de":
                mode, g, dn, L = _native.MODE_DE, 2.38 / math.sqrt(2 * npar), 1e-3, None
            else:
                mode, g, dn, L = _native.MODE_MALA, 0.0, 0.0, L0
            (d_ex, acc_ex, _), t_ex = timed(lambda: s.run(
                x0, sd0, ones, n_samp, seed + 7, mode, g, dn, L, rng=_native.RNG_PHILOX,
                out_draws=buf))
            e_ex = _ess_all(d_ex.reshape((n_samp, C, npar), order="F"))
            e0 = call.exact_evals
            (d_da, acc_da, _), t_da = timed(lambda: call(x0, sd0, n_samp, seed + 8, None, mode,
                                                         g, dn, L, out_draws=buf))
            frac = (call.exact_evals - e0) / (n_samp * C)
            e_da = _ess_all(np.asarray(d_da))
            r_ex, r_da = e_ex.min() / t_ex, e_da.min() / t_da
            out[meth] = {
                "exact": {"seconds": round(t_ex, 2), "accept": float(np.mean(acc_ex)),
                          "ess_min": float(e_ex.min()), "ess_per_s_min": r_ex},
                "da": {"seconds": round(t_da, 2), "accept": float(np.mean(acc_da)),
                       "exact_fraction": frac, "ess_min": float(e_da.min()),
                       "ess_per_s_min": r_da},
                "gain_ess_per_s_min": r_da / r_ex,
                "gain_ess_per_s_min_with_training":
                    e_da.min() / (t_da + out["train_s"]) / r_ex}
    finally:
        call.close()
    return out


def run_c5_da(a):
    import torch

    from gpumetropolis_b200 import _native
    from gpumetropolis_b200.build import build
    build()
    if not _native.available():
        raise SystemExit("gpum_b200: no usable sm_100 device")
    torch.cuda.set_device(0)
    print(json.dumps({"c5_da": c5_da_measure(a.c5_warmup, a.c5_iters)}), flush=True)


def run_profile_da(a, n_warm=200, n_samp=48, seed=11):
    """A small, self-contained target for profiler captures of the surrogate's
    training and of the two-stage loop on the logistic configuration (1024
    chains, N = 2^20): a short adaptive exact warmup whose second half is
    recorded, the surrogate trained inside an NVTX range "training", then
    n_samp two-stage iterations inside an NVTX range "da_sampling" (select
    them with ncu --nvtx --nvtx-include)."""
    import torch

    from gpumetropolis_b200 import _native, api
    from gpumetropolis_b200 import adaptive as AD
    from gpumetropolis_b200.build import build
    build()
    if not _native.available():
        raise SystemExit("gpum_b200: no usable sm_100 device")
    w = _workload(a.n_obs)
    m = w.model
    C, npar = a.chains, m.n_params
    call = api._Backend(m, w.data, w.n_obs, _native.RNG_PHILOX, dict(api.SURROGATE_DEFAULTS))
    try:
        call.record_at = n_warm // 2
        rng = np.random.default_rng(seed)
        init = w.truth["beta"] + rng.normal(0, 0.05, (C, npar))
        am = AD.am_orchestrate_warmup(call, npar, C, init, np.full((C, npar), 0.01), n_warm,
                                      seed)
        call.session.sync()
        torch.cuda.nvtx.range_push("training")
        t = time.perf_counter()
        call.start_da()
        t_train = time.perf_counter() - t
        torch.cuda.nvtx.range_pop()
        call.session.sync()
        torch.cuda.nvtx.range_push("da_sampling")
        t = time.perf_counter()
        call(am.final_init, am.final_proposal_sd, n_samp, seed + 2, None, _native.MODE_CHOL,
             0.0, 0.0, am.final_L)
        t_da = time.perf_counter() - t
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"profile_da": {"train_s": round(t_train, 4),
                                         "da_us_per_iter": round(1e6 * t_da / n_samp, 1),
                                         "surrogate": call.da_summary()}}), flush=True)
    finally:
        call.close()


def main():
    a = _args()
    if a.impl == "reference":
        run_reference(a)
    elif a.profile_da:
        run_profile_da(a)
    elif a.c5_da:
        run_c5_da(a)
    elif a.pt_da:
        run_pt_da(a)
    elif a.configs:
        run_configs(a)
    else:
        run_b200(a)


if __name__ == "__main__":
    main()
