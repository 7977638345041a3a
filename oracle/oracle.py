"""ctypes binding of the CPU oracle (gpum_oracle.c) -- TEST INFRASTRUCTURE ONLY.

The oracle restates the reference's f64 CPU backend (``src/rust/src/
cpu_native.rs``).  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg import this module; the B200 product path never
does.  Function names follow the reference's (``loglik_batch``,
``grad_batch``, ``loglik_pointwise``, ``run``, ``run_de_sync``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libgpum_oracle.so")
_lib = None

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
LOGLIK_FN = C.CFUNCTYPE(C.c_double, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64)


def build() -> str:
    """Compile the oracle with its Makefile; returns the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        sz = C.c_size_t
        L.gpo_triple32.restype = C.c_uint32
        L.gpo_triple32.argtypes = [C.c_uint32]
        L.gpo_uniform.restype = C.c_double
        L.gpo_uniform.argtypes = [C.c_uint32, C.c_uint32]
        L.gpo_seedmix.restype = C.c_uint32
        L.gpo_seedmix.argtypes = [C.c_uint32, C.c_uint32]
        L.gpo_lgamma.restype = C.c_double
        L.gpo_lgamma.argtypes = [C.c_double]
        L.gpo_digamma.restype = C.c_double
        L.gpo_digamma.argtypes = [C.c_double]
        L.gpo_eval.restype = C.c_double
        L.gpo_eval.argtypes = [_u32p, sz, _f64p, _f64p, C.c_void_p]
        for name in ("gpo_loglik_batch", "gpo_grad_batch", "gpo_loglik_pointwise"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [_u32p, sz, _f64p, sz, _f64p, sz, sz, _f64p, sz, _f64p]
        L.gpo_run.restype = C.c_int
        L.gpo_run.argtypes = [_u32p, sz, _f64p, _u32p, sz, _f64p, sz, _f64p, sz, sz,
                              _f64p, _f64p, _f64p, sz, sz, C.c_uint32, C.c_uint32,
                              C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_int,
                              _f32p, _f32p, _f64p]
        L.gpo_jit_batch.restype = None
        L.gpo_jit_batch.argtypes = [C.c_void_p, sz, _f64p, sz, sz, _f64p, sz, _f64p, C.c_int]
        L.gpo_grad_abs_batch.restype = C.c_int
        L.gpo_grad_abs_batch.argtypes = [_u32p, sz, _f64p, sz, _f64p, sz, sz, _f64p, sz, sz,
                                         _f64p, _f64p, C.c_int]
        L.gpo_run_de_sync.restype = C.c_int
        L.gpo_run_de_sync.argtypes = [_u32p, sz, _f64p, _u32p, sz, _f64p, sz, _f64p, sz,
                                      sz, _f64p, _f64p, sz, sz, C.c_uint32, C.c_double,
                                      C.c_double, C.c_void_p, _f32p, _f32p, _f64p]
        _lib = L
    return _lib


def _prog(code, consts):
    code = np.ascontiguousarray(code, dtype=np.uint32)
    consts = np.ascontiguousarray(consts, dtype=np.float64)
    if consts.size == 0:
        consts = np.zeros(1)
    return code, consts


def _data(data, n_cols, n_obs):
    d = np.ascontiguousarray(data, dtype=np.float64).reshape(-1)
    if d.size == 0:
        d = np.zeros(1)
    return d


def triple32(x: int) -> int:
    return lib().gpo_triple32(x & 0xFFFFFFFF)


def uniform(seedmix: int, ctr: int) -> float:
    return lib().gpo_uniform(seedmix & 0xFFFFFFFF, ctr & 0xFFFFFFFF)


def seedmix(seed: int, chain: int) -> int:
    return lib().gpo_seedmix(seed & 0xFFFFFFFF, chain & 0xFFFFFFFF)


def lgamma(x: float) -> float:
    return lib().gpo_lgamma(x)


def digamma(x: float) -> float:
    return lib().gpo_digamma(x)


def _batch(fname, code, consts, n_params, data, n_cols, n_obs, points, width):
    code, consts = _prog(code, consts)
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1)
    n_points = pts.size // n_params if n_params else 0
    out = np.zeros(max(n_points * width, 1))
    getattr(lib(), fname)(code, code.size // 2, consts, n_params,
                          _data(data, n_cols, n_obs), n_cols, n_obs,
                          pts if pts.size else np.zeros(1), n_points, out)
    return out[: n_points * width]


def loglik_batch(code, consts, n_params, data, n_cols, n_obs, points):
    """Summed log-likelihood per point (``cpu_native.rs:339-360``)."""
    return _batch("gpo_loglik_batch", code, consts, n_params, data, n_cols, n_obs,
                  points, 1)


def grad_batch(code, consts, n_params, data, n_cols, n_obs, points):
    """Point-major gradient of the data term (``cpu_native.rs:306-329``)."""
    return _batch("gpo_grad_batch", code, consts, n_params, data, n_cols, n_obs,
                  points, n_params)


def loglik_pointwise(code, consts, n_params, data, n_cols, n_obs, points):
    """``out[p * n_obs + i]`` per-observation log-likelihood (``:371-391``)."""
    return _batch("gpo_loglik_pointwise", code, consts, n_params, data, n_cols, n_obs,
                  points, n_obs)


def jit_batch(fn, n_params, data, n_cols, n_obs, points, n_threads=0):
    """A compiled evaluator (:func:`oracle.cjit.compile_loglik`) at each point,
    parallel over points: ``loglik_batch``'s value at full configuration
    sizes (the compiled code performs the interpreter's f64 operations in the
    same order).  Checker only; no reference counterpart."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1)
    n_points = pts.size // n_params
    out = np.zeros(max(n_points, 1))
    lib().gpo_jit_batch(C.cast(fn, C.c_void_p), n_params, _data(data, n_cols, n_obs), n_cols,
                        n_obs, pts if pts.size else np.zeros(1), n_points, out, n_threads)
    return out[:n_points]


def grad_abs_batch(code, consts, n_params, data, n_cols, n_obs, points, block=4096,
                   n_threads=0):
    """``grad_batch``'s gradient (``cpu_native.rs:306-329``) at each point and,
    per component, the sum over observations of the per-observation
    gradient's absolute value (the scale that bounds the rounding error of a
    sum that cancels).  Parallel over (point, block of observations), blocks
    added in order.  Returns ``(grad, abs_sum)``, both ``(n_points,
    n_params)``.  Checker only; no reference counterpart."""
    code, consts = _prog(code, consts)
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1)
    n_points = pts.size // n_params
    g = np.zeros(max(n_points * n_params, 1))
    a = np.zeros(max(n_points * n_params, 1))
    rc = lib().gpo_grad_abs_batch(code, code.size // 2, consts, n_params,
                                  _data(data, n_cols, n_obs), n_cols, n_obs,
                                  pts if pts.size else np.zeros(1), n_points, block, g, a,
                                  n_threads)
    if rc != 0:
        raise MemoryError("oracle grad_abs_batch failed to allocate")
    return (g[:n_points * n_params].reshape(n_points, n_params),
            a[:n_points * n_params].reshape(n_points, n_params))


def run(code, consts, prior_code, prior_consts, n_params, data, n_cols, n_obs, init,
        proposal_sd, temperatures, n_iter, seed, proposal_mode, gamma=0.0,
        de_noise=0.0, proposal_l=None, jit=None, n_threads=0):
    """Whole-chain sampler (``cpu_native.rs:510-825``).

    Returns ``(draws f32 (n_iter*C*np,) column-major (n_iter, C, np),
    accept_rate f32 (C,), last_log_post f64 (C,))``.  ``jit`` is an optional
    compiled data-term evaluator from :func:`oracle.cjit.compile_loglik`.
    """
    code, consts = _prog(code, consts)
    pcode, pconsts = _prog(prior_code, prior_consts)
    init = np.ascontiguousarray(init, dtype=np.float64).reshape(-1)
    n_chains = init.size // n_params
    sd = np.ascontiguousarray(proposal_sd, dtype=np.float64).reshape(-1)
    temps = np.ascontiguousarray(temperatures, dtype=np.float64).reshape(-1)
    L = None
    if proposal_l is not None and np.size(proposal_l) > 0:
        L = np.ascontiguousarray(proposal_l, dtype=np.float64).reshape(-1)
    draws = np.zeros(max(n_iter * n_chains * n_params, 1), np.float32)
    acc = np.zeros(n_chains, np.float32)
    last = np.zeros(n_chains, np.float64)
    rc = lib().gpo_run(code, code.size // 2, consts, pcode, pcode.size // 2, pconsts,
                       n_params, _data(data, n_cols, n_obs), n_cols, n_obs, init, sd,
                       temps, n_chains, n_iter, seed & 0xFFFFFFFF, proposal_mode,
                       gamma, de_noise, None if L is None else L.ctypes.data,
                       None if jit is None else C.cast(jit, C.c_void_p), n_threads,
                       draws, acc, last)
    if rc != 0:
        raise MemoryError("oracle run failed to allocate")
    return draws[: n_iter * n_chains * n_params], acc, last


def run_de_sync(code, consts, prior_code, prior_consts, n_params, data, n_cols, n_obs,
                init, proposal_sd, n_iter, seed, gamma, de_noise, jit=None):
    """Synchronous per-generation DE (``cpu_native.rs:400-506``)."""
    code, consts = _prog(code, consts)
    pcode, pconsts = _prog(prior_code, prior_consts)
    init = np.ascontiguousarray(init, dtype=np.float64).reshape(-1)
    n_chains = init.size // n_params
    sd = np.ascontiguousarray(proposal_sd, dtype=np.float64).reshape(-1)
    draws = np.zeros(max(n_iter * n_chains * n_params, 1), np.float32)
    acc = np.zeros(n_chains, np.float32)
    last = np.zeros(n_chains, np.float64)
    rc = lib().gpo_run_de_sync(code, code.size // 2, consts, pcode, pcode.size // 2,
                               pconsts, n_params, _data(data, n_cols, n_obs), n_cols,
                               n_obs, init, sd, n_chains, n_iter, seed & 0xFFFFFFFF,
                               gamma, de_noise,
                               None if jit is None else C.cast(jit, C.c_void_p),
                               draws, acc, last)
    if rc != 0:
        raise MemoryError("oracle de_sync failed to allocate")
    return draws[: n_iter * n_chains * n_params], acc, last
