"""ctypes binding of ``libgpum_b200.so`` (the C ABI in ``include/gpum_b200.h``).

The library is built in-tree (``gpumetropolis_b200/build.py``).  There is no
fallback: if the library is missing or cannot load, every call raises
:class:`BackendUnavailable`, and a GPU-side failure raises :class:`GpumError`
with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpum_b200.so")

OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_UNSUPPORTED, ERR_NODEVICE, ERR_DEVICE = range(7)
ENGINE_INTERP, ENGINE_COMPILED, ENGINE_AUTO = 0, 1, 2
MODE_RWM, MODE_DE, MODE_CHOL, MODE_MALA, MODE_DE_SYNC = 0, 1, 2, 3, 4
RNG_TRIPLE32, RNG_PHILOX = 0, 1
_ERRLEN = 1024


class BackendUnavailable(RuntimeError):
    """The b200 library is not built or cannot be loaded."""


class GpumError(RuntimeError):
    """A status code other than GPUM_OK from the C ABI."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"gpum_b200 error {code}: {msg}")
        self.code = code


_u32p = C.POINTER(C.c_uint32)
_f64p = C.POINTER(C.c_double)
_f32p = C.POINTER(C.c_float)
_sz = C.c_size_t
_errp = C.c_char_p

# name -> (restype, argtypes); the declarations of include/gpum_b200.h.
SIGNATURES = {
    "gpum_b200_available": (C.c_int, []),
    "gpum_b200_version": (C.c_char_p, []),
    "gpum_b200_validate_program": (C.c_int, [_u32p, _sz, _sz, C.c_uint32, C.c_uint32, C.c_int,
                                             C.POINTER(C.c_int), _errp, _sz]),
    "gpum_b200_run": (C.c_int, [_u32p, _sz, _f64p, _sz, _u32p, _sz, _f64p, _sz, C.c_uint32,
                                _f64p, C.c_uint32, C.c_uint64, _f64p, _f64p, _f64p, C.c_uint32,
                                C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_double,
                                _f64p, _sz, _f32p, _f32p, _f64p, _errp, _sz]),
    "gpum_b200_loglik_batch": (C.c_int, [_u32p, _sz, _f64p, _sz, C.c_uint32, _f64p,
                                         C.c_uint32, C.c_uint64, _f64p, _sz, _f64p, _errp,
                                         _sz]),
    "gpum_b200_loglik_pointwise": (C.c_int, [_u32p, _sz, _f64p, _sz, C.c_uint32, _f64p,
                                             C.c_uint32, C.c_uint64, _f64p, _sz, _f64p, _errp,
                                             _sz]),
    "gpum_b200_grad_batch": (C.c_int, [_u32p, _sz, _f64p, _sz, C.c_uint32, _f64p,
                                       C.c_uint32, C.c_uint64, _f64p, _sz, _f64p, _errp, _sz]),
    "gpum_b200_compile_check": (C.c_int, [_u32p, _sz, _f64p, _sz, _u32p, _sz, _f64p, _sz,
                                          C.c_uint32, C.c_uint32, C.POINTER(C.c_size_t), _errp,
                                          _sz]),
    "gpum_b200_session_set_engine": (C.c_int, [C.c_void_p, C.c_int, _errp, _sz]),
    "gpum_b200_session_engine": (C.c_int, [C.c_void_p]),
    "gpum_b200_session_tensor_cores": (C.c_int, [C.c_void_p]),
    "gpum_b200_session_grad_batch": (C.c_int, [C.c_void_p, _f64p, _sz, _f64p, _errp, _sz]),
    "gpum_b200_loglik_batch_noalloc": (C.c_int, [_u32p, _sz, _f64p, _sz, C.c_uint32,
                                                 C.c_void_p, C.c_uint64, C.c_uint32,
                                                 C.c_uint64, C.c_void_p, _sz, C.c_void_p,
                                                 C.c_void_p, _errp, _sz]),
    "gpum_b200_mlp_create": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                       C.POINTER(C.c_void_p), _errp, _sz]),
    "gpum_b200_mlp_destroy": (None, [C.c_void_p]),
    "gpum_b200_mlp_set_normalizer": (C.c_int, [C.c_void_p, _f64p, _f64p, C.c_double,
                                               C.c_double, _errp, _sz]),
    "gpum_b200_mlp_set_whitening": (C.c_int, [C.c_void_p, _f64p, _f64p, C.c_double,
                                              C.c_double, _errp, _sz]),
    "gpum_b200_mlp_train": (C.c_int, [C.c_void_p, _f64p, _f64p, _sz, C.c_uint32, C.c_double,
                                      _f32p, _errp, _sz]),
    "gpum_b200_mlp_train_stages": (C.c_int, [C.c_void_p, _f64p, _f64p, _sz, C.c_uint32,
                                             _u32p, _f64p, _f32p, _errp, _sz]),
    "gpum_b200_mlp_predict": (C.c_int, [C.c_void_p, _f64p, _sz, _f64p, _errp, _sz]),
    "gpum_b200_mlp_predict_grad": (C.c_int, [C.c_void_p, _f64p, _sz, _f64p, _f64p, _errp,
                                             _sz]),
    "gpum_b200_mlp_gradients": (C.c_int, [C.c_void_p, _f64p, _f64p, _sz, _f32p, _f32p, _errp,
                                          _sz]),
    "gpum_b200_mlp_get_params": (C.c_int, [C.c_void_p, _f32p, _errp, _sz]),
    "gpum_b200_mlp_gemm_check": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, _f32p, _f32p,
                                           _f32p, _errp, _sz]),
    "gpum_b200_session_create": (C.c_int, [_u32p, _sz, _f64p, _sz, _u32p, _sz, _f64p, _sz,
                                           C.c_uint32, _f64p, C.c_uint32, C.c_uint64,
                                           C.POINTER(C.c_void_p), _errp, _sz]),
    "gpum_b200_session_run": (C.c_int, [C.c_void_p, _f64p, _f64p, _f64p, C.c_uint32,
                                        C.c_uint32, C.c_uint32, C.c_uint32, C.c_double,
                                        C.c_double, _f64p, _sz, C.c_int, _f32p, _f32p, _f64p,
                                        _errp, _sz]),
    "gpum_b200_session_loglik_batch": (C.c_int, [C.c_void_p, _f64p, _sz, _f64p, _errp, _sz]),
    "gpum_b200_session_loglik_pointwise": (C.c_int, [C.c_void_p, _f64p, _sz, _f64p, _errp,
                                                     _sz]),
    "gpum_b200_session_prepare": (C.c_int, [C.c_void_p, _f64p, _f64p, _f64p, C.c_uint32,
                                            C.c_uint32, C.c_uint32, C.c_uint32, C.c_double,
                                            C.c_double, _f64p, _sz, C.c_int, _errp, _sz]),
    "gpum_b200_session_advance": (C.c_int, [C.c_void_p, C.c_uint32, _errp, _sz]),
    "gpum_b200_session_sync": (C.c_int, [C.c_void_p, _errp, _sz]),
    "gpum_b200_session_fetch": (C.c_int, [C.c_void_p, _f32p, _f32p, _f64p,
                                          C.POINTER(C.c_uint32), _errp, _sz]),
    "gpum_b200_session_launches": (C.c_uint64, [C.c_void_p]),
    "gpum_b200_session_selftest_wait": (C.c_int, [C.c_void_p, C.c_uint32, _errp, _sz]),
    "gpum_b200_session_stream": (C.c_void_p, [C.c_void_p]),
    "gpum_b200_session_destroy": (None, [C.c_void_p]),
    "gpum_b200_run_de_sync": (C.c_int, [_u32p, _sz, _f64p, _sz, C.c_uint32, _f64p, C.c_uint32,
                                        C.c_uint64, _u32p, _sz, _f64p, _sz, _f64p, _f64p,
                                        C.c_uint32, C.c_uint32, C.c_uint32, C.c_double,
                                        C.c_double, _f32p, _f32p, _f64p, _errp, _sz]),
    "gpum_b200_session_run_de_sync": (C.c_int, [C.c_void_p, _f64p, _f64p, C.c_uint32,
                                                C.c_uint32, C.c_uint32, C.c_double, C.c_double,
                                                C.c_int, _f32p, _f32p, _f64p, _errp, _sz]),
    "gpum_b200_session_set_exchange": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, _errp,
                                                 _sz]),
    "gpum_b200_session_exchange_stats": (C.c_int, [C.c_void_p, _u32p, _u32p, _u32p, _errp,
                                                   _sz]),
    "gpum_b200_session_draw_moments": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, _f64p,
                                                 _f64p, _f64p, _f64p, _errp, _sz]),
    "gpum_b200_session_state": (C.c_int, [C.c_void_p, _f64p, _errp, _sz]),
    "gpum_b200_session_set_likelihood_powers": (C.c_int, [C.c_void_p, _f64p, _sz, _errp,
                                                          _sz]),
    "gpum_b200_session_record": (C.c_int, [C.c_void_p, C.c_uint64, _errp, _sz]),
    "gpum_b200_session_recorded": (C.c_int, [C.c_void_p, _f32p, _f64p, C.c_uint64,
                                             C.POINTER(C.c_uint64), _errp, _sz]),
    "gpum_b200_session_train_surrogate": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32,
                                                    C.c_int, C.c_uint32, _u32p, _f64p, _f32p,
                                                    _f64p, _errp, _sz]),
    "gpum_b200_session_run_da": (C.c_int, [C.c_void_p, C.c_void_p, _f64p, _f64p, _f64p,
                                           C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                           C.c_double, C.c_double, _f64p, _sz, C.c_int, _f32p,
                                           _f32p, _f64p, _u32p, _errp, _sz]),
}

_lib = None
_lock = threading.Lock()


def load(path: str = LIB_PATH):
    """Load the library (once) and bind every declared symbol."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(path):
                raise BackendUnavailable(
                    f"{path} is not built; run `python -m gpumetropolis_b200.build`")
            try:
                lib = C.CDLL(path)
            except OSError as e:
                raise BackendUnavailable(f"cannot load {path}: {e}") from e
            for name, (res, args) in SIGNATURES.items():
                f = getattr(lib, name)
                f.restype = res
                f.argtypes = args
            _lib = lib
    return _lib


def available() -> bool:
    try:
        return bool(load().gpum_b200_available())
    except BackendUnavailable:
        return False


def _p(a, ctype):
    return None if a is None else a.ctypes.data_as(C.POINTER(ctype))


def _u32(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.int64).astype(np.uint32)).reshape(-1)
    return a


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64).reshape(-1)


def _check(rc: int, err) -> None:
    if rc != OK:
        raise GpumError(rc, err.value.decode(errors="replace"))


def validate_program(code, n_consts, n_params, n_cols, allow_data=True) -> int:
    code = _u32(code)
    err = C.create_string_buffer(_ERRLEN)
    depth = C.c_int(0)
    _check(load().gpum_b200_validate_program(_p(code, C.c_uint32), code.size, n_consts,
                                             n_params, n_cols, int(allow_data),
                                             C.byref(depth), err, _ERRLEN), err)
    return depth.value


def _out_f32(out, n):
    """A contiguous float32 array of at least max(n, 1) values: `out` itself
    when given (checked), else a new one."""
    if out is None:
        return np.empty(max(n, 1), np.float32)
    if not (isinstance(out, np.ndarray) and out.dtype == np.float32 and out.ndim == 1
            and out.flags.c_contiguous and out.size >= max(n, 1)):
        raise ValueError(f"out_draws must be a contiguous 1-D float32 array of >= {max(n, 1)} "
                         "values")
    return out


def run(code, consts, prior_code, prior_consts, n_params, data, n_cols, n_obs, init,
        proposal_sd, temperatures, n_iter, seed, proposal_mode, gamma=0.0, de_noise=0.0,
        proposal_l=None, out_draws=None):
    """One-shot sampler (``gpum_b200_run``); host arrays in, host arrays out
    (`out_draws`: optional float32 array receiving the draws)."""
    code, pcode = _u32(code), _u32(prior_code)
    consts, pconsts = _f64(consts), _f64(prior_consts)
    data, init = _f64(data), _f64(init)
    sd, temps = _f64(proposal_sd), _f64(temperatures)
    n_chains = init.size // n_params
    L = None if proposal_l is None or np.size(proposal_l) == 0 else _f64(proposal_l)
    draws = _out_f32(out_draws, n_iter * n_chains * n_params)
    acc = np.empty(n_chains, np.float32)
    last = np.empty(n_chains, np.float64)
    err = C.create_string_buffer(_ERRLEN)
    rc = load().gpum_b200_run(
        _p(code, C.c_uint32), code.size, _p(consts, C.c_double), consts.size,
        _p(pcode, C.c_uint32), pcode.size, _p(pconsts, C.c_double), pconsts.size, n_params,
        _p(data, C.c_double), n_cols, n_obs, _p(init, C.c_double), _p(sd, C.c_double),
        _p(temps, C.c_double), n_chains, n_iter, seed & 0xFFFFFFFF, proposal_mode, gamma,
        de_noise, _p(L, C.c_double), 0 if L is None else L.size, _p(draws, C.c_float),
        _p(acc, C.c_float), _p(last, C.c_double), err, _ERRLEN)
    _check(rc, err)
    return draws[: n_iter * n_chains * n_params], acc, last


def run_de_sync(code, consts, prior_code, prior_consts, n_params, data, n_cols, n_obs, init,
                proposal_sd, n_iter, seed, gamma, de_noise):
    """One-shot path-B DE (``gpum_b200_run_de_sync``, the argument order of
    ``rust_gpu_metropolis_de_sync``'s inputs)."""
    code, pcode = _u32(code), _u32(prior_code)
    consts, pconsts = _f64(consts), _f64(prior_consts)
    data, init, sd = _f64(data), _f64(init), _f64(proposal_sd)
    n_chains = init.size // n_params
    draws = np.empty(max(n_iter * n_chains * n_params, 1), np.float32)
    acc = np.empty(n_chains, np.float32)
    last = np.empty(n_chains, np.float64)
    err = C.create_string_buffer(_ERRLEN)
    rc = load().gpum_b200_run_de_sync(
        _p(code, C.c_uint32), code.size, _p(consts, C.c_double), consts.size, n_params,
        _p(data, C.c_double), n_cols, n_obs, _p(pcode, C.c_uint32), pcode.size,
        _p(pconsts, C.c_double), pconsts.size, _p(init, C.c_double), _p(sd, C.c_double),
        n_chains, n_iter, seed & 0xFFFFFFFF, float(gamma), float(de_noise),
        _p(draws, C.c_float), _p(acc, C.c_float), _p(last, C.c_double), err, _ERRLEN)
    _check(rc, err)
    return draws[: n_iter * n_chains * n_params], acc, last


def _batch(fname, code, consts, n_params, data, n_cols, n_obs, points, width):
    code, consts, data, pts = _u32(code), _f64(consts), _f64(data), _f64(points)
    n_points = pts.size // n_params
    out = np.empty(max(n_points * width, 1), np.float64)
    err = C.create_string_buffer(_ERRLEN)
    rc = getattr(load(), fname)(_p(code, C.c_uint32), code.size, _p(consts, C.c_double),
                                consts.size, n_params, _p(data, C.c_double), n_cols, n_obs,
                                _p(pts, C.c_double), n_points, _p(out, C.c_double), err,
                                _ERRLEN)
    _check(rc, err)
    return out[: n_points * width]


def loglik_batch(code, consts, n_params, data, n_cols, n_obs, points):
    return _batch("gpum_b200_loglik_batch", code, consts, n_params, data, n_cols, n_obs,
                  points, 1)


def loglik_pointwise(code, consts, n_params, data, n_cols, n_obs, points):
    return _batch("gpum_b200_loglik_pointwise", code, consts, n_params, data, n_cols, n_obs,
                  points, n_obs)


def grad_batch(code, consts, n_params, data, n_cols, n_obs, points):
    """Point-major gradient of the data term (``gpum_b200_grad_batch``)."""
    return _batch("gpum_b200_grad_batch", code, consts, n_params, data, n_cols, n_obs,
                  points, n_params)


def compile_check(code, consts, prior_code, prior_consts, n_params, n_cols) -> int:
    """NVRTC-build the compiled engine for a model (no GPU needed); returns
    the module size in bytes."""
    code, pcode = _u32(code), _u32(prior_code)
    consts, pconsts = _f64(consts), _f64(prior_consts)
    nbytes = C.c_size_t(0)
    err = C.create_string_buffer(8192)
    _check(load().gpum_b200_compile_check(
        _p(code, C.c_uint32), code.size, _p(consts, C.c_double), consts.size,
        _p(pcode, C.c_uint32), pcode.size, _p(pconsts, C.c_double), pconsts.size, n_params,
        n_cols, C.byref(nbytes), err, 8192), err)
    return nbytes.value


class Session:
    """A model + data resident on the GPU (``gpum_b200_session_*``)."""

    def __init__(self, code, consts, prior_code, prior_consts, n_params, data, n_cols, n_obs,
                 engine=ENGINE_AUTO):
        self._lib = load()
        code, pcode = _u32(code), _u32(prior_code)
        consts, pconsts = _f64(consts), _f64(prior_consts)
        data = _f64(data)
        self.n_params, self.n_cols, self.n_obs = n_params, n_cols, n_obs
        h = C.c_void_p()
        err = C.create_string_buffer(_ERRLEN)
        rc = self._lib.gpum_b200_session_create(
            _p(code, C.c_uint32), code.size, _p(consts, C.c_double), consts.size,
            _p(pcode, C.c_uint32), pcode.size, _p(pconsts, C.c_double), pconsts.size,
            n_params, _p(data, C.c_double), n_cols, n_obs, C.byref(h), err, _ERRLEN)
        _check(rc, err)
        self._h = h
        self.n_chains = 0
        if engine != ENGINE_AUTO:
            self.set_engine(engine)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gpum_b200_session_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def launches(self) -> int:
        return int(self._lib.gpum_b200_session_launches(self._h))

    @property
    def stream(self) -> int:
        """The session's cudaStream_t as an integer handle."""
        return int(self._lib.gpum_b200_session_stream(self._h) or 0)

    def run(self, init, proposal_sd, temperatures, n_iter, seed, proposal_mode, gamma=0.0,
            de_noise=0.0, proposal_l=None, rng=RNG_TRIPLE32, out_draws=None):
        """One run of n_iter iterations.  `out_draws` (optional): a float32 array
        of at least n_iter * n_chains * n_params values that receives the draws
        (e.g. pinned memory allocated once)."""
        init, sd, temps = _f64(init), _f64(proposal_sd), _f64(temperatures)
        n_chains = self.n_chains = init.size // self.n_params
        L = None if proposal_l is None or np.size(proposal_l) == 0 else _f64(proposal_l)
        draws = _out_f32(out_draws, n_iter * n_chains * self.n_params)
        acc = np.empty(n_chains, np.float32)
        last = np.empty(n_chains, np.float64)
        err = C.create_string_buffer(_ERRLEN)
        rc = self._lib.gpum_b200_session_run(
            self._h, _p(init, C.c_double), _p(sd, C.c_double), _p(temps, C.c_double), n_chains,
            n_iter, seed & 0xFFFFFFFF, proposal_mode, gamma, de_noise, _p(L, C.c_double),
            0 if L is None else L.size, rng, _p(draws, C.c_float), _p(acc, C.c_float),
            _p(last, C.c_double), err, _ERRLEN)
        _check(rc, err)
        return draws[: n_iter * n_chains * self.n_params], acc, last

    def run_de_sync(self, init, proposal_sd, n_iter, seed, gamma, de_noise, rng=RNG_TRIPLE32):
        """Per-generation DE (path B).  Returns (draws, accept, last_logpost)."""
        init, sd = _f64(init), _f64(proposal_sd)
        n_chains = self.n_chains = init.size // self.n_params
        draws = np.empty(max(n_iter * n_chains * self.n_params, 1), np.float32)
        acc = np.empty(n_chains, np.float32)
        last = np.empty(n_chains, np.float64)
        err = C.create_string_buffer(_ERRLEN)
        rc = self._lib.gpum_b200_session_run_de_sync(
            self._h, _p(init, C.c_double), _p(sd, C.c_double), n_chains, n_iter,
            seed & 0xFFFFFFFF, float(gamma), float(de_noise), rng, _p(draws, C.c_float),
            _p(acc, C.c_float), _p(last, C.c_double), err, _ERRLEN)
        _check(rc, err)
        return draws[: n_iter * n_chains * self.n_params], acc, last

    def set_exchange(self, ladder_len=0, swap_every=1):
        """Device replica exchange for later runs (ladder_len 0: off)."""
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_session_set_exchange(self._h, int(ladder_len),
                                                        int(swap_every), err, _ERRLEN), err)

    def exchange_stats(self):
        """(attempts (C,), accepted (C,), n_exchanges) of the prepared run."""
        att = np.zeros(self.n_chains, np.uint32)
        acc = np.zeros(self.n_chains, np.uint32)
        n = np.zeros(1, np.uint32)
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_session_exchange_stats(
            self._h, _p(att, C.c_uint32), _p(acc, C.c_uint32), _p(n, C.c_uint32), err,
            _ERRLEN), err)
        return att, acc, int(n[0])

    def draw_moments(self, t0, n):
        """(chain_mean (C, np), chain_m2 (C, np), pool_mean (np,), pool_m2 (np, np)) of
        the draws of iterations [t0, t0 + n) of the prepared run."""
        nc, d = self.n_chains, self.n_params
        cm, c2 = np.empty((nc, d)), np.empty((nc, d))
        pm, p2 = np.empty(d), np.empty((d, d))
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_session_draw_moments(
            self._h, int(t0), int(n), _p(cm, C.c_double), _p(c2, C.c_double),
            _p(pm, C.c_double), _p(p2, C.c_double), err, _ERRLEN), err)
        return cm, c2, pm, p2

    def selftest_wait(self, polls=1024):
        """Run the bounded-wait self-test (a wait that must run out); raises
        GpumError with code ERR_DEVICE, as a run whose device wait ran out."""
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_session_selftest_wait(self._h, int(polls), err, _ERRLEN), err)

    def state(self):
        """Current chain states (C, np)."""
        out = np.empty((self.n_chains, self.n_params))
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_session_state(self._h, _p(out, C.c_double), err, _ERRLEN),
               err)
        return out

    def set_likelihood_powers(self, beta=None):
        """Per-chain likelihood powers for later runs (None clears)."""
        err = C.create_string_buffer(_ERRLEN)
        if beta is None:
            _check(self._lib.gpum_b200_session_set_likelihood_powers(self._h, None, 0, err,
                                                                     _ERRLEN), err)
            return
        b = _f64(beta)
        _check(self._lib.gpum_b200_session_set_likelihood_powers(
            self._h, _p(b, C.c_double), b.size, err, _ERRLEN), err)

    def record(self, capacity):
        """Store the (theta, log-likelihood) pair of every exactly evaluated
        proposal of later exact runs, up to `capacity` pairs (0: off)."""
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_session_record(self._h, int(capacity), err, _ERRLEN), err)

    def recorded(self):
        """The recorded pairs: (theta float32 n x n_params, ll float64 n)."""
        n = C.c_uint64(0)
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_session_recorded(self._h, None, None, 0, C.byref(n), err,
                                                    _ERRLEN), err)
        theta = np.empty((max(n.value, 1), self.n_params), np.float32)
        ll = np.empty(max(n.value, 1), np.float64)
        _check(self._lib.gpum_b200_session_recorded(
            self._h, _p(theta, C.c_float), _p(ll, C.c_double), n.value, C.byref(n), err,
            _ERRLEN), err)
        return theta[: n.value], ll[: n.value]

    def recorded_count(self) -> int:
        """Pairs recorded so far."""
        n = C.c_uint64(0)
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_session_recorded(self._h, None, None, 0, C.byref(n), err,
                                                    _ERRLEN), err)
        return int(n.value)

    def train_surrogate(self, surrogate, stages, holdout_every=10, whiten=True):
        """Fit `surrogate` (a Surrogate with d = n_params) to the recorded
        pairs on the device: every `holdout_every`-th pair held out, the
        normaliser from the training pairs' moments (whitened inputs with
        `whiten`), Adam over `stages` [(steps, lr), ...].  Returns (losses,
        info) with info = {pairs, train_pairs, holdout_pairs,
        holdout_resid_sd, whitened}."""
        steps = np.ascontiguousarray([int(k) for k, _ in stages], dtype=np.uint32)
        lrs = np.ascontiguousarray([float(r) for _, r in stages], dtype=np.float64)
        total = int(steps.sum())
        losses = np.empty(max(total, 1), np.float32)
        info = np.full(5, np.nan)
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_session_train_surrogate(
            self._h, surrogate._h, int(holdout_every), int(bool(whiten)), steps.size,
            _p(steps, C.c_uint32), _p(lrs, C.c_double), _p(losses, C.c_float),
            _p(info, C.c_double), err, _ERRLEN), err)
        return losses[:total], {"pairs": int(info[0]), "train_pairs": int(info[1]),
                                "holdout_pairs": int(info[2]),
                                "holdout_resid_sd": float(info[3]),
                                "whitened": bool(info[4])}

    def run_da(self, surrogate, init, proposal_sd, temperatures, n_iter, seed, proposal_mode,
               gamma=0.0, de_noise=0.0, proposal_l=None, rng=RNG_TRIPLE32, out_draws=None):
        """Delayed-acceptance run with `surrogate` (a Surrogate) as stage 1.
        Returns (draws, accept, last_logpost, exact_evals per chain); `out_draws`
        as for run()."""
        init, sd, temps = _f64(init), _f64(proposal_sd), _f64(temperatures)
        n_chains = self.n_chains = init.size // self.n_params
        L = None if proposal_l is None or np.size(proposal_l) == 0 else _f64(proposal_l)
        draws = _out_f32(out_draws, n_iter * n_chains * self.n_params)
        acc = np.empty(n_chains, np.float32)
        last = np.empty(n_chains, np.float64)
        exact = np.empty(n_chains, np.uint32)
        err = C.create_string_buffer(_ERRLEN)
        rc = self._lib.gpum_b200_session_run_da(
            self._h, surrogate._h, _p(init, C.c_double), _p(sd, C.c_double),
            _p(temps, C.c_double), n_chains, n_iter, seed & 0xFFFFFFFF, proposal_mode, gamma,
            de_noise, _p(L, C.c_double), 0 if L is None else L.size, rng, _p(draws, C.c_float),
            _p(acc, C.c_float), _p(last, C.c_double), _p(exact, C.c_uint32), err, _ERRLEN)
        _check(rc, err)
        return draws[: n_iter * n_chains * self.n_params], acc, last, exact

    def prepare(self, init, proposal_sd, temperatures, max_iter, seed, proposal_mode,
                gamma=0.0, de_noise=0.0, proposal_l=None, rng=RNG_TRIPLE32):
        init, sd, temps = _f64(init), _f64(proposal_sd), _f64(temperatures)
        self.n_chains = init.size // self.n_params
        L = None if proposal_l is None or np.size(proposal_l) == 0 else _f64(proposal_l)
        err = C.create_string_buffer(_ERRLEN)
        rc = self._lib.gpum_b200_session_prepare(
            self._h, _p(init, C.c_double), _p(sd, C.c_double), _p(temps, C.c_double),
            self.n_chains, max_iter, seed & 0xFFFFFFFF, proposal_mode, gamma, de_noise,
            _p(L, C.c_double), 0 if L is None else L.size, rng, err, _ERRLEN)
        _check(rc, err)

    def advance(self, n_iter):
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_session_advance(self._h, n_iter, err, _ERRLEN), err)

    def sync(self):
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_session_sync(self._h, err, _ERRLEN), err)

    def fetch(self, want_draws=True):
        n = C.c_uint32(0)
        err = C.create_string_buffer(_ERRLEN)
        # First call learns n_done without copying draws.
        _check(self._lib.gpum_b200_session_fetch(self._h, None, None, None, C.byref(n), err,
                                                 _ERRLEN), err)
        nd = n.value
        draws = np.empty(max(nd * self.n_chains * self.n_params, 1), np.float32)
        acc = np.empty(self.n_chains, np.float32)
        last = np.empty(self.n_chains, np.float64)
        _check(self._lib.gpum_b200_session_fetch(
            self._h, _p(draws, C.c_float) if want_draws else None, _p(acc, C.c_float),
            _p(last, C.c_double), C.byref(n), err, _ERRLEN), err)
        return draws[: nd * self.n_chains * self.n_params], acc, last, nd

    def loglik_batch(self, points):
        pts = _f64(points)
        n = pts.size // self.n_params
        out = np.empty(max(n, 1))
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_session_loglik_batch(self._h, _p(pts, C.c_double), n,
                                                        _p(out, C.c_double), err, _ERRLEN), err)
        return out[:n]

    def set_engine(self, engine: int):
        err = C.create_string_buffer(8192)
        _check(self._lib.gpum_b200_session_set_engine(self._h, engine, err, 8192), err)

    @property
    def engine(self) -> int:
        return int(self._lib.gpum_b200_session_engine(self._h))

    @property
    def tensor_cores(self) -> bool:
        """Whether sums and value-only steps run the tensor-core value kernel."""
        return self._lib.gpum_b200_session_tensor_cores(self._h) == 1

    def grad_batch(self, points):
        pts = _f64(points)
        n = pts.size // self.n_params
        out = np.empty(max(n * self.n_params, 1))
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_session_grad_batch(self._h, _p(pts, C.c_double), n,
                                                      _p(out, C.c_double), err, _ERRLEN), err)
        return out[: n * self.n_params]

    def loglik_pointwise(self, points):
        pts = _f64(points)
        n = pts.size // self.n_params
        out = np.empty(max(n * self.n_obs, 1))
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_session_loglik_pointwise(self._h, _p(pts, C.c_double), n,
                                                            _p(out, C.c_double), err, _ERRLEN),
               err)
        return out[: n * self.n_obs]


def gemm_check(A, B):
    """C = bf16(A) . bf16(B)^T through the tcgen05 GEMM (test hook)."""
    A = np.ascontiguousarray(A, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float32)
    M, K = A.shape
    N = B.shape[0]
    out = np.empty((M, N), np.float32)
    err = C.create_string_buffer(_ERRLEN)
    _check(load().gpum_b200_mlp_gemm_check(M, N, K, _p(A, C.c_float), _p(B, C.c_float),
                                           _p(out, C.c_float), err, _ERRLEN), err)
    return out


class Surrogate:
    """The d-H-H-1 SiLU MLP surrogate trained on the GPU (``gpum_b200_mlp_*``)."""

    def __init__(self, d, hidden=256, batch=4096, seed=1):
        self._lib = load()
        h = C.c_void_p()
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_mlp_create(d, hidden, batch, seed, C.byref(h), err,
                                              _ERRLEN), err)
        self._h = h
        self.d, self.hidden, self.batch = d, hidden, batch
        self.dp = (d + 63) // 64 * 64
        self.n_params = hidden * self.dp + hidden + hidden * hidden + hidden + hidden + 1

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gpum_b200_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_normalizer(self, xmean, xsd, ymean, ysd):
        xm, xs = _f64(xmean), _f64(xsd)
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_mlp_set_normalizer(self._h, _p(xm, C.c_double),
                                                      _p(xs, C.c_double), float(ymean),
                                                      float(ysd), err, _ERRLEN), err)

    def set_whitening(self, xmean, xw, ymean, ysd):
        xm, w = _f64(xmean), _f64(xw)
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_mlp_set_whitening(self._h, _p(xm, C.c_double),
                                                     _p(w, C.c_double), float(ymean),
                                                     float(ysd), err, _ERRLEN), err)

    def fit_normalizer(self, theta, ll, whiten=False):
        """Standardise the target; inputs per coordinate, or (``whiten``)
        by the inverse Cholesky factor of their covariance."""
        theta = np.asarray(theta, dtype=np.float64).reshape(-1, self.d)
        ysd = float(np.std(ll)) or 1.0
        if whiten and self.d > 1:
            cov = np.cov(theta, rowvar=False)
            cov = cov + np.eye(self.d) * 1e-10 * max(float(np.mean(np.diag(cov))), 1e-300)
            try:
                Linv = np.linalg.inv(np.linalg.cholesky(cov))
            except np.linalg.LinAlgError:
                pass
            else:
                self.set_whitening(theta.mean(axis=0), Linv, float(np.mean(ll)), ysd)
                return
        sd = theta.std(axis=0)
        sd = np.where(sd > 0, sd, 1.0)
        self.set_normalizer(theta.mean(axis=0), sd, float(np.mean(ll)), ysd)

    def train(self, theta, ll, steps, lr=1e-3):
        th, y = _f64(theta), _f64(ll)
        losses = np.empty(max(steps, 1), np.float32)
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_mlp_train(self._h, _p(th, C.c_double), _p(y, C.c_double),
                                             y.size, steps, lr, _p(losses, C.c_float), err,
                                             _ERRLEN), err)
        return losses[:steps]

    def train_stages(self, theta, ll, stages):
        """Adam on the pairs with a learning-rate schedule, ``stages`` a list of
        (steps, lr); the pairs are uploaded once.  Returns every step's loss."""
        th, y = _f64(theta), _f64(ll)
        steps = np.ascontiguousarray([int(s) for s, _ in stages], dtype=np.uint32)
        lrs = np.ascontiguousarray([float(r) for _, r in stages], dtype=np.float64)
        total = int(steps.sum())
        losses = np.empty(max(total, 1), np.float32)
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_mlp_train_stages(
            self._h, _p(th, C.c_double), _p(y, C.c_double), y.size, steps.size,
            _p(steps, C.c_uint32), _p(lrs, C.c_double), _p(losses, C.c_float), err, _ERRLEN),
            err)
        return losses[:total]

    def predict(self, theta):
        th = _f64(theta)
        n = th.size // self.d
        out = np.empty(max(n, 1))
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_mlp_predict(self._h, _p(th, C.c_double), n,
                                               _p(out, C.c_double), err, _ERRLEN), err)
        return out[:n]

    def predict_grad(self, theta):
        """(log-likelihood (n,), gradient with respect to the parameters
        (n, d)) at n points: the drift of the Langevin delayed-acceptance
        proposal."""
        th = _f64(theta)
        n = th.size // self.d
        out = np.empty(max(n, 1))
        grad = np.empty(max(n * self.d, 1))
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_mlp_predict_grad(self._h, _p(th, C.c_double), n,
                                                    _p(out, C.c_double), _p(grad, C.c_double),
                                                    err, _ERRLEN), err)
        return out[:n], grad[:n * self.d].reshape(n, self.d)

    def gradients(self, theta, ll):
        th, y = _f64(theta), _f64(ll)
        g = np.empty(self.n_params, np.float32)
        loss = np.zeros(1, np.float32)
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_mlp_gradients(self._h, _p(th, C.c_double),
                                                 _p(y, C.c_double), y.size, _p(g, C.c_float),
                                                 _p(loss, C.c_float), err, _ERRLEN), err)
        return g, float(loss[0])

    def params(self):
        out = np.empty(self.n_params, np.float32)
        err = C.create_string_buffer(_ERRLEN)
        _check(self._lib.gpum_b200_mlp_get_params(self._h, _p(out, C.c_float), err, _ERRLEN),
               err)
        return out
