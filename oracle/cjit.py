"""Bytecode -> C -> gcc -> dlopen: the CPU compiled log-likelihood -- TEST AND CPU-BASELINE ONLY.

Restates the reference's Cranelift JIT (``src/rust/src/jit.rs:441-631``): the
per-observation program becomes straight-line f64 code inside the loop over
observations, summed sequentially, with libm ``exp``/``log``/``pow`` and the
oracle's Lanczos ``gpo_lgamma`` for the opcodes the JIT sends to shims
(``jit.rs:22-36``).  Compiled with ``-ffp-contract=off`` so no multiply-add is
fused, as Cranelift emits none, and with ``-fno-builtin`` so ``pow``/``exp``/
``log`` stay libm calls as the reference's shims are.  It is the timed CPU baseline's evaluator and
is only used by tests and ``bench.py``'s CPU-baseline leg.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
import subprocess
import tempfile

import numpy as np

from . import oracle as _oracle

_HERE = os.path.dirname(os.path.abspath(__file__))
_CACHE = os.path.join(_HERE, "_build", "jit")
_keep = {}


def _gcc() -> str:
    return "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"


def _c_double(v: float) -> str:
    if np.isnan(v):
        return "(0.0/0.0)"
    if np.isinf(v):
        return "(1.0/0.0)" if v > 0 else "(-1.0/0.0)"
    return repr(float(v))


def emit_c(code, consts, absolute=False) -> str:
    """C source of ``double gpum_jit_loglik(params, data, n_obs, n_cols)``;
    with ``absolute`` it returns the sum of the per-observation values'
    absolute values instead (the scale of the sum's rounding error when the
    terms cancel)."""
    code = np.asarray(code, dtype=np.uint32).reshape(-1)
    n = code.size // 2
    lines = [
        "#include <math.h>",
        "#include <stdint.h>",
        "extern double gpo_lgamma(double);",
        "double gpum_jit_loglik(const double* p, const double* data, int64_t n_obs,"
        " int64_t n_cols) {",
        "  double acc = 0.0;",
        "  for (int64_t i = 0; i < n_obs; ++i) {",
        "    const double* row = data + i * n_cols;",
    ]
    stack = []
    for pc in range(n):
        op, arg = int(code[2 * pc]), int(code[2 * pc + 1])
        v = f"v{pc}"
        if op == 0:
            lines.append(f"    const double {v} = {_c_double(consts[arg])};")
        elif op == 1:
            lines.append(f"    const double {v} = p[{arg}];")
        elif op == 2:
            lines.append(f"    const double {v} = row[{arg}];")
        elif op in (7, 8, 9, 10, 12):
            x = stack.pop()
            expr = {7: f"-{x}", 8: f"exp({x})", 9: f"log({x})", 10: f"sqrt({x})",
                    12: f"gpo_lgamma({x})"}[op]
            lines.append(f"    const double {v} = {expr};")
        else:
            r, l = stack.pop(), stack.pop()
            expr = {3: f"{l} + {r}", 4: f"{l} - {r}", 5: f"{l} * {r}",
                    6: f"{l} / {r}"}.get(op, f"pow({l}, {r})")
            lines.append(f"    const double {v} = {expr};")
        stack.append(v)
    term = stack[0] if n else "0.0"
    lines.append(f"    acc += fabs({term});" if absolute else f"    acc += {term};")
    lines += ["  }", "  return acc;", "}"]
    return "\n".join(lines) + "\n"


def compile_loglik(code, consts, absolute=False):
    """Compile and load; returns a ctypes function pointer usable by
    :func:`oracle.oracle.run` (``jit=``) and :func:`oracle.oracle.jit_batch`
    (``absolute``: the sum of absolute per-observation values)."""
    src = emit_c(code, consts, absolute)
    key = hashlib.sha1(src.encode()).hexdigest()[:16]
    if key in _keep:
        return _keep[key][1]
    os.makedirs(_CACHE, exist_ok=True)
    so = os.path.join(_CACHE, f"jit_{key}.so")
    if not os.path.exists(so):
        ora_dir = os.path.dirname(_oracle.build() if not os.path.exists(_oracle._SO)
                                  else _oracle._SO)
        with tempfile.NamedTemporaryFile("w", suffix=".c", delete=False) as f:
            f.write(src)
            cpath = f.name
        tmp = so + f".{os.getpid()}.tmp"
        subprocess.run([_gcc(), "-O2", "-fPIC", "-shared", "-ffp-contract=off",
                        "-fno-builtin",
                        "-o", tmp, cpath, f"-L{ora_dir}", "-lgpum_oracle",
                        f"-Wl,-rpath,{ora_dir}", "-lm"], check=True)
        os.replace(tmp, so)
        os.unlink(cpath)
    _oracle.lib()  # gpo_lgamma must be resolvable
    dll = C.CDLL(so)
    fn = _oracle.LOGLIK_FN(("gpum_jit_loglik", dll))
    _keep[key] = (dll, fn)
    return fn
