"""Model DSL: one-sided formulas compiled to gpumetropolis stack-machine bytecode.

This restates the reference's expression compiler (``R/dsl.R:13-134``) and its
model constructor (``R/api.R:87-116``) so that a ``gpum_model`` built here emits
exactly the bytecode the reference emits for the same formula:

* opcodes ``R/dsl.R:13-17`` (PUSH_CONST 0, PUSH_PARAM 1, PUSH_DATA 2, ADD 3,
  SUB 4, MUL 5, DIV 6, NEG 7, EXP 8, LOG 9, SQRT 10, POW 11, LGAMMA 12);
* postfix emission with (opcode, arg) pairs, binary ops carrying arg 0
  (``R/dsl.R:38-40,68-73``);
* a constant pool deduplicated by exact equality, first hit wins
  (``R/dsl.R:41-46``);
* peak stack depth tracked per push and checked against 32 (``R/dsl.R:20,
  34-37,115-119``).

Formulas are R source text (``"~ -((y - mu)^2) / 8"``), parsed with R's
operator precedence: ``^`` (right associative, binds tighter than unary minus),
then unary minus, then ``* /``, then ``+ -``.  Unary plus and any function
other than exp/log/sqrt/lgamma are rejected, as the reference rejects them.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Union

import numpy as np

OP = {
    "PUSH_CONST": 0, "PUSH_PARAM": 1, "PUSH_DATA": 2,
    "ADD": 3, "SUB": 4, "MUL": 5, "DIV": 6, "NEG": 7,
    "EXP": 8, "LOG": 9, "SQRT": 10, "POW": 11, "LGAMMA": 12,
}
STACK_SIZE = 32

_UNARY_FN = {"exp": OP["EXP"], "log": OP["LOG"], "sqrt": OP["SQRT"],
             "lgamma": OP["LGAMMA"]}


class DSLError(ValueError):
    """A formula the compiler refuses (the reference raises an R error)."""


# ---------------------------------------------------------------- parsing
@dataclass
class Num:
    value: float


@dataclass
class Sym:
    name: str


@dataclass
class Call:
    fn: str
    args: List["Node"] = field(default_factory=list)


Node = Union[Num, Sym, Call]

_TOKEN = re.compile(r"""
    (?P<ws>\s+)
  | (?P<num>(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?L?)
  | (?P<name>[A-Za-z.][A-Za-z0-9._]*)
  | (?P<op>[-+*/^(),~])
""", re.VERBOSE)


def _tokenize(src: str):
    pos, out = 0, []
    while pos < len(src):
        m = _TOKEN.match(src, pos)
        if not m:
            raise DSLError(f"cannot parse the log-density near: {src[pos:pos+12]!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        out.append((kind, m.group(kind)))
    out.append(("end", ""))
    return out


class _Parser:
    """Recursive descent over R's arithmetic grammar (``?Syntax``)."""

    def __init__(self, src: str):
        self.toks = _tokenize(src)
        self.i = 0

    def peek(self):
        return self.toks[self.i]

    def take(self, kind=None, val=None):
        tok = self.toks[self.i]
        if (kind and tok[0] != kind) or (val is not None and tok[1] != val):
            raise DSLError(f"unexpected token {tok[1]!r} in the log-density")
        self.i += 1
        return tok

    def parse(self) -> Node:
        node = self.sum()
        if self.peek()[0] != "end":
            raise DSLError(f"unexpected token {self.peek()[1]!r} in the log-density")
        return node

    def sum(self) -> Node:
        node = self.product()
        while self.peek() in (("op", "+"), ("op", "-")):
            op = self.take()[1]
            node = Call(op, [node, self.product()])
        return node

    def product(self) -> Node:
        node = self.unary()
        while self.peek() in (("op", "*"), ("op", "/")):
            op = self.take()[1]
            node = Call(op, [node, self.unary()])
        return node

    def unary(self) -> Node:
        if self.peek() in (("op", "-"), ("op", "+")):
            op = self.take()[1]
            return Call(op, [self.unary()])
        return self.power()

    def power(self) -> Node:
        base = self.primary()
        if self.peek() == ("op", "^"):
            self.take()
            return Call("^", [base, self.unary()])
        return base

    def primary(self) -> Node:
        kind, val = self.peek()
        if kind == "num":
            self.take()
            return Num(float(val.rstrip("L")))
        if kind == "name":
            self.take()
            if self.peek() == ("op", "("):
                self.take()
                args = []
                if self.peek() != ("op", ")"):
                    args.append(self.sum())
                    while self.peek() == ("op", ","):
                        self.take()
                        args.append(self.sum())
                self.take("op", ")")
                return Call(val, args)
            return Sym(val)
        if (kind, val) == ("op", "("):
            self.take()
            inner = self.sum()
            self.take("op", ")")
            return Call("(", [inner])
        raise DSLError(f"unexpected token {val!r} in the log-density")


def rhs(formula: str) -> Node:
    """Right-hand side of a one-sided formula ``"~ expr"`` (``R/dsl.R:126-134``)."""
    if not isinstance(formula, str):
        raise DSLError("expected a one-sided formula such as `~ expr`.")
    text = formula.strip()
    if not text.startswith("~"):
        raise DSLError("expected a one-sided formula such as `~ expr`.")
    return _Parser(text[1:]).parse()


# -------------------------------------------------------------- emission
@dataclass
class Program:
    """Compiled bytecode: flat (opcode, arg) u32 pairs, constant pool, depth."""
    code: np.ndarray
    consts: np.ndarray
    depth: int

    @property
    def n_instr(self) -> int:
        return len(self.code) // 2


def compile_expr(expr: Node, params: Sequence[str], data: Sequence[str]) -> Program:
    """Emit postfix bytecode for one expression (``R/dsl.R:28-122``)."""
    params, data = list(params), list(data)
    consts: List[float] = []
    code: List[int] = []
    depth = 0
    max_depth = 0

    def push_depth(delta):
        nonlocal depth, max_depth
        depth += delta
        max_depth = max(max_depth, depth)

    def const_index(v: float) -> int:
        for i, c in enumerate(consts):
            if c == v:
                return i
        consts.append(v)
        return len(consts) - 1

    def emit(node: Node):
        if isinstance(node, Num):
            code.extend((OP["PUSH_CONST"], const_index(float(node.value))))
            push_depth(1)
        elif isinstance(node, Sym):
            if node.name in params:
                code.extend((OP["PUSH_PARAM"], params.index(node.name)))
            elif node.name in data:
                code.extend((OP["PUSH_DATA"], data.index(node.name)))
            else:
                raise DSLError(f"unknown symbol in the log-density: '{node.name}'. "
                               "Declare it in `params` or `data`.")
            push_depth(1)
        else:
            fn, args = node.fn, node.args

            def binary(op):
                emit(args[0])
                emit(args[1])
                code.extend((op, 0))
                push_depth(-1)

            if fn == "(":
                emit(args[0])
            elif fn == "+" and len(args) == 2:
                binary(OP["ADD"])
            elif fn == "-" and len(args) == 2:
                binary(OP["SUB"])
            elif fn == "-" and len(args) == 1:
                emit(args[0])
                code.extend((OP["NEG"], 0))
            elif fn == "*" and len(args) == 2:
                binary(OP["MUL"])
            elif fn == "/" and len(args) == 2:
                binary(OP["DIV"])
            elif fn == "^" and len(args) == 2:
                binary(OP["POW"])
            elif fn in _UNARY_FN:
                if len(args) != 1:
                    raise DSLError(f"`{fn}` takes one argument in the log-density.")
                emit(args[0])
                code.extend((_UNARY_FN[fn], 0))
            else:
                raise DSLError(f"unsupported function in the log-density: '{fn}'. "
                               "Supported: + - * / ^ exp log sqrt lgamma.")

    emit(expr)
    if max_depth > STACK_SIZE:
        raise DSLError("the log-density expression is too deep for the interpreter "
                       f"(needs {max_depth} stack slots, limit {STACK_SIZE}).")
    return Program(np.asarray(code, dtype=np.uint32),
                   np.asarray(consts, dtype=np.float64), max_depth)


def empty_program() -> Program:
    return Program(np.zeros(0, np.uint32), np.zeros(0, np.float64), 0)


@dataclass
class GpumModel:
    """A compiled model (``R/api.R:87-116``): loglik + prior programs."""
    loglik: Program
    prior: Program
    params: List[str]
    data: List[str]

    @property
    def n_params(self) -> int:
        return len(self.params)

    @property
    def n_cols(self) -> int:
        return len(self.data)

    def __repr__(self) -> str:
        prior = (f"{self.prior.n_instr} instructions" if self.prior.n_instr else "flat")
        return (f"<gpum_model>\n  parameters : {', '.join(self.params)}\n"
                f"  data       : {', '.join(self.data) if self.data else '(none)'}\n"
                f"  loglik     : {self.loglik.n_instr} bytecode instructions\n"
                f"  prior      : {prior}")


def gpum_model(loglik: str, params, data=(), prior: Optional[str] = None) -> GpumModel:
    """Declare a model from one-sided formulas (``R/api.R:87-116``)."""
    if not isinstance(loglik, str) or not loglik.strip().startswith("~"):
        raise DSLError("`loglik` must be a one-sided formula such as `~ expr`.")
    params = [params] if isinstance(params, str) else [str(p) for p in params]
    data = [data] if isinstance(data, str) else [str(d) for d in data]
    if len(params) < 1:
        raise DSLError("`params` must name at least one parameter.")
    if len(set(params + data)) != len(params + data):
        raise DSLError("parameter and data names must be distinct.")
    ll = compile_expr(rhs(loglik), params, data)
    if prior is None:
        pr = empty_program()
    else:
        if not isinstance(prior, str) or not prior.strip().startswith("~"):
            raise DSLError("`prior` must be a one-sided formula or NULL.")
        pr = compile_expr(rhs(prior), params, [])
    return GpumModel(ll, pr, params, data)


def _fmt(v: float) -> str:
    if v == int(v) and abs(v) < 1e15:
        return str(int(v))
    return repr(float(v))


def linear_predictor(coefs: Sequence[str], covariates: Sequence[Optional[str]]) -> str:
    """Text of ``c0*x0 + c1*x1 + ...`` as a user writes it; a ``None``
    covariate is an intercept term (coefficient alone)."""
    terms = []
    for c, x in zip(coefs, covariates):
        terms.append(c if x is None else f"{c} * {x}")
    return " + ".join(terms)


def gaussian_prior(params: Sequence[str], sd: float, mean: float = 0.0) -> str:
    """``-p^2/(2 sd^2)`` summed over ``params`` (a user's N(mean, sd^2) prior)."""
    inv = 1.0 / (2.0 * sd * sd)
    terms = []
    for p in params:
        core = p if mean == 0 else f"({p} - {_fmt(mean)})"
        terms.append(f"{_fmt(inv)} * {core}^2")
    return "~ -(" + " + ".join(terms) + ")"


__all__ = ["OP", "STACK_SIZE", "DSLError", "Program", "GpumModel", "gpum_model",
           "compile_expr", "rhs", "empty_program", "linear_predictor", "gaussian_prior"]

