"""Initial-condition expressions on the CPU (TEST INFRASTRUCTURE ONLY: the
checker of the library's compiled programs, never shipped or measured).

The reference evaluates each material's initial condition with exprtk
(UserExpression, user_expression.cpp) cell by cell in
PrimeStateInitializer::GetInitialPrimeStates
(initial_condition/prime_state_initializer.cpp:41-84) and non-dimensionalises
the values with its UnitHandler (unit_handler.cpp:45-46, 67-98). exprtk (the
"expression_toolkit" submodule of the reference, not vendored and without a
recoverable pinned commit) is restated here only for the subset of its
published language that ALPACA's input files use:

* statements ``name := e`` (also ``: =``), ``+= -= *= /= %=``, ``var name := e``,
  ``if (c) S [else S]``, blocks ``{ ... }``, expression statements;
* expressions ``c ? a : b``, ``if (c, a, b)``, ``or | ||``, ``and & &&``,
  ``not !``, comparisons (``==`` / ``!=`` with exprtk's floating-point
  equality, ``|a - b| <= 1e-10 max(1, |a|, |b|)``), ``+ - * / %``, unary signs,
  ``^`` (not chained), implicit multiplication after a number or ``)``;
* functions abs ... trunc, atan2 hypot pow logn root, variadic min max; pi,
  true, false; comments ``//``, ``#``, ``/* */``.

Truth values are doubles; ``and`` / ``or`` evaluate both sides.

This module is independent of the library's compiler: its own tokenizer and
parser build a syntax tree that is evaluated over numpy arrays with masks.
``run_listing`` interprets the library's compiled program text so that the
compiler can be checked without a GPU.
"""
from __future__ import annotations

import math
import re

import numpy as np

F1 = {
    "abs": np.abs, "acos": np.arccos, "acosh": np.arccosh, "asin": np.arcsin,
    "asinh": np.arcsinh, "atan": np.arctan, "atanh": np.arctanh, "cbrt": np.cbrt,
    "ceil": np.ceil, "cos": np.cos, "cosh": np.cosh, "exp": np.exp, "expm1": np.expm1,
    "floor": np.floor, "frac": lambda a: a - np.trunc(a), "log": np.log, "log10": np.log10,
    "log1p": np.log1p, "log2": np.log2,
    # C round: halves away from zero
    "round": lambda a: np.where(np.abs(a - np.trunc(a)) >= 0.5, np.trunc(a) + np.sign(a),
                                np.trunc(a)),
    "sgn": np.sign, "sin": np.sin, "sinh": np.sinh, "sqrt": np.sqrt, "tan": np.tan,
    "tanh": np.tanh, "trunc": np.trunc,
    "deg2rad": lambda a: a * (math.pi / 180.0), "rad2deg": lambda a: a * (180.0 / math.pi),
}
F2 = {
    "atan2": np.arctan2, "hypot": np.hypot, "pow": np.power,
    "logn": lambda a, b: np.log(a) / np.log(b), "root": lambda a, b: np.power(a, 1.0 / b),
}
KEYWORDS = {"if", "else", "var", "and", "or", "not", "true", "false"}
PRIMES = ("density", "velocityX", "velocityY", "velocityZ", "pressure")


class ExprError(ValueError):
    pass


_TOKEN = re.compile(r"""
    (?P<ws>\s+|//[^\n]*|\#[^\n]*|/\*.*?\*/)
  | (?P<num>(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?)
  | (?P<id>[A-Za-z_]\w*)
  | (?P<assign>:[ \t]*=(?!=))
  | (?P<op>\+=|-=|\*=|/=|%=|<=|>=|==|!=|<>|&&|\|\||[-+*/%^<>=!&|(){},;?:\[\]])
""", re.X | re.S)


def tokenize(text: str):
    out, i = [], 0
    while i < len(text):
        m = _TOKEN.match(text, i)
        if not m:
            raise ExprError(f"unexpected character {text[i]!r} at {i}")
        if m.lastgroup == "num":
            out.append(("num", float(m.group()), i))
        elif m.lastgroup == "id":
            out.append(("id", m.group(), i))
        elif m.lastgroup == "assign":
            out.append(("op", ":=", i))
        elif m.lastgroup == "op":
            out.append(("op", m.group(), i))
        i = m.end()
    out.append(("end", None, len(text)))
    return out


class Parser:
    """Recursive descent to a tree of tuples:
    statements ('assign', name, op, e), ('var', name, e), ('if', c, S, S|None),
    ('block', [S]), ('expr', e); expressions ('num', v), ('var', name),
    ('bin', op, a, b), ('neg', e), ('not', e), ('f1', f, e), ('f2', f, a, b),
    ('minmax', f, [e]), ('sel', c, a, b)."""

    def __init__(self, text: str, inputs, outputs):
        self.t = tokenize(text)
        self.k = 0
        self.names = set(inputs) | set(outputs)
        self.inputs = set(inputs)

    # helpers
    def cur(self):
        return self.t[self.k]

    def is_op(self, o):
        return self.cur()[0] == "op" and self.cur()[1] == o

    def is_id(self, w):
        return self.cur()[0] == "id" and self.cur()[1] == w

    def expect(self, o):
        if not self.is_op(o):
            raise ExprError(f"expected {o!r} at {self.cur()[2]}")
        self.k += 1

    def program(self):
        out = []
        while self.cur()[0] != "end":
            out.append(self.statement())
        return ("block", out)

    def statement(self):
        if self.is_op(";"):
            self.k += 1
            return ("block", [])
        if self.is_op("{"):
            self.k += 1
            body = []
            while not self.is_op("}"):
                if self.cur()[0] == "end":
                    raise ExprError("expected '}'")
                body.append(self.statement())
            self.k += 1
            return ("block", body)
        if self.is_id("if") and self.t[self.k + 1][1] == "(" and not self._if_function():
            self.k += 2
            c = self.expression()
            self.expect(")")
            a = self.statement()
            b = None
            if self.is_id("else"):
                self.k += 1
                b = self.statement()
            return ("if", c, a, b)
        if self.is_id("var"):
            self.k += 1
            kind, name, _ = self.cur()
            if kind != "id" or name in KEYWORDS or name in self.names:
                raise ExprError("bad variable declaration")
            self.k += 1
            self.names.add(name)
            e = ("num", 0.0)
            if self.is_op(":="):
                self.k += 1
                e = self.expression()
            self._end()
            return ("assign", name, ":=", e)
        if self.cur()[0] == "id" and self.t[self.k + 1][0] == "op" and \
                self.t[self.k + 1][1] in (":=", "+=", "-=", "*=", "/=", "%="):
            name, op = self.cur()[1], self.t[self.k + 1][1]
            if name not in self.names or name in self.inputs:
                raise ExprError(f"cannot assign {name!r}")
            self.k += 2
            e = self.expression()
            self._end()
            return ("assign", name, op, e)
        e = self.expression()
        self._end()
        return ("expr", e)

    def _end(self):
        if self.is_op(";"):
            self.k += 1
        elif not (self.cur()[0] == "end" or self.is_op("}")):
            raise ExprError(f"expected ';' at {self.cur()[2]}")

    def _if_function(self):
        level = 0
        for kind, v, _ in self.t[self.k + 1:]:
            if kind == "end":
                return False
            if kind != "op":
                continue
            if v in "({[":
                level += 1
            elif v in ")}]":
                level -= 1
                if level == 0:
                    return False
            elif v == "," and level == 1:
                return True
        return False

    def expression(self):
        c = self.logical_or()
        if self.is_op("?"):
            self.k += 1
            a = self.expression()
            self.expect(":")
            b = self.expression()
            return ("sel", c, a, b)
        return c

    def logical_or(self):
        a = self.logical_and()
        while self.is_op("|") or self.is_op("||") or self.is_id("or"):
            self.k += 1
            a = ("bin", "or", a, self.logical_and())
        return a

    def logical_and(self):
        a = self.comparison()
        while self.is_op("&") or self.is_op("&&") or self.is_id("and"):
            self.k += 1
            a = ("bin", "and", a, self.comparison())
        return a

    def comparison(self):
        a = self.additive()
        ops = {"<": "<", "<=": "<=", ">": ">", ">=": ">=", "==": "==", "=": "==", "!=": "!=",
               "<>": "!="}
        while self.cur()[0] == "op" and self.cur()[1] in ops:
            op = ops[self.cur()[1]]
            self.k += 1
            a = ("bin", op, a, self.additive())
        return a

    def additive(self):
        a = self.multiplicative()
        while self.is_op("+") or self.is_op("-"):
            op = self.cur()[1]
            self.k += 1
            a = ("bin", op, a, self.multiplicative())
        return a

    def multiplicative(self):
        a, implicit = self.unary()
        while True:
            if self.cur()[0] == "op" and self.cur()[1] in "*/%" and len(self.cur()[1]) == 1:
                op = self.cur()[1]
                self.k += 1
                b, implicit = self.unary()
                a = ("bin", op, a, b)
            elif implicit and (self.is_op("(") or (self.cur()[0] == "id" and
                                                    self.cur()[1] not in KEYWORDS)):
                b, implicit = self.unary()
                a = ("bin", "*", a, b)
            else:
                return a

    def unary(self):
        if self.is_op("-"):
            self.k += 1
            a, implicit = self.unary()
            return ("neg", a), implicit
        if self.is_op("+"):
            self.k += 1
            return self.unary()
        if self.is_op("!") or self.is_id("not"):
            self.k += 1
            return ("not", self.unary()[0]), False
        a, implicit = self.primary()
        if self.is_op("^"):
            self.k += 1
            neg = False
            if self.is_op("-"):
                self.k += 1
                neg = True
            elif self.is_op("+"):
                self.k += 1
            b = self.primary()[0]
            a = ("bin", "^", a, ("neg", b) if neg else b)
            if self.is_op("^"):
                raise ExprError("chained '^'")
            return a, False
        return a, implicit

    def args(self):
        self.expect("(")
        out = []
        if not self.is_op(")"):
            out.append(self.expression())
            while self.is_op(","):
                self.k += 1
                out.append(self.expression())
        self.expect(")")
        return out

    def primary(self):
        kind, v, pos = self.cur()
        if kind == "num":
            self.k += 1
            return ("num", v), True
        if self.is_op("("):
            self.k += 1
            e = self.expression()
            self.expect(")")
            return e, True
        if kind != "id":
            raise ExprError(f"expected a value at {pos}")
        self.k += 1
        if v == "if":
            a = self.args()
            if len(a) != 3:
                raise ExprError("if(c, a, b) takes three arguments")
            return ("sel", a[0], a[1], a[2]), True
        if v == "pi":
            return ("num", math.pi), False
        if v in ("true", "false"):
            return ("num", 1.0 if v == "true" else 0.0), False
        if v in F1:
            a = self.args()
            if len(a) != 1:
                raise ExprError(f"{v} takes one argument")
            return ("f1", v, a[0]), True
        if v in F2:
            a = self.args()
            if len(a) != 2:
                raise ExprError(f"{v} takes two arguments")
            return ("f2", v, a[0], a[1]), True
        if v in ("min", "max"):
            a = self.args()
            if len(a) < 2:
                raise ExprError(f"{v} takes at least two arguments")
            return ("minmax", v, a), True
        if v in self.names and v not in KEYWORDS:
            return ("var", v), False
        raise ExprError(f"unknown symbol {v!r} at {pos}")


def _truth(b):
    return np.where(b, 1.0, 0.0)


def _feq(a, b):
    m = np.maximum(1.0, np.maximum(np.abs(a), np.abs(b)))
    return np.abs(a - b) <= 1e-10 * m


def _eval(e, env, shape):
    k = e[0]
    if k == "num":
        return np.full(shape, e[1])
    if k == "var":
        return env[e[1]]
    if k == "neg":
        return -_eval(e[1], env, shape)
    if k == "not":
        return _truth(_eval(e[1], env, shape) == 0.0)
    if k == "f1":
        return F1[e[1]](_eval(e[2], env, shape))
    if k == "f2":
        return F2[e[1]](_eval(e[2], env, shape), _eval(e[3], env, shape))
    if k == "minmax":
        vals = [_eval(a, env, shape) for a in e[2]]
        r = vals[0]
        for v in vals[1:]:
            r = np.fmin(r, v) if e[1] == "min" else np.fmax(r, v)
        return r
    if k == "sel":
        c = _eval(e[1], env, shape) != 0.0
        return np.where(c, _eval(e[2], env, shape), _eval(e[3], env, shape))
    op, a, b = e[1], _eval(e[2], env, shape), _eval(e[3], env, shape)
    return {
        "+": lambda: a + b, "-": lambda: a - b, "*": lambda: a * b, "/": lambda: a / b,
        "%": lambda: np.fmod(a, b), "^": lambda: np.power(a, b),
        "<": lambda: _truth(a < b), "<=": lambda: _truth(a <= b), ">": lambda: _truth(a > b),
        ">=": lambda: _truth(a >= b), "==": lambda: _truth(_feq(a, b)),
        "!=": lambda: _truth(~_feq(a, b)),
        "and": lambda: _truth((a != 0.0) & (b != 0.0)),
        "or": lambda: _truth((a != 0.0) | (b != 0.0)),
    }[op]()


def _exec(s, env, mask, shape):
    k = s[0]
    if k == "block":
        for t in s[1]:
            _exec(t, env, mask, shape)
    elif k == "if":
        c = _eval(s[1], env, shape) != 0.0
        _exec(s[2], env, mask & c, shape)
        if s[3] is not None:
            _exec(s[3], env, mask & ~c, shape)
    elif k == "assign":
        name, op, v = s[1], s[2], _eval(s[3], env, shape)
        old = env.get(name, np.zeros(shape))
        new = {":=": lambda: v, "+=": lambda: old + v, "-=": lambda: old - v,
               "*=": lambda: old * v, "/=": lambda: old / v,
               "%=": lambda: np.fmod(old, v)}[op]()
        env[name] = np.where(mask, new, old)
    else:  # expression statement: evaluated for its errors only
        _eval(s[1], env, shape)


def evaluate(text: str, inputs: dict, outputs=PRIMES) -> dict:
    """Runs a program on the points given by ``inputs`` (name -> array, all of
    one shape); returns every output variable (0 where never assigned), as
    UserExpression::GetValue does for each point."""
    shape = np.broadcast(*inputs.values()).shape if inputs else ()
    tree = Parser(text, list(inputs), list(outputs)).program()
    env = {n: np.broadcast_to(np.asarray(v, dtype=np.float64), shape).copy()
           for n, v in inputs.items()}
    for n in outputs:
        env[n] = np.zeros(shape)
    with np.errstate(all="ignore"):
        _exec(tree, env, np.ones(shape, dtype=bool), shape)
    return {n: env[n] for n in outputs}


def check_syntax(text: str, inputs=("x", "y", "z"), outputs=PRIMES) -> None:
    """Raises ExprError where the reference's UserExpression would throw."""
    Parser(text, list(inputs), list(outputs)).program()


def initial_prime_states(text: str, dim: int, origins, cell_size: float,
                         units=(1.0, 1.0, 1.0)) -> np.ndarray:
    """GetInitialPrimeStates for nodes of 16^dim cells with the given origins
    [nb, 3] and dimensional cell size: non-dimensional prime states in the
    reference's order (Density, Pressure, VelocityX.., field_details.h:201-212)
    as [nb, dim + 2, 16^dim], cells in C order."""
    rho_ref, vel_ref, _ = units
    origins = np.asarray(origins, dtype=np.float64).reshape(-1, 3)
    n = [16 if d < dim else 1 for d in range(3)]
    idx = np.indices(n).reshape(3, -1)
    out = np.empty((len(origins), dim + 2, idx.shape[1]))
    for b, o in enumerate(origins):
        xyz = {c: (o[d] + (idx[d] + 0.5) * cell_size if d < dim else np.zeros(idx.shape[1]))
               for d, c in enumerate("xyz")}
        v = evaluate(text, xyz)
        out[b, 0] = v["density"] / rho_ref
        out[b, 1] = v["pressure"] / (rho_ref * vel_ref * vel_ref)
        for d in range(dim):
            out[b, 2 + d] = v[("velocityX", "velocityY", "velocityZ")[d]] / vel_ref
    return out


def run_listing(lines, x, y, z, outputs=PRIMES) -> dict:
    """Interprets the library's compiled program text (alp_ic_program_listing)
    at the points (x, y, z), one point at a time."""
    prog = [ln.split(" ", 1) for ln in lines]
    x, y, z = (np.broadcast_to(np.asarray(a, dtype=np.float64), np.shape(x)).ravel()
               for a in (x, y, z))
    res = {n: np.zeros(len(x)) for n in outputs}
    binops = {
        "ADD": lambda a, b: a + b, "SUB": lambda a, b: a - b, "MUL": lambda a, b: a * b,
        "DIV": lambda a, b: float(np.float64(a) / np.float64(b)),
        "MOD": lambda a, b: float(np.fmod(np.float64(a), np.float64(b))),
        "POW": lambda a, b: float(np.power(np.float64(a), np.float64(b))),
        "LT": lambda a, b: float(a < b), "LE": lambda a, b: float(a <= b),
        "GT": lambda a, b: float(a > b), "GE": lambda a, b: float(a >= b),
        "EQ": lambda a, b: float(bool(_feq(a, b))), "NE": lambda a, b: float(not _feq(a, b)),
        "AND": lambda a, b: float(a != 0.0 and b != 0.0),
        "OR": lambda a, b: float(a != 0.0 or b != 0.0),
        "MIN": lambda a, b: float(np.fmin(a, b)), "MAX": lambda a, b: float(np.fmax(a, b)),
    }
    with np.errstate(all="ignore"):
        for p in range(len(x)):
            var = {"x": x[p], "y": y[p], "z": z[p]}
            st = []
            pc = 0
            while True:
                op = prog[pc][0]
                arg = prog[pc][1] if len(prog[pc]) > 1 else None
                pc += 1
                if op == "END":
                    break
                if op == "CONST":
                    st.append(float(arg))
                elif op == "LOAD":
                    st.append(var.get(arg, 0.0))
                elif op == "STORE":
                    var[arg] = st.pop()
                elif op == "POP":
                    st.pop()
                elif op == "NEG":
                    st[-1] = -st[-1]
                elif op == "NOT":
                    st[-1] = float(st[-1] == 0.0)
                elif op == "F1":
                    st[-1] = float(F1[arg](np.float64(st[-1])))
                elif op == "F2":
                    b = st.pop()
                    st[-1] = float(F2[arg](np.float64(st[-1]), np.float64(b)))
                elif op == "JZ":
                    if st.pop() == 0.0:
                        pc = int(arg)
                elif op == "JMP":
                    pc = int(arg)
                else:
                    b = st.pop()
                    st[-1] = float(binops[op](st[-1], b))
            for n in outputs:
                res[n][p] = var.get(n, 0.0)
    return res
