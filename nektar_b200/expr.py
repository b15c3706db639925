"""Analytic expressions of Nektar++ session files (boundary values, forcing,
exact solutions), evaluated on numpy arrays of point coordinates.

The grammar is the reference interpreter's (LibUtilities/Interpreter/
Interpreter.cpp:1150-1215), lowest precedence first:

    expression   = logical_or
    logical_or   = logical_and ('||' logical_and)*
    logical_and  = equality ('&&' equality)*
    equality     = lt_gt ('==' lt_gt)*
    lt_gt        = add_sub (('<=' | '>=' | '<' | '>') add_sub)*
    add_sub      = negate (('+' | '-') negate)*
    negate       = ['-'] mult_div_mod
    mult_div_mod = exponential (('*' | '/' | '%') exponential)*
    exponential  = base ['^' exponential]          (right associative)
    base         = number | function '(' args ')' | variable | constant
                   | parameter | '(' expression ')'

so `-x^2` is `-(x^2)` and a minus sign cannot follow `*` directly. The
constants and functions are the interpreter's tables (Interpreter.cpp:
192-238) except `awgn` (random noise) and `bessel`, which raise. Variables
are x, y, z, t; any other identifier is a session parameter. Comparisons
and logical operators give 1.0 / 0.0, as the interpreter does.

Expressions are parsed into closures over numpy arrays; nothing is passed
to Python's eval.
"""
import math
import re

import numpy as np

CONSTANTS = {
    "MEANINGLESS": 0.0, "E": math.e, "LOG2E": 1.0 / math.log(2.0), "LOG10E": 1.0 / math.log(10.0),
    "LN2": math.log(2.0), "LN10": math.log(10.0), "PI": math.pi, "PI_2": math.pi / 2,
    "PI_4": math.pi / 4, "1_PI": 1.0 / math.pi, "2_PI": 2.0 / math.pi,
    "2_SQRTPI": 2.0 / math.sqrt(math.pi), "SQRT2": math.sqrt(2.0), "SQRT1_2": math.sqrt(0.5),
    "GAMMA": 0.57721566490153286060, "DEG": 57.2957795130823208768,
    "PHI": 1.61803398874989484820,
}


def _sign(a):
    return np.where(a > 0, 1.0, np.where(a < 0, -1.0, 0.0))


def _ang(a, b):
    return np.arctan2(b, a)


FUNCTIONS = {
    "abs": (1, np.abs), "fabs": (1, np.abs), "asin": (1, np.arcsin), "acos": (1, np.arccos),
    "atan": (1, np.arctan), "atan2": (2, np.arctan2), "ang": (2, _ang), "ceil": (1, np.ceil),
    "cos": (1, np.cos), "cosh": (1, np.cosh), "exp": (1, np.exp), "floor": (1, np.floor),
    "fmax": (2, np.maximum), "fmin": (2, np.minimum), "max": (2, np.maximum),
    "min": (2, np.minimum), "fmod": (2, np.fmod), "log": (1, np.log), "log10": (1, np.log10),
    "rad": (2, lambda x, y: np.sqrt(x * x + y * y)), "sin": (1, np.sin), "sinh": (1, np.sinh),
    "sqrt": (1, np.sqrt), "tan": (1, np.tan), "tanh": (1, np.tanh), "sign": (1, _sign),
}
UNSUPPORTED = {"awgn", "bessel"}
VARIABLES = ("x", "y", "z", "t")

_TOKEN = re.compile(r"\s*(?:(?P<num>(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?)"
                    r"|(?P<id>[A-Za-z_$0-9][A-Za-z_$0-9]*)"
                    r"|(?P<op>\|\||&&|==|<=|>=|[-+*/%^()<>,]))")


class ExpressionError(ValueError):
    pass


def _tokenize(text):
    pos, out = 0, []
    text = text.strip()
    while pos < len(text):
        m = _TOKEN.match(text, pos)
        if not m or m.end() == pos:
            raise ExpressionError("cannot parse %r at %r" % (text, text[pos:]))
        kind = m.lastgroup
        out.append((kind, m.group(kind)))
        pos = m.end()
    return out


class _Parser:
    def __init__(self, text, params):
        self.text = text
        self.toks = _tokenize(text)
        self.i = 0
        self.params = params

    def peek(self):
        return self.toks[self.i] if self.i < len(self.toks) else (None, None)

    def take(self, op=None):
        t = self.peek()
        if op is not None and t[1] != op:
            raise ExpressionError("expected %r in %r" % (op, self.text))
        self.i += 1
        return t

    def parse(self):
        f = self.logical_or()
        if self.i != len(self.toks):
            raise ExpressionError("unexpected %r in %r" % (self.peek()[1], self.text))
        return f

    def _binary_chain(self, sub, ops):
        f = sub()
        while self.peek()[0] == "op" and self.peek()[1] in ops:
            op = self.take()[1]
            g = sub()
            f = self._combine(op, f, g)
        return f

    @staticmethod
    def _combine(op, f, g):
        fn = {
            "||": lambda a, b: np.where((a != 0) | (b != 0), 1.0, 0.0),
            "&&": lambda a, b: np.where((a != 0) & (b != 0), 1.0, 0.0),
            "==": lambda a, b: np.where(a == b, 1.0, 0.0),
            "<=": lambda a, b: np.where(a <= b, 1.0, 0.0),
            ">=": lambda a, b: np.where(a >= b, 1.0, 0.0),
            "<": lambda a, b: np.where(a < b, 1.0, 0.0),
            ">": lambda a, b: np.where(a > b, 1.0, 0.0),
            "+": np.add, "-": np.subtract, "*": np.multiply, "/": np.divide, "%": np.fmod,
            "^": np.power,
        }[op]
        return lambda env: fn(f(env), g(env))

    def logical_or(self):
        return self._binary_chain(self.logical_and, ("||",))

    def logical_and(self):
        return self._binary_chain(self.equality, ("&&",))

    def equality(self):
        return self._binary_chain(self.lt_gt, ("==",))

    def lt_gt(self):
        return self._binary_chain(self.add_sub, ("<=", ">=", "<", ">"))

    def add_sub(self):
        return self._binary_chain(self.negate, ("+", "-"))

    def negate(self):
        if self.peek() == ("op", "-"):
            self.take()
            f = self.mult_div_mod()
            return lambda env: np.negative(f(env))
        return self.mult_div_mod()

    def mult_div_mod(self):
        return self._binary_chain(self.exponential, ("*", "/", "%"))

    def exponential(self):
        b = self.base()
        if self.peek() == ("op", "^"):
            self.take()
            e = self.exponential()
            return lambda env: np.power(b(env), e(env))
        return b

    def base(self):
        kind, val = self.take()
        if kind == "num":
            v = float(val)
            return lambda env: v
        if kind == "op" and val == "(":
            f = self.logical_or()
            self.take(")")
            return f
        if kind == "id":
            if self.peek() == ("op", "(") and (val in FUNCTIONS or val in UNSUPPORTED):
                if val in UNSUPPORTED:
                    raise ExpressionError("function %s() is not supported" % val)
                nargs, fn = FUNCTIONS[val]
                self.take("(")
                args = [self.logical_or()]
                while self.peek() == ("op", ","):
                    self.take()
                    args.append(self.logical_or())
                self.take(")")
                if len(args) != nargs:
                    raise ExpressionError("%s() takes %d arguments" % (val, nargs))
                return lambda env: fn(*[a(env) for a in args])
            if val in VARIABLES:
                return lambda env: env[val]
            if val in CONSTANTS:
                c = CONSTANTS[val]
                return lambda env: c
            if val in self.params:
                p = float(self.params[val])
                return lambda env: p
            raise ExpressionError("unknown parameter %r in %r" % (val, self.text))
        raise ExpressionError("unexpected %r in %r" % (val, self.text))


class Expression:
    """One parsed expression; evaluate(x, y, z, t) broadcasts like numpy."""

    def __init__(self, text, params=None):
        self.text = text
        self._f = _Parser(text, params or {}).parse()

    def evaluate(self, x=0.0, y=0.0, z=0.0, t=0.0):
        x = np.asarray(x, dtype=np.float64)
        env = {"x": x, "y": np.asarray(y, dtype=np.float64), "z": np.asarray(z, dtype=np.float64),
               "t": np.asarray(t, dtype=np.float64)}
        v = self._f(env)
        return np.broadcast_to(np.asarray(v, dtype=np.float64),
                               np.broadcast(x, env["y"], env["z"], env["t"]).shape).copy()


def evaluate_parameters(pairs):
    """Session PARAMETERS in file order; each may use the ones before it
    (SessionReader::ReadParameters evaluates them as constant expressions)."""
    params = {}
    for name, text in pairs:
        params[name] = float(Expression(text, params).evaluate())
    return params
