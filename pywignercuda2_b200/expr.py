"""Parse and evaluate the C expression strings the reference's classes take.

The reference splices user strings such as ``kineticString``,
``potentialString`` (GPU_Wigner4D.py:249, 266) and ``potential_{0..3}_String``
(GPU_WignerDirac4D.py:498-514) into CUDA source.  Here they are parsed once
into an expression tree and evaluated in float64 with NumPy at plan creation,
to build the phase and coordinate tables the CUDA kernels consume.

Grammar (the C subset the reference's strings use): numbers, identifiers,
``+ - * / %``, unary ``+ -``, parentheses, and calls of the C math functions
below.  Integer literals keep C semantics: ``1/2`` is 0, ``7 % 3`` is 1.
"""
import math
import re

import numpy as np

__all__ = ["parse", "evaluate", "ExprError"]


class ExprError(ValueError):
    """The string is not an expression of the supported C subset."""


_FUNCS = {
    "pow": (2, np.power), "exp": (1, np.exp), "log": (1, np.log), "log10": (1, np.log10),
    "sqrt": (1, np.sqrt), "sin": (1, np.sin), "cos": (1, np.cos), "tan": (1, np.tan),
    "sinh": (1, np.sinh), "cosh": (1, np.cosh), "tanh": (1, np.tanh),
    "asin": (1, np.arcsin), "acos": (1, np.arccos), "atan": (1, np.arctan),
    "atan2": (2, np.arctan2), "fabs": (1, np.abs), "abs": (1, np.abs),
    "floor": (1, np.floor), "ceil": (1, np.ceil), "fmin": (2, np.minimum),
    "fmax": (2, np.maximum), "cbrt": (1, np.cbrt), "exp2": (1, np.exp2),
    "fmod": (2, np.fmod),
}
_CONSTS = {"M_PI": math.pi, "M_E": math.e, "M_SQRT2": math.sqrt(2.0)}

_TOK = re.compile(r"\s*(?:(?P<num>(?:\d+\.\d*|\.\d+)(?:[eE][-+]?\d+)?|\d+[eE][-+]?\d+|\d+)"
                  r"|(?P<name>[A-Za-z_]\w*)|(?P<op>[-+*/%(),]))")


class _Node:
    __slots__ = ("kind", "val", "args")

    def __init__(self, kind, val=None, args=()):
        self.kind, self.val, self.args = kind, val, tuple(args)


def _tokens(src):
    pos, out = 0, []
    src = src.strip()
    while pos < len(src):
        m = _TOK.match(src, pos)
        if m is None or m.end() == pos:
            raise ExprError("cannot parse %r at %r" % (src, src[pos:pos + 10]))
        pos = m.end()
        if m.group("num") is not None:
            t = m.group("num")
            is_int = re.fullmatch(r"\d+", t) is not None
            out.append(("num", int(t) if is_int else float(t)))
        elif m.group("name") is not None:
            out.append(("name", m.group("name")))
        else:
            out.append(("op", m.group("op")))
    return out


class _Parser:
    def __init__(self, toks):
        self.t, self.i = toks, 0

    def peek(self):
        return self.t[self.i] if self.i < len(self.t) else (None, None)

    def take(self, op=None):
        tok = self.peek()
        if op is not None and tok != ("op", op):
            raise ExprError("expected %r, got %r" % (op, tok[1]))
        self.i += 1
        return tok

    def expr(self):
        n = self.term()
        while self.peek() in (("op", "+"), ("op", "-")):
            op = self.take()[1]
            n = _Node("bin", op, (n, self.term()))
        return n

    def term(self):
        n = self.unary()
        while self.peek() in (("op", "*"), ("op", "/"), ("op", "%")):
            op = self.take()[1]
            n = _Node("bin", op, (n, self.unary()))
        return n

    def unary(self):
        if self.peek() in (("op", "-"), ("op", "+")):
            op = self.take()[1]
            return _Node("neg", None, (self.unary(),)) if op == "-" else self.unary()
        return self.primary()

    def primary(self):
        kind, val = self.take()
        if kind == "num":
            return _Node("num", val)
        if kind == "name":
            if self.peek() == ("op", "("):
                if val not in _FUNCS:
                    raise ExprError("unknown function %r" % val)
                self.take("(")
                args = [self.expr()]
                while self.peek() == ("op", ","):
                    self.take(",")
                    args.append(self.expr())
                self.take(")")
                if len(args) != _FUNCS[val][0]:
                    raise ExprError("%s takes %d arguments" % (val, _FUNCS[val][0]))
                return _Node("call", val, args)
            if val in _CONSTS:
                return _Node("num", _CONSTS[val])
            return _Node("var", val)
        if (kind, val) == ("op", "("):
            n = self.expr()
            self.take(")")
            return n
        raise ExprError("unexpected token %r" % (val,))


def parse(src):
    """Parse C expression ``src`` into a tree (raises ExprError)."""
    if not isinstance(src, str) or not src.strip():
        raise ExprError("empty expression")
    p = _Parser(_tokens(src))
    n = p.expr()
    if p.i != len(p.t):
        raise ExprError("trailing input in %r" % src)
    return n


def _is_int(v):
    return isinstance(v, int) and not isinstance(v, bool)


def _eval(n, env):
    k = n.kind
    if k == "num":
        return n.val
    if k == "var":
        if n.val not in env:
            raise ExprError("unknown variable %r" % n.val)
        return env[n.val]
    if k == "neg":
        return -_eval(n.args[0], env)
    if k == "call":
        args = [np.asarray(_eval(a, env), dtype=np.float64) for a in n.args]
        return _FUNCS[n.val][1](*args)
    a, b = _eval(n.args[0], env), _eval(n.args[1], env)
    op = n.val
    if _is_int(a) and _is_int(b):          # C integer arithmetic
        if op == "+":
            return a + b
        if op == "-":
            return a - b
        if op == "*":
            return a * b
        if b == 0:
            raise ExprError("integer division by zero")
        q = abs(a) // abs(b)
        q = q if (a >= 0) == (b >= 0) else -q
        return q if op == "/" else a - q * b
    a = np.asarray(a, dtype=np.float64) if not isinstance(a, float) else a
    b = np.asarray(b, dtype=np.float64) if not isinstance(b, float) else b
    if op == "+":
        return a + b
    if op == "-":
        return a - b
    if op == "*":
        return a * b
    if op == "/":
        return a / b
    return np.fmod(a, b)


def evaluate(src_or_tree, **env):
    """Evaluate an expression on NumPy arrays; the result broadcasts to the
    shape of the variables and is float64."""
    tree = parse(src_or_tree) if isinstance(src_or_tree, str) else src_or_tree
    val = _eval(tree, env)
    shape = np.broadcast_shapes(*[np.shape(v) for v in env.values()]) if env else ()
    return np.broadcast_to(np.asarray(val, dtype=np.float64), shape)


def variables(src_or_tree):
    """Names of the variables an expression reads."""
    tree = parse(src_or_tree) if isinstance(src_or_tree, str) else src_or_tree
    out, stack = set(), [tree]
    while stack:
        n = stack.pop()
        if n.kind == "var":
            out.add(n.val)
        stack.extend(n.args)
    return out
