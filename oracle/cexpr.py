"""Evaluate the reference's C-expression strings with NumPy (test infrastructure only).

The reference takes physics as C expression strings spliced into CUDA source
(``kineticString``/``potentialString``: GPU_Wigner4D.py:249, 266;
``potential_{0..3}_String``: GPU_WignerDirac4D.py:498-514).  The oracle
evaluates the same strings on NumPy arrays.  Integer literals keep C
semantics (``1/2 == 0``) through ``_CInt``; every other value is float64.
"""
import re

import numpy as np


class _CInt(int):
    """An int literal with C arithmetic (truncating division between ints)."""

    def _wrap(self, v):
        return _CInt(v) if isinstance(v, int) and not isinstance(v, bool) else v

    def __truediv__(self, o):
        if isinstance(o, _CInt):
            q = abs(int(self)) // abs(int(o))
            return _CInt(q if (int(self) >= 0) == (int(o) >= 0) else -q)
        return float(self) / o

    def __rtruediv__(self, o):
        return o / float(self)

    def __add__(self, o):
        return self._wrap(int(self) + o) if isinstance(o, _CInt) else float(self) + o

    __radd__ = __add__

    def __sub__(self, o):
        return self._wrap(int(self) - o) if isinstance(o, _CInt) else float(self) - o

    def __rsub__(self, o):
        return o - float(self)

    def __mul__(self, o):
        return self._wrap(int(self) * o) if isinstance(o, _CInt) else float(self) * o

    __rmul__ = __mul__

    def __neg__(self):
        return _CInt(-int(self))

    def __pos__(self):
        return self


_FUNCS = {
    "pow": np.power, "exp": np.exp, "log": np.log, "log10": np.log10,
    "sqrt": np.sqrt, "sin": np.sin, "cos": np.cos, "tan": np.tan,
    "sinh": np.sinh, "cosh": np.cosh, "tanh": np.tanh, "asin": np.arcsin,
    "acos": np.arccos, "atan": np.arctan, "atan2": np.arctan2,
    "fabs": np.abs, "abs": np.abs, "floor": np.floor, "ceil": np.ceil,
    "fmin": np.minimum, "fmax": np.maximum, "cbrt": np.cbrt,
    "M_PI": np.pi, "M_E": np.e,
}

_TOKEN = re.compile(r"\s*(?:(\d+\.\d*(?:[eE][-+]?\d+)?|\.\d+(?:[eE][-+]?\d+)?|\d+[eE][-+]?\d+)"
                    r"|(\d+)|([A-Za-z_]\w*)|(.))")


def _translate(src):
    out = []
    pos = 0
    src = src.strip()
    while pos < len(src):
        m = _TOKEN.match(src, pos)
        if m is None:
            break
        flt, integer, name, other = m.groups()
        if flt is not None:
            out.append("float(%r)" % flt)
        elif integer is not None:
            out.append("_CInt(%s)" % integer)
        elif name is not None:
            out.append(name)
        elif other is not None and not other.isspace():
            out.append(other)
        pos = m.end()
    return " ".join(out)


def evaluate(src, **variables):
    """Evaluate C expression ``src`` with the given NumPy variables."""
    code = _translate(src)
    env = dict(_FUNCS)
    env["_CInt"] = _CInt
    env["float"] = float
    env.update(variables)
    val = eval(code, {"__builtins__": {}}, env)  # noqa: S307 -- test oracle only
    shape = np.broadcast(*[np.asarray(v) for v in variables.values()]).shape if variables else ()
    return np.broadcast_to(np.asarray(val, dtype=np.float64), shape)
