"""Host logic: the C-expression evaluator and the pairwise factor tables."""
import numpy as np
import pytest

from oracle import cexpr
from pywignercuda2_b200 import expr, tables

EXPRS = ["0.5*(p_x*p_x  + p_y*p_y)/1.0", "0.5*pow(x,2) + 0.5*pow(y,2)",
         "0.5*(x*x + y*y) + 0.1*(pow(x,4) + pow(y,4)) + 0.05*x*y", "-y*0.26/2.",
         "x*0.26/2. + 0.05*pow(x,2)", "y*(x+16)/50.", "0.04*pow(x-5.,2)", "1/2 + x",
         "exp(-x*x)*cos(y) + sqrt(fabs(x)+1.)", "7 % 3 + x", "-(-x) - +y", "M_PI*x"]


@pytest.mark.parametrize("src", EXPRS)
def test_expr_matches_oracle(src):
    rng = np.random.default_rng(1)
    x, y = rng.normal(size=50), rng.normal(size=50)
    v = dict(x=x, y=y, p_x=x, p_y=y)
    a = expr.evaluate(src, **v)
    b = cexpr.evaluate(src, **v)
    assert np.allclose(a, b, rtol=1e-15, atol=1e-15)


def test_expr_c_integer_semantics():
    assert float(expr.evaluate("1/2")) == 0.0
    assert float(expr.evaluate("-7/2")) == -3.0
    assert float(expr.evaluate("7%3")) == 1.0
    assert float(expr.evaluate("1./2")) == 0.5


@pytest.mark.parametrize("bad", ["", "x +", "foo(x)", "x y", "pow(x)", "(x"])
def test_expr_rejects(bad):
    with pytest.raises(expr.ExprError):
        expr.evaluate(bad, x=np.zeros(3), y=np.zeros(3))


def _grid(n=12):
    return [0.3 * (np.arange(n) - n // 2), 0.5 * (np.arange(n) - n // 2),
            0.3 * (np.arange(n) - n // 2), 0.5 * (np.arange(n) - n // 2)]


def _phase(src, dt=0.01):
    t = expr.parse(src)
    return lambda ty, y, tx, x: (dt * expr.evaluate(t, x=x - 0.5 * tx, y=y - 0.5 * ty)
                                 - dt * expr.evaluate(t, x=x + 0.5 * tx, y=y + 0.5 * ty))


@pytest.mark.parametrize("src,separable", [
    ("0.5*(x*x + y*y) + 0.1*(pow(x,4) + pow(y,4)) + 0.05*x*y", True),
    ("0.04*pow(x-5.,2)", True), ("0.5*x", True),
    ("x*x*y*y", False), ("exp(-x*x-y*y)", False)])
def test_pairwise_tables_reconstruct(src, separable):
    v = _grid()
    fn = _phase(src)
    mags = [np.exp(-0.01 * v[0] ** 2), None, np.exp(-0.02 * v[2] ** 2), None]
    tabs, full = tables.build_factor(fn, mags, v)
    c = [a.reshape(s) for a, s in zip(v, [(-1, 1, 1, 1), (1, -1, 1, 1), (1, 1, -1, 1), (1, 1, 1, -1)])]
    want = np.exp(-1j * fn(*c)) * mags[0].reshape(-1, 1, 1, 1) * mags[2].reshape(1, 1, -1, 1)
    if separable:
        assert full is None and 0 < len(tabs) <= 10
        got = np.ones(want.shape, np.complex128)
        for a, b, t in tabs:
            sh = [1, 1, 1, 1]
            if b < 0:
                sh[a] = t.shape[0]
            else:
                sh[a], sh[b] = t.shape
            got = got * t.reshape(sh)
    else:
        assert full is not None and tabs == []
        got = full
    assert np.max(np.abs(got - want)) < 1e-13
