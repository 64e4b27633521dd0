"""Pin the oracle against the golden values the reference's notebooks print.

The reference has no tests; its Dirac/KvN notebooks print the trace norm
after the initial condition and at every Run() iteration (Normalize_4x4_GPU,
GPU_WignerDirac4D.py:1366-1369).  ``tests/golden/notebook_norms.json`` holds
them (extracted by ``tests/golden/make_golden.py``); the notebooks' frame
settings are in ``tests/golden/notebook_configs.py``.

The printed norms pin the FAFT scale 2 N d, the sign of its exponent for
both +delta and -delta, the centring, the wrappers' divisors (size and
sqrt(size)/100), the kinetic and potential sandwiches, the projector and the
absorbing mask.  They also show the notebooks ran with the mask constant 7
for p (the committed Run() passes 15, GPU_WignerDirac4D.py:1764).
"""
import json
import os

import numpy as np
import pytest

from golden.notebook_configs import NOTEBOOKS
from oracle_dirac_driver import prepare, run

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "notebook_norms.json")))


def _rel(a, b):
    return abs(a - b) / abs(b)


def test_golden_file_complete():
    for name in NOTEBOOKS:
        g = GOLD[name]
        assert len(g["init_norms"]) == 1
        assert len(g["run_norms"]) >= 11


@pytest.mark.parametrize("name", ["instances/WignerDirac4D_64_64/X.ipynb"])
def test_init_norm_fast(name):
    o, n0 = prepare(NOTEBOOKS[name])
    # the notebook prints 12 significant digits
    assert _rel(n0.real, GOLD[name]["init_norms"][0]) < 1e-11
    assert abs(n0.imag) < 1e-9 * abs(n0.real)


# Notebooks whose printed Run() norms the committed reference does not
# reproduce: their cells use attributes the committed GPU_WignerDirac4D.py
# lacks (skipFrames, no potential_3_String), i.e. they ran on other revisions
# of the reference.  Their initial norms match; the Run() norms differ at
# iteration 0 or 1, and these tests must keep failing until that changes.
OTHER_REVISION = {"instances/WignerDirac4D_64_64/Free.ipynb", "instances/WignerDirac4D_64_64/X2.ipynb",
                  "instances/WignerDirac4D_64_64/FreeFiltered.ipynb",
                  "instances/WignerDirac4D_64_64/SternGerlach.ipynb"}


def notebook_params(names):
    return [pytest.param(n, marks=pytest.mark.xfail(strict=True, reason="run on another revision of the reference"))
            if n in OTHER_REVISION else n for n in sorted(names)]


@pytest.mark.slow
@pytest.mark.parametrize("name", notebook_params(NOTEBOOKS))
def test_init_and_two_iterations(name):
    cfg = NOTEBOOKS[name]
    g = GOLD[name]
    o, n0 = prepare(cfg)
    assert _rel(n0.real, g["init_norms"][0]) < 1e-11
    norms, _ = run(o, cfg, 2, alias_w21=True, bound_p=7.0)
    for k in range(2):
        assert _rel(norms[k].real, g["run_norms"][k]) < 1e-10, (k, norms[k], g["run_norms"][k])
