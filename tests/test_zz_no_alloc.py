"""The allocation-free observables entry point against the plan-based one.

wig4d_observables_noalloc exists for callers that cannot call cudaMalloc
(a fixed memory pool, a footprint budget, pre-registered buffers only): it
takes every table as a device pointer the caller already owns and keeps its
partial sums in a fixed array inside the library.  This test calls it
through the C ABI twice in a row, on two different states, and checks each
result against wig4d_reduce (which uses the plan's own scratch) to the
tolerance of the other GPU parity tests.  It also checks the size limit.
The file name sorts last so that a run stopping at the first failure has
already run every other test; it also passes on its own.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from configs import cat_xp, config1, config2  # noqa: E402
from frames import make_frame, rel_err  # noqa: E402
from oracle.wigner4d import Wigner4DOracle  # noqa: E402
from pywignercuda2_b200 import GPU_Wigner4D, _lib, expr  # noqa: E402
from pywignercuda2_b200.device import stream_ptr  # noqa: E402


def _tables(f):
    """The frame's observable tables, as device tensors the caller owns."""
    cp = [torch.tensor(c, dtype=torch.float64, device="cuda") for c in f._coords]
    K = expr.evaluate(f.kineticString, p_x=f._coords[2][None, :], p_y=f._coords[0][:, None])
    V = expr.evaluate(f.potentialString, x=f._coords[3][None, :], y=f._coords[1][:, None])
    ep = torch.tensor(np.ascontiguousarray(K), dtype=torch.float64, device="cuda")
    ex = torch.tensor(np.ascontiguousarray(V), dtype=torch.float64, device="cuda")
    return cp, ep, ex


def _noalloc(f, W, cp, ep, ex, out):
    shape = (ctypes.c_int * 4)(*f.shape)
    return _lib.load().wig4d_observables_noalloc(
        W.data_ptr(), shape, f._desc.dtype, cp[0].data_ptr(), cp[1].data_ptr(), cp[2].data_ptr(),
        cp[3].data_ptr(), ep.data_ptr(), ex.data_ptr(), f._desc.dv_norm, f._desc.dv_obs, out.data_ptr(),
        stream_ptr())


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_noalloc_matches_plan_reduction_twice(dtype):
    params, c = config2(5, 64)
    f = make_frame(GPU_Wigner4D, params, complex_dtype=dtype)
    cp, ep, ex = _tables(f)
    out = torch.empty(2 * _lib.WIG4D_NOBS, dtype=torch.float64, device="cuda")
    tol = 1e-12
    states = [cat_xp(f._coords, c), cat_xp(f._coords, (0.3, -0.7, 0.2, 0.1), sep=1.0) * (1.0 + 0.2j)]
    for W0 in states:
        f.W_init_gpu.set(W0.astype(dtype))
        want = f._reduce(f.W_init_gpu)            # plan-based wig4d_reduce
        assert _noalloc(f, f.W_init_gpu.tensor, cp, ep, ex, out) == 0
        got = out.cpu().numpy()
        assert rel_err(got, want) < tol, (got, want)
        # and the oracle's norm and raw observables of the same (rounded) state
        o = Wigner4DOracle(params)
        Wh = W0.astype(dtype).astype(np.complex128)
        n = o.norm(Wh)
        assert abs(complex(got[0], got[1]) - n) < 1e-12 * abs(n)
        ob = o.observables(Wh)
        raw = got[_lib.WIG4D_NOBS:]
        names = ["average_x", "average_p_x", "average_x_square", "average_p_x_square", "average_y",
                 "average_p_y", "average_y_square", "average_p_y_square", "energy"]
        for k, name in enumerate(names):
            assert abs(raw[2 + k] - ob[name]) <= 1e-11 * max(abs(ob[name]), abs(n)), name


def test_noalloc_rejects_grids_above_the_limit():
    params, c = config1(0, 16)
    f = make_frame(GPU_Wigner4D, params)
    cp, ep, ex = _tables(f)
    out = torch.empty(2 * _lib.WIG4D_NOBS, dtype=torch.float64, device="cuda")
    lib = _lib.load()
    big = (ctypes.c_int * 4)(2, 256, 2, 128)      # N_y * N_x = 32768 > 16384
    st = lib.wig4d_observables_noalloc(f.W_init_gpu.ptr, big, f._desc.dtype, cp[0].data_ptr(),
                                       cp[1].data_ptr(), cp[2].data_ptr(), cp[3].data_ptr(), ep.data_ptr(),
                                       ex.data_ptr(), 1.0, 1.0, out.data_ptr(), stream_ptr())
    assert st == 7
    assert b"fixed limit" in lib.wig_last_error()
    # and a normal call still works afterwards
    assert _noalloc(f, f.W_init_gpu.tensor, cp, ep, ex, out) == 0
