"""GPU parity of the tensor-core transform engine (k_tc64, ``tensor_cores =
True``) and the 20-iteration oracle prefix of the 64^4 drop-in.

k_tc64 runs each 64-point transform as a dense complex GEMM on the tensor
cores with operands split into fp16 hi + lo (about 22 significant bits,
FP32 accumulation).  Measured against the complex128 form after 20
iterations of the 64^4 cat state: energy 9e-5, <x> 8e-6, max|dW|/max|W|
3e-5 relative; the tolerances below are three times those.  The complex128
drop-in itself is held to the parity bar (1e-12 observables, 1e-10
state) against the NumPy oracle over the same 20 iterations.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from configs import cat_xp, config1, config2  # noqa: E402
from frames import make_frame, rel_err  # noqa: E402
from oracle.wigner4d import Wigner4DOracle  # noqa: E402
from pywignercuda2_b200 import GPU_Wigner4D, _lib  # noqa: E402

OBS = ["average_x", "average_p_x", "average_x_square", "average_p_x_square", "average_y",
       "average_p_y", "average_y_square", "average_p_y_square", "energy"]
TC_TOL = {"energy": 3e-4, "state": 1e-4, "obs": 3e-4}


def _run(params, W0, iters, **kw):
    f = make_frame(GPU_Wigner4D, params, **kw)
    f.W_init_gpu.set(W0.astype(f.complex_dtype))
    f.timeSteps = iters - 1
    f.fileName = None
    f.Run()
    return f


def _notebook_windows(p):
    p.update(theta_x_amplitude=9.0, theta_y_amplitude=9.0, lambda_x_amplitude=9.0, lambda_y_amplitude=9.0)
    return p


def test_c128_and_tc_vs_oracle_20_iterations_64():
    """Config 2 (64^4 cat state): the complex128 drop-in and the tensor-core
    complex64 form against one 20-iteration oracle run."""
    p, c = config2(0, 64)
    o = Wigner4DOracle(p)
    f128 = make_frame(GPU_Wigner4D, p)
    W0 = cat_xp(f128._coords, c)
    Wo, obs = o.run(W0, 19)
    f128 = _run(p, W0, 20)
    assert f128.plan_info()["run64_kernel"] == "r4ring_pc"
    for name in OBS:
        assert rel_err(getattr(f128, name), obs[name]) < 1e-12, name
    assert rel_err(f128.norm, obs["norms"]) < 1e-12
    assert rel_err(f128.W_init_gpu.get(), Wo) < 1e-10
    ftc = _run(p, W0, 20, complex_dtype=np.complex64, tensor_cores=True)
    assert ftc.plan_info()["run64_kernel"] == "tc"
    assert rel_err(ftc.energy, obs["energy"]) < TC_TOL["energy"]
    for name in OBS:
        assert rel_err(getattr(ftc, name), obs[name]) < TC_TOL["obs"], name
    assert rel_err(ftc.norm, obs["norms"]) < 1e-9
    assert rel_err(ftc.W_init_gpu.get(), Wo) < TC_TOL["state"]


def test_tc_general_delta_vs_dense_c128_64():
    """Notebook windows (delta N = 0.716): k_tc64 with the fractional FAFT
    matrices against the complex128 dense half-steps (k_dense_half)."""
    p, c = config2(10, 64)
    p = _notebook_windows(p)
    f = make_frame(GPU_Wigner4D, p)
    W0 = cat_xp(f._coords, c)
    f128 = _run(p, W0, 10)
    ftc = _run(p, W0, 10, complex_dtype=np.complex64, tensor_cores=True)
    assert ftc.plan_info()["run64_kernel"] == "tc"
    for name in OBS:
        assert rel_err(getattr(ftc, name), getattr(f128, name)) < TC_TOL["obs"], name
    assert rel_err(ftc.W_init_gpu.get(), f128.W_init_gpu.get()) < TC_TOL["state"]


def test_tc_timed_run_matches_graph_run():
    """The event-bracketed Run() launches the same k_tc64 kernels as the
    graph: the same bits."""
    p, c = config2(1, 64)
    f = make_frame(GPU_Wigner4D, p, complex_dtype=np.complex64, tensor_cores=True)
    W0 = cat_xp(f._coords, c).astype(np.complex64)
    iters = 6
    h1 = torch.empty((iters, _lib.WIG4D_NOBS), dtype=torch.float64, device="cuda")
    h2 = torch.empty_like(h1)
    f.W_init_gpu.set(W0)
    f.run_device(f.W_init_gpu, iters, h1)
    W1 = f.W_init_gpu.get()
    f.W_init_gpu.set(W0)
    ms = f.run_device_timed(f.W_init_gpu, iters, h2)
    assert np.array_equal(h1.cpu().numpy(), h2.cpu().numpy())
    assert np.array_equal(W1, f.W_init_gpu.get())
    assert all(m > 0 for m in ms)


@pytest.mark.parametrize("dtype,n", [(np.complex128, 64), (np.complex64, 32)])
def test_tc_rejects_unsupported_plans(dtype, n):
    p, c = config1(0, n)
    with pytest.raises(_lib.WignerError) as e:
        make_frame(GPU_Wigner4D, p, complex_dtype=dtype, tensor_cores=True)
    assert e.value.status == 2


@pytest.mark.parametrize("kernel", ["r4ring_mx", "r4_mixed"])
def test_mixed_form_vs_oracle_20_iterations_64(kernel, monkeypatch):
    """complex64 storage with FP64 transforms (fp64_transforms = True), on
    the plane-contiguous ring kernel (default) or on k_r4 (WIG_MIXED_KERNEL
    = r4): the only rounding left is the state's float32 storage, relative
    to each value, so the energy stays within 1e-6 of the oracle."""
    if kernel == "r4_mixed":
        monkeypatch.setenv("WIG_MIXED_KERNEL", "r4")
    p, c = config2(0, 64)
    o = Wigner4DOracle(p)
    f = make_frame(GPU_Wigner4D, p, complex_dtype=np.complex64, fp64_transforms=True)
    assert f.plan_info()["run64_kernel"] == kernel
    W0 = cat_xp(f._coords, c)
    Wo, obs = o.run(W0.astype(np.complex64).astype(np.complex128), 19)
    f = _run(p, W0, 20, complex_dtype=np.complex64, fp64_transforms=True)
    for name in OBS:
        assert rel_err(getattr(f, name), obs[name]) < 1e-6, name
    assert rel_err(f.norm, obs["norms"]) < 1e-9
    assert rel_err(f.W_init_gpu.get(), Wo) < 1e-6
