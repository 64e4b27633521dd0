"""GPU parity of the scalar Wigner4D path against the NumPy oracle.

Tolerances: complex128 (the drop-in) must match the oracle to 1e-12
relative in norms and observables and 1e-10 in max|dW| / max|W| (the
parity bar of the drop-in).  complex64 (the precision form) is held to about three
times the error it reaches on each case (measured on B200): 2e-5 to 4e-5
relative on the observables and 1e-6 to 3e-6 on the state against the
oracle over these short runs, and below 1e-6 where two complex64 paths are
compared with each other.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from configs import config1, config2, w4d_params  # noqa: E402
from frames import make_frame, rel_err  # noqa: E402
from oracle.faft import faft  # noqa: E402
from oracle.wigner4d import Wigner4DOracle  # noqa: E402
from pywignercuda2_b200 import GPU_Wigner4D, GPUArray, _lib  # noqa: E402


def _rand(shape, seed, dtype=np.complex128):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("shape", [(16, 16, 32, 32), (32, 16, 16, 64), (16, 32, 16, 16), (48, 16, 48, 16)])
@pytest.mark.parametrize("axis", [0, 1, 2, 3])
@pytest.mark.parametrize("dn", [1.0, -1.0, 0.7, -0.83])
def test_faft_kernel(dtype, shape, axis, dn):
    a = _rand(shape, 3 + axis, dtype)
    n = shape[axis]
    d, delta = 0.37, dn / n
    g = GPUArray.to_gpu(a)
    sh = (ctypes.c_int * 4)(*shape)
    wd = _lib.C128 if dtype == np.complex128 else _lib.C64
    _lib.call("wig_faft", g.ptr, sh, wd, axis, d, delta, 0.5, None)
    torch.cuda.synchronize()
    want = 0.5 * faft(a.astype(np.complex128), axis, d, delta)
    tol = 1e-13 if dtype == np.complex128 else 2e-6
    assert rel_err(g.get(), want) < tol


def test_faft_reference_shim_64():
    a = _rand((64, 64, 64, 64), 9)
    g = GPUArray.to_gpu(a)
    _lib.call("FAFT64_4D_Z2Z", g.ptr, 0.25, 1.0 / 64, 0, 2, 1.0)
    torch.cuda.synchronize()
    assert rel_err(g.get(), faft(a, 2, 0.25, 1.0 / 64)) < 1e-13


def _pair(params, dtype=np.complex128, **kw):
    f = make_frame(GPU_Wigner4D, params, complex_dtype=dtype, **kw)
    o = Wigner4DOracle(params)
    return f, o


@pytest.mark.parametrize("n", [16, 32])
def test_init_kernels(n):
    p, c = config1(0, n)
    f, o = _pair(p)
    f.HOscillatorGound_GPU(f.W_init_gpu, c[0], c[1], c[2], c[3], 1.0, 1.0, 1.0)
    assert rel_err(f.W_init_gpu.get(), o.ho_ground(c[0], c[1], c[2], c[3], 1.0, 1.0, 1.0)) < 1e-15
    f.Gaussian_GPU(f.W_init_gpu, 0.1, -0.2, 0.3, 0.4, 1.1, 0.9, 1.3, 0.7)
    assert rel_err(f.W_init_gpu.get(), o.gaussian(0.1, -0.2, 0.3, 0.4, 1.1, 0.9, 1.3, 0.7)) < 1e-15


@pytest.mark.parametrize("n", [16, 32, 64])
def test_fused_halfsteps(n):
    p, c = config1(1, n)
    f, o = _pair(p)
    W0 = o.ho_ground(c[0], c[1], c[2], c[3], 1.0, 1.0, 1.0) + 0.01 * _rand(f.shape, 5)
    g = GPUArray.to_gpu(W0)
    f.kinetic_halfstep(g)
    want = o.x_to_lambda(o.x_to_lambda(W0) * o.kinetic_factor(), -1)
    assert rel_err(g.get(), want) < 1e-12
    g.set(W0)
    f.potential_halfstep(g)
    want = o.p_to_theta(o.p_to_theta(W0) * o.potential_factor(), -1)
    assert rel_err(g.get(), want) < 1e-12


def test_unfused_wrappers_and_phase_kernels():
    p, c = config1(2, 16)
    f, o = _pair(p)
    W0 = _rand(f.shape, 11)
    g = GPUArray.to_gpu(W0)
    f.Fourier_X_To_Lambda_64_64_GPU(g)
    f.exp_p_lambda_GPU(g)
    f.Fourier_Lambda_To_X_64_64_GPU(g)
    f.Fourier_P_To_Theta_64_64_GPU(g)
    f.exp_x_theta_GPU(g)
    f.Fourier_Theta_To_P_64_64_GPU(g)
    want = o.x_to_lambda(o.x_to_lambda(W0) * o.kinetic_factor(), -1)
    want = o.p_to_theta(o.p_to_theta(want) * o.potential_factor(), -1)
    assert rel_err(g.get(), want) < 1e-12


def test_reductions():
    p, c = config1(3, 32)
    f, o = _pair(p)
    W0 = o.ho_ground(c[0], c[1], c[2], c[3], 1.0, 1.0, 1.0) * (1.0 + 0.3j)
    g = GPUArray.to_gpu(W0)
    assert abs(f.Norm_GPU(g) - o.norm(W0)) < 1e-13 * abs(o.norm(W0))
    ob = o.observables(W0)
    for name in ["average_x", "average_p_x", "average_x_square", "average_p_x_square", "average_y",
                 "average_p_y", "average_y_square", "average_p_y_square"]:
        got = getattr(f, name.replace("average", "Average") + "_GPU")(g).get()
        assert abs(got - ob[name]) <= 1e-12 * max(1.0, abs(ob[name])), name
    assert abs(f.Energy_GPU(g).get() - ob["energy"]) <= 1e-12 * abs(ob["energy"])


def _run_both(params, init, iters, dtype=np.complex128):
    f, o = _pair(params, dtype)
    W0 = init(f, o)
    f.W_init_gpu.set(W0.astype(dtype))
    f.timeSteps = iters - 1
    f.fileName = None
    f.Run()
    Wo, obs = o.run(W0.astype(np.complex64).astype(np.complex128) if dtype == np.complex64 else W0, iters - 1)
    return f, Wo, obs


OBS = ["average_x", "average_p_x", "average_x_square", "average_p_x_square", "average_y",
       "average_p_y", "average_y_square", "average_p_y_square", "energy"]


@pytest.mark.parametrize("n", [16, 32])
def test_run_config1_parity(n):
    p, c = config1(0, n)
    init = lambda f, o: o.ho_ground(c[0], c[1], c[2], c[3], 1.0, 1.0, 1.0) / np.pi ** 2
    f, Wo, obs = _run_both(p, init, 21)
    for name in OBS:
        assert rel_err(getattr(f, name), obs[name]) < 1e-12, name
    assert rel_err(f.norm, obs["norms"]) < 1e-12
    assert rel_err(f.W_init_gpu.get(), Wo) < 1e-10


def test_run_general_delta_unfused():
    """Notebook-style windows (delta N != 1) take the dense unfused path."""
    p = w4d_params(16, D=0.01, dt=0.01)
    p.update(theta_x_amplitude=9.0, theta_y_amplitude=9.0, lambda_x_amplitude=9.0, lambda_y_amplitude=9.0)
    init = lambda f, o: o.ho_ground(0.5, -0.5, 1.0, 1.0, 1.0, 1.0, 1.0)
    f, Wo, obs = _run_both(p, init, 6)
    for name in OBS:
        assert rel_err(getattr(f, name), obs[name]) < 1e-12, name
    assert rel_err(f.W_init_gpu.get(), Wo) < 1e-10


def test_run_precision_form_c64():
    p, c = config1(4, 32)
    init = lambda f, o: o.ho_ground(c[0], c[1], c[2], c[3], 1.0, 1.0, 1.0)
    f, Wo, obs = _run_both(p, init, 21, np.complex64)
    for name in OBS:                          # reached: 4.1e-5 (observables), 2.8e-6 (state)
        assert rel_err(getattr(f, name), obs[name]) < 1e-4, name
    assert rel_err(f.W_init_gpu.get(), Wo) < 1e-5


def test_run_cat_state_config2_prefix():
    from configs import cat_xp
    p, c = config2(0, 32)
    f, o = _pair(p)
    W0 = cat_xp(f._coords, c)
    f.W_init_gpu.set(W0)
    f.timeSteps = 9
    f.fileName = None
    f.Run()
    Wo, obs = o.run(W0, 9)
    assert (W0.real < 0).any()
    for name in OBS:
        assert rel_err(getattr(f, name), obs[name]) < 1e-12, name
    assert rel_err(f.W_init_gpu.get(), Wo) < 1e-10


def test_nonfinite_state_raises():
    p, c = config1(0, 16)
    f, o = _pair(p)
    W0 = o.ho_ground(c[0], c[1], c[2], c[3], 1.0, 1.0, 1.0)
    W0[3, 3, 3, 3] = np.nan
    f.W_init_gpu.set(W0)
    f.timeSteps = 1
    f.fileName = None
    with pytest.raises(FloatingPointError):
        f.Run()


def test_run_fast64_vs_oracle():
    """64^4 takes k_r4 on the LA / LB layouts (3 iterations; the 20-iteration
    prefix is in test_gpu_tc.py)."""
    from configs import cat_xp
    p, c = config2(0, 64)
    f, o = _pair(p)
    W0 = cat_xp(f._coords, c)
    f.W_init_gpu.set(W0)
    f.timeSteps = 2
    f.fileName = None
    f.Run()
    Wo, obs = o.run(W0, 2)
    for name in OBS:
        assert rel_err(getattr(f, name), obs[name]) < 1e-12, name
    assert rel_err(f.W_init_gpu.get(), Wo) < 1e-10


@pytest.mark.parametrize("dtype,tol,wtol", [(np.complex128, 1e-12, 1e-10), (np.complex64, 5e-5, 1e-5)])
def test_fast64_matches_generic_kernels(dtype, tol, wtol, monkeypatch):
    from configs import cat_xp
    p, c = config2(3, 64)
    f1 = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
    monkeypatch.setenv("WIG_NO_FAST64", "1")
    f2 = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
    monkeypatch.delenv("WIG_NO_FAST64")
    W0 = cat_xp(f1._coords, c).astype(dtype)
    for f in (f1, f2):
        f.W_init_gpu.set(W0)
        f.timeSteps = 19
        f.fileName = None
        f.Run()
    for name in OBS:
        assert rel_err(getattr(f1, name), getattr(f2, name)) < tol, name
    assert rel_err(f1.W_init_gpu.get(), f2.W_init_gpu.get()) < wtol      # complex64 reached 3.4e-6


@pytest.mark.parametrize("n,dtype", [(32, np.complex128), (64, np.complex128), (64, np.complex64)])
def test_run_timed_matches_run(n, dtype):
    """The event-bracketed Run() launches the same kernels as the graph."""
    from configs import cat_xp
    p, c = config2(1, n)
    f = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
    W0 = cat_xp(f._coords, c).astype(dtype)
    iters = 70                      # more than the 64-slot event ring
    h1 = torch.empty((iters, _lib.WIG4D_NOBS), dtype=torch.float64, device="cuda")
    h2 = torch.empty_like(h1)
    f.W_init_gpu.set(W0)
    f.run_device(f.W_init_gpu, iters, h1)
    W1 = f.W_init_gpu.get()
    f.W_init_gpu.set(W0)
    ms = f.run_device_timed(f.W_init_gpu, iters, h2)
    W2 = f.W_init_gpu.get()
    assert rel_err(h2.cpu().numpy(), h1.cpu().numpy()) < 1e-14
    assert rel_err(W2, W1) < 1e-14
    assert all(m > 0 for m in ms)


@pytest.mark.parametrize("kernel", ["r4", "r4ring_f32"])
def test_run_r4_c64_vs_oracle(kernel, monkeypatch):
    """complex64 at 64^4 runs k_r4 on the LA / LB layouts (default) or the
    float32 ring on the plane-contiguous layouts (WIG_FAST64_KERNEL =
    r4ring_f32); the state comes back in the reference layout.  Float32 bar:
    2e-5 relative after 3 steps."""
    from configs import cat_xp
    if kernel == "r4ring_f32":
        monkeypatch.setenv("WIG_FAST64_KERNEL", kernel)
    p, c = config2(2, 64)
    f, o = _pair(p, np.complex64)
    assert f.plan_info()["run64_kernel"] == kernel
    W0 = cat_xp(f._coords, c)
    f.W_init_gpu.set(W0.astype(np.complex64))
    f.timeSteps = 2
    f.fileName = None
    f.Run()
    Wo, obs = o.run(W0.astype(np.complex64).astype(np.complex128), 2)
    for name in OBS:
        assert rel_err(getattr(f, name), obs[name]) < 2e-5, name
    assert rel_err(f.norm, obs["norms"]) < 2e-5
    assert rel_err(f.W_init_gpu.get(), Wo) < 2e-5


@pytest.mark.parametrize("dtype,tol,wtol", [(np.complex128, 1e-12, 1e-10), (np.complex64, 1e-4, 5e-6)])
def test_run_48_radix3_parity(dtype, tol, wtol):
    """48 = 3 x 16 points per axis: fused half-steps with a radix-3 pass."""
    p, c = config1(5, 48)
    init = lambda f, o: o.ho_ground(c[0], c[1], c[2], c[3], 1.0, 1.0, 1.0) / np.pi ** 2
    f, Wo, obs = _run_both(p, init, 6, dtype)
    assert f._plan_fused() == (True, True)
    for name in OBS:                          # complex64 reached 3.2e-5 (observables), 1.3e-6 (state)
        assert rel_err(getattr(f, name), obs[name]) < tol, name
    assert rel_err(f.W_init_gpu.get(), Wo) < wtol


@pytest.mark.parametrize("dtype,tol", [(np.complex128, 1e-13), (np.complex64, 2e-5)])
def test_k48_matches_generic(dtype, tol, monkeypatch):
    """The register-blocked 48 x 48 kinetic half-step (k_kin48: 3 x 3 DFTs,
    then 16 x 16 sub-plane DFTs) against the generic k_kinetic (WIG_NO_K48)."""
    p, c = config1(6, 48)
    f1 = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
    monkeypatch.setenv("WIG_NO_K48", "1")
    f2 = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
    W0 = (np.random.default_rng(3).standard_normal(f1.shape) * 1e-3).astype(dtype)
    out = []
    for f, env in ((f1, False), (f2, True)):
        if env:
            monkeypatch.setenv("WIG_NO_K48", "1")
        else:
            monkeypatch.delenv("WIG_NO_K48", raising=False)
        f.W_init_gpu.set(W0)
        f.timeSteps = 4
        f.fileName = None
        f.Run()
        out.append((f.norm, f.energy, f.W_init_gpu.get()))
    monkeypatch.delenv("WIG_NO_K48", raising=False)
    for a, b in zip(out[0], out[1]):
        assert rel_err(a, b) < tol


@pytest.mark.parametrize("variant", ["r4", "r4cluster", "r4ring_ts"])
def test_r4_variants_match_default(variant, monkeypatch):
    """complex128: k_r4 with plain (r4) or cluster (r4cluster) stores and
    k_r4ring on LA / LB with TMA tensor stores (r4ring_ts), against the
    default, k_r4ring on the plane-contiguous layouts: the same arithmetic
    (the ring kernels sum each plane's observables in another order)."""
    from configs import cat_xp
    p, c = config2(7, 64)
    f1 = make_frame(GPU_Wigner4D, p)
    monkeypatch.setenv("WIG_FAST64_KERNEL", variant)
    f2 = make_frame(GPU_Wigner4D, p)
    monkeypatch.delenv("WIG_FAST64_KERNEL")
    label = {"r4cluster": "r4"}.get(variant, variant)
    assert (f1.plan_info()["run64_kernel"], f2.plan_info()["run64_kernel"]) == ("r4ring_pc", label)
    W0 = cat_xp(f1._coords, c)
    for f in (f1, f2):
        f.W_init_gpu.set(W0)
        f.timeSteps = 9
        f.fileName = None
        f.Run()
    for name in OBS:
        assert rel_err(getattr(f1, name), getattr(f2, name)) < 1e-13, name
    assert rel_err(f1.W_init_gpu.get(), f2.W_init_gpu.get()) < 1e-12


def _notebook_windows(p):
    """The reference notebooks' ambiguity windows (delta N != 1)."""
    p.update(theta_x_amplitude=9.0, theta_y_amplitude=9.0, lambda_x_amplitude=9.0, lambda_y_amplitude=9.0)
    return p


def test_general_delta_fused_vs_oracle_32():
    """General delta on a 32^4 grid: both half-steps in k_dense_half."""
    p, c = config1(9, 32)
    p = _notebook_windows(p)
    init = lambda f, o: o.ho_ground(c[0], c[1], c[2], c[3], 1.0, 1.0, 1.0) / np.pi ** 2
    f, Wo, obs = _run_both(p, init, 4)
    for name in OBS:
        assert rel_err(getattr(f, name), obs[name]) < 1e-12, name
    assert rel_err(f.W_init_gpu.get(), Wo) < 1e-10


@pytest.mark.parametrize("dtype,tol", [(np.complex128, 1e-12), (np.complex64, 2e-6)])
def test_general_delta_fused_matches_unfused_64(dtype, tol, monkeypatch):
    """k_dense_half against the unfused FAFT passes on the notebook windows at 64^4."""
    from configs import cat_xp
    p, c = config2(10, 64)
    p = _notebook_windows(p)
    f1 = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
    monkeypatch.setenv("WIG_NO_DENSE_FUSED", "1")
    f2 = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
    monkeypatch.delenv("WIG_NO_DENSE_FUSED")
    W0 = cat_xp(f1._coords, c).astype(dtype)
    for f in (f1, f2):
        f.W_init_gpu.set(W0)
        f.timeSteps = 3
        f.fileName = None
        f.Run()
    for name in OBS:
        assert rel_err(getattr(f1, name), getattr(f2, name)) < tol, name
    # complex64 reached 6.2e-7 (observables) and 6.9e-7 (state)
    assert rel_err(f1.W_init_gpu.get(), f2.W_init_gpu.get()) < (1e-10 if dtype == np.complex128 else 2e-6)


@pytest.mark.parametrize("n", [32, 64])
def test_cat_state_initialiser(n):
    """CatState_GPU (psi-based W in (x, theta), then theta -> p) against the
    oracle's construction (1e-12), and at 64^4 against the analytic Wigner
    function of the cat state (tests/configs.cat_xp) after normalisation (at
    32^4 the theta window, |theta| < 6.3, cuts the interference term off)."""
    from configs import cat_xp
    p, c = config2(0, n)
    f, o = _pair(p)
    f.CatState_GPU(f.W_init_gpu, c[0], c[1], c[2], c[3], 1.5, 0.0)
    got = f.W_init_gpu.get()
    want = o.p_to_theta(o.cat_xtheta(c[0], c[1], c[2], c[3], 1.5, 0.0), -1)
    assert rel_err(got, want) < 1e-12
    assert (got.real < -1e-3 * got.real.max()).any()           # interference region
    if n == 64:
        ana = cat_xp(f._coords, c)
        assert rel_err(got / o.norm(got), ana / o.norm(ana)) < 1e-6


def test_faft_kernel_128_axis():
    """128-point axes (the p axes of the 64x128 grids), radix and fractional."""
    for dtype, tol in ((np.complex128, 1e-13), (np.complex64, 2e-6)):
        for axis, shape in ((0, (128, 8, 16, 16)), (1, (8, 128, 16, 8)), (2, (8, 16, 128, 16)), (3, (4, 16, 8, 128))):
            for dn in (1.0, -1.0, 0.71):
                a = _rand(shape, 17 + axis, dtype)
                g = GPUArray.to_gpu(a)
                sh = (ctypes.c_int * 4)(*shape)
                wd = _lib.C128 if dtype == np.complex128 else _lib.C64
                _lib.call("wig_faft", g.ptr, sh, wd, axis, 0.125, dn / 128, 1.0, None)
                torch.cuda.synchronize()
                want = faft(a.astype(np.complex128), axis, 0.125, dn / 128)
                assert rel_err(g.get(), want) < tol, (dtype, axis, dn)


def _frame_64_128():
    """The reference's 64x128 frame (instances/Wigner4D_64_128): shape
    (N_py, N_y, N_px, N_x) = (64, 64, 128, 128)."""
    p = dict(gridDIM_p_y=64, gridDIM_y=64, gridDIM_p_x=128, gridDIM_x=128, dt=0.05, timeSteps=0, mass=1.0,
             p_y_amplitude=7.0, y_amplitude=7.0, p_x_amplitude=8.0, x_amplitude=8.0,
             theta_y_amplitude=9.0, lambda_y_amplitude=9.0, theta_x_amplitude=9.0, lambda_x_amplitude=9.0,
             kineticString="0.5*(p_x*p_x + p_y*p_y)", potentialString="0.5*pow(x,2) + 0.5*pow(y,2)",
             D_theta_x=1e-4, D_theta_y=1e-4, D_lambda_x=1e-4, D_lambda_y=1e-4)
    return make_frame(GPU_Wigner4D, p)


def test_faft128_256_shims_and_64_128_wrappers():
    """FAFT128_4D_Z2Z / FAFT256_4D_Z2Z on the (64, 64, 128, 128) array, bound
    as cuda_faft64 / cuda_faft128 by the reference's 64x128 wrappers
    (GPU_Wigner4D.py:387-405): the package's Fourier_*_64_128_GPU against the
    wrappers' own call sequence through the shims, and one shim call against
    the oracle's FAFT."""
    f = _frame_64_128()
    assert f.shape == (64, 64, 128, 128)
    a = (_rand(f.shape, 21) * 1e-3).astype(np.complex128)
    size = float(np.prod(f.shape))
    seqs = {
        "Fourier_X_To_Lambda_64_128_GPU": [("FAFT256_4D_Z2Z", f.dp_x, f.delta_p_x, 1), ("FAFT128_4D_Z2Z", f.dp_y, f.delta_p_y, 2)],
        "Fourier_Lambda_To_X_64_128_GPU": [("FAFT256_4D_Z2Z", f.dp_x, -f.delta_p_x, 1), ("FAFT128_4D_Z2Z", f.dp_y, -f.delta_p_y, 2)],
        "Fourier_P_To_Theta_64_128_GPU": [("FAFT256_4D_Z2Z", f.dp_x, f.delta_p_x, 0), ("FAFT128_4D_Z2Z", f.dp_y, f.delta_p_y, 3)],
        "Fourier_Theta_To_P_64_128_GPU": [("FAFT256_4D_Z2Z", f.dp_x, -f.delta_p_x, 0), ("FAFT128_4D_Z2Z", f.dp_y, -f.delta_p_y, 3)],
    }
    for wrapper, calls in seqs.items():
        g1 = GPUArray.to_gpu(a)
        getattr(f, wrapper)(g1)
        g2 = GPUArray.to_gpu(a)
        for name, d, delta, axis in calls:
            _lib.call(name, g2.ptr, d, delta, 0, axis, 1.0)
        torch.cuda.synchronize()
        want = g2.get() / size
        assert rel_err(g1.get(), want) < 1e-14, wrapper
    g = GPUArray.to_gpu(a)
    _lib.call("FAFT128_4D_Z2Z", g.ptr, f.dp_y, f.delta_p_y, 0, 3, 1.0)
    torch.cuda.synchronize()
    assert rel_err(g.get(), faft(a, 3, f.dp_y, f.delta_p_y)) < 1e-12


def test_run_config3_grid_vs_oracle():
    """Config 3's grid: 64 (x) x 128 (p_x) x 64 (y) x 128 (p_y), i.e. shape
    (128, 64, 128, 64), config-1 potential and initial state, dt = 0.005,
    delta = 1/N per axis: three Run() iterations of the complex128 drop-in
    (1e-12) and of the complex64 form (5e-5) against one oracle run."""
    p = w4d_params(64, q=0.1, kappa=0.05, D=0.01, dt=0.005, n_p=128)
    o = Wigner4DOracle(p)
    W0 = o.ho_ground(0.4, -0.3, 0.2, -0.1, 1.0, 1.0, 1.0)
    Wo, obs = o.run(W0, 2)
    # delta = 1/N on every axis, so the energy of the ground state moves slowly
    assert np.all(np.abs(np.diff(obs["energy"])) < 0.01 * abs(obs["energy"][0]))
    for dtype, tol in ((np.complex128, 1e-12), (np.complex64, 5e-5)):
        f = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
        assert f.shape == (128, 64, 128, 64)
        f.W_init_gpu.set(W0.astype(dtype))
        f.timeSteps = 2
        f.fileName = None
        f.Run()
        for name in OBS:
            assert rel_err(getattr(f, name), obs[name]) < tol, (dtype, name)
        assert rel_err(f.W_init_gpu.get(), Wo) < (1e-10 if dtype == np.complex128 else 10 * tol), dtype
        del f
