"""GPU parity of the scalar Wigner4D path against the NumPy oracle.

Tolerances: complex128 (the drop-in) must match the oracle to 1e-12
relative in norms and observables and 1e-10 in max|dW| / max|W|, the
north-star bar.  complex64 (the precision form) is held to 1e-4 relative on
the observables over the short runs here: its float32 state and transforms
drift from the float64 result by about 1e-6 per step on these grids.
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
    for name in OBS:
        assert rel_err(getattr(f, name), obs[name]) < 1e-4, name
    assert rel_err(f.W_init_gpu.get(), Wo) < 1e-3


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
    """64^4 takes the register-resident ping-pong kernels (k_kin64 / k_pot64)."""
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


@pytest.mark.parametrize("dtype,tol", [(np.complex128, 1e-12), (np.complex64, 1e-4)])
def test_fast64_matches_generic_kernels(dtype, tol, monkeypatch):
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
    assert rel_err(f1.W_init_gpu.get(), f2.W_init_gpu.get()) < (100 * tol if tol < 1e-6 else 10 * tol)


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


def test_run_quad64_c64_vs_oracle():
    """complex64 at 64^4 runs k_quad64 on the LA / LB layouts; the state comes
    back in the reference layout.  Float32 bar: 2e-5 relative after 3 steps."""
    from configs import cat_xp
    p, c = config2(2, 64)
    f, o = _pair(p, np.complex64)
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


@pytest.mark.parametrize("dtype,tol", [(np.complex128, 1e-12), (np.complex64, 1e-4)])
def test_run_48_radix3_parity(dtype, tol):
    """48 = 3 x 16 points per axis: fused half-steps with a radix-3 pass."""
    p, c = config1(5, 48)
    init = lambda f, o: o.ho_ground(c[0], c[1], c[2], c[3], 1.0, 1.0, 1.0) / np.pi ** 2
    f, Wo, obs = _run_both(p, init, 6, dtype)
    assert f._plan_fused() == (True, True)
    for name in OBS:
        assert rel_err(getattr(f, name), obs[name]) < tol, name
    assert rel_err(f.W_init_gpu.get(), Wo) < (1e-10 if tol < 1e-6 else 1e-3)


@pytest.mark.parametrize("pot48", [False, True])
@pytest.mark.parametrize("dtype,tol", [(np.complex128, 1e-13), (np.complex64, 2e-5)])
def test_k48_matches_generic(dtype, tol, pot48, monkeypatch):
    """The register-blocked 48 x 48 kinetic half-step (k_kin48: 3 x 3 DFTs,
    then 16 x 16 sub-plane DFTs), and with WIG_POT48 the potential one
    (k_pot48), against the generic k_kinetic / k_potential_g (WIG_NO_K48)."""
    if pot48:
        monkeypatch.setenv("WIG_POT48", "1")
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


@pytest.mark.parametrize("dtype,tol", [(np.complex128, 1e-12), (np.complex64, 1e-4)])
def test_r4_matches_pair_kernels(dtype, tol, monkeypatch):
    """The default 64^4 kernels (k_r4 with cluster stores) against
    k_half64 / k_quad64."""
    from configs import cat_xp
    p, c = config2(6, 64)
    f1 = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
    monkeypatch.setenv("WIG_FAST64_KERNEL", "pair")
    f2 = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
    monkeypatch.delenv("WIG_FAST64_KERNEL")
    assert f1.plan_info()["run64_kernel"] == "r4"
    assert f2.plan_info()["run64_kernel"] == ("half64" if dtype == np.complex128 else "quad64")
    W0 = cat_xp(f1._coords, c).astype(dtype)
    for f in (f1, f2):
        f.W_init_gpu.set(W0)
        f.timeSteps = 9
        f.fileName = None
        f.Run()
    for name in OBS:
        assert rel_err(getattr(f1, name), getattr(f2, name)) < tol, name
    assert rel_err(f1.W_init_gpu.get(), f2.W_init_gpu.get()) < (100 * tol if tol < 1e-6 else 10 * tol)


@pytest.mark.parametrize("variant", ["r4t", "r4"])
def test_r4_variants_match_default(variant, monkeypatch):
    """complex128: k_r4 with TMA plane loads (r4t) and k_r4 with plain stores
    (r4) against the default k_r4 with cluster stores: the same arithmetic."""
    from configs import cat_xp
    p, c = config2(7, 64)
    f1 = make_frame(GPU_Wigner4D, p)
    monkeypatch.setenv("WIG_FAST64_KERNEL", variant)
    f2 = make_frame(GPU_Wigner4D, p)
    monkeypatch.delenv("WIG_FAST64_KERNEL")
    assert (f1.plan_info()["run64_kernel"], f2.plan_info()["run64_kernel"]) == ("r4", variant)
    W0 = cat_xp(f1._coords, c)
    for f in (f1, f2):
        f.W_init_gpu.set(W0)
        f.timeSteps = 9
        f.fileName = None
        f.Run()
    for name in OBS:
        assert rel_err(getattr(f1, name), getattr(f2, name)) < 1e-13, name
    assert rel_err(f1.W_init_gpu.get(), f2.W_init_gpu.get()) < 1e-12


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_r4p_matches_r4(dtype, monkeypatch):
    """The persistent k_r4p (next plane prefetched) runs k_r4's arithmetic
    plane by plane: the same history and state."""
    from configs import cat_xp
    p, c = config2(8, 64)
    f1 = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
    monkeypatch.setenv("WIG_FAST64_KERNEL", "r4p")
    f2 = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
    monkeypatch.delenv("WIG_FAST64_KERNEL")
    assert (f1.plan_info()["run64_kernel"], f2.plan_info()["run64_kernel"]) == ("r4", "r4p")
    W0 = cat_xp(f1._coords, c).astype(dtype)
    for f in (f1, f2):
        f.W_init_gpu.set(W0)
        f.timeSteps = 9
        f.fileName = None
        f.Run()
    for name in OBS:
        assert rel_err(getattr(f1, name), getattr(f2, name)) < 1e-13, name
    assert rel_err(f1.W_init_gpu.get(), f2.W_init_gpu.get()) < 1e-13


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_r4_split_bitwise(dtype, monkeypatch):
    """k_r4 as two launches per half-step (WIG_R4_SPLIT: forward half to a
    scratch buffer, inverse half from it) runs the same arithmetic: the same
    bits in the history and the state."""
    from configs import cat_xp
    p, c = config2(12, 64)
    f1 = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
    monkeypatch.setenv("WIG_R4_SPLIT", "1")
    f2 = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
    monkeypatch.delenv("WIG_R4_SPLIT")
    W0 = cat_xp(f1._coords, c).astype(dtype)
    for f in (f1, f2):
        f.W_init_gpu.set(W0)
        f.timeSteps = 7
        f.fileName = None
        f.Run()
    for name in OBS:
        assert np.array_equal(getattr(f1, name), getattr(f2, name)), name
    assert np.array_equal(f1.W_init_gpu.get(), f2.W_init_gpu.get())


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


@pytest.mark.parametrize("dtype,tol", [(np.complex128, 1e-12), (np.complex64, 1e-4)])
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
    assert rel_err(f1.W_init_gpu.get(), f2.W_init_gpu.get()) < (1e-10 if tol < 1e-6 else 1e-3)
