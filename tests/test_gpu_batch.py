"""Batched Run() (WignerBatch / wig4d_run_batch) against each instance's own Run().

The batch replays the same kernels per instance inside one graph per step,
so every instance must end bit-for-bit where its own Run() ends (checked to
1e-13 relative, histories and final states).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from configs import config4, gaussian_xp  # noqa: E402
from frames import make_frame, rel_err  # noqa: E402
from pywignercuda2_b200 import GPU_Wigner4D, WignerBatch  # noqa: E402


def _frames(sizes, dtypes, steps, seed=3):
    out = []
    for (params, c), dt in zip(config4(seed, sizes), dtypes):
        params = dict(params, timeSteps=steps)
        f = make_frame(GPU_Wigner4D, params, complex_dtype=dt)
        f.fileName = None
        W0 = gaussian_xp(f._coords, c).astype(dt)
        out.append((f, W0))
    return out


def test_batch_matches_single_runs():
    sizes = (16, 32, 48, 64, 32, 64)
    dtypes = (np.complex128, np.complex64, np.complex64, np.complex64, np.complex128, np.complex128)
    steps = 7
    ref = []
    for f, W0 in _frames(sizes, dtypes, steps):
        f.W_init_gpu.set(W0)
        f.Run()
        ref.append((f.W_init_gpu.get(), np.array(f.energy), np.array(f.norm), np.array(f.average_x)))
    fr = _frames(sizes, dtypes, steps)
    for f, W0 in fr:
        f.W_init_gpu.set(W0)
    WignerBatch([f for f, _ in fr]).Run()
    for (f, _), (W, e, n, x) in zip(fr, ref):
        assert len(f.energy) == steps + 1
        assert rel_err(f.energy, e) < 1e-13
        assert rel_err(f.norm, n) < 1e-13
        assert rel_err(f.average_x, x) < 1e-13
        assert rel_err(f.W_init_gpu.get(), W) < 1e-13


def test_batch_rejects_repeated_frame():
    (f, W0), = _frames((16,), (np.complex128,), 2)
    with pytest.raises(ValueError):
        WignerBatch([f, f])


def test_batch_unequal_steps_rejected():
    fr = _frames((16, 16), (np.complex128, np.complex128), 2)
    fr[1][0].timeSteps = 3
    with pytest.raises(ValueError):
        WignerBatch([f for f, _ in fr]).Run()


def test_autotune_choices_and_cache():
    """wig4d_autotune: the tuned plan gives the untuned plan's results, the
    choice is reported, and a second plan with the same key takes the cached
    choice without timing."""
    from configs import config1, config2, cat_xp
    from frames import rel_err
    out = {}
    for n, dtype, tc in ((48, np.complex128, False), (64, np.complex64, "auto")):
        p, c = (config1(2, n) if n == 48 else config2(2, n))
        ref = make_frame(GPU_Wigner4D, p, complex_dtype=dtype)
        f = make_frame(GPU_Wigner4D, p, complex_dtype=dtype, autotune="force", tensor_cores=tc)
        ch = f.autotune_choice
        assert ch is not None and ch["timed"] >= 1
        g = make_frame(GPU_Wigner4D, p, complex_dtype=dtype, autotune=True, tensor_cores=tc)
        assert g.autotune_choice["timed"] == 0 and g.autotune_choice["engine"] == ch["engine"]
        W0 = cat_xp(f._coords, c).astype(dtype)
        for fr in (ref, f):
            fr.W_init_gpu.set(W0)
            fr.timeSteps = 4
            fr.fileName = None
            fr.Run()
        tol = 1e-12 if dtype == np.complex128 else 3e-4
        assert rel_err(f.energy, ref.energy) < tol
        assert rel_err(f.W_init_gpu.get(), ref.W_init_gpu.get()) < (1e-10 if dtype == np.complex128 else 1e-4)
        out[n] = ch
    assert out[64]["engine"] in ("k_r4 plain stores", "k_r4 cluster stores", "k_tc64")
    assert out[48]["engine"] == "per-size kernels"
