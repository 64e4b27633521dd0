"""Run() with snapshots and checkpoint/resume against a plain Run().

Chunked runs (WIG_RUN_KEEP_NORM between chunks) must reproduce the
observables and the final state of one Run() (1e-13 relative), and each
snapshot must be the normalised state a shorter Run() reaches.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from configs import cat_xp, config2  # noqa: E402
from frames import make_frame, rel_err  # noqa: E402
from pywignercuda2_b200 import GPU_Wigner4D  # noqa: E402

OBS = ["average_x", "average_p_x", "average_x_square", "average_p_x_square", "average_y",
       "average_p_y", "average_y_square", "average_p_y_square", "energy"]


def _frame(n, dtype, steps, **kw):
    p, c = config2(4, n)
    f = make_frame(GPU_Wigner4D, dict(p, timeSteps=steps), complex_dtype=dtype, **kw)
    f.fileName = None
    W0 = cat_xp(f._coords, c).astype(dtype)
    f.W_init_gpu.set(W0)
    return f, W0


@pytest.mark.parametrize("n,dtype", [(32, np.complex128), (64, np.complex128), (64, np.complex64)])
def test_snapshots_do_not_change_the_run(n, dtype):
    # complex64: the chunks' first steps divide by norms that differ in the
    # last float32 places, which the float32 noise floor turns into 1e-6-level
    # differences of the edge-weighted moments after a few steps
    tol = 1e-13 if dtype == np.complex128 else 1e-4
    a, _ = _frame(n, dtype, 11)
    a.Run()
    b, W0 = _frame(n, dtype, 11, snapshotEvery=4)
    b.Run()
    for name in OBS:
        assert rel_err(getattr(b, name), getattr(a, name)) < tol, name
    assert len(b.energy) == 12
    assert rel_err(b.W_init_gpu.get(), a.W_init_gpu.get()) < tol
    assert [t for t, _ in b.snapshots] == pytest.approx([0.0, 4 * b.dt, 8 * b.dt])
    # snapshot 1 (after 4 steps) is the state a 4-step Run() ends in (Run()
    # renormalises at the end, as the snapshot is normalised)
    c, _ = _frame(n, dtype, 3)
    c.Run()
    assert rel_err(b.snapshots[1][1], c.W_init_gpu.get()) < (1e-12 if tol < 1e-6 else 1e-4)
    assert rel_err(b.snapshots[0][1], W0 / complex(a.norm[0])) < tol


def test_checkpoint_resume(tmp_path):
    a, _ = _frame(32, np.complex128, 9)
    a.Run()
    b, _ = _frame(32, np.complex128, 4)
    b.Run()
    b.save_checkpoint(str(tmp_path / "ck.npz"))
    c, _ = _frame(32, np.complex128, 4)
    c.W_init_gpu.set(np.zeros(c.shape, np.complex128))
    c.load_checkpoint(str(tmp_path / "ck.npz"))
    c.Run()
    # rows 5..9 of the uninterrupted run are rows 0..4 of the resumed one
    for name in OBS:
        assert rel_err(getattr(c, name), np.asarray(getattr(a, name))[5:]) < 1e-12, name
    assert rel_err(c.W_init_gpu.get(), a.W_init_gpu.get()) < 1e-12
    assert c.time_offset == pytest.approx(5 * b.dt)
    assert c.timeRange[0] == pytest.approx(5 * b.dt)


def test_snapshot_times_after_resume(tmp_path):
    """Snapshots of a resumed run carry the checkpoint's time offset, as its
    Ehrenfest timeRange does."""
    b, _ = _frame(32, np.complex128, 4)
    b.Run()
    b.save_checkpoint(str(tmp_path / "ck.npz"))
    c, _ = _frame(32, np.complex128, 8, snapshotEvery=4)
    c.load_checkpoint(str(tmp_path / "ck.npz"))
    c.Run()
    t0 = 5 * b.dt
    assert [t for t, _ in c.snapshots] == pytest.approx([t0, t0 + 4 * c.dt, t0 + 8 * c.dt])
    assert c.timeRange[0] == pytest.approx(t0)
    assert c.snapshots[0][0] == pytest.approx(c.timeRange[0])
