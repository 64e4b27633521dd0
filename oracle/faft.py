"""Restatement of the reference's FAFT transform (test infrastructure only).

The reference calls ``FAFT{64,128}_4D_Z2Z(ptr, d, delta, segment, axis, NF)``
(GPU_Wigner4D.py:32-58; call sites GPU_Wigner4D.py:409-427,
GPU_WignerDirac4D.py:1428-1458).  The library is absent; its contract, pinned
against the notebook norms, is the scaled centred fractional DFT along one
axis of a 4D complex128 array, in place::

    F[k] = 2 N d * sum_n f[n] exp(-2 pi i delta (n - N/2)(k - N/2))

with ``delta`` signed (the "inverse" call passes ``-delta``).  ``segment`` and
``NF`` are always 0 and 1 at the call sites and carry no meaning here.
"""
import numpy as np

# threads for the FFT path (1 = NumPy's single-threaded pocketfft; more uses
# scipy.fft with that many workers) -- set by bench.py's CPU legs only
FFT_WORKERS = 1


def faft_matrix(n, d, delta):
    """Dense N x N matrix M[k, n] of the transform above."""
    idx = np.arange(n, dtype=np.float64) - n // 2
    return (2.0 * n * d) * np.exp(-2j * np.pi * delta * np.outer(idx, idx))


def faft(a, axis, d, delta):
    """Apply the FAFT along ``axis`` of ``a`` (returns a new array).

    A dense product, exact for any delta.  When ``|delta| * N == 1`` and
    ``N % 4 == 0`` it is a centred DFT and NumPy's FFT gives the same numbers
    faster: F = 2Nd (-1)^k FFT((-1)^n f) for delta>0, and with the inverse FFT
    times N for delta<0.
    """
    n = a.shape[axis]
    if abs(abs(delta) * n - 1.0) < 1e-15 and n % 4 == 0:
        return _faft_fft(a, axis, d, delta > 0)
    m = faft_matrix(n, d, delta)
    b = np.ascontiguousarray(np.moveaxis(a, axis, -1))
    out = (b.reshape(-1, n) @ m.T).reshape(b.shape)
    return np.moveaxis(out, -1, axis)


def _faft_fft(a, axis, d, forward):
    n = a.shape[axis]
    shape = [1] * a.ndim
    shape[axis] = n
    sgn = ((-1.0) ** np.arange(n)).reshape(shape)
    if FFT_WORKERS > 1:
        import scipy.fft as sf
        if forward:
            out = sf.fft(a * sgn, axis=axis, workers=FFT_WORKERS)
        else:
            out = sf.ifft(a * sgn, axis=axis, workers=FFT_WORKERS) * n
    elif forward:
        out = np.fft.fft(a * sgn, axis=axis)
    else:
        out = np.fft.ifft(a * sgn, axis=axis) * n
    return out * sgn * (2.0 * n * d)
