"""Low-rank tables for fields evaluated at Bopp-shifted points.

The Dirac potential propagator needs A1, A2, A3 at x -+ theta/2, y -+ theta/2
at every point of the (x, theta) grid (GPU_WignerDirac4D.py:580-604).  With
u = x -+ theta_x/2 (a function of the two indices ix, itheta_x) and
v = y -+ theta_y/2 (of iy, itheta_y), the values form the matrix
M[(ix, itx), (iy, ity)] = A(u, v).  Adaptive cross approximation with
complete pivoting writes it as sum_r F_r(ix, itx) G_r(iy, ity) with the
smallest rank that reproduces M to ``tol`` relative on every entry; the
kernel then evaluates A with ``rank`` fused multiply-adds.  Any polynomial
of degree d in one of the coordinates has rank <= d + 1 (the reference's
notebooks need rank 1 or 2); the construction is checked on the full matrix
and raises if the rank would exceed ``max_rank``.
"""
import numpy as np


class RankError(ValueError):
    """The field is not of low rank on this grid."""


def cross_approximation(M, tol=1e-14, max_rank=16):
    """Complete-pivot ACA of a dense matrix: returns (F, G) with
    M ~= F @ G, F of shape (m, r), G of shape (r, n)."""
    M = np.asarray(M, dtype=np.float64)
    R = np.array(M, copy=True)
    m, n = R.shape
    scale = float(np.max(np.abs(R))) if R.size else 0.0
    Fs, Gs = [], []
    if scale == 0.0:
        return np.zeros((m, 0)), np.zeros((0, n))
    while True:
        k = int(np.argmax(np.abs(R)))
        i, j = divmod(k, n)
        piv = R[i, j]
        if abs(piv) <= tol * scale:
            break
        if len(Fs) == max_rank:
            raise RankError("rank above %d (residual %.3e)" % (max_rank, abs(piv) / scale))
        f = R[:, j].copy()
        g = R[i, :].copy() / piv
        R -= np.outer(f, g)
        Fs.append(f)
        Gs.append(g)
    F = np.stack(Fs, axis=1) if Fs else np.zeros((m, 0))
    G = np.stack(Gs, axis=0) if Gs else np.zeros((0, n))
    err = float(np.max(np.abs(M - F @ G)))
    if err > 64 * tol * scale:
        raise RankError("cross approximation residual %.3e" % (err / scale))
    return F, G


def field_tables(fn, U, V, tol=1e-14, max_rank=16):
    """fn(u, v) on u = U (2-D array over (ix, itx)) and v = V (over (iy, ity)).

    Returns (F, G): F of shape (r, *U.shape), G of shape (r, *V.shape)."""
    M = np.asarray(fn(U.reshape(-1, 1), V.reshape(1, -1)), np.float64)
    M = np.broadcast_to(M, (U.size, V.size))
    F, G = cross_approximation(M, tol, max_rank)
    r = F.shape[1]
    return F.T.reshape((r,) + U.shape), G.reshape((r,) + V.shape)
