"""Factor tables for the fused half-step kernels.

A half-step multiplies the transformed state by r * exp(-i phi) at every
point of a 4-D grid (exp_p_lambda_GPU, GPU_Wigner4D.py:251-262;
exp_x_theta_GPU, GPU_Wigner4D.py:269-281).  Instead of evaluating the user's
expression per point on the GPU, the phase is split once, on the host in
float64, into a sum of terms that each depend on two grid axes:

    phi(i0, i1, i2, i3) = sum_{a<b} g_ab(i_a, i_b)

(the anchored second-order decomposition: every g_ab is phi with the other
two indices at an anchor, minus the one-axis terms).  The kernels then
multiply by the product of at most six N_a x N_b complex tables, each a few
kilobytes that stay in L1.  The split is exact whenever the Bopp difference
of the potential has no three-axis interaction -- true for any potential of
the form f(x) + g(y) + c x y, any kinetic energy K1(p_x) + K2(p_y) and the
reference's notebooks.  It is verified against the direct evaluation on the
full grid; when it does not hold the factor falls back to one full 4-D
table (one extra read per half-step).
"""
import numpy as np

PAIRS = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]


def _coords(vals, axes):
    """Broadcastable coordinate arrays for the listed axes (others length 1)."""
    out = []
    for a in range(4):
        sh = [1, 1, 1, 1]
        if a in axes:
            sh[a] = len(vals[a])
            out.append(np.asarray(vals[a], np.float64).reshape(sh))
        else:
            out.append(None)
    return out


def _eval_on(fn, vals, fixed):
    """fn evaluated with axis a at all values if a not in fixed, else at vals[a][fixed[a]]."""
    args = []
    for a in range(4):
        sh = [1, 1, 1, 1]
        if a in fixed:
            args.append(np.full(sh, vals[a][fixed[a]], np.float64))
        else:
            sh[a] = len(vals[a])
            args.append(np.asarray(vals[a], np.float64).reshape(sh))
    return fn(*args)


def pairwise_phase(fn, vals, anchor=None):
    """Anchored pairwise split of phi = fn(c0, c1, c2, c3).

    Returns {(a, b): 2-D array g_ab} with phi ~= sum g_ab.  The one-axis and
    constant parts are folded into the first pair containing their axis.
    """
    n = [len(v) for v in vals]
    if anchor is None:
        anchor = [k // 2 for k in n]
    f0 = float(np.asarray(_eval_on(fn, vals, {a: anchor[a] for a in range(4)})).reshape(()))
    h = []
    for a in range(4):
        fixed = {b: anchor[b] for b in range(4) if b != a}
        h.append(np.asarray(_eval_on(fn, vals, fixed), np.float64).reshape(n[a]))
    g = {}
    for a, b in PAIRS:
        fixed = {c: anchor[c] for c in range(4) if c not in (a, b)}
        g[(a, b)] = np.asarray(_eval_on(fn, vals, fixed), np.float64).reshape(n[a], n[b]).copy()
    # phi ~= sum g_ab - 2 sum h_a + 3 f0
    done = set()
    for a, b in PAIRS:
        for c in (a, b):
            if c not in done:
                if c == a:
                    g[(a, b)] -= 2.0 * h[c][:, None]
                else:
                    g[(a, b)] -= 2.0 * h[c][None, :]
                done.add(c)
    g[PAIRS[0]] += 3.0 * f0
    return g


def _pair_sum(g, slab, n):
    """sum of the pair terms over axis-0 slab [i0s] x full other axes."""
    tot = 0.0
    for (a, b), t in g.items():
        if a == 0:
            part = t[slab]
            sh = [part.shape[0], 1, 1, 1]
            sh[b] = n[b]
            tot = tot + part.reshape(sh)
        else:
            sh = [1, 1, 1, 1]
            sh[a], sh[b] = n[a], n[b]
            tot = tot + t.reshape(sh)
    return tot


def build_factor(phase_fn, mags, vals, tol=1e-11, chunk=8):
    """Factor tables for r * exp(-i phi).

    phase_fn(c0, c1, c2, c3) -> phi on broadcast coordinate arrays (float64).
    mags: list of 4 arrays (or None) of per-axis real magnitudes whose
    product is r.  vals: the 4 coordinate vectors.

    Returns (tables, full) where tables is a list of (axis_a, axis_b,
    complex128 2-D array) and full is None, or tables == [] and full is the
    complex128 4-D factor when the phase is not pairwise separable.
    """
    n = [len(v) for v in vals]
    g = pairwise_phase(phase_fn, vals)
    # verify on the full grid, a slab of axis 0 at a time
    ok = True
    maxphi = 0.0
    for s0 in range(0, n[0], chunk):
        sl = slice(s0, min(n[0], s0 + chunk))
        c = [np.asarray(vals[0][sl], np.float64).reshape(-1, 1, 1, 1)]
        for a in (1, 2, 3):
            sh = [1, 1, 1, 1]
            sh[a] = n[a]
            c.append(np.asarray(vals[a], np.float64).reshape(sh))
        phi = np.asarray(phase_fn(*c), np.float64)
        phi = np.broadcast_to(phi, (sl.stop - sl.start, n[1], n[2], n[3]))
        approx = _pair_sum(g, sl, n)
        err = np.max(np.abs(phi - approx)) if phi.size else 0.0
        maxphi = max(maxphi, float(np.max(np.abs(phi))) if phi.size else 0.0)
        if not np.isfinite(err) or err > tol * max(1.0, maxphi):
            ok = False
            break
    if ok:
        tables = []
        mag_done = set()
        for a, b in PAIRS:
            t = np.exp(-1j * g[(a, b)])
            for c in (a, b):
                if mags[c] is not None and c not in mag_done:
                    m = np.asarray(mags[c], np.float64)
                    t = t * (m[:, None] if c == a else m[None, :])
                    mag_done.add(c)
            if np.max(np.abs(t - 1.0)) > 0.0:
                tables.append((a, b, np.ascontiguousarray(t, np.complex128)))
        return tables, None
    # full 4-D table
    full = np.empty(tuple(n), np.complex128)
    for s0 in range(0, n[0], chunk):
        sl = slice(s0, min(n[0], s0 + chunk))
        c = [np.asarray(vals[0][sl], np.float64).reshape(-1, 1, 1, 1)]
        for a in (1, 2, 3):
            sh = [1, 1, 1, 1]
            sh[a] = n[a]
            c.append(np.asarray(vals[a], np.float64).reshape(sh))
        phi = np.broadcast_to(np.asarray(phase_fn(*c), np.float64), (sl.stop - sl.start, n[1], n[2], n[3]))
        r = np.ones_like(phi)
        for a in range(4):
            if mags[a] is not None:
                sh = [1, 1, 1, 1]
                sh[a] = n[a]
                m = np.asarray(mags[a], np.float64)
                r = r * (m[sl].reshape(-1, 1, 1, 1) if a == 0 else m.reshape(sh))
        full[sl] = r * np.exp(-1j * phi)
    return [], full
