"""Factor tables for the fused half-step kernels.

A half-step multiplies the transformed state by r * exp(-i phi) at every
point of a 4-D grid (exp_p_lambda_GPU, GPU_Wigner4D.py:251-262;
exp_x_theta_GPU, GPU_Wigner4D.py:269-281).  Instead of evaluating the user's
expression per point on the GPU, the phase is split once, on the host in
float64, into a sum of terms that each depend on two grid axes:

    phi(i0, i1, i2, i3) = sum_{a<b} g_ab(i_a, i_b)

(the anchored second-order decomposition: the value at an anchor point,
one-axis terms with the other three indices at the anchor, and pair terms
with the one-axis parts removed).  The kernels then multiply by the product
of a few small complex tables (1-D for the one-axis terms and the damping
magnitudes, 2-D only for real two-axis interactions), a few kilobytes that
stay in L1.  The split is exact whenever the Bopp difference
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
    """Anchored second-order (ANOVA) split of phi = fn(c0, c1, c2, c3).

    Returns (e0, singles, pairs): phi ~= e0 + sum_a singles[a](i_a)
    + sum_{a<b} pairs[(a, b)](i_a, i_b), where with f0 = phi(anchor),
    h_a = phi with only axis a free and g_ab = phi with only a, b free:
    singles[a] = h_a - f0 and pairs[(a, b)] = g_ab - h_a - h_b + f0.
    """
    n = [len(v) for v in vals]
    if anchor is None:
        anchor = [k // 2 for k in n]
    f0 = float(np.asarray(_eval_on(fn, vals, {a: anchor[a] for a in range(4)})).reshape(()))
    h = []
    for a in range(4):
        fixed = {b: anchor[b] for b in range(4) if b != a}
        h.append(np.asarray(_eval_on(fn, vals, fixed), np.float64).reshape(n[a]))
    pairs = {}
    for a, b in PAIRS:
        fixed = {c: anchor[c] for c in range(4) if c not in (a, b)}
        g = np.asarray(_eval_on(fn, vals, fixed), np.float64).reshape(n[a], n[b])
        pairs[(a, b)] = g - h[a][:, None] - h[b][None, :] + f0
    singles = [h[a] - f0 for a in range(4)]
    return f0, singles, pairs


def _split_sum(split, slab, n):
    """The split evaluated over axis-0 slab [slab] x full other axes."""
    e0, singles, pairs = split
    tot = e0
    for a in range(4):
        sh = [1, 1, 1, 1]
        if a == 0:
            part = singles[0][slab]
            sh[0] = part.shape[0]
        else:
            part = singles[a]
            sh[a] = n[a]
        tot = tot + part.reshape(sh)
    for (a, b), t in pairs.items():
        if a == 0:
            part = t[slab]
            sh = [part.shape[0], 1, 1, 1]
            sh[b] = n[b]
        else:
            part = t
            sh = [1, 1, 1, 1]
            sh[a], sh[b] = n[a], n[b]
        tot = tot + part.reshape(sh)
    return tot


def build_factor(phase_fn, mags, vals, tol=1e-11, chunk=8):
    """Factor tables for r * exp(-i phi).

    phase_fn(c0, c1, c2, c3) -> phi on broadcast coordinate arrays (float64).
    mags: list of 4 arrays (or None) of per-axis real magnitudes whose
    product is r.  vals: the 4 coordinate vectors.

    Returns (tables, full) where tables is a list of (axis_a, axis_b,
    complex128 array): a 1-D table over axis_a when axis_b == -1, else a
    2-D table over (axis_a, axis_b); full is None.  When the phase is not
    pairwise separable, tables == [] and full is the complex128 4-D factor.
    One-axis terms (and the magnitudes) are 1-D tables, so a pair table
    appears only for a real two-axis interaction.
    """
    n = [len(v) for v in vals]
    split = pairwise_phase(phase_fn, vals)
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
        approx = _split_sum(split, sl, n)
        err = np.max(np.abs(phi - approx)) if phi.size else 0.0
        maxphi = max(maxphi, float(np.max(np.abs(phi))) if phi.size else 0.0)
        if not np.isfinite(err) or err > tol * max(1.0, maxphi):
            ok = False
            break
    if ok:
        e0, singles, pairs = split
        tables = []
        first_single = True
        for a in range(4):
            ph = singles[a] + (e0 if first_single else 0.0)
            t = np.exp(-1j * ph)
            if mags[a] is not None:
                t = t * np.asarray(mags[a], np.float64)
            if np.max(np.abs(t - 1.0)) > 1e-14 or (first_single and e0 != 0.0):
                tables.append((a, -1, np.ascontiguousarray(t, np.complex128)))
                first_single = False
        if first_single and e0 != 0.0:
            tables.append((0, -1, np.full(n[0], np.exp(-1j * e0), np.complex128)))
        for a, b in PAIRS:
            t = np.exp(-1j * pairs[(a, b)])
            # a pair that differs from 1 only by rounding of the split (a few
            # ulps) is no interaction; keeping it would cost a per-point lookup
            if np.max(np.abs(t - 1.0)) > 1e-14:
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
