"""Workloads of the parity tests and the bench: the W4D configurations.

``config1`` is the 32^4 complex128 case (V = 0.5(x^2+y^2) + 0.1(x^4+y^4)
+ 0.05 x y, seeded Gaussian Wigner state, D = 0.01, dt = 0.01); ``config2``
the 64^4 case with seeded quartic / coupling coefficients and a two-Gaussian
cat state.  Ambiguity windows are chosen so that delta = 1/N on every axis
(lambda_amp = pi/dx, theta_amp = pi/dp).
"""
import math

import numpy as np


def w4d_params(n, amp=8.0, q=0.1, kappa=0.05, D=0.01, dt=0.01, n_p=None):
    """delta = 1/N on every axis.  The reference steps theta with the x grid
    size and lambda with the p grid size (dtheta = 2 theta_amp / N_x,
    dlambda = 2 lambda_amp / N_p, GPU_Wigner4D.py:95-98), so on an N_x x N_p
    grid delta_p = dp dtheta / 2 pi = 1/N_p needs theta_amp = pi N_x / (N_p dp)
    and delta_x = 1/N_x needs lambda_amp = pi N_p / (N_x dx)."""
    n_p = n if n_p is None else n_p
    dx = 2 * amp / n
    dp = 2 * amp / n_p
    return dict(
        gridDIM_p_y=n_p, gridDIM_y=n, gridDIM_p_x=n_p, gridDIM_x=n,
        p_y_amplitude=amp, y_amplitude=amp, p_x_amplitude=amp, x_amplitude=amp,
        theta_y_amplitude=math.pi * n / (n_p * dp), theta_x_amplitude=math.pi * n / (n_p * dp),
        lambda_y_amplitude=math.pi * n_p / (n * dx), lambda_x_amplitude=math.pi * n_p / (n * dx),
        dt=dt, mass=1.0, timeSteps=0,
        kineticString="0.5*(p_x*p_x + p_y*p_y)",
        potentialString="0.5*(x*x + y*y) + %r*(pow(x,4) + pow(y,4)) + %r*x*y" % (q, kappa),
        D_theta_x=D, D_theta_y=D, D_lambda_x=D, D_lambda_y=D)


def centres(seed):
    rng = np.random.default_rng(seed)
    x0, y0 = rng.uniform(-2, 2, size=2)
    px0, py0 = rng.uniform(-1, 1, size=2)
    return float(x0), float(y0), float(px0), float(py0)


def config1(seed=0, n=32):
    return w4d_params(n, q=0.1, kappa=0.05, D=0.01, dt=0.01), centres(seed)


def config2(seed=0, n=64):
    rng = np.random.default_rng(seed + 1000)
    q = float(rng.uniform(0.05, 0.2))
    kappa = float(rng.uniform(0.0, 0.1))
    return w4d_params(n, q=q, kappa=kappa, D=0.005, dt=0.005), centres(seed)


def gaussian_xp(coords, c):
    """(1/pi^2) exp(-sum (q - q0)^2) on the (x, p) grid; coords = (p_y, y, p_x, x)."""
    x0, y0, px0, py0 = c
    py, y, px, x = [np.asarray(v).reshape(s) for v, s in zip(
        coords, [(-1, 1, 1, 1), (1, -1, 1, 1), (1, 1, -1, 1), (1, 1, 1, -1)])]
    return (np.exp(-(x - x0) ** 2 - (px - px0) ** 2 - (y - y0) ** 2 - (py - py0) ** 2)
            / np.pi ** 2).astype(np.complex128)


def cat_xp(coords, c, sep=1.5):
    """Two displaced Gaussians in superposition, as a Wigner function in (x, p):
    W = G(q - a) + G(q + a) + 2 G(q) cos(2 (p . a_x - x . a_p)) (interference),
    normalisation irrelevant (Run() renormalises)."""
    x0, y0, px0, py0 = c
    py, y, px, x = [np.asarray(v).reshape(s) for v, s in zip(
        coords, [(-1, 1, 1, 1), (1, -1, 1, 1), (1, 1, -1, 1), (1, 1, 1, -1)])]
    g = lambda dx, dy: np.exp(-(x - x0 - dx) ** 2 - (px - px0) ** 2 - (y - y0 - dy) ** 2 - (py - py0) ** 2)
    w = g(sep, 0.0) + g(-sep, 0.0) + 2 * g(0.0, 0.0) * np.cos(2 * sep * (px - px0))
    return (w / np.pi ** 2).astype(np.complex128)


def config4(seed=0, sizes=(32,) * 16 + (48,) * 16 + (64,) * 16):
    """The batched workload: one instance per entry of ``sizes``, each with its
    own quartic / coupling coefficients, Gaussian centre, D ~ U[0.001, 0.02]
    and dt in {0.005, 0.01}.  Returns [(params, centre), ...]."""
    rng = np.random.default_rng(seed + 4000)
    out = []
    for i, n in enumerate(sizes):
        q = float(rng.uniform(0.05, 0.2))
        kappa = float(rng.uniform(0.0, 0.1))
        D = float(rng.uniform(0.001, 0.02))
        dt = float(rng.choice([0.005, 0.01]))
        out.append((w4d_params(n, q=q, kappa=kappa, D=D, dt=dt), centres(seed * 1000 + i)))
    return out
