"""NumPy restatement of ``GPU_Wigner4D`` (test infrastructure only).

Follows GPU_Wigner4D.py (cited as W4D) of cabrer7/PyWignerCUDA2:

* grid / ambiguity steps and deltas ................ W4D:91-124
* device constants printed with '%f' ............... W4D:126-152
* HOscillatorGound_GPU / Gaussian_GPU .............. W4D:216-245
* exp_p_lambda_GPU (kinetic phase, lambda damping) . W4D:249-262
* exp_x_theta_GPU (Bopp potential phase) ........... W4D:266-281
* observables (ReductionKernel map_expr) ........... W4D:285-358
* Norm_GPU .......................................... W4D:367-369
* Fourier_*_64_64_GPU wrappers ..................... W4D:409-427
* Run() loop ........................................ W4D:431-541

State layout is the reference's: a complex128 array of shape
(N_py, N_y, N_px, N_x), x fastest.  Axis i of the array is FAFT axis i.
"""
import numpy as np

from . import cexpr
from .faft import faft


def dev(v, rounding=True):
    """A host float as the reference's CUDA preamble sees it ('%f', W4D:128-150)."""
    return float("%f" % v) if rounding else float(v)


class Wigner4DOracle:
    """Holds the same attributes as a ``GPU_Wigner4D`` frame (W4D:71-124).

    ``params`` keys: gridDIM_{p_y,y,p_x,x}, {p_y,y,p_x,x}_amplitude,
    {theta,lambda}_{x,y}_amplitude, dt, mass, kineticString, potentialString,
    D_{theta,lambda}_{x,y}.
    """

    def __init__(self, params, round_constants=True):
        for k, v in params.items():
            setattr(self, k, v)
        self.rc = round_constants
        # W4D:91-106
        self.dp_y = 2 * self.p_y_amplitude / float(self.gridDIM_p_y)
        self.dy = 2 * self.y_amplitude / float(self.gridDIM_y)
        self.dp_x = 2 * self.p_x_amplitude / float(self.gridDIM_p_x)
        self.dx = 2 * self.x_amplitude / float(self.gridDIM_x)
        self.dtheta_y = 2 * self.theta_y_amplitude / float(self.gridDIM_y)
        self.dlambda_y = 2 * self.lambda_y_amplitude / float(self.gridDIM_p_y)
        self.dtheta_x = 2 * self.theta_x_amplitude / float(self.gridDIM_x)
        self.dlambda_x = 2 * self.lambda_x_amplitude / float(self.gridDIM_p_x)
        self.delta_p_y = self.dp_y * self.dtheta_y / (2 * np.pi)
        self.delta_y = self.dy * self.dlambda_y / (2 * np.pi)
        self.delta_p_x = self.dp_x * self.dtheta_x / (2 * np.pi)
        self.delta_x = self.dx * self.dlambda_x / (2 * np.pi)
        self.shape = (self.gridDIM_p_y, self.gridDIM_y, self.gridDIM_p_x, self.gridDIM_x)
        self.size = int(np.prod(self.shape))
        for name in ("D_theta_x", "D_theta_y", "D_lambda_x", "D_lambda_y"):
            if not hasattr(self, name):
                setattr(self, name, 0.0)

    # ---- device-side coordinates (W4D:167-212: q = d_q * (i_q - N/2)) ----
    def _axis(self, ax, step):
        n = self.shape[ax]
        v = dev(step, self.rc) * (np.arange(n) - n // 2)
        sh = [1, 1, 1, 1]
        sh[ax] = n
        return v.reshape(sh)

    def dc(self, name):
        return dev(getattr(self, name), self.rc)

    # ---- initial states -------------------------------------------------
    def ho_ground(self, x_mu, y_mu, p_x_mu, p_y_mu, omega_x, omega_y, mass):
        """HOscillatorGound_GPU, W4D:233-245."""
        x, px = self._axis(3, self.dx), self._axis(2, self.dp_x)
        y, py = self._axis(1, self.dy), self._axis(0, self.dp_y)
        t = (mass * (omega_x * (x - x_mu)) ** 2 + (px - p_x_mu) ** 2 / mass) / omega_x
        t = t + (mass * (omega_y * (y - y_mu)) ** 2 + (py - p_y_mu) ** 2 / mass) / omega_y
        return np.exp(-t).astype(np.complex128)

    def gaussian(self, mu_p_y, mu_y, mu_p_x, mu_x, s_p_y, s_y, s_p_x, s_x):
        """Gaussian_GPU, W4D:216-230."""
        x, px = self._axis(3, self.dx), self._axis(2, self.dp_x)
        y, py = self._axis(1, self.dy), self._axis(0, self.dp_y)
        t = np.exp(-0.5 * (x - mu_x) ** 2 / s_x ** 2)
        t = t * np.exp(-0.5 * (y - mu_y) ** 2 / s_y ** 2)
        t = t * np.exp(-0.5 * (px - mu_p_x) ** 2 / s_p_x ** 2)
        t = t * np.exp(-0.5 * (py - mu_p_y) ** 2 / s_p_y ** 2)
        return t.astype(np.complex128)

    def cat_xtheta(self, x_mu, y_mu, p_x_mu, p_y_mu, a_x, a_y):
        """Two displaced Gaussians in superposition on the (x, theta) grid,
        W = psi(x - theta/2) conj(psi(x + theta/2)) -- the construction of
        WignerDiracGaussian_ParticleUp_GPU (WD4D:939-968) applied to
        psi = [g(q - q_mu - a) + g(q - q_mu + a)] exp(i p_mu . q),
        g = exp(-|q|^2 / 2).  p_to_theta(W, -1) then gives (x, p)."""
        x, tx = self._axis(3, self.dx), self._axis(2, self.dtheta_x)
        y, ty = self._axis(1, self.dy), self._axis(0, self.dtheta_y)

        def psi(u, v):
            g = (np.exp(-0.5 * ((u - x_mu - a_x) ** 2 + (v - y_mu - a_y) ** 2))
                 + np.exp(-0.5 * ((u - x_mu + a_x) ** 2 + (v - y_mu + a_y) ** 2)))
            return g * np.exp(1j * (p_x_mu * u + p_y_mu * v))

        return (psi(x - 0.5 * tx, y - 0.5 * ty) * np.conj(psi(x + 0.5 * tx, y + 0.5 * ty))).astype(np.complex128)

    # ---- reductions -----------------------------------------------------
    def norm(self, W):
        """Norm_GPU, W4D:367-369 (host-precision dV, complex)."""
        return W.sum() * self.dx * self.dp_x * self.dy * self.dp_y

    def observables(self, W):
        """The nine ReductionKernels of W4D:294-358, in Run()'s order (W4D:486-498).

        Returns a dict: average_x, average_p_x, average_x_square,
        average_p_x_square, average_y, average_p_y, average_y_square,
        average_p_y_square, energy.
        """
        dV = self.dc("dx") * self.dc("dy") * self.dc("dp_x") * self.dc("dp_y")
        x, px = self._axis(3, self.dx), self._axis(2, self.dp_x)
        y, py = self._axis(1, self.dy), self._axis(0, self.dp_y)
        wr = W.real
        out = {
            "average_x": (x * dV * wr).sum(),
            "average_p_x": (px * dV * wr).sum(),
            "average_x_square": (x * x * dV * wr).sum(),
            "average_p_x_square": (px * px * dV * wr).sum(),
            "average_y": (y * dV * wr).sum(),
            "average_p_y": (py * dV * wr).sum(),
            "average_y_square": (y * y * dV * wr).sum(),
            "average_p_y_square": (py * py * dV * wr).sum(),
        }
        e = (cexpr.evaluate(self.kineticString, p_x=px, p_y=py)
             + cexpr.evaluate(self.potentialString, x=x, y=y))
        out["energy"] = (e * dV * wr).sum()
        return out

    # ---- transforms (W4D:409-427) ---------------------------------------
    def x_to_lambda(self, W, sign=+1):
        W = faft(W, 1, self.dx, sign * self.delta_x)
        W = faft(W, 3, self.dy, sign * self.delta_y)
        return W / self.size

    def p_to_theta(self, W, sign=+1):
        W = faft(W, 0, self.dp_x, sign * self.delta_p_x)
        W = faft(W, 2, self.dp_y, sign * self.delta_p_y)
        return W / self.size

    # ---- phase kernels --------------------------------------------------
    def kinetic_factor(self):
        """exp_p_lambda_GPU multiplier on the (lambda, p) grid, W4D:251-262."""
        dt = self.dc("dt")
        Dly = self.dc("D_lambda_y")
        lx, px = self._axis(3, self.dlambda_x), self._axis(2, self.dp_x)
        ly, py = self._axis(1, self.dlambda_y), self._axis(0, self.dp_y)
        r = np.exp(-dt * Dly * lx * lx) * np.exp(-dt * Dly * ly * ly)
        ph = (dt * cexpr.evaluate(self.kineticString, p_x=px + 0.5 * lx, p_y=py + 0.5 * ly)
              - dt * cexpr.evaluate(self.kineticString, p_x=px - 0.5 * lx, p_y=py - 0.5 * ly))
        return r * np.cos(ph) - 1j * r * np.sin(ph)

    def potential_factor(self):
        """exp_x_theta_GPU multiplier on the (x, theta) grid, W4D:269-281."""
        dt = self.dc("dt")
        Dty = self.dc("D_theta_y")
        x, tx = self._axis(3, self.dx), self._axis(2, self.dtheta_x)
        y, ty = self._axis(1, self.dy), self._axis(0, self.dtheta_y)
        ph = (dt * cexpr.evaluate(self.potentialString, x=x - 0.5 * tx, y=y - 0.5 * ty)
              - dt * cexpr.evaluate(self.potentialString, x=x + 0.5 * tx, y=y + 0.5 * ty))
        r = np.exp(-dt * Dty * tx * tx - dt * Dty * ty * ty)
        return r * np.cos(ph) - 1j * r * np.sin(ph)

    # ---- one Run() iteration (W4D:479-513) -------------------------------
    def step(self, W, kin=None, pot=None, record=None):
        """Renormalise, record observables, then K and V half-steps.

        Returns the new W.  ``record`` (a list) receives
        ``(norm, observables)`` for this iteration.
        """
        kin = self.kinetic_factor() if kin is None else kin
        pot = self.potential_factor() if pot is None else pot
        n = self.norm(W)
        W = W / n
        if record is not None:
            record.append((n, self.observables(W)))
        W = self.x_to_lambda(W, +1)
        W = W * kin
        W = self.x_to_lambda(W, -1)
        W = self.p_to_theta(W, +1)
        W = W * pot
        W = self.p_to_theta(W, -1)
        return W

    def run(self, W, time_steps):
        """Run(), W4D:431-541: ``time_steps + 1`` iterations then a final renormalisation."""
        kin, pot = self.kinetic_factor(), self.potential_factor()
        rec = []
        for _ in range(time_steps + 1):
            W = self.step(W, kin, pot, rec)
        W = W / self.norm(W)
        obs = {k: np.array([r[1][k] for r in rec]) for k in rec[0][1]}
        obs["norms"] = np.array([r[0] for r in rec])
        return W, obs
