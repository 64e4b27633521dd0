"""NumPy restatement of ``GPU_WignerDirac4D`` / ``GPU_WignerDiracKvN4D`` (test infrastructure only).

Cites GPU_WignerDirac4D.py as WD4D and GPU_WignerDiracKvN4D.py as KvN:

* grids, deltas, '%f' device constants ......... WD4D:91-155
* Real_GPU ....................................... WD4D:240-244
* boundary_p_GPU / boundary_xp_GPU .............. WD4D:292-366 (KvN:327-366: constants 7, 0.005)
* kinetic sandwich exp_p_lambda_GPU ............. WD4D:377-481 (KvN:388-476: p+- = +-lambda/2)
* Potential_Propagator_Kernel ................... WD4D:492-708 (KvN:~486-690)
* WignerDiracGaussian_ParticleUp_GPU ............ WD4D:908-968
* WignerLandaoGround_GPU ........................ WD4D:975-999 (KvN:776-795)
* WignerDiracGaussian_Majorana_GPU .............. WD4D:1003-1032
* ParticleProjector_GPU ......................... WD4D:1040-1148 (KvN:853-945: p+- = p)
* reductions ..................................... WD4D:1156-1342 (KvN:955-1140)
* Norm_4x4_GPU / Normalize_4x4_GPU .............. WD4D:1359-1388
* Fourier_*_64_64_GPU wrappers .................. WD4D:1428-1458
* Run() ........................................... WD4D:1678-1899 (KvN:1475-1669)

The sixteen components are sixteen separate complex128 arrays of shape
(N_py, N_y, N_px, N_x), exactly as in the reference, and every kernel writes
them in place in the reference's statement order.  That makes the
reference's pointer aliasing (``W21 = self.W22`` in Run(), WD4D:1716,
KvN:1513) reproduce itself when ``alias_w21`` is set: the 16-way wrappers then
transform W22 twice, Normalize divides it twice, boundary_xp multiplies it by
the mask twice, and the sandwich kernels read W22 in place of W21.
"""
import numpy as np

from . import cexpr
from .faft import faft
from .wigner4d import dev

COMP = [(a, b) for a in range(4) for b in range(4)]
NAMES = ["W%d%d" % (a + 1, b + 1) for a, b in COMP]


class DiracOracle:
    """Holds the attributes of a ``GPU_WignerDirac4D`` frame (WD4D:71-155).

    ``kvn=True`` selects the GPU_WignerDiracKvN4D variant.
    """

    def __init__(self, params, kvn=False, round_constants=True, a3_mode="sin_a3"):
        for k, v in params.items():
            setattr(self, k, v)
        self.kvn = kvn
        self.rc = round_constants
        # "sin_a3": U13 = i sin(A3 c dt) as committed (GPU_WignerDirac4D.py:601-604);
        # "sinF": the commented-out form i A3 sin(c dt F / hbar) / F (WD4D:596-599)
        self.a3_mode = a3_mode
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
        for name in ("potential_0_String", "potential_1_String", "potential_2_String",
                     "potential_3_String", "D_1_potential_0_String",
                     "D_1_potential_1_String", "D_1_potential_2_String"):
            if not hasattr(self, name):
                setattr(self, name, "0.")
        self.W = [np.zeros(self.shape, np.complex128) for _ in range(16)]

    def dc(self, name):
        return dev(getattr(self, name), self.rc)

    def _axis(self, ax, step):
        n = self.shape[ax]
        v = dev(step, self.rc) * (np.arange(n) - 0.5 * n)
        sh = [1, 1, 1, 1]
        sh[ax] = n
        return v.reshape(sh)

    # --- coordinate sets ---------------------------------------------------
    def xp(self):
        return (self._axis(3, self.dx), self._axis(2, self.dp_x),
                self._axis(1, self.dy), self._axis(0, self.dp_y))

    def lambda_p(self):
        return (self._axis(3, self.dlambda_x), self._axis(2, self.dp_x),
                self._axis(1, self.dlambda_y), self._axis(0, self.dp_y))

    def x_theta(self):
        return (self._axis(3, self.dx), self._axis(2, self.dtheta_x),
                self._axis(1, self.dy), self._axis(0, self.dtheta_y))

    # --- elementwise kernels ------------------------------------------------
    @staticmethod
    def real(W):
        """Real_GPU, WD4D:240-244 (in place)."""
        W.imag[...] = 0.0

    def _mask(self, bound_p, bound_x):
        x, px, y, py = self.xp()
        dpx, dpy, dx, dy = self.dc("dp_x"), self.dc("dp_y"), self.dc("dx"), self.dc("dy")
        npx, npy, nx, ny = self.shape[2], self.shape[0], self.shape[3], self.shape[1]
        r = 1.0 - np.exp(-bound_p * (px - 0.5 * dpx * npx) ** 4)
        r = r * (1.0 - np.exp(-bound_p * (px + 0.5 * dpx * (npx - 1)) ** 4))
        r = r * (1.0 - np.exp(-bound_p * (py - 0.5 * dpy * npy) ** 4))
        r = r * (1.0 - np.exp(-bound_p * (py + 0.5 * dpy * (npy - 1)) ** 4))
        if bound_x is not None:
            r = r * (1.0 - np.exp(-bound_x * (x - 0.5 * dx * nx) ** 4))
            r = r * (1.0 - np.exp(-bound_x * (x + 0.5 * dx * (nx - 1)) ** 4))
            r = r * (1.0 - np.exp(-bound_x * (y - 0.5 * dy * ny) ** 4))
            r = r * (1.0 - np.exp(-bound_x * (y + 0.5 * dy * (ny - 1)) ** 4))
        return r

    def boundary_p(self, Ws):
        """boundary_p_GPU, WD4D:292-325 (mask constant 7, p only)."""
        r = self._mask(7.0, None)
        for W in Ws:
            W *= r

    def boundary_xp(self, Ws, bound_x=0.005, bound_p=15.0):
        """boundary_xp_GPU, WD4D:327-366; KvN:327-366 hard-codes 7 and 0.005."""
        if self.kvn:
            bound_x, bound_p = 0.005, 7.0
        r = self._mask(bound_p, bound_x)
        for W in Ws:
            W *= r

    def _kin_mats(self, px, py, dt):
        """K11, K14 of WD4D:377-388 -> the left/right 4x4 factors' entries."""
        c, hb = self.dc("c"), self.dc("HBar")
        m = self.dc("mass")
        om = c / hb * np.sqrt((m * c) ** 2 + px ** 2 + py ** 2)
        s = np.sin(dt * om)
        k11 = np.cos(dt * om) - 1j * (c ** 2 * m * s) / (om * hb)
        k14 = -(c * py * s) / (om * hb) - 1j * (c * px * s) / (om * hb)
        return k11, k14

    @staticmethod
    def _spin_matrix(a, b, conj_offdiag=-1.0):
        """[[a,0,0,b],[0,a,s*conj(b),0],[0,b,conj(a),0],[s*conj(b),0,0,conj(a)]] with s=conj_offdiag."""
        cb = conj_offdiag * np.conj(b)
        return [[a, None, None, b], [None, a, cb, None], [None, b, np.conj(a), None],
                [cb, None, None, np.conj(a)]]

    @staticmethod
    def _sandwich(L, Win, R, scale=1.0):
        # structural zeros of the 4x4 factors are None and skipped
        out = []
        for a, b in COMP:
            acc = 0.0
            for k in range(4):
                if L[a][k] is None:
                    continue
                for l in range(4):
                    if R[l][b] is None or not Win[4 * k + l].any():
                        continue
                    acc = acc + L[a][k] * Win[4 * k + l] * R[l][b]
            out.append(scale * acc)
        return out

    def kinetic(self, Ws):
        """exp_p_lambda_GPU, WD4D:392-481: W <- r * KL W KR on the (lambda, p) grid."""
        lx, px, ly, py = self.lambda_p()
        hb, dt = self.dc("HBar"), self.dc("dt")
        if self.kvn:   # KvN:396-399
            pxp, pyp, pxm, pym = 0.5 * lx, 0.5 * ly, -0.5 * lx, -0.5 * ly
        else:
            pxp, pyp = px + 0.5 * hb * lx, py + 0.5 * hb * ly
            pxm, pym = px - 0.5 * hb * lx, py - 0.5 * hb * ly
        r = np.exp(-dt * self.dc("D_lambda_x") * lx ** 2 - dt * self.dc("D_lambda_y") * ly ** 2)
        a, b = self._kin_mats(pxp, pyp, dt)
        cc, d = self._kin_mats(pxm, pym, -dt)
        L = self._spin_matrix(a, b)
        R = self._spin_matrix(cc, d)
        Win = [W.copy() for W in Ws]
        out = self._sandwich(L, Win, R)
        for W, o in zip(Ws, out):
            W[...] = r * o

    def _U(self, x, y, dt, m, right):
        """The 4x4 U of Potential_Propagator_Kernel (WD4D:580-604, KvN:584-597)."""
        c, hb = self.dc("c"), self.dc("HBar")
        A1 = cexpr.evaluate(self.potential_1_String, t=0.0, x=x, y=y)
        A2 = cexpr.evaluate(self.potential_2_String, t=0.0, x=x, y=y)
        z = np.zeros(np.broadcast(x, y).shape, np.complex128)
        if self.kvn:
            F = np.sqrt((m * c) ** 2 + A1 ** 2 + A2 ** 2)
            s = np.sin(c * dt * F / hb)
            co = np.cos(c * dt * F / hb)
            if not right:
                u11 = co + 1j * (-m * c * np.sin(-c * dt * F / hb) / F)
                u33 = co + 1j * (m * c * np.sin(-c * dt * F / hb) / F)
                sm = np.sin(-c * dt * F / hb) / F
                u14 = (-A2 - 1j * A1) * sm
                u41 = (A2 - 1j * A1) * sm
                u23 = (A2 - 1j * A1) * sm
                u32 = (-A2 - 1j * A1) * sm
            else:
                u11 = co + 1j * (m * c * np.sin(-c * dt * F / hb) / F)
                u33 = co + 1j * (-m * c * np.sin(-c * dt * F / hb) / F)
                sp = s / F
                u14 = (-A2 - 1j * A1) * sp
                u41 = (A2 - 1j * A1) * sp
                u23 = (A2 - 1j * A1) * sp
                u32 = (-A2 - 1j * A1) * sp
            return [[u11, None, None, u14], [None, u11, u23, None], [None, u32, u33, None],
                    [u41, None, None, u33]]
        A3 = cexpr.evaluate(self.potential_3_String, t=0.0, x=x, y=y)
        F = np.sqrt((m * c) ** 2 + A1 ** 2 + A2 ** 2 + A3 ** 2)
        s = np.sin(c * dt * F / hb)
        u11 = np.cos(c * dt * F / hb) + 1j * (m * c * s / F)
        u33 = np.cos(c * dt * F / hb) - 1j * (m * c * s / F)
        u14 = (A2 + 1j * A1) * s / F
        u23 = -(-A2 + 1j * A1) * s / F
        u32 = -(A2 + 1j * A1) * s / F
        u41 = (-A2 + 1j * A1) * s / F
        s3 = np.sin(A3 * c * dt) if self.a3_mode == "sin_a3" else A3 * s / F
        u13 = 1j * s3 + z
        u24 = -1j * s3 + z
        return [[u11, None, u13, u14], [None, u11, u23, u24], [u13, u32, u33, None],
                [u41, u24, None, u33]]

    def potential(self, Ws):
        """Potential_Propagator_Kernel on the (x, theta) grid: W <- e^{-i dt dA0/hbar} U- W U+."""
        x, tx, y, ty = self.x_theta()
        hb, dt = self.dc("HBar"), self.dc("dt")
        if self.kvn:     # KvN:527-531
            xm, xp_, ym, yp = -0.5 * tx, 0.5 * tx, -0.5 * ty, 0.5 * ty
            m = 1e-6     # KvN:536
        else:            # WD4D:531-535 (no hbar in the shift)
            xm, xp_, ym, yp = x - 0.5 * tx, x + 0.5 * tx, y - 0.5 * ty, y + 0.5 * ty
            m = 1e-12    # WD4D:542
        UL = self._U(xm, ym, dt, m, right=False)
        UR = self._U(xp_, yp, -dt if not self.kvn else dt, m, right=True)
        Win = [W.copy() for W in Ws]
        out = self._sandwich(UL, Win, UR)
        ph = (cexpr.evaluate(self.potential_0_String, t=0.0, x=xm, y=ym)
              - cexpr.evaluate(self.potential_0_String, t=0.0, x=xp_, y=yp))
        ev = np.cos(dt * ph / hb) - 1j * np.sin(dt * ph / hb)
        for W, o in zip(Ws, out):
            W[...] = ev * o

    def projector(self, Ws, sign):
        """ParticleProjector_GPU, WD4D:1040-1148 (KvN:853-945 uses p+- = p)."""
        lx, px, ly, py = self.lambda_p()
        hb, c, m = self.dc("HBar"), self.dc("c"), self.dc("mass")
        if self.kvn:
            pxm, pym, pxp, pyp = px, py, px, py
        else:
            pxm, pym = px - 0.5 * hb * lx, py - 0.5 * hb * ly
            pxp, pyp = px + 0.5 * hb * lx, py + 0.5 * hb * ly

        def P(qx, qy):
            K = c * np.sqrt((m * c) ** 2 + qx ** 2 + qy ** 2)
            p11 = 1.0 + (c ** 2 * m * sign) / K + 0j
            p33 = 1.0 - (c ** 2 * m * sign) / K + 0j
            p14 = (sign * (c * qx) - 1j * sign * (c * qy)) / K
            return [[p11, None, None, p14], [None, p11, np.conj(p14), None],
                    [None, p14, p33, None], [np.conj(p14), None, None, p33]]

        Win = [W / 4.0 for W in Ws]
        out = self._sandwich(P(pxp, pyp), Win, P(pxm, pym))
        for W, o in zip(Ws, out):
            W[...] = o

    # --- initial states -----------------------------------------------------
    def _shifted(self, x_mu, y_mu):
        x, tx, y, ty = self.x_theta()
        hb = self.dc("HBar")
        return (x - 0.5 * hb * tx - x_mu, y - 0.5 * hb * ty - y_mu,
                x + 0.5 * hb * tx - x_mu, y + 0.5 * hb * ty - y_mu)

    def _psi(self, x, y, ux, uy, sx, sy):
        c, m = self.dc("c"), self.dc("mass")
        u0 = np.sqrt(ux ** 2 + uy ** 2 + c * c)
        ph = m * (x * ux + y * uy)
        g = np.exp(-0.5 * (x / sx) ** 2 - 0.5 * (y / sy) ** 2)
        psi1 = g * (c + u0) * (np.cos(ph) + 1j * np.sin(ph))
        psi4 = g * ((np.cos(ph) * ux - np.sin(ph) * uy) + 1j * (np.sin(ph) * ux + np.cos(ph) * uy))
        return psi1, psi4

    def particle_up(self, ux, uy, x_mu, y_mu, sx, sy):
        """WignerDiracGaussian_ParticleUp_GPU, WD4D:940-968: writes W11, W14, W41, W44."""
        xm, ym, xp_, yp = self._shifted(x_mu, y_mu)
        p1m, p4m = self._psi(xm, ym, ux, uy, sx, sy)
        p1p, p4p = self._psi(xp_, yp, ux, uy, sx, sy)
        self.W[0][...] = p1m * np.conj(p1p)
        self.W[3][...] = p1m * np.conj(p4p)
        self.W[12][...] = p4m * np.conj(p1p)
        self.W[15][...] = p4m * np.conj(p4p)

    def majorana(self, ux, uy, x_mu, y_mu, sx, sy):
        """WignerDiracGaussian_Majorana_GPU, WD4D:1003-1032."""
        xm, ym, xp_, yp = self._shifted(x_mu, y_mu)
        p1m, p4m = self._psi(xm, ym, ux, uy, sx, sy)
        p1p, p4p = self._psi(xp_, yp, ux, uy, sx, sy)
        a_m, b_m = p1m - np.conj(p4m), p4m - np.conj(p1m)
        a_p, b_p = p1p - np.conj(p4p), p4p - np.conj(p1p)
        self.W[0][...] = a_m * np.conj(a_p)
        self.W[3][...] = a_m * np.conj(b_p)
        self.W[12][...] = b_m * np.conj(a_p)
        self.W[15][...] = b_m * np.conj(b_p)

    def landau_ground(self, B, x_off=0.0, y_off=0.0):
        """WignerLandaoGround_GPU, WD4D:975-999 (KvN has no offsets)."""
        xm, ym, xp_, yp = self._shifted(x_off, y_off)
        f = lambda x, y: np.exp(-B * 0.25 * x ** 2 - B * 0.25 * y ** 2)
        self.W[0][...] = f(xm, ym) * f(xp_, yp)

    # --- transforms (WD4D:1428-1458) ----------------------------------------
    def _pair(self, W, a0, d0, dl0, a1, d1, dl1, div):
        if W.any():
            t = faft(W, a0, d0, dl0)
            t = faft(t, a1, d1, dl1)
            W[...] = t
        W /= div

    def x_to_lambda(self, W):
        self._pair(W, 3, self.dx, self.delta_x, 1, self.dy, self.delta_y, self.size)

    def lambda_to_x(self, W):
        self._pair(W, 3, self.dx, -self.delta_x, 1, self.dy, -self.delta_y, np.sqrt(self.size) / 100.0)

    def p_to_theta(self, W, div=None):
        self._pair(W, 2, self.dp_x, self.delta_p_x, 0, self.dp_y, self.delta_p_y,
                   self.size if div is None else div)

    def theta_to_p(self, W, div=None):
        self._pair(W, 2, self.dp_x, -self.delta_p_x, 0, self.dp_y, -self.delta_p_y,
                   np.sqrt(self.size) / 100.0 if div is None else div)

    # --- reductions -----------------------------------------------------------
    def norm4(self, Ws):
        """Norm_4x4_GPU, WD4D:1359-1364 (host dV)."""
        n = Ws[0].sum() + Ws[5].sum() + Ws[10].sum() + Ws[15].sum()
        return n * self.dx * self.dp_x * self.dy * self.dp_y

    def normalize(self, Ws):
        """Normalize_4x4_GPU, WD4D:1366-1388; returns the printed norm."""
        n = self.norm4(Ws)
        for W in Ws:
            W /= n
        return n

    def observables(self, Ws):
        """The Run() reductions (WD4D:1174-1342, KvN:973-1140) at their (x, p) coordinates."""
        x, px, y, py = self.xp()
        dV = self.dc("dx") * self.dc("dy") * self.dc("dp_x") * self.dc("dp_y")
        c, m = self.dc("c"), self.dc("mass")
        W11, W14, W41, W44 = Ws[0], Ws[3], Ws[12], Ws[15]
        W22, W23, W32, W33 = Ws[5], Ws[6], Ws[9], Ws[10]
        W13, W24, W31, W42 = Ws[2], Ws[7], Ws[8], Ws[13]
        tr = (W11 + W22 + W33 + W44).real
        a1 = (W14 + W41 + W23 + W32).real
        a2 = -(W14 - W41 + W32 - W23).imag
        ev = lambda s: cexpr.evaluate(s, t=0.0, x=x, y=y)
        A0, A1, A2 = ev(self.potential_0_String), ev(self.potential_1_String), ev(self.potential_2_String)
        o = {
            "average_x": (dV * x * tr).sum(), "average_p_x": (dV * px * tr).sum(),
            "average_x_square": (dV * x ** 2 * tr).sum(),
            "average_p_x_square": (dV * px * px * tr).sum(),
            "average_y": (dV * y * tr).sum(), "average_p_y": (dV * py * tr).sum(),
            "average_y_square": (dV * y * y * tr).sum(),
            "average_p_y_square": (dV * py * py * tr).sum(),
            "average_Alpha_1": (dV * a1).sum(), "average_Alpha_2": (dV * a2).sum(),
            "average_Alpha_1_x": (dV * x * a1).sum(), "average_Alpha_2_y": (dV * y * a2).sum(),
        }
        o["energyKinetic"] = ((c * dV * px * (W14 + W41 + W32 + W23).real)
                              - c * dV * py * (W14 - W41 + W32 - W23).imag
                              + dV * m * c * c * (W11 + W22 - W33 - W44).real).sum()
        D10 = ev(self.D_1_potential_0_String)
        D11 = ev(self.D_1_potential_1_String)
        D12 = ev(self.D_1_potential_2_String)
        if self.kvn:   # KvN:1107-1109, 1137
            o["energyPotential"] = (dV * A1 * c * (W14 + W41 + W23 + W32).real
                                    - dV * A2 * c * (W14 - W41 - W23 + W32).imag
                                    + c * A0 * dV * tr).sum()
            o["average_D_1_A_2"] = (c * D12 * dV * (W14 - W41 - W23 + W32).real).sum()
        else:          # WD4D:1309-1312, 1340
            A3 = ev(self.potential_3_String)
            o["energyPotential"] = (dV * A1 * c * (-W14 - W23 - W32 - W41).real
                                    - dV * A2 * c * (-W14 + W23 - W32 + W41).imag
                                    + dV * A3 * c * (-W13 + W24 - W31 + W42).real
                                    + c * A0 * dV * tr).sum()
            o["average_D_1_A_2"] = (-dV * D12 * c * (-W14 + W23 - W32 + W41).imag).sum()
        o["average_D_1_A_0"] = (c * D10 * dV * tr).sum()
        o["average_D_1_A_1"] = (c * D11 * dV * a1).sum()
        return o

    # --- Run() ------------------------------------------------------------------
    def pointers(self, alias_w21):
        Ws = list(self.W)
        if alias_w21:
            Ws[4] = self.W[5]          # W21 = self.W22, WD4D:1716 / KvN:1513
        return Ws

    def run_iteration(self, Ws, filter_particle=False, bound_x=0.005, bound_p=15.0,
                      observe=True):
        """One iteration of Run() (WD4D:1767-1851).  Returns (printed norm, observables)."""
        self.boundary_xp(Ws, bound_x, bound_p)
        for k in (0, 5, 10, 15):
            self.real(Ws[k])
        n = self.normalize(Ws)
        obs = self.observables(Ws) if observe else None
        for W in Ws:
            self.x_to_lambda(W)
        if filter_particle:
            self.projector(Ws, 1)
        self.kinetic(Ws)
        for W in Ws:
            self.lambda_to_x(W)
        for W in Ws:
            self.p_to_theta(W)
        self.potential(Ws)
        for W in Ws:
            self.theta_to_p(W)
        return n, obs
