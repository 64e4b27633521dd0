"""``GPU_Wigner4D``: drop-in for the reference class of the same name.

Mirrors GPU_Wigner4D.py (cabrer7/PyWignerCUDA2) -- a user subclass sets the
same attributes and calls ``GPU_Wigner4D.__init__(self)``, then an initial
condition, then ``Run()`` -- with every device operation a kernel of
libwigner_b200.so (sm_100a):

* constructor .............. GPU_Wigner4D.py:71-358 (grids, '%f' device
                             constants, state allocation, kernels -> a plan)
* Gaussian_GPU, HOscillatorGound_GPU ....... GPU_Wigner4D.py:216-245
* exp_p_lambda_GPU, exp_x_theta_GPU ........ GPU_Wigner4D.py:251-281
* Average_*_GPU, Energy_GPU, Norm_GPU ...... GPU_Wigner4D.py:294-369
* Fourier_*_64_64_GPU / _64_128_GPU ........ GPU_Wigner4D.py:372-427
* Run() .................................... GPU_Wigner4D.py:431-541

Extra attributes a frame may set (defaults reproduce the reference):

* ``complex_dtype``: ``numpy.complex128`` (the drop-in) or
  ``numpy.complex64`` (the precision form: complex64 state, phase factors
  built in float64 and rounded once, float64 reductions).
* ``tensor_cores``: True (complex64 64^4 grids, any delta) runs Run()'s
  64-point transforms as dense FAFT GEMMs on the tensor cores (fp16 hi + lo
  operands, FP32 accumulation; k_tc64) instead of the CUDA-core kernels;
  "auto" makes them a candidate of the autotuner.
* ``fp64_transforms``: True (complex64 64^4 grids, delta = 1/N) keeps the
  complex64 state in memory but runs the transforms and factors in FP64.
* ``autotune``: True times the plan's kernel choices once per (grid, dtype,
  kernel path) in the process (wig4d_autotune) and keeps the fastest; the
  choice is in ``self.autotune_choice``.  "force" times it again.
* ``round_constants``: True reproduces the reference's '%f' formatting of the
  device constants (GPU_Wigner4D.py:128-150); False uses full precision.
* ``snapshotEvery``: K > 0 makes Run() keep the normalised state every K
  iterations in ``self.snapshots`` (list of (time, array)) and write them
  beside the Ehrenfest data (``/Snapshots/W_<i>``); the observables and the
  final state are those of a Run() without snapshots.

``save_checkpoint(fname)`` / ``load_checkpoint(fname)`` store and restore the
state so that a later Run() continues the run (no counterpart in the
reference).
"""
import ctypes
import os

import numpy as np
import torch

from . import _lib, expr, tables
from .device import DeviceScalar, GPUArray, ptr_of, require_cuda, stream_ptr, wdtype_of


def dev_const(v, rounding=True):
    """A float as the reference's CUDA preamble sees it ('%f', GPU_Wigner4D.py:128-150)."""
    return float("%f" % v) if rounding else float(v)


class GPU_Wigner4D:
    """Split-operator propagation of W(x, p_x, y, p_y); see the module docstring."""

    complex_dtype = np.complex128
    round_constants = True
    tensor_cores = False
    autotune = False
    fp64_transforms = False

    def __init__(self):
        require_cuda()
        # ---- GPU_Wigner4D.py:74-124 ----
        self.FAFT_axes0, self.FAFT_axes1, self.FAFT_axes2, self.FAFT_axes3 = 0, 1, 2, 3
        self.FAFT_segment_axes0 = self.FAFT_segment_axes1 = 0
        self.FAFT_segment_axes2 = self.FAFT_segment_axes3 = 0
        self.NF = 1
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
        self.p_y_range = np.linspace(-self.p_y_amplitude, self.p_y_amplitude - self.dp_y, self.gridDIM_p_y)
        self.y_range = np.linspace(-self.y_amplitude, self.y_amplitude - self.dy, self.gridDIM_y)
        self.p_x_range = np.linspace(-self.p_x_amplitude, self.p_x_amplitude - self.dp_x, self.gridDIM_p_x)
        self.x_range = np.linspace(-self.x_amplitude, self.x_amplitude - self.dx, self.gridDIM_x)
        self.theta_y_range = np.linspace(-self.theta_y_amplitude, self.theta_y_amplitude - self.dtheta_y, self.gridDIM_y)
        self.lambda_y_range = np.linspace(-self.lambda_y_amplitude, self.lambda_y_amplitude - self.dlambda_y, self.gridDIM_p_y)
        self.theta_x_range = np.linspace(-self.theta_x_amplitude, self.theta_x_amplitude - self.dtheta_x, self.gridDIM_x)
        self.lambda_x_range = np.linspace(-self.lambda_x_amplitude, self.lambda_x_amplitude - self.dlambda_x, self.gridDIM_p_x)
        self.y = self.y_range[np.newaxis, :, np.newaxis, np.newaxis]
        self.p_y = self.p_y_range[:, np.newaxis, np.newaxis, np.newaxis]
        self.p_x = self.p_x_range[np.newaxis, np.newaxis, :, np.newaxis]
        self.x = self.x_range[np.newaxis, np.newaxis, np.newaxis, :]
        for name in ("D_theta_x", "D_theta_y", "D_lambda_x", "D_lambda_y"):
            if not hasattr(self, name):
                setattr(self, name, 0.0)
        self.shape = (self.gridDIM_p_y, self.gridDIM_y, self.gridDIM_p_x, self.gridDIM_x)
        self.W_init_gpu = GPUArray.zeros(self.shape, self.complex_dtype)
        self._plan = None
        self._build_plan()

    # ------------------------------------------------------------------------
    def _c(self, name):
        return dev_const(getattr(self, name), self.round_constants)

    def _axis_coords(self, step, n):
        """q = d_q (i - N/2) with the device-constant step (GPU_Wigner4D.py:167-212)."""
        return dev_const(step, self.round_constants) * (np.arange(n) - n // 2)

    def _build_plan(self):
        N0, N1, N2, N3 = self.shape
        dt = self._c("dt")
        K = expr.parse(self.kineticString)
        V = expr.parse(self.potentialString)
        # (lambda, p) representation: axes p_y, lambda_y, p_x, lambda_x
        kv = [self._axis_coords(self.dp_y, N0), self._axis_coords(self.dlambda_y, N1),
              self._axis_coords(self.dp_x, N2), self._axis_coords(self.dlambda_x, N3)]

        def kin_phase(py, ly, px, lx):
            return (dt * expr.evaluate(K, p_x=px + 0.5 * lx, p_y=py + 0.5 * ly)
                    - dt * expr.evaluate(K, p_x=px - 0.5 * lx, p_y=py - 0.5 * ly))

        Dly = self._c("D_lambda_y")   # used for both axes, GPU_Wigner4D.py:255-256
        kmag = [None, np.exp(-dt * Dly * kv[1] * kv[1]), None, np.exp(-dt * Dly * kv[3] * kv[3])]
        ktabs, kfull = tables.build_factor(kin_phase, kmag, kv)
        # (x, theta) representation: axes theta_y, y, theta_x, x
        vv = [self._axis_coords(self.dtheta_y, N0), self._axis_coords(self.dy, N1),
              self._axis_coords(self.dtheta_x, N2), self._axis_coords(self.dx, N3)]

        def pot_phase(ty, y, tx, x):
            return (dt * expr.evaluate(V, x=x - 0.5 * tx, y=y - 0.5 * ty)
                    - dt * expr.evaluate(V, x=x + 0.5 * tx, y=y + 0.5 * ty))

        Dty = self._c("D_theta_y")    # used for both axes, GPU_Wigner4D.py:275
        vmag = [np.exp(-dt * Dty * vv[0] * vv[0]), None, np.exp(-dt * Dty * vv[2] * vv[2]), None]
        vtabs, vfull = tables.build_factor(pot_phase, vmag, vv)
        self._factor_mode = ("pairwise" if kfull is None else "full",
                             "pairwise" if vfull is None else "full")
        # observables: coordinates of the reduction kernels (x(i) = dx (i - N/2))
        self._coords = [self._axis_coords(self.dp_y, N0), self._axis_coords(self.dy, N1),
                        self._axis_coords(self.dp_x, N2), self._axis_coords(self.dx, N3)]
        ep = np.ascontiguousarray(expr.evaluate(
            K, p_x=self._coords[2][None, :], p_y=self._coords[0][:, None]), np.float64)
        ex = np.ascontiguousarray(expr.evaluate(
            V, x=self._coords[3][None, :], y=self._coords[1][:, None]), np.float64)
        size = float(N0 * N1 * N2 * N3)
        d = _lib.Desc4D()
        d.shape[:] = list(self.shape)
        d.dtype = _lib.C128 if np.dtype(self.complex_dtype) == np.complex128 else _lib.C64
        # FAFT (d, delta) per axis exactly as the 64x64 wrappers pass them
        # (GPU_Wigner4D.py:409-427): axis 1 <- (dx, delta_x), axis 3 <- (dy,
        # delta_y), axis 0 <- (dp_x, delta_p_x), axis 2 <- (dp_y, delta_p_y).
        d.d[:] = [self.dp_x, self.dx, self.dp_y, self.dy]
        d.delta[:] = [self.delta_p_x, self.delta_x, self.delta_p_y, self.delta_y]
        d.kin_post_scale = 1.0 / (size * size)
        d.pot_post_scale = 1.0 / (size * size)
        keep = []

        def fill(dst, tabs, full):
            if full is not None:
                arr = np.ascontiguousarray(full).view(np.float64)
                keep.append(arr)
                dst[0].axis_a, dst[0].axis_b, dst[0].host_data = -1, -1, _lib.dptr(arr)
                return 1
            for i, (a, b, t) in enumerate(tabs):
                arr = np.ascontiguousarray(t).view(np.float64)
                keep.append(arr)
                dst[i].axis_a, dst[i].axis_b, dst[i].host_data = a, b, _lib.dptr(arr)
            return len(tabs)

        d.n_kin = fill(d.kin, ktabs, kfull)
        d.n_pot = fill(d.pot, vtabs, vfull)
        cs = [np.ascontiguousarray(c, np.float64) for c in self._coords]
        keep += cs + [ep, ex]
        for i in range(4):
            d.coord[i] = _lib.dptr(cs[i])
        d.energy_p = _lib.dptr(ep)
        d.energy_x = _lib.dptr(ex)
        d.dv_norm = self.dx * self.dp_x * self.dy * self.dp_y
        d.dv_obs = self._c("dx") * self._c("dy") * self._c("dp_x") * self._c("dp_y")
        plan = ctypes.c_void_p()
        if self.fp64_transforms:
            d.transform = 3
        else:
            d.transform = 2 if self.tensor_cores == "auto" else (1 if self.tensor_cores else 0)
        _lib.call("wig4d_plan_create", ctypes.byref(d), ctypes.byref(plan))
        self._plan = plan
        self.autotune_choice = None
        if self.autotune:
            ch = (ctypes.c_int * 4)()
            _lib.call("wig4d_autotune", plan, 3, 1 if self.autotune == "force" else 0, stream_ptr(), ch)
            engines = {0: "k_r4 plain stores", 1: "k_r4 cluster stores", 3: "k_tc64",
                       4: "per-size kernels", 6: "k_r4ring TMA stores",
                       7: "k_r4ring plane-contiguous"}
            self.autotune_choice = {"engine": engines[ch[0]], "k_kin48": bool(ch[1]), "pot_columns": ch[2],
                                    "timed": ch[3]}
        self._desc = d
        self._obs_buf = torch.empty(2 * _lib.WIG4D_NOBS, dtype=torch.float64, device="cuda")

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value and _lib._lib is not None:
            try:
                _lib._lib.wig4d_plan_destroy(plan)
            except Exception:
                pass
            self._plan = None

    def _check(self, W):
        if tuple(W.tensor.shape if isinstance(W, GPUArray) else W.shape) != self.shape:
            raise ValueError("state shape %s != grid %s" % (W.shape, self.shape))
        if wdtype_of(W) != self._desc.dtype:
            raise TypeError("state dtype does not match the plan's complex_dtype")
        return ptr_of(W)

    # ---- initial states (GPU_Wigner4D.py:216-245) ----------------------------
    def Gaussian_GPU(self, W, mu_p_y, mu_y, mu_p_x, mu_x, sigma_p_y, sigma_y, sigma_p_x, sigma_x):
        _lib.call("wig4d_init_gaussian", self._plan, self._check(W), mu_p_y, mu_y, mu_p_x, mu_x,
                  sigma_p_y, sigma_y, sigma_p_x, sigma_x, stream_ptr())

    def CatState_GPU(self, W, x_mu, y_mu, p_x_mu, p_y_mu, a_x, a_y):
        """Two displaced Gaussians in superposition (no reference initialiser):
        the wave function psi = [g(q - q_mu - a) + g(q - q_mu + a)] exp(i p_mu . q),
        g = exp(-|q|^2 / 2), turned into W(x, theta) = psi(x - theta/2)
        conj(psi(x + theta/2)) on the device, then Fourier_Theta_To_P_GPU into
        the (x, p) grid -- the pattern of WignerDiracGaussian_ParticleUp_GPU
        and the notebooks' preparation (GPU_WignerDirac4D.py:939-968).  The
        result is real up to rounding and negative where the two Gaussians
        interfere; Run() normalises it."""
        _lib.call("wig4d_init_cat_xtheta", self._plan, self._check(W), self._c("dtheta_y"), self._c("dtheta_x"),
                  x_mu, y_mu, p_x_mu, p_y_mu, a_x, a_y, stream_ptr())
        self.Fourier_Theta_To_P_GPU(W)

    def HOscillatorGound_GPU(self, W, x_mu, y_mu, p_x_mu, p_y_mu, omega_x, omega_y, mass):
        _lib.call("wig4d_init_ho_ground", self._plan, self._check(W), x_mu, y_mu, p_x_mu, p_y_mu,
                  omega_x, omega_y, mass, stream_ptr())

    # ---- reductions (GPU_Wigner4D.py:294-369) ----------------------------------
    def _reduce(self, W):
        _lib.call("wig4d_reduce", self._plan, self._check(W), self._obs_buf.data_ptr(), stream_ptr())
        return self._obs_buf.cpu().numpy()

    def Norm_GPU(self, W):
        r = self._reduce(W)
        return complex(r[0], r[1])

    def _raw(self, k):
        return lambda W: DeviceScalar(self._reduce(W)[_lib.WIG4D_NOBS + k])

    @property
    def Average_x_GPU(self):
        return self._raw(2)

    @property
    def Average_p_x_GPU(self):
        return self._raw(3)

    @property
    def Average_x_square_GPU(self):
        return self._raw(4)

    @property
    def Average_p_x_square_GPU(self):
        return self._raw(5)

    @property
    def Average_y_GPU(self):
        return self._raw(6)

    @property
    def Average_p_y_GPU(self):
        return self._raw(7)

    @property
    def Average_y_square_GPU(self):
        return self._raw(8)

    @property
    def Average_p_y_square_GPU(self):
        return self._raw(9)

    @property
    def Energy_GPU(self):
        return self._raw(10)

    # ---- transforms (GPU_Wigner4D.py:372-427) ----------------------------------
    def _faft(self, W, d, delta, axis, post=1.0):
        shape = (ctypes.c_int * 4)(*self.shape)
        _lib.call("wig_faft", self._check(W), shape, wdtype_of(W), axis, d, delta, post, stream_ptr())

    def _pair(self, W, a, b, sign):
        size = float(np.prod(self.shape))
        self._faft(W, self._desc.d[a], sign * self._desc.delta[a], a)
        self._faft(W, self._desc.d[b], sign * self._desc.delta[b], b, 1.0 / size)

    def Fourier_X_To_Lambda_64_64_GPU(self, W):
        self._pair(W, 1, 3, +1)

    def Fourier_Lambda_To_X_64_64_GPU(self, W):
        self._pair(W, 1, 3, -1)

    def Fourier_P_To_Theta_64_64_GPU(self, W):
        self._pair(W, 0, 2, +1)

    def Fourier_Theta_To_P_64_64_GPU(self, W):
        self._pair(W, 0, 2, -1)

    # the reference's 64x128 wrappers (GPU_Wigner4D.py:387-405) pass these
    # (d, delta, axis) triples verbatim
    def Fourier_X_To_Lambda_64_128_GPU(self, W):
        size = float(np.prod(self.shape))
        self._faft(W, self.dp_x, self.delta_p_x, 1)
        self._faft(W, self.dp_y, self.delta_p_y, 2, 1.0 / size)

    def Fourier_Lambda_To_X_64_128_GPU(self, W):
        size = float(np.prod(self.shape))
        self._faft(W, self.dp_x, -self.delta_p_x, 1)
        self._faft(W, self.dp_y, -self.delta_p_y, 2, 1.0 / size)

    def Fourier_P_To_Theta_64_128_GPU(self, W):
        size = float(np.prod(self.shape))
        self._faft(W, self.dp_x, self.delta_p_x, 0)
        self._faft(W, self.dp_y, self.delta_p_y, 3, 1.0 / size)

    def Fourier_Theta_To_P_64_128_GPU(self, W):
        size = float(np.prod(self.shape))
        self._faft(W, self.dp_x, -self.delta_p_x, 0)
        self._faft(W, self.dp_y, -self.delta_p_y, 3, 1.0 / size)

    # general names (any grid)
    Fourier_X_To_Lambda_GPU = Fourier_X_To_Lambda_64_64_GPU
    Fourier_Lambda_To_X_GPU = Fourier_Lambda_To_X_64_64_GPU
    Fourier_P_To_Theta_GPU = Fourier_P_To_Theta_64_64_GPU
    Fourier_Theta_To_P_GPU = Fourier_Theta_To_P_64_64_GPU

    # ---- phase kernels (GPU_Wigner4D.py:251-281) -------------------------------
    def exp_p_lambda_GPU(self, W):
        _lib.call("wig4d_apply_factor", self._plan, self._check(W), 0, stream_ptr())

    def exp_x_theta_GPU(self, W):
        _lib.call("wig4d_apply_factor", self._plan, self._check(W), 1, stream_ptr())

    def plan_info(self):
        """Kernels the plan runs: fused_kinetic, fused_potential, fast64, run64_kernel."""
        info = (ctypes.c_int * 4)()
        _lib.call("wig4d_plan_info", self._plan, info)
        run64 = {0: None, 3: "r4", 6: "tc", 7: "r4_mixed", 9: "r4ring_ts", 10: "r4ring_pc",
                 11: "r4ring_mx", 12: "r4ring_f32"}[info[3]]
        return {"fused_kinetic": bool(info[0]), "fused_potential": bool(info[1]), "fast64": bool(info[2]),
                "run64_kernel": run64}

    def _plan_fused(self):
        i = self.plan_info()
        return i["fused_kinetic"], i["fused_potential"]

    # ---- fused half-steps ---------------------------------------------------------
    def kinetic_halfstep(self, W):
        """Fourier_X_To_Lambda + exp_p_lambda_GPU + Fourier_Lambda_To_X in one kernel."""
        _lib.call("wig4d_kinetic", self._plan, self._check(W), None, stream_ptr())

    def potential_halfstep(self, W):
        """Fourier_P_To_Theta + exp_x_theta_GPU + Fourier_Theta_To_P in one kernel."""
        _lib.call("wig4d_potential", self._plan, self._check(W), stream_ptr())

    # ---- Run (GPU_Wigner4D.py:431-541) -------------------------------------------
    def run_device(self, W, iterations, history):
        """``iterations`` Run() iterations on device; ``history`` is a float64
        CUDA tensor of shape (iterations, 11) (no host synchronisation)."""
        _lib.call("wig4d_run", self._plan, self._check(W), int(iterations), history.data_ptr(),
                  stream_ptr())

    def run_device_timed(self, W, iterations, history):
        """run_device without the CUDA graph, each kernel bracketed by CUDA
        events; returns the summed milliseconds of the kinetic half-steps,
        potential half-steps and finalize kernels (synchronises)."""
        ms = (ctypes.c_double * 3)()
        _lib.call("wig4d_run_timed", self._plan, self._check(W), int(iterations), history.data_ptr(),
                  stream_ptr(), ms)
        return tuple(ms)

    def Run(self):
        iterations = self.timeSteps + 1
        W = self.W_init_gpu
        every = int(getattr(self, "snapshotEvery", 0) or 0)
        if every <= 0 or every >= iterations:
            hist = torch.empty((max(iterations, 1), _lib.WIG4D_NOBS), dtype=torch.float64, device="cuda")
            self.run_device(W, iterations, hist)
            self._store_history(hist.cpu().numpy()[:iterations])
            return
        # Snapshots: the loop runs in chunks of `every` iterations; between
        # chunks the final renormalisation is skipped (WIG_RUN_KEEP_NORM), so
        # the chunks continue one Run().  Snapshot t is the state whose
        # observables row t records, normalised as Run() normalises it.
        rows, self.snapshots = [], []
        self._W0_copy = W.get()
        t = 0
        while t < iterations:
            n = min(every, iterations - t)
            last = t + n >= iterations
            hist = torch.empty((n, _lib.WIG4D_NOBS), dtype=torch.float64, device="cuda")
            _lib.call("wig4d_run_ex", self._plan, self._check(W), n, hist.data_ptr(),
                      0 if last else _lib.WIG_RUN_KEEP_NORM, stream_ptr())
            h = hist.cpu().numpy()
            # the state that entered this chunk, normalised by its row-0 norm
            t0 = float(getattr(self, "time_offset", 0.0))
            self.snapshots.append((t0 + t * self.dt, self._snapshot_from(self._W0_copy, h[0])))
            rows.append(h)
            t += n
            if not last:
                self._W0_copy = W.get()
        self._store_history(np.concatenate(rows)[:iterations])
        self._write_snapshots()

    def _snapshot_from(self, Wh, row):
        return Wh / complex(row[0], row[1])

    def _write_snapshots(self):
        fname = getattr(self, "fileName", None)
        if fname and self.snapshots:
            write_snapshots(fname, self.snapshots)

    # ---- checkpoint / resume (no counterpart in the reference) -----------------
    def save_checkpoint(self, fname):
        """Save the current state and the result attributes of the last Run()
        to ``fname`` (.npz).  A frame built with the same attributes continues
        the run after ``load_checkpoint``: its Run() starts from this state."""
        data = {"W": self.W_init_gpu.get(), "shape": np.array(self.shape),
                "dt": np.array(self.dt), "time_offset": np.array(self._time_offset_next())}
        for k in RESULT_NAMES:
            if hasattr(self, k):
                data[k] = np.asarray(getattr(self, k))
        np.savez(fname, **data)

    def load_checkpoint(self, fname):
        """Restore a state saved by ``save_checkpoint`` into ``W_init_gpu``."""
        with np.load(fname) as z:
            if tuple(z["shape"]) != self.shape:
                raise ValueError("checkpoint grid %s != %s" % (tuple(z["shape"]), self.shape))
            self.W_init_gpu.set(z["W"].astype(self.W_init_gpu.dtype))
            self.time_offset = float(z["time_offset"])

    def _time_offset_next(self):
        # the state after the last Run() is len(energy) steps past its start
        t0 = float(getattr(self, "time_offset", 0.0))
        return t0 + len(getattr(self, "energy", ())) * self.dt

    def _store_history(self, h):
        """Run()'s result attributes (and the Ehrenfest file) from the history rows."""
        iterations = h.shape[0]
        if not np.all(np.isfinite(h)):
            raise FloatingPointError("Run(): non-finite norm or observable")
        self.norm = h[:, 0] + 1j * h[:, 1]
        self.average_x, self.average_p_x = h[:, 2], h[:, 3]
        self.average_x_square, self.average_p_x_square = h[:, 4], h[:, 5]
        self.average_y, self.average_p_y = h[:, 6], h[:, 7]
        self.average_y_square, self.average_p_y_square = h[:, 8], h[:, 9]
        self.energy = h[:, 10]
        self.timeRange = float(getattr(self, "time_offset", 0.0)) + np.arange(iterations) * self.dt
        fname = getattr(self, "fileName", None)
        if fname:
            write_ehrenfest(fname, {
                "energy": self.energy, "average_x": self.average_x, "average_p_x": self.average_p_x,
                "average_y": self.average_y, "average_p_y": self.average_p_y,
                "average_x_square": self.average_x_square,
                "average_p_x_square": self.average_p_x_square,
                "average_y_square": self.average_y_square,
                "average_p_y_square": self.average_p_y_square})


RESULT_NAMES = ("norm", "average_x", "average_p_x", "average_x_square", "average_p_x_square", "average_y",
                "average_p_y", "average_y_square", "average_p_y_square", "energy", "timeRange")


def write_snapshots(fname, snaps):
    """Run()'s snapshots as ``/Snapshots/W_<i>`` with ``/Snapshots/time``:
    added to the HDF5 file when h5py is importable, else written to
    ``<fileName>.snapshots.npz`` with keys ``time`` and ``W_<i>``."""
    times = np.array([t for t, _ in snaps])
    try:
        import h5py
    except ImportError:
        np.savez(fname + ".snapshots.npz", time=times, **{"W_%d" % i: w for i, (_, w) in enumerate(snaps)})
        return fname + ".snapshots.npz"
    with h5py.File(fname, "a") as f:
        f["/Snapshots/time"] = times
        for i, (_, w) in enumerate(snaps):
            f["/Snapshots/W_%d" % i] = w
    return fname


def write_ehrenfest(fname, data):
    """The reference's ``/Ehrenfest/<name>`` datasets (GPU_Wigner4D.py:531-540):
    an HDF5 file when h5py is importable, else ``<fileName>.npz`` with the
    same dataset paths as keys."""
    try:
        os.remove(fname)
    except OSError:
        pass
    try:
        import h5py  # noqa: F401
    except ImportError:
        np.savez(fname + ".npz", **{"/Ehrenfest/" + k: v for k, v in data.items()})
        return fname + ".npz"
    with h5py.File(fname, "w") as f:
        for k, v in data.items():
            f["/Ehrenfest/" + k] = v
    return fname
