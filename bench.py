"""Benchmark: 4D Wigner split-operator steps/s at 64^4 on B200.

Workload (one "step" = one Run() iteration: renormalise, observables,
kinetic half-step x<->lambda, potential half-step p<->theta): the plain
complex128 GPU_Wigner4D drop-in on a 64x64x64x64 grid (268 MB state,
larger than the 126 MB L2, so no flush is needed between steps), seeded
quartic/coupling coefficients and a two-Gaussian cat state, D = 0.005,
dt = 0.005, delta = 1/N windows.  Beside it the same step in the complex64
precision form.  Synthetic seeded data; nothing is read from disk.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints ONE JSON line (rank 0).  ``--impl reference`` times the reference's
algorithm on the host cores instead: the NumPy/SciPy restatement of
GPU_Wigner4D.Run() in oracle/ (the reference itself is Python 2 + PyCUDA +
an absent FAFT library and cannot run here), multi-threaded, on the same
workload.  N > 1 runs N independent replicas (the path does not shard; one
process per GPU under torchrun).
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "4D Wigner steps/s at 64^4: FP32-TC batched vs FP64 plain, same B200, <=1e-6 err"
WORKLOAD = "GPU_Wigner4D plain complex128 Run() iteration, 64x64x64x64, cat state, V=0.5r^2+q r^4+k xy"


def _dist():
    from pywignercuda2_b200.replicas import rank_info
    return rank_info()


def _clock_sampler(local):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        p = subprocess.Popen(["nvidia-smi", "-i", str(local), "--query-gpu=" + q,
                              "--format=csv,noheader,nounits", "-lms", "100"],
                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
        return None
    time.sleep(1.0)   # nvidia-smi needs a moment before its first sample
    return p


def _clock_summary(proc):
    if proc is None:
        return None
    proc.terminate()
    try:
        out, _ = proc.communicate(timeout=5)
    except subprocess.TimeoutExpired:
        proc.kill()
        out, _ = proc.communicate()
    rows = [r.split(",") for r in out.strip().splitlines() if r.count(",") >= 8]
    if not rows:
        return None
    sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
    mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
    return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
            "reasons": reasons, "samples": len(rows)}


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def _traffic():
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)
    from the committed ncu summary profiles/dram_traffic.txt: lines of
    ``<kernel> <workload> <bytes>``."""
    out = {}
    try:
        for ln in open(os.path.join(ROOT, "profiles", "dram_traffic.txt")):
            f = ln.split()
            if len(f) == 3 and not ln.startswith("#"):
                out[(f[0], f[1])] = float(f[2])
    except OSError:
        pass
    return out


def _frame(dtype, **kw):
    """The 64^4 workload: config 2's coefficients, the cat state built by the
    product initialiser (psi-based W in (x, theta), then theta -> p)."""
    from configs import config2
    from frames import make_frame
    from pywignercuda2_b200 import GPU_Wigner4D
    params, c = config2(seed=0, n=64)
    f = make_frame(GPU_Wigner4D, params, complex_dtype=dtype, **kw)
    f.CatState_GPU(f.W_init_gpu, c[0], c[1], c[2], c[3], 1.5, 0.0)
    W0 = f.W_init_gpu.get()
    return f, W0


def _hist_err(h, ref):
    """Relative errors of a Run() history against a reference history."""
    def rel(a, b):
        return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
    return {"norm_rel_max": rel(h[:, 0], ref[:, 0]), "energy_rel_max": rel(h[:, 10], ref[:, 10]),
            "energy_rel_last": float(abs(h[-1, 10] - ref[-1, 10]) / abs(ref[-1, 10])),
            "x_rel_max": rel(h[:, 2], ref[:, 2]), "p_x_rel_max": rel(h[:, 3], ref[:, 3]),
            "x2_rel_max": rel(h[:, 4], ref[:, 4])}


def accuracy_1000(steps=1000):
    """The FP32 forms after `steps` Run() iterations against the complex128
    drop-in from the same initial state (the drop-in matches the FP64 oracle
    to 1e-12 over 20 iterations at 64^4 and 3 iterations on config 3's grid,
    tests/test_gpu_tc.py and tests/test_gpu_w4d.py): the radix complex64
    kernels, the tensor-core kernels and complex64 storage with FP64
    transforms at 64^4 (config 2), and the complex64
    form on config 3's 64 x 128 x 64 x 128 grid."""
    import torch
    from configs import w4d_params
    from frames import make_frame
    from pywignercuda2_b200 import GPU_Wigner4D, _lib
    out = {"steps": steps, "reference": "complex128 drop-in on the same GPU (oracle-pinned)"}

    def run(f, W0):
        h = torch.empty((steps, _lib.WIG4D_NOBS), dtype=torch.float64, device="cuda")
        f.W_init_gpu.set(W0.astype(f.complex_dtype))
        f.run_device(f.W_init_gpu, steps, h)
        return h.cpu().numpy(), f.W_init_gpu.tensor.to(torch.complex128)

    f, W0 = _frame(np.complex128)
    h128, w128 = run(f, W0)
    del f
    for name, kw in (("c64_radix", {}), ("c64_tensor_cores", {"tensor_cores": True}),
                     ("c64_storage_fp64_transforms", {"fp64_transforms": True})):
        g, _ = _frame(np.complex64, **kw)
        h, w = run(g, W0)
        e = _hist_err(h, h128)
        e["max_dW_rel"] = (w - w128).abs().max().item() / w128.abs().max().item()
        out["64^4_" + name] = e
        del g, w
    del w128
    p = w4d_params(64, q=0.1, kappa=0.05, D=0.01, dt=0.005, n_p=128)
    fa = make_frame(GPU_Wigner4D, p)
    fa.HOscillatorGound_GPU(fa.W_init_gpu, 0.4, -0.3, 0.2, -0.1, 1.0, 1.0, 1.0)
    W3 = fa.W_init_gpu.get()
    h3, _ = run(fa, W3)
    del fa
    fb = make_frame(GPU_Wigner4D, p, complex_dtype=np.complex64)
    h3b, _ = run(fb, W3)
    del fb
    out["config3_64x128x64x128_c64_radix"] = _hist_err(h3b, h3)
    torch.cuda.empty_cache()
    return out


def cpu_baseline_port(steps, workers, budget_s=20.0):
    """The oracle's Run() iteration at 64^4 on the host (bounded sample)."""
    from configs import cat_xp, config2
    from oracle.wigner4d import Wigner4DOracle
    import oracle.faft as of
    params, c = config2(seed=0, n=64)
    o = Wigner4DOracle(params)
    coords = [o._axis(0, o.dp_y).ravel(), o._axis(1, o.dy).ravel(), o._axis(2, o.dp_x).ravel(),
              o._axis(3, o.dx).ravel()]
    W = cat_xp(coords, c)
    kin, pot = o.kinetic_factor(), o.potential_factor()
    of.FFT_WORKERS = workers
    W = o.step(W, kin, pot)     # warm-up (plans, page faults)
    n, t0 = 0, time.perf_counter()
    while n < steps:
        W = o.step(W, kin, pot)
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    of.FFT_WORKERS = 1
    return n / dt, n, dt


def bench_batched(steps):
    """The batched workload: 48 instances (16 each at 32^4, 48^4, 64^4, own
    coefficients, centres, D and dt) advanced together in complex64 through
    WignerBatch, against the same 48 run one at a time in the plain complex128
    form.  Aggregate grid-point steps per second, CUDA events.  With N ranks
    the instances are split among them (no collective on the data path): the
    job's time is the slowest rank's, its points the sum over ranks."""
    import torch
    from configs import config4, gaussian_xp
    from frames import make_frame
    from pywignercuda2_b200 import GPU_Wigner4D, WignerBatch, replicas
    ws, rank, _ = replicas.rank_info()
    cfg = replicas.shard(config4(0), rank, ws)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    frames = []
    tuned = {}
    for params, c in cfg:
        f = make_frame(GPU_Wigner4D, dict(params, timeSteps=steps - 1), complex_dtype=np.complex64,
                       autotune=True)
        f.W_init_gpu.set(gaussian_xp(f._coords, c).astype(np.complex64))
        frames.append(f)
        if f.autotune_choice["timed"]:
            tuned["%d^4" % f.shape[0]] = f.autotune_choice
    pts_rank = sum(int(np.prod(f.shape)) for f in frames)
    pts = int(replicas.sum_over_ranks(pts_rank))
    batch = WignerBatch(frames)
    hists = [torch.empty((steps, 11), dtype=torch.float64, device="cuda") for _ in frames]
    batch.run_device(3, hists)
    torch.cuda.synchronize()
    replicas.barrier()
    e0.record()
    batch.run_device(steps, hists)
    e1.record()
    torch.cuda.synchronize()
    ms_batch = replicas.max_over_ranks(e0.elapsed_time(e1))
    finite = all(bool(torch.isfinite(h).all()) for h in hists)
    del batch, frames, hists
    ms_plain = 0.0
    for params, c in cfg:
        f = make_frame(GPU_Wigner4D, dict(params, timeSteps=steps - 1), autotune=True)
        f.W_init_gpu.set(gaussian_xp(f._coords, c))
        h = torch.empty((steps, 11), dtype=torch.float64, device="cuda")
        f.run_device(f.W_init_gpu, 3, h)
        torch.cuda.synchronize()
        e0.record()
        f.run_device(f.W_init_gpu, steps, h)
        e1.record()
        torch.cuda.synchronize()
        ms_plain += e0.elapsed_time(e1)
        del f, h
    ms_plain = replicas.max_over_ranks(ms_plain)
    return {"workload": "48 instances: 16 x 32^4, 16 x 48^4, 16 x 64^4, seeded q, kappa, centre, "
                        "D in U[0.001, 0.02], dt in {0.005, 0.01}", "steps": steps,
            "grid_points": pts, "dtype": "c64", "ranks": ws,
            "scaling": "strong", "parallelism": "instances split over ranks" if ws > 1 else "single",
            "gp_steps_per_s": pts * steps / (ms_batch / 1e3), "ms": ms_batch, "finite": finite,
            "one_at_a_time_plain_c128": {"gp_steps_per_s": pts * steps / (ms_plain / 1e3), "ms": ms_plain},
            "speedup_vs_one_at_a_time_plain": ms_plain / ms_batch,
            "autotune": tuned}


def _dirac_frame(steps, complex_dtype=np.complex128):
    """The Wigner-Dirac workload: 64^4 grid x 16 components (4.3 GB in
    complex128), V = 0.3 (x^2 + y^2), symmetric-gauge field B in U[0.1, 0.5],
    D_lambda = 0.005, dt = 0.002, delta = 1/N windows."""
    import math
    from frames import make_frame
    from pywignercuda2_b200 import GPU_WignerDirac4D
    rng = np.random.default_rng(5000)
    B = float(rng.uniform(0.1, 0.5))
    x0, y0 = (float(v) for v in rng.uniform(-2, 2, size=2))
    n, amp_x, amp_p = 64, 8.0, 8.0
    dx, dp = 2 * amp_x / n, 2 * amp_p / n
    params = dict(gridDIM_p_y=n, gridDIM_y=n, gridDIM_p_x=n, gridDIM_x=n, dt=0.002, timeSteps=steps - 1,
                  p_y_amplitude=amp_p, y_amplitude=amp_x, p_x_amplitude=amp_p, x_amplitude=amp_x,
                  theta_y_amplitude=math.pi / dp, theta_x_amplitude=math.pi / dp,
                  lambda_y_amplitude=math.pi / dx, lambda_x_amplitude=math.pi / dx,
                  c=1.0, HBar=1.0, mass=1.0, potential_0_String="0.3*(x*x + y*y)",
                  potential_1_String="-%r*y/2." % B, potential_2_String="%r*x/2." % B,
                  potential_3_String="0.", D_1_potential_0_String="0.6*x", D_1_potential_1_String="0.",
                  D_1_potential_2_String="%r/2." % B, D_theta_x=0.0, D_theta_y=0.0,
                  D_lambda_x=0.005, D_lambda_y=0.005)
    f = make_frame(GPU_WignerDirac4D, params, complex_dtype=complex_dtype)
    f.fileName = None
    return f, B, (x0, y0)


def dirac_passes(f, reps=5):
    """Milliseconds of each pass of one Dirac Run() iteration on the frame's
    state (CUDA events around `reps` launches of each)."""
    import torch
    from pywignercuda2_b200 import _lib
    from pywignercuda2_b200.device import stream_ptr
    from pywignercuda2_b200.dirac4d import NAMES
    Ws = [getattr(f, k) for k in NAMES]
    slots = f._slots(Ws)
    obs = torch.zeros(64, dtype=torch.float64, device="cuda")
    plan = f._plan
    stages = [
        ("boundary", lambda: _lib.call("wigd_mask", plan, slots, 1, stream_ptr())),
        ("real", lambda: _lib.call("wigd_real_diag", plan, slots, stream_ptr())),
        ("sums", lambda: _lib.call("wigd_reduce", plan, slots, obs.data_ptr(), 0, stream_ptr())),
        ("x_to_lambda", lambda: f._transform(Ws, 0)),
        ("kinetic", lambda: _lib.call("wigd_kinetic", plan, slots, 0, 1, stream_ptr())),
        ("lambda_to_x", lambda: f._transform(Ws, 1)),
        ("p_to_theta", lambda: f._transform(Ws, 2)),
        ("potential", lambda: _lib.call("wigd_potential", plan, slots, stream_ptr())),
        ("theta_to_p", lambda: f._transform(Ws, 3)),
    ]
    out = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for name, fn in stages:
        fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1) / reps
    return out


def bench_dirac(steps):
    """The Wigner-Dirac workload (`_dirac_frame`) from a positive-energy
    Gaussian spinor.  Steps/s of Run() in the reference's call sequence (the
    W21 alias, the default) and of the fused device loop (alias off), CUDA
    events, and the milliseconds of each pass."""
    import torch
    from pywignercuda2_b200.dirac4d import NAMES
    f, B, (x0, y0) = _dirac_frame(steps)
    n = 64
    out = {"workload": "WignerDirac4D 64^4 x 16 components, complex128, B=%.3f, dt=0.002" % B,
           "state_bytes": 16 * n ** 4 * 16, "steps": steps}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    Ws = [getattr(f, k) for k in NAMES]
    for alias in (True, False):
        f.alias_w21 = alias
        def init():                            # the notebooks' preparation: (x, theta) -> (x, p)
            f.WignerDiracGaussian_ParticleUp_GPU(*Ws, 0.0, 0.0, x0, y0, 1.0, 1.0)
            f._Fourier_Theta_To_P_64_64_4x4_GPU(*Ws)
        init()
        f.timeSteps = 1
        f.Run()                                # warm-up (plans, graphs)
        init()
        f.timeSteps = steps - 1
        torch.cuda.synchronize()
        e0.record()
        f.Run()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        key = "reference_sequence" if alias else "fused_loop"
        out[key] = {"steps_per_s": steps / (ms / 1e3), "ms_per_step": ms / steps,
                    "hbm_gbs_per_sweep_equivalent": 2 * out["state_bytes"] / (ms / steps / 1e3) / 1e9,
                    "finite": bool(np.all(np.isfinite(f.energyKinetic)))}
    out["pass_ms"] = dirac_passes(f)
    del f
    torch.cuda.empty_cache()
    # the complex64 form of the same workload (fused loop), beside the plain one
    f, _, _ = _dirac_frame(steps, np.complex64)
    Ws = [getattr(f, k) for k in NAMES]
    f.alias_w21 = False

    def init32():
        f.WignerDiracGaussian_ParticleUp_GPU(*Ws, 0.0, 0.0, x0, y0, 1.0, 1.0)
        f._Fourier_Theta_To_P_64_64_4x4_GPU(*Ws)
    init32()
    f.timeSteps = 1
    f.Run()
    init32()
    f.timeSteps = steps - 1
    torch.cuda.synchronize()
    e0.record()
    f.Run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out["fused_loop_c64"] = {"steps_per_s": steps / (ms / 1e3), "ms_per_step": ms / steps,
                             "state_bytes": 16 * n ** 4 * 8,
                             "finite": bool(np.all(np.isfinite(f.energyKinetic))),
                             "energy_kinetic_last": float(f.energyKinetic[-1])}
    del f
    return out


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    cores = len(os.sched_getaffinity(0))
    steps = max(1, min(args.steps, 5))
    v, n, dt = cpu_baseline_port(steps, workers=cores, budget_s=120.0)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": n, "warmup": 1, "ms_per_step": 1e3 * dt / n, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": [64, 64, 64, 64], "parallelism": "replicas",
                       "cache": "inputs larger than L2"},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": cores, "kind": "port",
                             "sample": "%d Run() iterations of oracle/wigner4d.py at 64^4, scipy.fft "
                                       "workers=%d" % (n, cores)},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched 48-instance line")
    ap.add_argument("--batch-steps", type=int, default=100)
    ap.add_argument("--no-dirac", action="store_true", help="skip the Wigner-Dirac line")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the 1000-step accuracy block")
    ap.add_argument("--profile-form", choices=["c128", "c64", "tc", "tc-general", "mixed"],
                    help="only run two Run() iterations of one 64^4 form (a small case for ncu) and exit")
    ap.add_argument("--dirac-steps", type=int, default=20)
    ap.add_argument("--dirac-passes", choices=["c128", "c64"],
                    help="only time each pass of one Wigner-Dirac iteration in this dtype and exit")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_form:
        kw = {"c128": {}, "c64": {"complex_dtype": np.complex64},
              "tc": {"complex_dtype": np.complex64, "tensor_cores": True},
              "tc-general": {"complex_dtype": np.complex64, "tensor_cores": True},
              "mixed": {"complex_dtype": np.complex64, "fp64_transforms": True}}[args.profile_form]
        from configs import config2
        from frames import make_frame
        from pywignercuda2_b200 import GPU_Wigner4D
        params, c = config2(seed=0, n=64)
        if args.profile_form == "tc-general":     # the notebooks' windows, delta N = 0.716
            params.update(theta_x_amplitude=9.0, theta_y_amplitude=9.0, lambda_x_amplitude=9.0,
                          lambda_y_amplitude=9.0)
        f = make_frame(GPU_Wigner4D, params, complex_dtype=kw.pop("complex_dtype", np.complex128), **kw)
        f.CatState_GPU(f.W_init_gpu, c[0], c[1], c[2], c[3], 1.5, 0.0)
        f.timeSteps = 1
        f.fileName = None
        f.Run()
        print(json.dumps({"profile_form": args.profile_form, "kernels": f.plan_info(),
                          "energy": [float(e) for e in f.energy]}), flush=True)
        return 0
    if args.dirac_passes:
        from pywignercuda2_b200.dirac4d import NAMES
        f, _, (x0, y0) = _dirac_frame(2, np.complex64 if args.dirac_passes == "c64" else np.complex128)
        Ws = [getattr(f, k) for k in NAMES]
        f.WignerDiracGaussian_ParticleUp_GPU(*Ws, 0.0, 0.0, x0, y0, 1.0, 1.0)
        f._Fourier_Theta_To_P_64_64_4x4_GPU(*Ws)
        print(json.dumps({"dirac_pass_ms": dirac_passes(f), "dtype": args.dirac_passes}), flush=True)
        return 0

    import torch
    import torch.distributed as dist
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from pywignercuda2_b200 import _lib, replicas

    K, Wm = args.steps, args.warmup
    f, W0 = _frame(np.complex128)
    f.W_init_gpu.set(W0)
    st = torch.cuda.current_stream()
    hist = torch.empty((K + Wm + 2, _lib.WIG4D_NOBS), dtype=torch.float64, device="cuda")

    def barrier():
        replicas.barrier()
        torch.cuda.synchronize()

    # ---- device-resident throughput (value) ---------------------------------
    f.run_device(f.W_init_gpu, Wm, hist)
    barrier()
    clk = _clock_sampler(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(st)
    f.run_device(f.W_init_gpu, K, hist)
    e1.record(st)
    barrier()
    ms = e0.elapsed_time(e1)
    clocks = _clock_summary(clk)
    ms = replicas.max_over_ranks(ms)
    value = ws * K / (ms / 1e3)
    h128 = hist[:K].cpu().numpy()
    finite = bool(np.all(np.isfinite(h128)))
    W128 = f.W_init_gpu.tensor.clone()

    # ---- precision form (complex64) on the same workload and step count -------
    f32, _ = _frame(np.complex64)
    f32.W_init_gpu.set(W0.astype(np.complex64))        # the same initial state, rounded
    hist32 = torch.empty_like(hist)
    f32.run_device(f32.W_init_gpu, Wm, hist32)
    torch.cuda.synchronize()
    e0.record(st)
    f32.run_device(f32.W_init_gpu, K, hist32)
    e1.record(st)
    torch.cuda.synchronize()
    ms32 = e0.elapsed_time(e1)
    h32 = hist32[:K].cpu().numpy()
    dW = (f32.W_init_gpu.tensor.to(torch.complex128) - W128).abs().max().item()
    scale_W = W128.abs().max().item()
    del W128

    def rel(a, b):
        return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
    names = ["norm_re", "norm_im", "x", "p_x", "x2", "p_x2", "y", "p_y", "y2", "p_y2", "energy"]
    last = {n: float(abs(h32[-1, i] - h128[-1, i]) / max(abs(h128[-1, i]), 1e-300))
            for i, n in enumerate(names) if n != "norm_im"}
    precision = {"dtype": "c64", "steps_per_s": K / (ms32 / 1e3),
                 "speedup_vs_plain": (K / (ms32 / 1e3)) / (K / (ms / 1e3)),
                 "error_vs_c128": {"steps": Wm + K,
                                   "norm_rel_max": rel(h32[:, 0], h128[:, 0]),
                                   "energy_rel_max": rel(h32[:, 10], h128[:, 10]),
                                   "x_rel_max": rel(h32[:, 2], h128[:, 2]),
                                   "p_x_rel_max": rel(h32[:, 3], h128[:, 3]),
                                   "rel_at_last_step": last,
                                   "max_dW_rel": dW / scale_W,
                                   "reference": "the complex128 plain form on the same GPU, same "
                                                "initial state and steps (itself matched to the "
                                                "FP64 oracle to 1e-12 by the parity tests)"}}

    # ---- dominant-kernel roofline ----------------------------------------------
    # The same K iterations again, launched one by one with CUDA events around
    # each kernel on the launching stream: average duration of each launch.
    P = int(np.prod(f.shape))
    state_bytes = P * 16
    kin_ms, pot_ms, fin_ms = [m / K for m in f.run_device_timed(f.W_init_gpu, K, hist)]
    run64 = f.plan_info()["run64_kernel"]
    names = {"r4": ("k_r4<kin>", "k_r4<pot>"), "r4ring_ts": ("k_r4ring<kin>", "k_r4ring<pot>"),
             "r4ring_pc": ("k_r4ring<kin>", "k_r4ring<pot>")}.get(run64, ("k_kinetic", "k_potential"))
    dom_name, dom_ms = (names[1], pot_ms) if pot_ms >= kin_ms else (names[0], kin_ms)
    peaks = _peaks()
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    alg_bytes = 2 * state_bytes            # one read + one write of the state per launch
    achieved = alg_bytes / (dom_ms / 1e3) / 1e9
    tr = _traffic().get((dom_name, "64x64x64x64_c128"))
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": tr, "kernel": dom_name,
                "peak_source": peak_src, "algorithmic_bytes_per_launch": alg_bytes,
                "kinetic_ms": kin_ms, "potential_ms": pot_ms, "finalize_ms": fin_ms,
                "step_frac": (4 * state_bytes / (ms / K / 1e3) / 1e9) / peak}
    k32, p32, _ = [m / K for m in f32.run_device_timed(f32.W_init_gpu, K, hist32)]
    d32 = max(k32, p32)
    kname = "k_r4ring_mx" if f32.plan_info()["run64_kernel"] == "r4ring_f32" else "k_r4"
    precision["roofline"] = {"bound": "hbm", "kernel": kname + ("<pot>" if p32 >= k32 else "<kin>"),
                             "achieved": state_bytes / (d32 / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": state_bytes / (d32 / 1e3) / 1e9 / peak,
                             "algorithmic_bytes_per_launch": state_bytes,
                             "kinetic_ms": k32, "potential_ms": p32,
                             "traffic": _traffic().get((kname + ("<pot>" if p32 >= k32 else "<kin>"),
                                                        "64x64x64x64_c64"))}
    del f32

    # ---- mixed form: complex64 state in memory, FP64 transforms and factors ----
    fmx, _ = _frame(np.complex64, fp64_transforms=True)
    fmx.W_init_gpu.set(W0.astype(np.complex64))
    histmx = torch.empty_like(hist)
    fmx.run_device(fmx.W_init_gpu, Wm, histmx)
    torch.cuda.synchronize()
    e0.record(st)
    fmx.run_device(fmx.W_init_gpu, K, histmx)
    e1.record(st)
    torch.cuda.synchronize()
    msmx = e0.elapsed_time(e1)
    hmx = histmx[:K].cpu().numpy()
    kmx, pmx, _ = [m / K for m in fmx.run_device_timed(fmx.W_init_gpu, K, histmx)]
    dmx = max(kmx, pmx)
    mx_kernel = {"r4ring_mx": "k_r4ring_mx", "r4_mixed": "k_r4<double2, ., ., float2>"}.get(
        fmx.plan_info()["run64_kernel"], fmx.plan_info()["run64_kernel"])
    mixed_form = {"dtype": "c64 state, FP64 transforms and factors", "kernel": mx_kernel,
                  "steps_per_s": K / (msmx / 1e3), "speedup_vs_plain": (K / (msmx / 1e3)) / (K / (ms / 1e3)),
                  "kinetic_ms": kmx, "potential_ms": pmx,
                  "roofline": {"bound": "hbm", "achieved": state_bytes / (dmx / 1e3) / 1e9, "peak": peak,
                               "unit": "GB/s", "frac": state_bytes / (dmx / 1e3) / 1e9 / peak,
                               "algorithmic_bytes_per_launch": state_bytes,
                               "traffic": _traffic().get((mx_kernel + ("<pot>" if pmx >= kmx else "<kin>"),
                                                          "64x64x64x64_c64"))},
                  "error_vs_c128": dict(_hist_err(hmx, h128), steps=Wm + K)}
    del fmx

    # ---- tensor-core form (k_tc64: the 64-point transforms as dense GEMMs on
    # tcgen05, split fp16, FP32 accumulation) on the same workload ---------------
    ftc, _ = _frame(np.complex64, tensor_cores=True)
    ftc.W_init_gpu.set(W0.astype(np.complex64))
    histtc = torch.empty_like(hist)
    ftc.run_device(ftc.W_init_gpu, Wm, histtc)
    torch.cuda.synchronize()
    e0.record(st)
    ftc.run_device(ftc.W_init_gpu, K, histtc)
    e1.record(st)
    torch.cuda.synchronize()
    mstc = e0.elapsed_time(e1)
    htc = histtc[:K].cpu().numpy()
    ktc, ptc, _ = [m / K for m in ftc.run_device_timed(ftc.W_init_gpu, K, histtc)]
    dtc = max(ktc, ptc)
    # issued tensor FLOPs per launch: 2048 plane pairs x 4 stages x 3 products
    # x (2 x 128 x 128 x 128); the dense-DFT algorithmic count is 4 transforms
    # x 8 N flops per point
    tc_flops = 2048 * 4 * 3 * 2 * 128 ** 3
    dft_flops = 4 * 8 * 64 * P
    tpeak = peaks.get("bf16_tflops_sustained") or 1400.0
    tensor_form = {"dtype": "c64 state, fp16 hi+lo operands, FP32 accumulation", "kernel": "k_tc64",
                   "steps_per_s": K / (mstc / 1e3), "speedup_vs_plain": (K / (mstc / 1e3)) / (K / (ms / 1e3)),
                   "kinetic_ms": ktc, "potential_ms": ptc,
                   "roofline": {"bound": "tensor", "kernel": "k_tc64<pot>" if ptc >= ktc else "k_tc64<kin>",
                                "achieved": tc_flops / (dtc / 1e3) / 1e12, "peak": tpeak, "unit": "TFLOP/s",
                                "frac": tc_flops / (dtc / 1e3) / 1e12 / tpeak,
                                "peak_source": "measured bf16 dense, sustained" if peaks.get("bf16_tflops_sustained")
                                else "fallback",
                                "issued_tensor_flops_per_launch": tc_flops,
                                "dense_dft_flops_per_launch": dft_flops,
                                "hbm_frac": state_bytes / (dtc / 1e3) / 1e9 / peak,
                                "traffic": _traffic().get(("k_tc64<pot>" if ptc >= ktc else "k_tc64<kin>",
                                                           "64x64x64x64_c64"))},
                   "error_vs_c128": dict(_hist_err(htc, h128), steps=Wm + K)}
    del ftc

    # ---- end to end through the public API with host buffers ---------------------
    host_in = torch.from_numpy(W0).pin_memory()
    host_out = torch.empty(f.shape, dtype=torch.complex128).pin_memory()
    f.timeSteps = K - 1
    f.fileName = None
    barrier()
    t0 = time.perf_counter()
    e0.record(st)
    f.W_init_gpu.tensor.copy_(host_in, non_blocking=True)
    f.Run()                                     # history read back inside Run()
    host_out.copy_(f.W_init_gpu.tensor, non_blocking=True)
    e1.record(st)
    barrier()
    e2e_ms = replicas.max_over_ranks(e0.elapsed_time(e1))
    h2d = state_bytes
    d2h = state_bytes + K * _lib.WIG4D_NOBS * 8

    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws, "steps": K,
            "warmup": Wm, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": list(f.shape), "state_bytes": state_bytes,
                       "parallelism": "replicas" if ws > 1 else "single",
                       "cache": "inputs larger than L2 (268 MB state vs 126 MB L2), no flush",
                       "factor_mode": list(f._factor_mode)},
            "value_form": "FP64 plain drop-in (complex128, oracle-exact)",
            "grid_point_steps_per_s": value * P,
            "precision_form": precision,
            "tensor_core_form": tensor_form,
            "mixed_form": mixed_form,
            "gpu_launches": (4 * K + 4) if run64 in ("r4", "r4ring_ts", "r4ring_pc") else (3 * K + 3),
            "finite": finite, "roofline": roofline, "clocks": clocks,
            "e2e": {"value": ws * K / (e2e_ms / 1e3), "unit": "steps/s", "h2d_bytes_per_step": h2d / K,
                    "d2h_bytes_per_step": d2h / K,
                    "note": "one Run() of K iterations: pinned H2D of the state, history and "
                            "final state read back"}}
    if not args.no_batch:
        line["batched_form"] = bench_batched(args.batch_steps)
    if not args.no_accuracy:
        line["accuracy_1000_steps"] = accuracy_1000(1000)
    line["metric_ratio"] = {
        "tensor_core_vs_plain": tensor_form["speedup_vs_plain"],
        "fp32_radix_vs_plain": precision["speedup_vs_plain"],
        "c64_storage_fp64_transforms_vs_plain": mixed_form["speedup_vs_plain"],
        "batched_fp32_vs_one_at_a_time_plain": line.get("batched_form", {}).get("speedup_vs_one_at_a_time_plain"),
        "note": "steps/s ratios at 64^4 on the same GPU and step count; errors after 1000 steps are in "
                "accuracy_1000_steps (target <= 1e-6 in norm and energy)"}
    if not args.no_dirac:
        line["dirac_form"] = bench_dirac(args.dirac_steps)
    if rank == 0 and not args.no_cpu_baseline:
        v, n, dt = cpu_baseline_port(3, workers=1, budget_s=20.0)
        line["cpu_baseline"] = {"value": v, "unit": "steps/s", "cores": 1, "kind": "port",
                                "sample": "%d Run() iterations of oracle/wigner4d.py at 64^4 "
                                          "(numpy pocketfft, 1 thread), %.1f s" % (n, dt)}
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
