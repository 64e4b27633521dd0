/*
 * wigner_b200.h -- C ABI of the B200 (sm_100a) split-operator Wigner propagator.
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t
 * passed as void*, and returns an int status (WIG_OK == 0).  No C++ or
 * PyTorch type crosses this boundary; the library never frees caller memory.
 *
 * Reference interfaces replaced (cabrer7/PyWignerCUDA2):
 *   FAFT64_4D_Z2Z / IFAFT64_4D_Z2Z / FAFT128_4D_Z2Z / FAFT256_4D_Z2Z
 *       ctypes bindings of the external FAFT library, GPU_Wigner4D.py:29-58
 *       (same in GPU_WignerDirac4D.py:29-58, GPU_WignerDiracKvN4D.py:29-58).
 *   wig_faft            the general form of the above (any shape, axis, N).
 *   wig4d_*             GPU_Wigner4D's JIT kernels and Run() loop,
 *                       GPU_Wigner4D.py:216-541.
 *   wigd_*              GPU_WignerDirac4D / GPU_WignerDiracKvN4D kernels and
 *                       Run(), GPU_WignerDirac4D.py:240-1899,
 *                       GPU_WignerDiracKvN4D.py:240-1669.
 *
 * Array convention (the reference's): a 4-D complex array of shape
 * shape[4] = {N_py, N_y, N_px, N_x}, C order, x fastest.  "axis" is the
 * NumPy axis index into that shape.  dtype 0 = complex128, 1 = complex64.
 */
#ifndef WIGNER_B200_H
#define WIGNER_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define WIG_OK                 0
#define WIG_ERR_INVALID_ARG    1   /* null pointer, bad axis, bad dtype       */
#define WIG_ERR_UNSUPPORTED    2   /* shape not supported by this build       */
#define WIG_ERR_CUDA           3   /* a CUDA runtime call failed              */
#define WIG_ERR_ALLOC          4   /* device allocation failed                */
#define WIG_ERR_NONFINITE      5   /* a reduction saw NaN or Inf              */
#define WIG_ERR_ALIAS          6   /* two component pointers alias            */
#define WIG_ERR_TOO_LARGE      7   /* size above a fixed limit of the call    */
#define WIG_ERR_TIMEOUT        8   /* a bounded device wait gave up           */

#define WIG_C128 0
#define WIG_C64  1

/* Human-readable text for a status code (static storage). */
const char* wig_status_string(int status);

/* Text of the last CUDA error seen by this library on the calling thread. */
const char* wig_last_error(void);

/* Library version as an integer, major*10000 + minor*100 + patch. */
int wig_version(void);

/* ---- the fractional centred transform (FAFT) ---------------------------- */
/*
 * In place along one axis:
 *   F[k] = post_scale * 2 N d * sum_n f[n] exp(-2 pi i delta (n - N/2)(k - N/2))
 * delta is signed (the reference's "inverse" passes -delta).  |delta| N == 1
 * runs a radix FFT when N is 16, 32, 64 or 128; any other N or delta runs the
 * dense transform.  Replaces one FAFT*_4D_Z2Z call (GPU_Wigner4D.py:409-427)
 * plus, through post_scale, the wrapper's "W /= size" pass.
 */
int wig_faft(void* data, const int shape[4], int dtype, int axis,
             double d, double delta, double post_scale, void* stream);

/*
 * Drop-in shims with the exact ctypes signature the reference binds
 * (GPU_Wigner4D.py:34-35, 43-44, 51-55):
 *   int FAFTxx_4D_Z2Z(void* dev_ptr, double d, double delta,
 *                     int segment, int axes, double NF);
 * FAFT64_4D_Z2Z and IFAFT64_4D_Z2Z act on a 64^4 complex128 array (the
 * reference's 64x64 frames); FAFT128_4D_Z2Z and FAFT256_4D_Z2Z on the
 * (64, 64, 128, 128) array of its 64x128 frames, where the reference binds
 * them as cuda_faft64 and cuda_faft128 and calls them only from the
 * FAFT_64_128 / Fourier_*_64_128_GPU wrappers (GPU_Wigner4D.py:372-405).
 * The transform length is the array's extent along `axes`.  IFAFT64_4D_Z2Z is FAFT64_4D_Z2Z with delta negated (the reference
 * binds but never calls it).  segment must be 0 and NF 1, the only values
 * the reference passes.  They run on the legacy default stream.
 */
int FAFT64_4D_Z2Z(void* dev_ptr, double d, double delta, int segment, int axes, double NF);
int IFAFT64_4D_Z2Z(void* dev_ptr, double d, double delta, int segment, int axes, double NF);
int FAFT128_4D_Z2Z(void* dev_ptr, double d, double delta, int segment, int axes, double NF);
int FAFT256_4D_Z2Z(void* dev_ptr, double d, double delta, int segment, int axes, double NF);

/* ---- elementwise helpers ------------------------------------------------- */
/* data[i] *= (s_re + i s_im) for n complex elements. */
int wig_scale(void* data, long long n, int dtype, double s_re, double s_im, void* stream);
/* data[i] /= *d_norm, where d_norm points at one complex128 on the device. */
int wig_divide_by_device_scalar(void* data, long long n, int dtype,
                                const double* d_norm, void* stream);
/* data[i] = Re(data[i])  (Real_GPU, GPU_WignerDirac4D.py:240-244). */
int wig_real(void* data, long long n, int dtype, void* stream);

/* ---- factor tables ------------------------------------------------------- */
/*
 * A multiplicative phase factor is the product of up to WIG_MAX_FACTORS
 * complex tables, each indexed by two array axes (axis_a, axis_b):
 * value = data[i_a * shape[axis_b] + i_b].  axis_b < 0 gives a table over
 * axis_a alone; axis_a < 0 gives a full 4-D table in the array's layout.
 * Host data is interleaved (re, im) float64; the plan copies it to the GPU
 * (rounded to complex64 for WIG_C64 plans).
 */
#define WIG_MAX_FACTORS 12
typedef struct {
    int axis_a;
    int axis_b;
    const double* host_data;
} wig_factor;

/* ---- scalar Wigner4D plan ------------------------------------------------ */
typedef struct wig4d_plan wig4d_plan;

typedef struct {
    int shape[4];              /* N_py, N_y, N_px, N_x                          */
    int dtype;                 /* WIG_C128 (drop-in) or WIG_C64 (precision)     */
    /* FAFT parameters per array axis for the two half-steps.  Axes 1, 3 are
       transformed by the kinetic half-step (x <-> lambda), axes 0, 2 by the
       potential one (p <-> theta).  The forward call uses +delta, the inverse
       -delta, both with the same d (GPU_Wigner4D.py:409-427).                */
    double d[4];
    double delta[4];
    double kin_post_scale;     /* wrapper divisors of the kinetic pair, e.g. 1/size^2  */
    double pot_post_scale;     /* same for the potential pair                          */
    int n_kin;                 /* factor tables of exp_p_lambda (GPU_Wigner4D.py:251-262) */
    wig_factor kin[WIG_MAX_FACTORS];
    int n_pot;                 /* factor tables of exp_x_theta (GPU_Wigner4D.py:269-281)  */
    wig_factor pot[WIG_MAX_FACTORS];
    /* observables (GPU_Wigner4D.py:285-369): coordinates of each axis as the
       reduction kernels see them, host float64, lengths shape[axis].          */
    const double* coord[4];    /* p_y, y, p_x, x                                  */
    const double* energy_p;    /* K(p_x, p_y) on [N_py][N_px]                     */
    const double* energy_x;    /* V(x, y)     on [N_y][N_x]                       */
    double dv_norm;            /* dV of Norm_GPU (host precision)                 */
    double dv_obs;             /* dV of the ReductionKernels (device constants)   */
    /* Transform engine of the Run() entry points (no counterpart in the
       reference, whose transforms are the FAFT calls of GPU_Wigner4D.py:
       409-427): 0 the CUDA-core kernels (radix for |delta| N = 1, dense
       otherwise); 1 k_tc64, every 64-point transform of a half-step as a
       dense complex GEMM on the tensor cores (tcgen05.mma kind::f16,
       operands split into fp16 hi + lo, three products, FP32 accumulation
       in tensor memory; the factor as float-float products of FP64
       vectors; FP64 sums above the row level), for any delta.  1 needs
       WIG_C64 on a 64^4 grid, factor tables that do not span both in-plane
       axes of a half-step, positive deltas and the same |delta| on the two
       in-plane axes of each half-step (else WIG_ERR_UNSUPPORTED).  2 sets
       k_tc64 up as a candidate of wig4d_autotune and starts with 0.  3 (a
       WIG_C64 plan on the 64^4 radix path) keeps the complex64 state in
       memory but runs the transforms and factors in FP64 (k_r4 with
       complex128 arithmetic on complex64 storage).                       */
    int transform;
} wig4d_desc;

/* Number of float64 values wig4d_reduce and one wig4d_run iteration write. */
#define WIG4D_NOBS 11
/* Order: norm_re, norm_im, <x>, <p_x>, <x^2>, <p_x^2>, <y>, <p_y>, <y^2>,
   <p_y^2>, energy  -- the moments of the state divided by its complex norm,
   exactly as Run() records them after "W /= norm" (GPU_Wigner4D.py:483-498). */

int wig4d_plan_create(const wig4d_desc* desc, wig4d_plan** plan);
int wig4d_plan_destroy(wig4d_plan* plan);

/* Fused kinetic half-step, in place: X->Lambda, exp_p_lambda, Lambda->X
   (GPU_Wigner4D.py:501-506), times *d_inv_norm if non-null (a complex128
   device scalar the state is divided by first, as in W4D:484). */
int wig4d_kinetic(wig4d_plan* plan, void* W, const double* d_norm, void* stream);
/* Fused potential half-step, in place: P->Theta, exp_x_theta, Theta->P
   (GPU_Wigner4D.py:508-513). */
int wig4d_potential(wig4d_plan* plan, void* W, void* stream);
/* The factor of one half-step applied alone, in place, on a state already in
   the (lambda, p) (which = 0) or (x, theta) (which = 1) representation:
   exp_p_lambda_GPU / exp_x_theta_GPU (GPU_Wigner4D.py:251-281). */
int wig4d_apply_factor(wig4d_plan* plan, void* W, int which, void* stream);
/* Norm and observables of W (not modified) into d_out[2 * WIG4D_NOBS]
   (device): row 0 as Run() records them (moments of W / norm), row 1 the
   raw Re(sum q W dV) each of the reference's ReductionKernels returns for W
   as given (GPU_Wigner4D.py:294-358); both rows start with the complex norm. */
int wig4d_reduce(wig4d_plan* plan, const void* W, double* d_out, void* stream);
/*
 * Run() (GPU_Wigner4D.py:431-541) on the device: `iterations` times
 * {renormalise, record observables, kinetic half-step, potential half-step},
 * then a final renormalisation.  d_history receives iterations rows of
 * WIG4D_NOBS float64 (device memory, caller-owned).  No host synchronisation
 * happens inside; the launches are replayed from a CUDA graph.
 */
int wig4d_run(wig4d_plan* plan, void* W, int iterations, double* d_history, void* stream);
/*
 * wig4d_run with flags (no counterpart in the reference).  WIG_RUN_KEEP_NORM
 * skips the final renormalisation, so that consecutive calls continue one
 * Run() exactly: the next call's first history row is the norm the skipped
 * division would have used, and its first step divides by it.  Run() with
 * snapshots is split this way.
 */
#define WIG_RUN_KEEP_NORM 1
int wig4d_run_ex(wig4d_plan* plan, void* W, int iterations, double* d_history, int flags, void* stream);

/*
 * wig4d_run with per-kernel timing (no counterpart in the reference): the
 * same launches, issued one by one rather than from a graph, each iteration's
 * kinetic half-step, potential half-step and finalize bracketed by CUDA
 * events on `stream`.  ms_out (host, 3 doubles) receives the summed
 * milliseconds of the three parts over all iterations.  Returns after the
 * stream has finished the last iteration.
 */
int wig4d_run_timed(wig4d_plan* plan, void* W, int iterations, double* d_history, void* stream,
                    double* ms_out);

/*
 * Batched Run() (no counterpart in the reference): n independent instances,
 * each with its own plan, state (device, the plan's shape and dtype) and
 * history (iterations rows of WIG4D_NOBS float64), advanced `iterations`
 * Run() iterations together.  Every step is one CUDA graph launch whose
 * branches are the instances' iterations, so instances of different sizes
 * run concurrently.  Plans and states must be distinct (WIG_ERR_ALIAS).
 * Each instance ends exactly as wig4d_run would leave it.
 */
int wig4d_run_batch(wig4d_plan* const* plans, void* const* states, int n, int iterations,
                    double* const* d_histories, void* stream);

/* Initial states on the (x, p) grid, coordinates from desc.coord:
   HOscillatorGound_GPU (GPU_Wigner4D.py:233-245) and Gaussian_GPU (216-230). */
int wig4d_init_ho_ground(wig4d_plan* plan, void* W, double x_mu, double y_mu,
                         double p_x_mu, double p_y_mu, double omega_x,
                         double omega_y, double mass, void* stream);
int wig4d_init_gaussian(wig4d_plan* plan, void* W, double mu_p_y, double mu_y,
                        double mu_p_x, double mu_x, double s_p_y, double s_y,
                        double s_p_x, double s_x, void* stream);
/*
 * Two displaced Gaussians in superposition on the (x, theta) grid (no
 * reference initialiser; built as WignerDiracGaussian_ParticleUp_GPU builds
 * its spinor, GPU_WignerDirac4D.py:939-968):
 *   W = psi(x - theta/2) conj(psi(x + theta/2)),
 *   psi = [g(x - x_mu - a_x, y - y_mu - a_y) + g(x - x_mu + a_x, y - y_mu + a_y)]
 *         exp(i (p_x_mu x + p_y_mu y)),  g(u, v) = exp(-(u^2 + v^2) / 2),
 * theta_q = dtheta_q (i_q - N_q/2) along axes 0 (theta_y) and 2 (theta_x).
 * Fourier_Theta_To_P afterwards gives the Wigner function on the (x, p) grid.
 */
int wig4d_init_cat_xtheta(wig4d_plan* plan, void* W, double dtheta_y, double dtheta_x,
                          double x_mu, double y_mu, double p_x_mu, double p_y_mu,
                          double a_x, double a_y, void* stream);

/*
 * Observables of a state without any device allocation.  This entry point
 * has no counterpart in the reference.  It is for callers that cannot call
 * cudaMalloc (a fixed memory pool, a footprint budget, pre-registered
 * buffers only) and therefore cannot create a plan either: it computes what
 * wig4d_reduce computes -- d_out[2 * WIG4D_NOBS], the Run()-style row then
 * the raw row -- from device tables the caller already holds: the four axis
 * coordinate vectors, K(p_x, p_y) on [N_py][N_px] and V(x, y) on [N_y][N_x]
 * (see wig4d_desc).  Its partial sums live in a fixed array inside the
 * library (WIG4D_NOALLOC_MAX_COLUMNS * 12 doubles, 1.5 MiB, held by every GPU
 * that loads the library until the process exits); grids with
 * N_y * N_x > WIG4D_NOALLOC_MAX_COLUMNS return WIG_ERR_TOO_LARGE.  The first
 * call on a device looks up the array's device address (again after the
 * device's context was reset), so make it before any stream capture.  All calls share the array: calls whose kernels
 * overlap on the GPU race; calls ordered on one stream do not.
 */
#define WIG4D_NOALLOC_MAX_COLUMNS 16384
int wig4d_observables_noalloc(const void* W, const int shape[4], int dtype,
                              const double* d_coord_py, const double* d_coord_y,
                              const double* d_coord_px, const double* d_coord_x,
                              const double* d_energy_p, const double* d_energy_x,
                              double dv_norm, double dv_obs, double* d_out, void* stream);

/* Which kernels a plan runs (no counterpart in the reference): info[0] fused
   kinetic half-step, info[1] fused potential half-step, info[2] the 64^4
   radix Run() kernels (1 or 0 each); info[3] the 64^4 Run() kernels: 0 none,
   3 k_r4 (16 points per thread: the complex64 default; complex128 with
   WIG_FAST64_KERNEL=r4 or r4cluster), 6 k_tc64 (tensor-core transforms,
   wig4d_desc.transform = 1), 7 k_r4 with FP64 transforms on complex64
   storage (wig4d_desc.transform = 3 with WIG_MIXED_KERNEL=r4), 9 k_r4ring
   (complex128 persistent ring of TMA-loaded planes) on the LA / LB layouts
   with TMA tensor stores (WIG_FAST64_KERNEL=r4ring_ts), 10 k_r4ring on the
   plane-contiguous layouts with bulk stores (the complex128 default), 11
   k_r4ring_mx (the mixed form of wig4d_desc.transform = 3 on the
   plane-contiguous layouts; WIG_MIXED_KERNEL=r4 selects 7), 12 the same
   ring with float32 arithmetic for complex64 (WIG_FAST64_KERNEL=r4ring_f32). */
int wig4d_plan_info(const wig4d_plan* plan, int info[4]);


/*
 * The project's autotuner (no counterpart in the reference): times the
 * kernel choices this plan has on a scratch copy of a Gaussian state
 * (`iterations` Run() iterations each, CUDA events on `stream`) and keeps
 * the fastest.  The candidates are the 64^4 engines (k_r4 with cluster or
 * plain stores, complex128 k_r4ring on either layout, and k_tc64 when the plan was made with
 * wig4d_desc.transform = 2) or, for the other kernels, k_kin48 against
 * k_kinetic on 48 x 48 planes and the columns per CTA of k_potential_g
 * (8, 4, 2, or k_potential).  The choice is cached per (shape, dtype,
 * kernel path) for the process: later plans with the same key take it
 * without timing unless flags has WIG_TUNE_FORCE.  choice_out (host, 4
 * ints, may be NULL) receives the engine (0 k_r4 plain, 1 k_r4 cluster,
 * 3 k_tc64, 4 the per-size kernels, 6 k_r4ring on LA / LB with TMA stores,
 * 7 k_r4ring on plane-contiguous layouts), k_kin48 (1/0), the columns
 * per CTA and the number of candidates timed.  Allocates a scratch state;
 * synchronous; call it outside any stream capture.
 */
#define WIG_TUNE_FORCE 1
int wig4d_autotune(wig4d_plan* plan, int iterations, int flags, void* stream, int* choice_out);

/* Bytes of device memory the plan holds (tables, partial sums). */
long long wig4d_plan_device_bytes(const wig4d_plan* plan);

/* ---- 4 x 4 spinor Wigner-Dirac / KvN plan -------------------------------- */
/*
 * The sixteen components W11..W44 are passed as an array of sixteen device
 * pointers ("slots", row-major: slot 4a+b is W_{a+1,b+1}), each a 4-D array
 * of the plan's shape.  The elementwise entry points (mask, real, divide,
 * kinetic, potential, reduce, init) keep the reference's per-point order
 * and accept repeated pointers, reproducing the reference's Run(), which
 * binds W21 to W22 (GPU_WignerDirac4D.py:1716).  wigd_transform and
 * wigd_run reject repeated pointers (WIG_ERR_ALIAS).
 */
typedef struct wigd_plan wigd_plan;

typedef struct {
    int shape[4];              /* N_py, N_y, N_px, N_x                            */
    int dtype;                 /* WIG_C128 or WIG_C64                             */
    int kvn;                   /* 0: GPU_WignerDirac4D, 1: GPU_WignerDiracKvN4D   */
    double d[4], delta[4];     /* FAFT (d, delta) per axis, forward sign           */
    double post[4];            /* divisors of X->Lambda, Lambda->X, P->Theta,
                                  Theta->P (GPU_WignerDirac4D.py:1428-1458)       */
    double c, hbar, mass, dt;  /* device constants (as the CUDA preamble has them) */
    double m_pot;              /* mass of the potential propagator: 1e-12 Dirac
                                  (WD4D:542), 1e-6 KvN (KvN:536)                  */
    double d_lambda_x, d_lambda_y;   /* kinetic dephasing (WD4D:403)               */
    const double* coord[4];    /* (x, p) grid: p_y, y, p_x, x                      */
    const double* acoord[4];   /* ambiguity grid: theta_y, lambda_y, theta_x, lambda_x */
    const double* mask_xp[4];  /* boundary_xp_GPU factor per axis (WD4D:327-366)   */
    const double* mask_p[4];   /* boundary_p_GPU factor per axis (WD4D:292-325)    */
    int n_phase;               /* A0 Bopp phase exp(-i dt (A0(x-) - A0(x+))/hbar)   */
    wig_factor phase[WIG_MAX_FACTORS];   /* over (theta_y, y, theta_x, x)          */
    int a_rank;                /* A1, A2, A3 at x -+ theta/2 as sums of a_rank     */
    const double* a_tabs;      /* products F(ix, itheta_x) G(iy, itheta_y):
                                  [3][2 sides][a_rank][N_x*N_px + N_y*N_py]        */
    const double* obs_xy;      /* [7][N_y][N_x]: A0 A1 A2 A3 D1A0 D1A1 D1A2        */
    double dv_norm, dv_obs;
    /* Fields without a low-rank form (a_rank = 0): A1, A2, A3 at x -+ theta/2
       on every point of the (x, theta) grid, [3][2 sides][N_py*N_y*N_px*N_x]
       in the state's layout; NULL when the rank tables are used.  The
       reference evaluates any expression there (GPU_WignerDirac4D.py:580-604). */
    const double* a_full;
} wigd_desc;

/* values per observables row: norm_re, norm_im, <x>, <p_x>, <x^2>, <p_x^2>, <y>,
   <p_y>, <y^2>, <p_y^2>, Alpha_1, Alpha_2, Alpha_1_x, Alpha_2_y, energyKinetic,
   energyPotential, D_1_A_0, D_1_A_1, D_1_A_2 (GPU_WignerDirac4D.py:1784-1822). */
#define WIGD_NOBS 19

int wigd_plan_create(const wigd_desc* desc, wigd_plan** plan);
int wigd_plan_destroy(wigd_plan* plan);
/* which: 0 X->Lambda, 1 Lambda->X, 2 P->Theta, 3 Theta->P on nslots
   components (Fourier_*_64_64_4x4_GPU); d_norm (optional): complex128
   device scalar divided out. */
int wigd_transform(wigd_plan* plan, void* const* slots, int nslots, int which,
                   const double* d_norm, void* stream);
/* kind 1: boundary_xp_GPU, 2: boundary_p_GPU. */
int wigd_mask(wigd_plan* plan, void* const* slots, int kind, void* stream);
/* replace the factors of mask `kind` (four host float64 vectors, one per axis,
   e.g. for other bound_x / bound_p values); synchronous. */
int wigd_set_mask(wigd_plan* plan, int kind, const double* const* factors);
/* Real_GPU on W11, W22, W33, W44. */
int wigd_real_diag(wigd_plan* plan, void* const* slots, void* stream);
/* every slot /= *d_norm, slot by slot (Normalize_4x4_GPU). */
int wigd_divide(wigd_plan* plan, void* const* slots, const double* d_norm, void* stream);
/* trace norm and observables into d_out[WIGD_NOBS]; divide != 0 divides the
   observables by the norm.  The norm also goes to the plan's device scalar
   (wigd_norm_ptr). */
int wigd_reduce(wigd_plan* plan, void* const* slots, double* d_out, int divide, void* stream);
const double* wigd_norm_ptr(wigd_plan* plan);
/* ParticleProjector_GPU(sign) when projector_sign != 0, then the kinetic
   sandwich exp_p_lambda_GPU when kinetic != 0, on the (lambda, p) grid. */
int wigd_kinetic(wigd_plan* plan, void* const* slots, int projector_sign, int kinetic, void* stream);
/* Potential_Propagator_Kernel on the (x, theta) grid. */
int wigd_potential(wigd_plan* plan, void* const* slots, void* stream);
/* initial states on the (x, theta) grid (GPU_WignerDirac4D.py:908-1032) */
int wigd_init_particle_up(wigd_plan* plan, void* const* slots, double u_x, double u_y,
                          double x_mu, double y_mu, double x_sigma, double y_sigma, void* stream);
int wigd_init_majorana(wigd_plan* plan, void* const* slots, double u_x, double u_y,
                       double x_mu, double y_mu, double x_sigma, double y_sigma, void* stream);
int wigd_init_landau(wigd_plan* plan, void* const* slots, double B, double x_offset,
                     double y_offset, void* stream);
/* Run() (GPU_WignerDirac4D.py:1767-1851) with distinct component pointers:
   iterations x {boundary_xp, Real, normalise + observables row, X->Lambda,
   [projector], kinetic, Lambda->X, P->Theta, potential, Theta->P}. */
int wigd_run(wigd_plan* plan, void* const* slots, int iterations, int filter,
             double* d_history, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* WIGNER_B200_H */
