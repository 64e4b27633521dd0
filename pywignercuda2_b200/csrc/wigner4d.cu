// wigner4d.cu -- scalar 4-D Wigner split-operator step for sm_100a.
//
// Replaces GPU_Wigner4D's Run() loop (GPU_Wigner4D.py:431-541): per
// iteration, 2 x FAFT + "/= size" + exp_p_lambda + 2 x FAFT + "/= size"
// (x <-> lambda), the same around exp_x_theta (p <-> theta), and ten host-
// synchronising reductions.  Here one iteration is three kernels:
//
//   k_kinetic   one CTA per (p_y, p_x): loads the (y, x) plane, forward 2-D
//               transform in shared memory, multiplies by the kinetic factor
//               (phase, lambda damping, wrapper scales and the previous
//               iteration's 1/norm folded into one complex number per
//               point), inverse transform, stores.  1 read + 1 write.
//   k_potential one CTA per (y, x): the same over the (p_y, p_x) plane with
//               the Bopp potential factor; its epilogue also forms the
//               partial sums of the next iteration's norm and observables.
//   k_finalize  one CTA: reduces the partial sums in a fixed order, writes
//               the observables row and the complex norm the next kinetic
//               step divides by.
//
// The (-1)^n centring of the FAFT cancels between a forward and an inverse
// transform of the same axis except on the plane's input and output, where
// it is a sign flip; the 2 N d scales and wrapper divisors are one scalar.
#include <cuda.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

#include <cooperative_groups.h>

#include "common.cuh"
#include "fft_smem.cuh"

void* wig_dense_matrix(int n, double delta, int dtype, cudaStream_t st);

// ---------------------------------------------------------------------------
// Factor tables
// ---------------------------------------------------------------------------
template <class C>
struct FactorSet {
    int n;
    const C* data[WIG_MAX_FACTORS];
    int ia[WIG_MAX_FACTORS];
    int ib[WIG_MAX_FACTORS];
    int nb[WIG_MAX_FACTORS];
};

__device__ __forceinline__ int sel4(int a, int i0, int i1, int i2, int i3) {
    return a == 0 ? i0 : (a == 1 ? i1 : (a == 2 ? i2 : i3));
}

// Product of the factor tables at point (i0, i1, i2, i3); lin is the point's
// linear index in the array (used by full 4-D tables).
// The loop over the tables stays rolled: kernels call this at every point
// they hold, and the unrolled form (WIG_MAX_FACTORS bodies per call) made
// them miss in the instruction cache.
template <class C>
__device__ __forceinline__ C factor_at(const FactorSet<C>& F, int i0, int i1, int i2, int i3,
                                       long long lin, C acc) {
#pragma unroll 1
    for (int t = 0; t < F.n; ++t) {
        long long idx;
        if (F.ia[t] < 0) idx = lin;
        else if (F.ib[t] < 0) idx = sel4(F.ia[t], i0, i1, i2, i3);
        else idx = (long long)sel4(F.ia[t], i0, i1, i2, i3) * F.nb[t] + sel4(F.ib[t], i0, i1, i2, i3);
        acc = cmul(acc, __ldg(F.data[t] + idx));
    }
    return acc;
}

// The same product with the table loop unrolled (constant table indices):
// faster where a kernel calls it at few sites (the potential kernels).
template <class C>
__device__ __forceinline__ C factor_at_unrolled(const FactorSet<C>& F, int i0, int i1, int i2, int i3,
                                                long long lin, C acc) {
#pragma unroll
    for (int t = 0; t < WIG_MAX_FACTORS; ++t) {
        if (t < F.n) {
            long long idx;
            if (F.ia[t] < 0) idx = lin;
            else if (F.ib[t] < 0) idx = sel4(F.ia[t], i0, i1, i2, i3);
            else idx = (long long)sel4(F.ia[t], i0, i1, i2, i3) * F.nb[t] + sel4(F.ib[t], i0, i1, i2, i3);
            acc = cmul(acc, __ldg(F.data[t] + idx));
        }
    }
    return acc;
}

struct ObsTabs {
    const double* cx;    // x[N_x]
    const double* cy;    // y[N_y]
    const double* cpx;   // p_x[N_px]
    const double* cpy;   // p_y[N_py]
    const double* ep;    // K(p_x, p_y) [N_py][N_px]
    const double* ex;    // V(x, y) [N_y][N_x]
};

#define NPART 12   // partial sums per CTA: sum W, p_x W, p_x^2 W, p_y W, p_y^2 W, K W (complex)

// Block reduction of NPART doubles; thread 0 writes out[0..NPART).
template <int NT>
__device__ __forceinline__ void block_sum_partials(double (&a)[NPART], double* smem, double* out) {
#pragma unroll
    for (int i = 0; i < NPART; ++i) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a[i] += __shfl_down_sync(0xffffffffu, a[i], o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
#pragma unroll
        for (int i = 0; i < NPART; ++i) smem[w * NPART + i] = a[i];
    }
    __syncthreads();
    if (threadIdx.x < NPART) {
        double s = 0.0;
        for (int k = 0; k < NT / 32; ++k) s += smem[k * NPART + threadIdx.x];
        out[threadIdx.x] = s;
    }
}

// ---------------------------------------------------------------------------
// Plane layout in shared memory: rows of the plane are padded by one element
// (row stride NX + 1) so that a warp walking down a column, or across the
// rows at a fixed column, touches every bank once; every FFT pass then maps
// consecutive threads to consecutive lines (LINE_FAST) and is conflict-free.
// Loads and stores issue all of a thread's global accesses before touching
// shared memory, so each thread keeps PER requests in flight.
// ---------------------------------------------------------------------------
template <int NY, int NX, int NT>
struct PlaneCfg {
    static constexpr int LD = NX + 1;                 // padded row stride
    static constexpr int PTS = NY * NX;
    static constexpr int PER = (PTS + NT - 1) / NT;   // points per thread
    // two CTAs per SM while a thread holds at most 8 (512 threads) or 16
    // (256 threads) points
    static constexpr int MINB = ((NT >= 512 && PER <= 8) || (NT == 256 && PER <= 16)) ? 2 : 1;
};

template <class C, int NY, int NX>
static constexpr size_t plane_bytes() {
    return sizeof(C) * ((size_t)NY * (NX + 1) + NX + NY);
}

// ---------------------------------------------------------------------------
// Fused kinetic half-step: CTA = one (p_y, p_x) plane of NY x NX points.
// ---------------------------------------------------------------------------
template <class C, int NY, int NX, int NT>
__global__ void __launch_bounds__(NT, PlaneCfg<NY, NX, NT>::MINB) k_kinetic(C* __restrict__ W, int npy, int npx,
                                                const __grid_constant__ FactorSet<C> F, double2 scale,
                                                const double* __restrict__ d_norm) {
    typedef PlaneCfg<NY, NX, NT> P;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* s = reinterpret_cast<C*>(smraw);
    C* twx = s + NY * P::LD;
    C* twy = twx + NX;
    const int ipx = blockIdx.x % npx, ipy = blockIdx.x / npx;
    make_twiddles(twx, NX);
    if (NY != NX) make_twiddles(twy, NY);
    const C* ty = (NY != NX) ? twy : twx;

    const long long rowstride = (long long)npx * NX;
    C* g = W + ((long long)ipy * NY * npx + ipx) * NX;
    {
        C v[P::PER];
#pragma unroll
        for (int i = 0; i < P::PER; ++i) {
            const int e = threadIdx.x + i * NT;
            if (P::PTS % NT == 0 || e < P::PTS) v[i] = g[(e / NX) * rowstride + (e % NX)];
        }
#pragma unroll
        for (int i = 0; i < P::PER; ++i) {
            const int e = threadIdx.x + i * NT;
            if (P::PTS % NT == 0 || e < P::PTS) {
                const int y = e / NX, x = e % NX;
                s[y * P::LD + x] = ((x + y) & 1) ? cneg(v[i]) : v[i];
            }
        }
    }
    __syncthreads();
    const LineMap rows{1, P::LD, 0, 1}, cols{1, 1, 0, P::LD};
    fft_lines<C, NX, NY, NT, true, true>(s, rows, twx);
    fft_lines<C, NY, NX, NT, true, true>(s, cols, ty);

    double2 c0 = scale;
    if (d_norm) c0 = zmul(c0, zinv(make_double2(d_norm[0], d_norm[1])));
    const C cc = to_c<C>(c0);
    const long long lin0 = ((long long)ipy * NY * npx + ipx) * NX;
#pragma unroll
    for (int i = 0; i < P::PER; ++i) {
        const int e = threadIdx.x + i * NT;
        if (P::PTS % NT == 0 || e < P::PTS) {
            const int y = e / NX, x = e % NX;
            C f = factor_at(F, ipy, y, ipx, x, lin0 + y * rowstride + x, cc);
            s[y * P::LD + x] = cmul(s[y * P::LD + x], f);
        }
    }
    __syncthreads();
    fft_lines<C, NY, NX, NT, false, true>(s, cols, ty);
    fft_lines<C, NX, NY, NT, false, true>(s, rows, twx);
#pragma unroll
    for (int i = 0; i < P::PER; ++i) {
        const int e = threadIdx.x + i * NT;
        if (P::PTS % NT == 0 || e < P::PTS) {
            const int y = e / NX, x = e % NX;
            C v = s[y * P::LD + x];
            g[y * rowstride + x] = ((x + y) & 1) ? cneg(v) : v;
        }
    }
}

// ---------------------------------------------------------------------------
// Fused potential half-step: CTA = one (y, x) column, the (p_y, p_x) plane.
// Epilogue: partial sums of the next iteration's reductions.
// ---------------------------------------------------------------------------
template <class C, int NPY, int NPX, int NT>
__global__ void __launch_bounds__(NT, PlaneCfg<NPY, NPX, NT>::MINB) k_potential(C* __restrict__ W, int ny, int nx,
                                                  const __grid_constant__ FactorSet<C> F, double2 scale, ObsTabs ob,
                                                  double* __restrict__ partials) {
    typedef PlaneCfg<NPY, NPX, NT> P;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* s = reinterpret_cast<C*>(smraw);
    C* twx = s + NPY * P::LD;
    C* twy = twx + NPX;
    const int ix = blockIdx.x % nx, iy = blockIdx.x / nx;
    make_twiddles(twx, NPX);
    if (NPY != NPX) make_twiddles(twy, NPY);
    const C* ty = (NPY != NPX) ? twy : twx;

    const long long pxs = nx;                       // stride of p_x
    const long long pys = (long long)ny * NPX * nx; // stride of p_y
    C* g = W + (long long)iy * NPX * nx + ix;
    {
        C v[P::PER];
#pragma unroll
        for (int i = 0; i < P::PER; ++i) {
            const int e = threadIdx.x + i * NT;
            if (P::PTS % NT == 0 || e < P::PTS) v[i] = g[(e / NPX) * pys + (e % NPX) * pxs];
        }
#pragma unroll
        for (int i = 0; i < P::PER; ++i) {
            const int e = threadIdx.x + i * NT;
            if (P::PTS % NT == 0 || e < P::PTS) {
                const int py = e / NPX, px = e % NPX;
                s[py * P::LD + px] = ((px + py) & 1) ? cneg(v[i]) : v[i];
            }
        }
    }
    __syncthreads();
    const LineMap rows{1, P::LD, 0, 1}, cols{1, 1, 0, P::LD};
    fft_lines<C, NPX, NPY, NT, true, true>(s, rows, twx);
    fft_lines<C, NPY, NPX, NT, true, true>(s, cols, ty);
    const C cc = to_c<C>(scale);
    const long long lin0 = (long long)iy * NPX * nx + ix;
#pragma unroll
    for (int i = 0; i < P::PER; ++i) {
        const int e = threadIdx.x + i * NT;
        if (P::PTS % NT == 0 || e < P::PTS) {
            const int py = e / NPX, px = e % NPX;
            C f = factor_at_unrolled(F, py, iy, px, ix, lin0 + py * pys + px * pxs, cc);
            s[py * P::LD + px] = cmul(s[py * P::LD + px], f);
        }
    }
    __syncthreads();
    fft_lines<C, NPY, NPX, NT, false, true>(s, cols, ty);
    fft_lines<C, NPX, NPY, NT, false, true>(s, rows, twx);

    double a[NPART];
#pragma unroll
    for (int i = 0; i < NPART; ++i) a[i] = 0.0;
#pragma unroll
    for (int i = 0; i < P::PER; ++i) {
        const int e = threadIdx.x + i * NT;
        if (P::PTS % NT == 0 || e < P::PTS) {
            const int py = e / NPX, px = e % NPX;
            C v = s[py * P::LD + px];
            if ((px + py) & 1) v = cneg(v);
            g[py * pys + px * pxs] = v;
            if (partials) {
                const double2 w = to_d2(v);
                const double qx = __ldg(ob.cpx + px), qy = __ldg(ob.cpy + py);
                const double k = __ldg(ob.ep + py * NPX + px);
                a[0] += w.x; a[1] += w.y;
                a[2] = fma(qx, w.x, a[2]); a[3] = fma(qx, w.y, a[3]);
                a[4] = fma(qx * qx, w.x, a[4]); a[5] = fma(qx * qx, w.y, a[5]);
                a[6] = fma(qy, w.x, a[6]); a[7] = fma(qy, w.y, a[7]);
                a[8] = fma(qy * qy, w.x, a[8]); a[9] = fma(qy * qy, w.y, a[9]);
                a[10] = fma(k, w.x, a[10]); a[11] = fma(k, w.y, a[11]);
            }
        }
    }
    if (partials) {
        __syncthreads();   // smem reused for the block reduction
        block_sum_partials<NT>(a, reinterpret_cast<double*>(smraw), partials + (long long)blockIdx.x * NPART);
    }
}

// ---------------------------------------------------------------------------
// Fused potential half-step over G neighbouring (y, x) columns per CTA.
//
// A (p_y, p_x) plane at fixed (y, x) is a gather at stride N_x; taking the
// planes x0 .. x0+G-1 together makes every access a run of G elements
// (G * 16 or G * 8 = 64 bytes), and cp.async moves them straight into shared
// memory.  There are no centring sign flips: with S = (-1)^(p_x + p_y),
// S IFFT2(F FFT2(S w)) = IFFT2(F' FFT2(w)), F'[k] = F[k + N/2], so the factor
// is read at frequencies shifted by N/2.  One partial row per column, as
// k_potential writes.
// ---------------------------------------------------------------------------
template <class C, int NPY, int NPX, int G>
struct PotCfg {
    static constexpr int NT = 256;
    // complex64 planes of at most 48 x 48 points: two CTAs per SM (the
    // dispatch halves G); complex128 would spill at that register budget
    static constexpr int MINB = (sizeof(C) == 8 && NPY * NPX <= 48 * 48) ? 2 : 1;
    static constexpr int LD = NPX + 1;                              // row stride
    static constexpr int PSP = ((NPY * LD + 13) / 16) * 16 + 2;     // plane stride, = 2 (mod 16)
    static constexpr int PTS = NPY * NPX;
    static constexpr size_t bytes() {
        return sizeof(C) * ((size_t)G * PSP + NPX + NPY) + sizeof(double) * NPART * (NT / 32);
    }
};


template <class C, int NPY, int NPX, int G>
__global__ void __launch_bounds__(256, (PotCfg<C, NPY, NPX, G>::MINB)) k_potential_g(C* __restrict__ W, int ny, int nx, const __grid_constant__ FactorSet<C> F,
                                                        double2 scale, ObsTabs ob, double* __restrict__ partials) {
    typedef PotCfg<C, NPY, NPX, G> P;
    constexpr int NT = P::NT;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* s = reinterpret_cast<C*>(smraw);
    C* twx = s + G * P::PSP;
    C* twy = twx + NPX;
    double* red = reinterpret_cast<double*>(twy + NPY);
    const int nxg = nx / G;
    const int x0 = (blockIdx.x % nxg) * G, iy = blockIdx.x / nxg;
    make_twiddles(twx, NPX);
    if (NPY != NPX) make_twiddles(twy, NPY);
    const C* ty = (NPY != NPX) ? twy : twx;
    const long long pys = (long long)ny * NPX * nx;     // stride of p_y
    C* gb = W + (long long)iy * NPX * nx + x0;          // element (p_y, p_x, g): gb[p_y*pys + p_x*nx + g]
    for (int e = threadIdx.x; e < G * P::PTS; e += NT) {
        const int g = e % G, px = (e / G) % NPX, py = e / (G * NPX);
        cp_async_elem(s + g * P::PSP + py * P::LD + px, gb + py * pys + (long long)px * nx + g);
    }
    cp_async_wait_all();
    __syncthreads();
    // the planes' transforms one after another (registers as for one plane)
    const LineMap rows{1, P::LD, 0, 1}, cols{1, 1, 0, P::LD};
    for (int g = 0; g < G; ++g) {
        fft_lines<C, NPX, NPY, NT, true, true>(s + g * P::PSP, rows, twx);
        fft_lines<C, NPY, NPX, NT, true, true>(s + g * P::PSP, cols, ty);
    }
    const C cc = to_c<C>(scale);
    for (int e = threadIdx.x; e < G * P::PTS; e += NT) {
        const int g = e / P::PTS, r = e % P::PTS, py = r / NPX, px = r % NPX;
        const int ky = (py + NPY / 2) % NPY, kx = (px + NPX / 2) % NPX, ix = x0 + g;
        const long long lin = ky * pys + (long long)iy * NPX * nx + (long long)kx * nx + ix;
        C* q = s + g * P::PSP + py * P::LD + px;
        *q = cmul(*q, factor_at_unrolled(F, ky, iy, kx, ix, lin, cc));
    }
    __syncthreads();
    for (int g = 0; g < G; ++g) {
        fft_lines<C, NPY, NPX, NT, false, true>(s + g * P::PSP, cols, ty);
        fft_lines<C, NPX, NPY, NT, false, true>(s + g * P::PSP, rows, twx);
    }
    for (int e = threadIdx.x; e < G * P::PTS; e += NT) {
        const int g = e % G, px = (e / G) % NPX, py = e / (G * NPX);
        gb[py * pys + (long long)px * nx + g] = s[g * P::PSP + py * P::LD + px];
    }
    if (partials) {
        // plane-major: NT / G threads per column, in whole warps
        constexpr int TPP = NT / G;
        const int g = threadIdx.x / TPP, t = threadIdx.x % TPP;
        double a[NPART];
#pragma unroll
        for (int i = 0; i < NPART; ++i) a[i] = 0.0;
        for (int r = t; r < P::PTS; r += TPP) {
            const int py = r / NPX, px = r % NPX;
            const double2 w = to_d2(s[g * P::PSP + py * P::LD + px]);
            const double qx = __ldg(ob.cpx + px), qy = __ldg(ob.cpy + py), k = __ldg(ob.ep + py * NPX + px);
            a[0] += w.x; a[1] += w.y;
            a[2] = fma(qx, w.x, a[2]); a[3] = fma(qx, w.y, a[3]);
            a[4] = fma(qx * qx, w.x, a[4]); a[5] = fma(qx * qx, w.y, a[5]);
            a[6] = fma(qy, w.x, a[6]); a[7] = fma(qy, w.y, a[7]);
            a[8] = fma(qy * qy, w.x, a[8]); a[9] = fma(qy * qy, w.y, a[9]);
            a[10] = fma(k, w.x, a[10]); a[11] = fma(k, w.y, a[11]);
        }
#pragma unroll
        for (int i = 0; i < NPART; ++i)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) a[i] += __shfl_down_sync(0xffffffffu, a[i], o);
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        if (l == 0)
#pragma unroll
            for (int i = 0; i < NPART; ++i) red[w * NPART + i] = a[i];
        __syncthreads();
        if (threadIdx.x < G * NPART) {
            const int gg = threadIdx.x / NPART, i = threadIdx.x % NPART;
            double sum = 0.0;
            for (int k = 0; k < TPP / 32; ++k) sum += red[(gg * (TPP / 32) + k) * NPART + i];
            partials[((long long)iy * nx + x0 + gg) * NPART + i] = sum;
        }
    }
}

// ---------------------------------------------------------------------------
// Per-plane factor vectors of the 64^4 Run() kernels.
//
// * No centring sign flips in the radix kernels: with S = (-1)^(x+y),
//   S IFFT2(F FFT2(S w)) equals IFFT2(F' FFT2(w)) where F'[k] = F[k + N/2]
//   (indices mod N), so the factor is read at frequencies shifted by N/2.
// * The factor of a plane is the product of a vector along each in-plane
//   axis, built once per plan from the pairwise tables.
// ---------------------------------------------------------------------------
#define NSUM 22   // sum W, xW, x^2 W, p_x W, p_x^2 W, yW, y^2 W, p_y W, p_y^2 W, K W, V W (complex)
#define FOLD_BLOCKS 64   // first-stage rows of the Run() reduction over columns

// Per-plane factor vectors, built once at plan creation: for plane (f0, f1)
// the row-frequency vector PV[plane][0][k] and the column-frequency vector
// PV[plane][1][k] (k shifted by `shift`: N/2 for the radix kernels, which
// leave out the centring signs; 0 for k_tc64's centred matrices), whose outer product is the
// separable part of the factor.  Tables over both in-plane axes or full
// tables stay per point (the kernels test `pp`).
template <class C>
__global__ void k_plane_vectors(const __grid_constant__ FactorSet<C> F, int ay, int ax, int f0, int f1, int n_f1, int nplanes,
                                C* __restrict__ PV, int shift) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)nplanes * 128) return;
    const int plane = (int)(t >> 7), j = (int)(t & 127);
    const bool along_y = j < 64;
    const int k = j & 63, kk = (k + shift) & 63;
    const int i_f0 = plane / n_f1, i_f1 = plane % n_f1;
    const int axis = along_y ? ay : ax;
    double2 acc = make_double2(1.0, 0.0);
    for (int m = 0; m < F.n; ++m) {
        const int a = F.ia[m], b = F.ib[m];
        if (a < 0) continue;
        const bool ina = (a == ay || a == ax), inb = (b >= 0) && (b == ay || b == ax);
        if (ina && inb) continue;
        const bool touches = (a == axis) || (b == axis);
        const bool scalar = !ina && !inb;
        if (!(touches || (scalar && along_y))) continue;
        auto idx_of = [&](int ax_) { return ax_ == axis ? kk : (ax_ == f0 ? i_f0 : i_f1); };
        const long long idx = (b < 0) ? idx_of(a) : (long long)idx_of(a) * F.nb[m] + idx_of(b);
        acc = zmul(acc, to_d2(F.data[m][idx]));
    }
    PV[t] = to_c<C>(acc);
}

// Finalize of NSUM-wide partial rows (k_fold_columns' output).  One warp
// per sum: lanes stride over the rows, then a fixed shuffle tree.
__global__ void __launch_bounds__(32 * NSUM) k_finalize_sums(const double* __restrict__ part, int nrows,
                                                            double dv_norm, double dv_obs, double* out,
                                                            int* counter, int max_rows, double* cur_norm,
                                                            int* flag) {
    __shared__ double S[NSUM];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    double t = 0.0;
    for (int r = l; r < nrows; r += 32) t += part[(long long)r * NSUM + w];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (l == 0) S[w] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        const double2 n = make_double2(S[0] * dv_norm, S[1] * dv_norm);
        const double2 inv = zinv(n);
        auto obs = [&](int k) { return dv_obs * (S[k] * inv.x - S[k + 1] * inv.y); };
        double row[WIG4D_NOBS];
        row[0] = n.x; row[1] = n.y;
        row[2] = obs(2); row[3] = obs(6); row[4] = obs(4); row[5] = obs(8);
        row[6] = obs(10); row[7] = obs(14); row[8] = obs(12); row[9] = obs(16);
        row[10] = dv_obs * ((S[18] + S[20]) * inv.x - (S[19] + S[21]) * inv.y);
        double* dst = out;
        if (counter) {
            const int r = *counter;
            dst = (r < max_rows) ? out + (long long)r * WIG4D_NOBS : nullptr;
            *counter = r + 1;
        }
        bool bad = false;
        for (int i = 0; i < WIG4D_NOBS; ++i) bad |= !isfinite(row[i]);
        if (bad && flag) *flag = WIG_ERR_NONFINITE;
        if (dst)
            for (int i = 0; i < WIG4D_NOBS; ++i) dst[i] = row[i];
        if (cur_norm) { cur_norm[0] = n.x; cur_norm[1] = n.y; }
    }
}

#include "ff.cuh"
#include "dense_half.cuh"
#include "r4.cuh"
#include "tc64.cuh"

// First stage of the Run() reduction for one partial row per column (y, x):
// CTA b folds the columns b*per .. b*per + per - 1, weighted by x, y and V of
// each column, into one NSUM row (the layout k_finalize_sums reads).  Two
// small launches instead of one single-CTA pass over every column.
__global__ void __launch_bounds__(256) k_fold_columns(const double* __restrict__ part, int ncols, int nx, int per,
                                                      ObsTabs ob, double* __restrict__ rows) {
    __shared__ double red[NSUM][8];
    double a[NSUM];
#pragma unroll
    for (int i = 0; i < NSUM; ++i) a[i] = 0.0;
    const int c0 = blockIdx.x * per, c1 = min(ncols, c0 + per);
    for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
        const int ix = c % nx, iy = c / nx;
        const double x = __ldg(ob.cx + ix), y = __ldg(ob.cy + iy), V = __ldg(ob.ex + c);
        const double* p = part + (long long)c * NPART;
        const double wr = p[0], wi = p[1];
        a[0] += wr;               a[1] += wi;                 // W
        a[2] = fma(x, wr, a[2]);  a[3] = fma(x, wi, a[3]);    // x W
        a[4] = fma(x * x, wr, a[4]); a[5] = fma(x * x, wi, a[5]);
        a[6] += p[2];             a[7] += p[3];               // p_x W
        a[8] += p[4];             a[9] += p[5];               // p_x^2 W
        a[10] = fma(y, wr, a[10]); a[11] = fma(y, wi, a[11]); // y W
        a[12] = fma(y * y, wr, a[12]); a[13] = fma(y * y, wi, a[13]);
        a[14] += p[6];            a[15] += p[7];              // p_y W
        a[16] += p[8];            a[17] += p[9];              // p_y^2 W
        a[18] += p[10];           a[19] += p[11];             // K W
        a[20] = fma(V, wr, a[20]); a[21] = fma(V, wi, a[21]); // V W
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < NSUM; ++i) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a[i] += __shfl_down_sync(0xffffffffu, a[i], o);
        if (l == 0) red[i][w] = a[i];
    }
    __syncthreads();
    if (threadIdx.x < NSUM) {
        double t = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) t += red[threadIdx.x][k];
        rows[(long long)blockIdx.x * NSUM + threadIdx.x] = t;
    }
}

// Standalone reduction of a state in the (x, p) representation: same CTA
// shape and partial layout as k_potential's epilogue.
template <class C, int NT>
__global__ void __launch_bounds__(NT) k_reduce_xp(const C* __restrict__ W, int npy, int ny, int npx,
                                                  int nx, ObsTabs ob, double* __restrict__ partials) {
    __shared__ double sm[NPART * (NT / 32)];
    const int ix = blockIdx.x % nx, iy = blockIdx.x / nx;
    const long long pxs = nx, pys = (long long)ny * npx * nx;
    const C* g = W + (long long)iy * npx * nx + ix;
    double a[NPART];
#pragma unroll
    for (int i = 0; i < NPART; ++i) a[i] = 0.0;
    for (int e = threadIdx.x; e < npy * npx; e += NT) {
        const int py = e / npx, px = e % npx;
        const double2 w = to_d2(g[py * pys + px * pxs]);
        const double qx = ob.cpx[px], qy = ob.cpy[py], k = ob.ep[py * npx + px];
        a[0] += w.x; a[1] += w.y;
        a[2] = fma(qx, w.x, a[2]); a[3] = fma(qx, w.y, a[3]);
        a[4] = fma(qx * qx, w.x, a[4]); a[5] = fma(qx * qx, w.y, a[5]);
        a[6] = fma(qy, w.x, a[6]); a[7] = fma(qy, w.y, a[7]);
        a[8] = fma(qy * qy, w.x, a[8]); a[9] = fma(qy * qy, w.y, a[9]);
        a[10] = fma(k, w.x, a[10]); a[11] = fma(k, w.y, a[11]);
    }
    block_sum_partials<NT>(a, sm, partials + (long long)blockIdx.x * NPART);
}

// Final reduction: one CTA of 1024 threads, fixed summation order.
// Writes out[WIG4D_NOBS] (row of the history, or of wig4d_reduce) and the
// complex norm into cur_norm.  Row index comes from *counter when non-null.
__global__ void __launch_bounds__(1024) k_finalize(const double* __restrict__ part, int nblk, int nx,
                                                   ObsTabs ob, double dv_norm, double dv_obs,
                                                   double* out, int* counter, int max_rows,
                                                   double* cur_norm, int* flag, double* raw_out) {
    constexpr int NS = 22;
    __shared__ double sm[NS * 32];
    double a[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) a[i] = 0.0;
    for (int c = threadIdx.x; c < nblk; c += 1024) {
        const int ix = c % nx, iy = c / nx;
        const double x = ob.cx[ix], y = ob.cy[iy], V = ob.ex[iy * nx + ix];
        const double* p = part + (long long)c * NPART;
        const double wr = p[0], wi = p[1];
        a[0] += wr; a[1] += wi;                              // sum W
        a[2] = fma(x, wr, a[2]); a[3] = fma(x, wi, a[3]);    // x W
        a[4] += p[2]; a[5] += p[3];                          // p_x W
        a[6] = fma(x * x, wr, a[6]); a[7] = fma(x * x, wi, a[7]);
        a[8] += p[4]; a[9] += p[5];                          // p_x^2 W
        a[10] = fma(y, wr, a[10]); a[11] = fma(y, wi, a[11]);
        a[12] += p[6]; a[13] += p[7];                        // p_y W
        a[14] = fma(y * y, wr, a[14]); a[15] = fma(y * y, wi, a[15]);
        a[16] += p[8]; a[17] += p[9];                        // p_y^2 W
        a[18] += p[10]; a[19] += p[11];                      // K W
        a[20] = fma(V, wr, a[20]); a[21] = fma(V, wi, a[21]); // V W
    }
#pragma unroll
    for (int i = 0; i < NS; ++i) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a[i] += __shfl_down_sync(0xffffffffu, a[i], o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
#pragma unroll
        for (int i = 0; i < NS; ++i) sm[w * NS + i] = a[i];
    }
    __syncthreads();
    __shared__ double S[NS];
    if (threadIdx.x < NS) {                          // one thread per sum, fixed order
        double t = 0.0;
#pragma unroll 8
        for (int k = 0; k < 32; ++k) t += sm[k * NS + threadIdx.x];
        S[threadIdx.x] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double2 n = make_double2(S[0] * dv_norm, S[1] * dv_norm);
        const double2 inv = zinv(n);
        auto obs = [&](int k) { return dv_obs * (S[k] * inv.x - S[k + 1] * inv.y); };
        double row[WIG4D_NOBS];
        row[0] = n.x; row[1] = n.y;
        row[2] = obs(2); row[3] = obs(4); row[4] = obs(6); row[5] = obs(8);
        row[6] = obs(10); row[7] = obs(12); row[8] = obs(14); row[9] = obs(16);
        row[10] = dv_obs * ((S[18] + S[20]) * inv.x - (S[19] + S[21]) * inv.y);
        double* dst = out;
        if (counter) {
            int r = *counter;
            dst = (r < max_rows) ? out + (long long)r * WIG4D_NOBS : nullptr;
            *counter = r + 1;
        }
        bool bad = false;
        for (int i = 0; i < WIG4D_NOBS; ++i) bad |= !isfinite(row[i]);
        if (bad && flag) *flag = WIG_ERR_NONFINITE;
        if (dst)
            for (int i = 0; i < WIG4D_NOBS; ++i) dst[i] = row[i];
        if (cur_norm) { cur_norm[0] = n.x; cur_norm[1] = n.y; }
        if (raw_out) {   // Re(dV sum q W) of the state as given, as a ReductionKernel returns it
            raw_out[0] = n.x; raw_out[1] = n.y;
            for (int q = 0; q < 8; ++q) raw_out[2 + q] = dv_obs * S[2 + 2 * q];
            raw_out[10] = dv_obs * (S[18] + S[20]);
        }
    }
}

// Factor applied alone (unfused path): elementwise over the whole array.
template <class C>
__global__ void k_apply_factor(C* W, int n0, int n1, int n2, int n3, const __grid_constant__ FactorSet<C> F, double2 scale) {
    const long long tot = (long long)n0 * n1 * n2 * n3;
    const C cc = to_c<C>(scale);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot;
         i += (long long)gridDim.x * blockDim.x) {
        const int i3 = i % n3;
        const int i2 = (i / n3) % n2;
        const int i1 = (i / ((long long)n3 * n2)) % n1;
        const int i0 = i / ((long long)n3 * n2 * n1);
        W[i] = cmul(W[i], factor_at(F, i0, i1, i2, i3, i, cc));
    }
}

// Initial states (GPU_Wigner4D.py:216-245) on the (x, p) grid.
template <class C>
__global__ void k_init_ho(C* W, int n0, int n1, int n2, int n3, ObsTabs ob, double x_mu, double y_mu,
                          double px_mu, double py_mu, double wx, double wy, double mass) {
    const long long tot = (long long)n0 * n1 * n2 * n3;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot;
         i += (long long)gridDim.x * blockDim.x) {
        const int i3 = i % n3, i2 = (i / n3) % n2, i1 = (i / ((long long)n3 * n2)) % n1;
        const int i0 = i / ((long long)n3 * n2 * n1);
        const double x = ob.cx[i3], px = ob.cpx[i2], y = ob.cy[i1], py = ob.cpy[i0];
        double t = (mass * pow(wx * (x - x_mu), 2.0) + pow(px - px_mu, 2.0) / mass) / wx;
        t += (mass * pow(wy * (y - y_mu), 2.0) + pow(py - py_mu, 2.0) / mass) / wy;
        W[i] = to_c<C>(make_double2(exp(-t), 0.0));
    }
}
template <class C>
__global__ void k_init_gauss(C* W, int n0, int n1, int n2, int n3, ObsTabs ob, double mpy, double my,
                             double mpx, double mx, double spy, double sy, double spx, double sx) {
    const long long tot = (long long)n0 * n1 * n2 * n3;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot;
         i += (long long)gridDim.x * blockDim.x) {
        const int i3 = i % n3, i2 = (i / n3) % n2, i1 = (i / ((long long)n3 * n2)) % n1;
        const int i0 = i / ((long long)n3 * n2 * n1);
        const double x = ob.cx[i3], px = ob.cpx[i2], y = ob.cy[i1], py = ob.cpy[i0];
        double t = exp(-0.5 * (x - mx) * (x - mx) / (sx * sx));
        t *= exp(-0.5 * (y - my) * (y - my) / (sy * sy));
        t *= exp(-0.5 * (px - mpx) * (px - mpx) / (spx * spx));
        t *= exp(-0.5 * (py - mpy) * (py - mpy) / (spy * spy));
        W[i] = to_c<C>(make_double2(t, 0.0));
    }
}

// Two displaced Gaussians in superposition ("cat state") on the (x, theta)
// grid [theta_y][y][theta_x][x], built from the wave function as
// WignerDiracGaussian_ParticleUp_GPU builds its spinor (GPU_WignerDirac4D.py:
// 939-968): W = psi(x - theta/2) conj(psi(x + theta/2)) with
//   psi(x, y) = [g(x - x0 - ax, y - y0 - ay) + g(x - x0 + ax, y - y0 + ay)]
//               exp(i (px0 x + py0 y)),   g(u, v) = exp(-(u^2 + v^2) / 2).
// The theta -> p transform (Fourier_Theta_To_P) then gives the Wigner
// function, negative in the interference region.
template <class C>
__global__ void k_init_cat(C* W, int n0, int n1, int n2, int n3, ObsTabs ob, double dty, double dtx, double x0,
                           double y0, double px0, double py0, double ax, double ay) {
    const long long tot = (long long)n0 * n1 * n2 * n3;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot;
         i += (long long)gridDim.x * blockDim.x) {
        const int i3 = i % n3, i2 = (i / n3) % n2, i1 = (i / ((long long)n3 * n2)) % n1;
        const int i0 = i / ((long long)n3 * n2 * n1);
        const double x = ob.cx[i3], y = ob.cy[i1];
        const double tx = dtx * (i2 - n2 / 2), ty = dty * (i0 - n0 / 2);
        auto psi = [&](double u, double v) {
            const double g = exp(-0.5 * ((u - x0 - ax) * (u - x0 - ax) + (v - y0 - ay) * (v - y0 - ay))) +
                             exp(-0.5 * ((u - x0 + ax) * (u - x0 + ax) + (v - y0 + ay) * (v - y0 + ay)));
            double s, c;
            sincos(px0 * u + py0 * v, &s, &c);
            return make_double2(g * c, g * s);
        };
        const double2 a = psi(x - 0.5 * tx, y - 0.5 * ty), b = psi(x + 0.5 * tx, y + 0.5 * ty);
        W[i] = to_c<C>(zmul(a, make_double2(b.x, -b.y)));
    }
}

// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------
struct wig4d_plan {
    int shape[4];
    int dtype;
    double d[4], delta[4];
    double kin_scale, pot_scale;   // total scalar of each fused half-step
    bool fused_kin, fused_pot;     // fused fast kernels usable
    double dv_norm, dv_obs;
    long long npts;
    // device memory
    void* tabs;                    // all factor tables (one allocation)
    long long tab_bytes;
    FactorSet<double2> kin_d, pot_d;
    FactorSet<float2> kin_f, pot_f;
    double* obs_mem;               // coords + energy tables
    ObsTabs ob;
    double* partials;              // NPART per (y, x) column
    double* cur_norm;              // complex128 norm of the current state
    int* counter;                  // history row of the next finalize
    int* flag;                     // WIG_ERR_NONFINITE when seen
    bool fast64;                   // 64^4 grid with separable factors: Run() uses k_r4
    void* pingpong;                // second state buffer (layout [y][x][p_y][p_x])
    void* pv;                      // per-plane factor vectors of the two half-steps
    bool r4;                       // 64^4 Run(): k_r4 (16 points per thread) on its LA / LB layouts
    bool r4_cluster;               // k_r4 launched as clusters with full-sector stores
    bool kin48;                    // 48 x 48 kinetic planes: k_kin48 (else k_kinetic)
    int pot_gmax;                  // k_potential_g: at most this many columns per CTA (< 2: k_potential)
    bool tc_ready;                 // k_tc64's buffers exist (wig4d_desc.transform 1 or 2)
    int tuned;                     // wig4d_autotune has set the choices above
    bool r4ring;                   // complex128 64^4 Run(): persistent k_r4ring (TMA plane ring)
    bool r4ring_ready;             // k_r4ring's tensor map and attributes are set
    bool r4ring_pc;                // k_r4ring on the plane-contiguous layouts LK / LP (bulk stores)
    bool r4_mixed;                 // complex64 64^4: k_r4 with FP64 transforms on complex64 storage
    bool mx_ring;                  // the mixed form with k_r4ring_mx on the plane-contiguous layouts
    bool mx_f32;                   // ... with float32 arithmetic: the complex64 radix form on those layouts
    CUtensorMap map_t_load_mx;     // k_r4ring_mx: unit boxes of the ping-pong buffer (LK)
    CUtensorMap map_w_load_mx;     // and of the caller's state (LP)
    const void* map_w_mx_ptr;      // state map_w_load_mx describes
    void* tw64d;                   // its FP64 twiddle table
    int dense_n;                   // > 0: general-delta half-steps fused (k_dense_half, N^4 grids)
    const void* dmat[4];           // FAFT matrices per axis (|delta|), when dense_n > 0
    void* tw64;                    // k_r4 twiddle table (64 complex of the plan's dtype)
    double* fold;                  // k_fold_columns output: FOLD_BLOCKS rows of NSUM
    bool tc;                       // complex64 64^4 Run(): k_tc64 (tensor-core DFTs) on the LK / LP layouts
    void* tc_bimg[2];              // k_tc64's embedded FAFT matrices of the two half-steps (shared-memory images)
    void* tc_pv;                   // k_tc64's FP64 per-plane factor vectors (unshifted frequencies)
    CUtensorMap map_t_load;        // LA view of the ping-pong buffer (kinetic source)
    CUtensorMap map_w_load;        // LB view of the caller's state (potential source)
    CUtensorMap map_t_store;       // k_r4ring stores: the ping-pong buffer (potential destination, LA)
    CUtensorMap map_w_store;       // k_r4ring stores: the caller's state (kinetic destination, LB)
    CUtensorMap map_t_load_pc;     // k_r4ring plane-contiguous layouts: LK view of the ping-pong buffer
    CUtensorMap map_w_load_pc;     // and LP view of the caller's state
    const void* map_w_ptr;                 // state the W maps describe
    // CUDA graph of one Run() iteration, cached per (W, history, stream)
    cudaGraphExec_t graph;
    void* graph_W;
    double* graph_hist;
    int graph_rows;
};

static bool pow2_16_128(int n) { return wig_radix_size(n); }

// k_tc64's B operand: the centred 64-point FAFT matrix
//   M[k][n] = exp(-2 pi i delta (n - 32)(k - 32))
// embedded as the real 128 x 128 matrix B[(ri', k)][(ri, n)] (Re/Im of the
// output, Re/Im of the input), times 2^B_EXP, split into fp16 hi + lo, in
// the K-major no-swizzle layout of the kernel's shared memory: element
// (row, col) at byte (col/8)*2048 + (row/8)*128 + (row%8)*16 + (col%8)*2.
// The phase is reduced to [0, 1) turns in FP64 before the sine and cosine.
static int build_tc_bimg(double delta, void** out) {
    std::vector<__half> img(2 * 128 * 128);
    for (int row = 0; row < 128; ++row)
        for (int col = 0; col < 128; ++col) {
            const int rio = row >> 6, k = row & 63, ri = col >> 6, n = col & 63;
            double turns = delta * (double)((n - 32) * (k - 32));
            turns -= floor(turns);
            const double ang = 2.0 * M_PI * turns;
            const double c = cos(ang), s = sin(ang);   // M = c - i s
            const double b = ldexp((rio == ri) ? c : (ri == 1 ? s : -s), tc64::B_EXP);
            const __half hi = __float2half_rn((float)b);
            const __half lo = __float2half_rn((float)(b - (double)__half2float(hi)));
            const int off = ((col >> 3) * 2048 + (row >> 3) * 128 + (row & 7) * 16 + (col & 7) * 2) / 2;
            img[off] = hi;
            img[128 * 128 + off] = lo;
        }
    if (cudaMalloc(out, img.size() * sizeof(__half)) != cudaSuccess) return WIG_ERR_ALLOC;
    WIG_CUDA(cudaMemcpy(*out, img.data(), img.size() * sizeof(__half), cudaMemcpyHostToDevice));
    return WIG_OK;
}

// Threads per CTA of the fused kernels: one radix-8 butterfly per thread and
// pass for a 64 x 64 plane; smaller planes use fewer threads.
template <int A, int B> struct FusedNT { static constexpr int v = (A * B / 8 >= 512) ? 512 : (A * B / 8 >= 256 ? 256 : 128); };

template <class C> static FactorSet<C>& kin_set(wig4d_plan* p);
template <> FactorSet<double2>& kin_set<double2>(wig4d_plan* p) { return p->kin_d; }
template <> FactorSet<float2>& kin_set<float2>(wig4d_plan* p) { return p->kin_f; }
template <class C> static FactorSet<C>& pot_set(wig4d_plan* p);
template <> FactorSet<double2>& pot_set<double2>(wig4d_plan* p) { return p->pot_d; }
template <> FactorSet<float2>& pot_set<float2>(wig4d_plan* p) { return p->pot_f; }

#include "k48.cuh"

// Dispatch a fused kernel over the supported plane sizes.
#define WIG_PLANE_CASES(X) X(16, 16) X(32, 32) X(48, 48) X(64, 64) X(128, 128) X(64, 128) X(128, 64)

template <class C>
static int launch_kinetic(wig4d_plan* p, C* W, const double* d_norm, cudaStream_t st) {
    const int NY = p->shape[1], NX = p->shape[3];
    const int npy = p->shape[0], npx = p->shape[2];
    const unsigned grid = (unsigned)(npy * npx);
    const double2 sc = make_double2(p->kin_scale, 0.0);
    if (NY == 48 && NX == 48 && p->kin48) {                 // 48 x 48 planes in registers
        const size_t sm = k48::smem_bytes<C>();
        WIG_CUDA(cudaFuncSetAttribute(k_kin48<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_kin48<C><<<grid, k48::NT, sm, st>>>(W, npy, npx, kin_set<C>(p), sc, d_norm);
        WIG_LAUNCHED("k_kin48");
        return WIG_OK;
    }
#define KCASE(a, b)                                                                      \
    if (NY == a && NX == b) {                                                            \
        constexpr int NT = FusedNT<a, b>::v;                                             \
        auto kern = k_kinetic<C, a, b, NT>;                                              \
        size_t sm = plane_bytes<C, a, b>();                                              \
        WIG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)); \
        kern<<<grid, NT, sm, st>>>(W, npy, npx, kin_set<C>(p), sc, d_norm);              \
        WIG_LAUNCHED("k_kinetic");                                                       \
        return WIG_OK;                                                                   \
    }
    WIG_PLANE_CASES(KCASE)
#undef KCASE
    return WIG_ERR_UNSUPPORTED;
}

// The G-column potential kernel, when G columns fit in shared memory and N_x
// is a multiple of G (G = 4 for complex128, 8 for complex64, halved until the
// CTA fits).  Returns false when it does not apply.
template <class C, int NPY, int NPX, int G>
static bool launch_potential_gn(wig4d_plan* p, C* W, double* partials, cudaStream_t st, double2 sc) {
    if constexpr (G < 2) {
        return false;
    } else {
        typedef PotCfg<C, NPY, NPX, G> P;
        if (G > p->pot_gmax || P::bytes() > 227 * 1024 || p->shape[3] % G != 0)
            return launch_potential_gn<C, NPY, NPX, G / 2>(p, W, partials, st, sc);
        auto kern = k_potential_g<C, NPY, NPX, G>;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P::bytes()) != cudaSuccess)
            return false;
        const unsigned grid = (unsigned)(p->shape[1] * (p->shape[3] / G));
        kern<<<grid, P::NT, P::bytes(), st>>>(W, p->shape[1], p->shape[3], pot_set<C>(p), sc, p->ob, partials);
        return cudaGetLastError() == cudaSuccess;
    }
}
template <class C, int NPY, int NPX>
static bool launch_potential_g(wig4d_plan* p, C* W, double* partials, cudaStream_t st, double2 sc) {
    if (p->pot_gmax < 2) return false;
    constexpr int G0 = sizeof(C) == 16 ? 4 : (NPY * NPX <= 48 * 48 ? 4 : 8);
    return launch_potential_gn<C, NPY, NPX, G0>(p, W, partials, st, sc);
}

template <class C>
static int launch_potential(wig4d_plan* p, C* W, double* partials, cudaStream_t st) {
    const int NPY = p->shape[0], NPX = p->shape[2];
    const int ny = p->shape[1], nx = p->shape[3];
    const unsigned grid = (unsigned)(ny * nx);
    const double2 sc = make_double2(p->pot_scale, 0.0);
#define PCASE(a, b)                                                                      \
    if (NPY == a && NPX == b) {                                                          \
        if (launch_potential_g<C, a, b>(p, W, partials, st, sc)) return WIG_OK;           \
        constexpr int NT = FusedNT<a, b>::v;                                             \
        auto kern = k_potential<C, a, b, NT>;                                            \
        size_t sm = plane_bytes<C, a, b>();                                              \
        if (sm < NPART * (NT / 32) * sizeof(double)) sm = NPART * (NT / 32) * sizeof(double); \
        WIG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)); \
        kern<<<grid, NT, sm, st>>>(W, ny, nx, pot_set<C>(p), sc, p->ob, partials);       \
        WIG_LAUNCHED("k_potential");                                                     \
        return WIG_OK;                                                                   \
    }
    WIG_PLANE_CASES(PCASE)
#undef PCASE
    return WIG_ERR_UNSUPPORTED;
}

static unsigned grid_for(long long n) {
    long long b = (n + 255) / 256, cap = (long long)wig_num_sms() * 16;
    return (unsigned)(b < cap ? (b > 0 ? b : 1) : cap);
}

// Unfused fallback of one half-step: FAFT pair, factor, inverse pair.
template <class C>
static int halfstep_unfused(wig4d_plan* p, C* W, int which, const double* d_norm, cudaStream_t st) {
    const int a0 = which == 0 ? 1 : 0, a1 = which == 0 ? 3 : 2;
    int s;
    if ((s = wig_faft(W, p->shape, p->dtype, a0, p->d[a0], p->delta[a0], 1.0, st))) return s;
    if ((s = wig_faft(W, p->shape, p->dtype, a1, p->d[a1], p->delta[a1], 1.0, st))) return s;
    if (d_norm) {
        if ((s = wig_divide_by_device_scalar(W, p->npts, p->dtype, d_norm, st))) return s;
    }
    const double post = which == 0 ? p->kin_scale : p->pot_scale;
    // kin_scale holds the FAFT 2Nd factors of both directions; the transforms
    // above and below already apply them, so only the wrapper divisors remain.
    double f = post;
    for (int a : {a0, a1}) f /= (2.0 * p->shape[a] * p->d[a]) * (2.0 * p->shape[a] * p->d[a]);
    FactorSet<C>& F = which == 0 ? kin_set<C>(p) : pot_set<C>(p);
    k_apply_factor<C><<<grid_for(p->npts), 256, 0, st>>>(W, p->shape[0], p->shape[1], p->shape[2],
                                                         p->shape[3], F, make_double2(f, 0.0));
    WIG_LAUNCHED("k_apply_factor");
    if ((s = wig_faft(W, p->shape, p->dtype, a0, p->d[a0], -p->delta[a0], 1.0, st))) return s;
    if ((s = wig_faft(W, p->shape, p->dtype, a1, p->d[a1], -p->delta[a1], 1.0, st))) return s;
    return WIG_OK;
}

// Fused general-delta half-step (k_dense_half), N^4 grids with N = 16, 32, 64.
template <class C, bool KIN>
static int launch_dense(wig4d_plan* p, C* W, const double* d_norm, double* partials, cudaStream_t st) {
    const int ar = KIN ? 1 : 0, ac = KIN ? 3 : 2;          // row / column axes of the plane
    const C* Mr = reinterpret_cast<const C*>(p->dmat[ar]);
    const C* Mc = reinterpret_cast<const C*>(p->dmat[ac]);
    const int n = p->dense_n;
    const unsigned grid = (unsigned)(n * n);
    const double2 sc = make_double2(KIN ? p->kin_scale : p->pot_scale, 0.0);
    FactorSet<C>& F = KIN ? kin_set<C>(p) : pot_set<C>(p);
#define DENSE_CASE(N)                                                                                  \
    if (n == N) {                                                                                      \
        auto kern = k_dense_half<C, N, KIN>;                                                           \
        const size_t sm = dense_half_smem_bytes<C, N>(Mr != Mc);                                      \
        WIG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));    \
        kern<<<grid, dense_half::NT, sm, st>>>(W, n, Mr, Mc, p->delta[ar] < 0, p->delta[ac] < 0, F, sc, d_norm, \
                                               p->ob, partials, n);                                    \
        WIG_LAUNCHED("k_dense_half");                                                                  \
        return WIG_OK;                                                                                 \
    }
    DENSE_CASE(16) DENSE_CASE(32) DENSE_CASE(64)
#undef DENSE_CASE
    return WIG_ERR_UNSUPPORTED;
}

template <class C>
static int kinetic_impl(wig4d_plan* p, C* W, const double* d_norm, cudaStream_t st) {
    if (p->fused_kin) return launch_kinetic<C>(p, W, d_norm, st);
    if (p->dense_n) return launch_dense<C, true>(p, W, d_norm, nullptr, st);
    return halfstep_unfused<C>(p, W, 0, d_norm, st);
}

template <class C>
static int potential_impl(wig4d_plan* p, C* W, double* partials, cudaStream_t st) {
    if (p->fused_pot) return launch_potential<C>(p, W, partials, st);
    if (p->dense_n) return launch_dense<C, false>(p, W, nullptr, partials, st);
    int s = halfstep_unfused<C>(p, W, 1, nullptr, st);
    if (s || !partials) return s;
    k_reduce_xp<C, 256><<<p->shape[1] * p->shape[3], 256, 0, st>>>(
        W, p->shape[0], p->shape[1], p->shape[2], p->shape[3], p->ob, partials);
    WIG_LAUNCHED("k_reduce_xp");
    return WIG_OK;
}

static int finalize(wig4d_plan* p, double* out, int* counter, int max_rows, cudaStream_t st,
                    double* raw_out = nullptr) {
    k_finalize<<<1, 1024, 0, st>>>(p->partials, p->shape[1] * p->shape[3], p->shape[3], p->ob,
                                   p->dv_norm, p->dv_obs, out, counter, max_rows, p->cur_norm, p->flag,
                                   raw_out);
    WIG_LAUNCHED("k_finalize");
    return WIG_OK;
}

template <class C>
static int reduce_impl(wig4d_plan* p, const C* W, cudaStream_t st) {
    k_reduce_xp<C, 256><<<p->shape[1] * p->shape[3], 256, 0, st>>>(
        W, p->shape[0], p->shape[1], p->shape[2], p->shape[3], p->ob, p->partials);
    WIG_LAUNCHED("k_reduce_xp");
    return WIG_OK;
}

static void free_plan(wig4d_plan* p) {
    if (!p) return;
    if (p->graph) cudaGraphExecDestroy(p->graph);
    cudaFree(p->tabs);
    cudaFree(p->obs_mem);
    cudaFree(p->partials);
    cudaFree(p->cur_norm);
    cudaFree(p->pingpong);
    cudaFree(p->pv);
    cudaFree(p->tw64);
    cudaFree(p->fold);
    cudaFree(p->tw64d);
    cudaFree(p->tc_bimg[0]);
    cudaFree(p->tc_bimg[1]);
    cudaFree(p->tc_pv);
    delete p;
}

// Tensor maps of a 64^4 complex128 array viewed as 4-D float64 [d3][d2][d1][d0]
// with d0 = 128 (64 complex values): rows of 1 KB, planes of 64 KB.
// cuTensorMapEncodeTiled through the runtime's driver entry point, so that the
// library does not link the driver and still loads where no driver exists.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(f);
    });
    return fn;
}

// 5-D view of a 64^4 complex128 array in the LA / LB layouts of k_r4 (IL = 2):
// (4 float64 = 2 points, f1, f0, c/2, r) with strides 32 B, 2 KB, 128 KB, 4 MB;
// the box is one plane of either half-step.
static int encode_plane_map(CUtensorMap* m, const void* base) {
    const cuuint64_t dims[5] = {4, 64, 64, 32, 64};
    const cuuint64_t strides[4] = {32, 2048, 128 * 1024, 4 * 1024 * 1024};
    const cuuint32_t box[5] = {4, 1, 1, 32, 64};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    EncodeTiledFn enc = encode_tiled_fn();
    if (!enc) {
        snprintf(wig_last_error_buffer(), 256, "cuTensorMapEncodeTiled is not available from the driver");
        return WIG_ERR_CUDA;
    }
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<void*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        snprintf(wig_last_error_buffer(), 256, "cuTensorMapEncodeTiled failed (%d)", (int)r);
        return WIG_ERR_CUDA;
    }
    return WIG_OK;
}

// Destination view of a 64^4 complex128 array in the LA / LB layouts for the
// tensor stores of k_r4ring: (2 float64 = 1 point, f1 % 2, c, r, unit) with
// strides 16 B, 32 B, 2 KB, 128 KB (unit = f0 * 32 + f1 / 2); the box is one
// plane, written into every other 16-byte slot of 64 x 64 sectors.
static int encode_store_map(CUtensorMap* m, const void* base) {
    const cuuint64_t dims[5] = {2, 2, 64, 64, 2048};
    const cuuint64_t strides[4] = {16, 32, 2048, 128 * 1024};
    const cuuint32_t box[5] = {2, 1, 64, 64, 1};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    EncodeTiledFn enc = encode_tiled_fn();
    if (!enc) {
        snprintf(wig_last_error_buffer(), 256, "cuTensorMapEncodeTiled is not available from the driver");
        return WIG_ERR_CUDA;
    }
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<void*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        snprintf(wig_last_error_buffer(), 256, "cuTensorMapEncodeTiled failed (%d)", (int)r);
        return WIG_ERR_CUDA;
    }
    return WIG_OK;
}

// Plane-contiguous layouts of k_r4ring (LK = [y][x][p_y][p_x], LP =
// [p_y][p_x][y][x]): a plane (f0, f1) of either half-step reads point (r, c)
// at ((r * 64 + c) * 64 + f0) * 64 + f1, i.e. (2 float64 = 1 point, f1, f0, c,
// r) with strides 16 B, 1 KB, 64 KB, 4 MB; the box is one plane.
static int encode_plane_map_pc(CUtensorMap* m, const void* base) {
    const cuuint64_t dims[5] = {2, 64, 64, 64, 64};
    const cuuint64_t strides[4] = {16, 1024, 64 * 1024, 4 * 1024 * 1024};
    const cuuint32_t box[5] = {2, 1, 1, 64, 64};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    EncodeTiledFn enc = encode_tiled_fn();
    if (!enc) {
        snprintf(wig_last_error_buffer(), 256, "cuTensorMapEncodeTiled is not available from the driver");
        return WIG_ERR_CUDA;
    }
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<void*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        snprintf(wig_last_error_buffer(), 256, "cuTensorMapEncodeTiled failed (%d)", (int)r);
        return WIG_ERR_CUDA;
    }
    return WIG_OK;
}

// The mixed form's unit boxes on LK / LP (complex64): the two planes f1 = 2m,
// 2m + 1 of one f0 as rows of two points, (4 float32, f1 / 2, f0, c, r) with
// strides 16 B, 512 B, 32 KB, 2 MB; the box is one unit (64 KB).
static int encode_unit_map_mx(CUtensorMap* m, const void* base) {
    const cuuint64_t dims[5] = {4, 32, 64, 64, 64};
    const cuuint64_t strides[4] = {16, 512, 32 * 1024, 2 * 1024 * 1024};
    const cuuint32_t box[5] = {4, 1, 1, 64, 64};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    EncodeTiledFn enc = encode_tiled_fn();
    if (!enc) {
        snprintf(wig_last_error_buffer(), 256, "cuTensorMapEncodeTiled is not available from the driver");
        return WIG_ERR_CUDA;
    }
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, const_cast<void*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        snprintf(wig_last_error_buffer(), 256, "cuTensorMapEncodeTiled failed (%d)", (int)r);
        return WIG_ERR_CUDA;
    }
    return WIG_OK;
}

// LB maps of the caller's state W (the potential half-step's source, the
// kinetic half-step's destination), and its LP map.
static int ensure_w_maps(wig4d_plan* p, const void* W) {
    if (p->map_w_ptr == W) return WIG_OK;
    int s;
    if ((s = encode_plane_map(&p->map_w_load, W))) return s;
    if ((s = encode_store_map(&p->map_w_store, W))) return s;
    if ((s = encode_plane_map_pc(&p->map_w_load_pc, W))) return s;
    p->map_w_ptr = W;
    return WIG_OK;
}

// k_r4ring (complex128): the LA / LK maps and the LA store map of the
// ping-pong buffer (the caller's state gets its maps at the first run).
static int ensure_r4ring(wig4d_plan* p) {
    if (p->r4ring_ready) return WIG_OK;
    int r;
    if ((r = encode_plane_map(&p->map_t_load, p->pingpong))) return r;
    if ((r = encode_store_map(&p->map_t_store, p->pingpong))) return r;
    if ((r = encode_plane_map_pc(&p->map_t_load_pc, p->pingpong))) return r;
    const int sm = (int)r4ring::Cfg<double2>::SMEM;
    WIG_CUDA(cudaFuncSetAttribute(k_r4ring<double2, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    WIG_CUDA(cudaFuncSetAttribute(k_r4ring<double2, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    WIG_CUDA(cudaFuncSetAttribute(k_r4ring<double2, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    WIG_CUDA(cudaFuncSetAttribute(k_r4ring<double2, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    p->r4ring_ready = true;
    return WIG_OK;
}

extern "C" int wig4d_plan_create(const wig4d_desc* desc, wig4d_plan** out) {
    if (!desc || !out) return WIG_ERR_INVALID_ARG;
    *out = nullptr;
    if (desc->dtype != WIG_C128 && desc->dtype != WIG_C64) return WIG_ERR_INVALID_ARG;
    if (desc->transform < 0 || desc->transform > 3) return WIG_ERR_INVALID_ARG;
    for (int a = 0; a < 4; ++a) {
        if (desc->shape[a] < 2 || desc->shape[a] > 1024 || (desc->shape[a] & 1)) return WIG_ERR_UNSUPPORTED;
        if (!desc->coord[a]) return WIG_ERR_INVALID_ARG;
    }
    if (!desc->energy_p || !desc->energy_x) return WIG_ERR_INVALID_ARG;
    if (desc->n_kin < 0 || desc->n_kin > WIG_MAX_FACTORS || desc->n_pot < 0 ||
        desc->n_pot > WIG_MAX_FACTORS)
        return WIG_ERR_INVALID_ARG;
    wig4d_plan* p = new wig4d_plan();
    memset(p, 0, sizeof(*p));
    memcpy(p->shape, desc->shape, sizeof(p->shape));
    p->dtype = desc->dtype;
    memcpy(p->d, desc->d, sizeof(p->d));
    memcpy(p->delta, desc->delta, sizeof(p->delta));
    p->npts = (long long)p->shape[0] * p->shape[1] * p->shape[2] * p->shape[3];
    p->dv_norm = desc->dv_norm;
    p->dv_obs = desc->dv_obs;
    // kernel choices (wig4d_autotune may change them; the variables override
    // the defaults for comparisons in tests)
    p->kin48 = getenv("WIG_NO_K48") == nullptr;
    p->pot_gmax = getenv("WIG_NO_POT_G") ? 1 : 8;
    // total scalar of a fused half-step: (2 N d)^2 per transformed axis (the
    // forward and the inverse FAFT) times the wrapper divisors.
    p->kin_scale = desc->kin_post_scale;
    p->pot_scale = desc->pot_post_scale;
    for (int a : {1, 3}) p->kin_scale *= (2.0 * p->shape[a] * p->d[a]) * (2.0 * p->shape[a] * p->d[a]);
    for (int a : {0, 2}) p->pot_scale *= (2.0 * p->shape[a] * p->d[a]) * (2.0 * p->shape[a] * p->d[a]);
    auto fast_axis = [&](int a) {
        return pow2_16_128(p->shape[a]) && fabs(fabs(p->delta[a]) * p->shape[a] - 1.0) < 1e-12;
    };
    const size_t esz = desc->dtype == WIG_C128 ? 16 : 8;
    const size_t max_smem = 227 * 1024;
    p->fused_kin = fast_axis(1) && fast_axis(3) &&
                   esz * ((size_t)p->shape[1] * (p->shape[3] + 1) + p->shape[1] + p->shape[3]) <= max_smem;
    p->fused_pot = fast_axis(0) && fast_axis(2) &&
                   esz * ((size_t)p->shape[0] * (p->shape[2] + 1) + p->shape[0] + p->shape[2]) <= max_smem;
    auto plane_ok = [](int a, int b) {
        return (a == b && pow2_16_128(a)) || (a == 64 && b == 128) || (a == 128 && b == 64);
    };
    p->fused_kin = p->fused_kin && plane_ok(p->shape[1], p->shape[3]);
    p->fused_pot = p->fused_pot && plane_ok(p->shape[0], p->shape[2]);

    // ---- factor tables: one device allocation ----
    auto tab_elems = [&](const wig_factor& f) -> long long {
        if (f.axis_a < 0) return p->npts;
        if (f.axis_b < 0) return p->shape[f.axis_a];
        return (long long)p->shape[f.axis_a] * p->shape[f.axis_b];
    };
    long long tot = 0;
    for (int i = 0; i < desc->n_kin; ++i) tot += tab_elems(desc->kin[i]);
    for (int i = 0; i < desc->n_pot; ++i) tot += tab_elems(desc->pot[i]);
    for (int i = 0; i < desc->n_kin; ++i) if (!desc->kin[i].host_data) { delete p; return WIG_ERR_INVALID_ARG; }
    for (int i = 0; i < desc->n_pot; ++i) if (!desc->pot[i].host_data) { delete p; return WIG_ERR_INVALID_ARG; }
    p->tab_bytes = tot * (long long)esz;
    if (tot > 0 && cudaMalloc(&p->tabs, (size_t)p->tab_bytes) != cudaSuccess) { free_plan(p); return WIG_ERR_ALLOC; }
    long long off = 0;
    auto upload = [&](const wig_factor& f, const void** dst, int* ia, int* ib, int* nb) -> int {
        const long long n = tab_elems(f);
        char* base = reinterpret_cast<char*>(p->tabs) + off * esz;
        if (desc->dtype == WIG_C128) {
            if (cudaMemcpy(base, f.host_data, n * 16, cudaMemcpyHostToDevice) != cudaSuccess) return WIG_ERR_CUDA;
        } else {
            std::vector<float> tmp(2 * n);
            for (long long i = 0; i < 2 * n; ++i) tmp[i] = (float)f.host_data[i];
            if (cudaMemcpy(base, tmp.data(), n * 8, cudaMemcpyHostToDevice) != cudaSuccess) return WIG_ERR_CUDA;
        }
        *dst = base;
        *ia = f.axis_a;
        *ib = f.axis_b;
        *nb = f.axis_b >= 0 ? p->shape[f.axis_b] : 1;
        off += n;
        return WIG_OK;
    };
    p->kin_d.n = p->kin_f.n = desc->n_kin;
    p->pot_d.n = p->pot_f.n = desc->n_pot;
    for (int i = 0; i < desc->n_kin; ++i) {
        const void* dp;
        int r = upload(desc->kin[i], &dp, &p->kin_d.ia[i], &p->kin_d.ib[i], &p->kin_d.nb[i]);
        if (r) { free_plan(p); return r; }
        p->kin_d.data[i] = (const double2*)dp; p->kin_f.data[i] = (const float2*)dp;
        p->kin_f.ia[i] = p->kin_d.ia[i]; p->kin_f.ib[i] = p->kin_d.ib[i]; p->kin_f.nb[i] = p->kin_d.nb[i];
    }
    for (int i = 0; i < desc->n_pot; ++i) {
        const void* dp;
        int r = upload(desc->pot[i], &dp, &p->pot_d.ia[i], &p->pot_d.ib[i], &p->pot_d.nb[i]);
        if (r) { free_plan(p); return r; }
        p->pot_d.data[i] = (const double2*)dp; p->pot_f.data[i] = (const float2*)dp;
        p->pot_f.ia[i] = p->pot_d.ia[i]; p->pot_f.ib[i] = p->pot_d.ib[i]; p->pot_f.nb[i] = p->pot_d.nb[i];
    }
    // ---- observable tables ----
    const int N0 = p->shape[0], N1 = p->shape[1], N2 = p->shape[2], N3 = p->shape[3];
    const long long nobs = N0 + N1 + N2 + N3 + (long long)N0 * N2 + (long long)N1 * N3;
    if (cudaMalloc(&p->obs_mem, nobs * sizeof(double)) != cudaSuccess) { free_plan(p); return WIG_ERR_ALLOC; }
    double* q = p->obs_mem;
    p->ob.cpy = q; cudaMemcpy(q, desc->coord[0], N0 * 8, cudaMemcpyHostToDevice); q += N0;
    p->ob.cy = q;  cudaMemcpy(q, desc->coord[1], N1 * 8, cudaMemcpyHostToDevice); q += N1;
    p->ob.cpx = q; cudaMemcpy(q, desc->coord[2], N2 * 8, cudaMemcpyHostToDevice); q += N2;
    p->ob.cx = q;  cudaMemcpy(q, desc->coord[3], N3 * 8, cudaMemcpyHostToDevice); q += N3;
    p->ob.ep = q;  cudaMemcpy(q, desc->energy_p, (size_t)N0 * N2 * 8, cudaMemcpyHostToDevice); q += (long long)N0 * N2;
    p->ob.ex = q;  cudaMemcpy(q, desc->energy_x, (size_t)N1 * N3 * 8, cudaMemcpyHostToDevice);
    // ---- reduction scratch: partials, current norm, row counter, flag ----
    const size_t npart = (size_t)N1 * N3 * NPART;
    if (cudaMalloc(&p->partials, npart * sizeof(double)) != cudaSuccess) { free_plan(p); return WIG_ERR_ALLOC; }
    if (cudaMalloc(&p->cur_norm, 4 * sizeof(double)) != cudaSuccess) { free_plan(p); return WIG_ERR_ALLOC; }
    p->counter = reinterpret_cast<int*>(p->cur_norm + 2);
    p->flag = p->counter + 1;
    cudaMemset(p->cur_norm, 0, 4 * sizeof(double));
    // dense matrices for the unfused general-delta path are created now, so
    // that no allocation happens during graph capture
    for (int a = 0; a < 4; ++a) {
        const bool fast = pow2_16_128(p->shape[a]) && fabs(fabs(p->delta[a]) * p->shape[a] - 1.0) < 1e-12;
        if (!fast && !wig_dense_matrix(p->shape[a], fabs(p->delta[a]), p->dtype, 0)) { free_plan(p); return WIG_ERR_ALLOC; }
    }
    // general delta on an N^4 grid (N = 16, 32, 64): both half-steps fused
    // (k_dense_half) when neither is on the radix path
    {
        const int n = p->shape[0];
        const bool square = p->shape[1] == n && p->shape[2] == n && p->shape[3] == n;
        if (square && (n == 16 || n == 32 || n == 64) && !p->fused_kin && !p->fused_pot &&
            getenv("WIG_NO_DENSE_FUSED") == nullptr) {
            bool ok = true;
            for (int a = 0; a < 4; ++a) {
                p->dmat[a] = wig_dense_matrix(n, fabs(p->delta[a]), p->dtype, 0);
                ok = ok && p->dmat[a];
            }
            if (!ok) { free_plan(p); return WIG_ERR_ALLOC; }
            p->dense_n = n;
        }
    }
    // the 64^4 kernels take the factor as per-plane outer products: no full
    // 4-D table and no table over both in-plane axes of a half-step
    auto separable = [](const wig_factor* f, int n, int ay, int ax) {
        for (int i = 0; i < n; ++i) {
            if (f[i].axis_a < 0) return false;
            const bool ina = f[i].axis_a == ay || f[i].axis_a == ax;
            const bool inb = f[i].axis_b >= 0 && (f[i].axis_b == ay || f[i].axis_b == ax);
            if (ina && inb) return false;
        }
        return true;
    };
    p->fast64 = p->fused_kin && p->fused_pot && p->shape[0] == 64 && p->shape[1] == 64 &&
                p->shape[2] == 64 && p->shape[3] == 64 && separable(desc->kin, desc->n_kin, 1, 3) &&
                separable(desc->pot, desc->n_pot, 0, 2) && getenv("WIG_NO_FAST64") == nullptr;
    if (p->fast64) {
        // k_r4 on the LA / LB layouts: a ping-pong buffer, FP64 per-plane
        // factor vectors (from FP64 copies of the host tables for a
        // complex64 plan, which keeps only float32 tables), the twiddles
        if (cudaMalloc(&p->pingpong, (size_t)p->npts * esz) != cudaSuccess) { free_plan(p); return WIG_ERR_ALLOC; }
        const int npl_k = p->shape[0] * p->shape[2], npl_p = p->shape[1] * p->shape[3];
        if (cudaMalloc(&p->pv, (size_t)(npl_k + npl_p) * 128 * sizeof(double2)) != cudaSuccess) {
            free_plan(p); return WIG_ERR_ALLOC;
        }
        double2* pv = (double2*)p->pv;
        if (desc->dtype == WIG_C128) {
            k_plane_vectors<double2><<<(npl_k * 128 + 255) / 256, 256>>>(p->kin_d, 1, 3, 0, 2, p->shape[2], npl_k, pv, 32);
            k_plane_vectors<double2><<<(npl_p * 128 + 255) / 256, 256>>>(p->pot_d, 0, 2, 1, 3, p->shape[3], npl_p,
                                                                        pv + (size_t)npl_k * 128, 32);
        } else {
            long long n64 = 0;
            for (int i = 0; i < desc->n_kin; ++i) n64 += tab_elems(desc->kin[i]);
            for (int i = 0; i < desc->n_pot; ++i) n64 += tab_elems(desc->pot[i]);
            double2* t64 = nullptr;
            if (n64 > 0 && cudaMalloc(&t64, (size_t)n64 * sizeof(double2)) != cudaSuccess) {
                free_plan(p); return WIG_ERR_ALLOC;
            }
            FactorSet<double2> k64 = p->kin_d, p64 = p->pot_d;
            long long o64 = 0;
            bool ok = true;
            for (int i = 0; i < desc->n_kin; ++i) {
                const long long n = tab_elems(desc->kin[i]);
                ok = ok && cudaMemcpy(t64 + o64, desc->kin[i].host_data, n * 16, cudaMemcpyHostToDevice) == cudaSuccess;
                k64.data[i] = t64 + o64; o64 += n;
            }
            for (int i = 0; i < desc->n_pot; ++i) {
                const long long n = tab_elems(desc->pot[i]);
                ok = ok && cudaMemcpy(t64 + o64, desc->pot[i].host_data, n * 16, cudaMemcpyHostToDevice) == cudaSuccess;
                p64.data[i] = t64 + o64; o64 += n;
            }
            if (ok) {
                k_plane_vectors<double2><<<(npl_k * 128 + 255) / 256, 256>>>(k64, 1, 3, 0, 2, p->shape[2], npl_k, pv, 32);
                k_plane_vectors<double2><<<(npl_p * 128 + 255) / 256, 256>>>(p64, 0, 2, 1, 3, p->shape[3], npl_p,
                                                                            pv + (size_t)npl_k * 128, 32);
                ok = cudaDeviceSynchronize() == cudaSuccess;
            }
            cudaFree(t64);
            if (!ok) { wig_set_cuda_error(cudaGetLastError(), "plane vectors"); free_plan(p); return WIG_ERR_CUDA; }
        }
        // complex128: k_r4ring on the plane-contiguous layouts (default);
        // complex64: k_r4 with cluster stores.  WIG_FAST64_KERNEL overrides: r4
        // (k_r4, plain stores), r4cluster (k_r4, cluster stores), and for
        // complex128 r4ring_ts (the ring on LA / LB, TMA tensor stores), r4ring_pc
        const char* env_kern = getenv("WIG_FAST64_KERNEL");
        const char* kern = env_kern ? env_kern : (desc->dtype == WIG_C128 ? "r4ring_pc" : "r4cluster");
        p->r4 = true;
        if (desc->dtype == WIG_C128 && (strcmp(kern, "r4ring_ts") == 0 || strcmp(kern, "r4ring_pc") == 0)) {
            int r;
            if ((r = ensure_r4ring(p))) { free_plan(p); return r; }
            p->r4ring = true;
            p->r4ring_pc = strcmp(kern, "r4ring_pc") == 0;
        }
        p->r4_cluster = strcmp(kern, "r4") != 0;
        if (desc->dtype == WIG_C64 && strcmp(kern, "r4ring_f32") == 0) {
            int r;
            if ((r = encode_unit_map_mx(&p->map_t_load_mx, p->pingpong))) { free_plan(p); return r; }
            cudaFuncSetAttribute(k_r4ring_mx<float2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)r4mx::SMEM);
            cudaFuncSetAttribute(k_r4ring_mx<float2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)r4mx::SMEM);
            p->mx_ring = true;
            p->mx_f32 = true;
        }
        if (cudaMalloc(&p->tw64, 64 * esz) != cudaSuccess) { free_plan(p); return WIG_ERR_ALLOC; }
        if (cudaMalloc(&p->fold, FOLD_BLOCKS * NSUM * sizeof(double)) != cudaSuccess) { free_plan(p); return WIG_ERR_ALLOC; }
        if (desc->dtype == WIG_C128) k_make_r4_twiddles<double2><<<1, 64>>>((double2*)p->tw64);
        else k_make_r4_twiddles<float2><<<1, 64>>>((float2*)p->tw64);
        const int rsm = (int)(desc->dtype == WIG_C128 ? r4_smem_bytes<double2>() : r4_smem_bytes<float2>());
        if (desc->dtype == WIG_C128) {
            cudaFuncSetAttribute(k_r4<double2, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm);
            cudaFuncSetAttribute(k_r4<double2, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm);
            cudaFuncSetAttribute(k_r4<double2, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm);
            cudaFuncSetAttribute(k_r4<double2, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm);
        } else {
            cudaFuncSetAttribute(k_r4<float2, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm);
            cudaFuncSetAttribute(k_r4<float2, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm);
            cudaFuncSetAttribute(k_r4<float2, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm);
            cudaFuncSetAttribute(k_r4<float2, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm);
        }
    }
    // tensor-core transforms (k_tc64): complex64 64^4, separable factors,
    // positive deltas, the same |delta| on both in-plane axes of each half-step
    if (desc->transform == 1 || desc->transform == 2) {
        const bool ok64 = desc->dtype == WIG_C64 && p->shape[0] == 64 && p->shape[1] == 64 && p->shape[2] == 64 &&
                          p->shape[3] == 64;
        bool ok = ok64 && separable(desc->kin, desc->n_kin, 1, 3) && separable(desc->pot, desc->n_pot, 0, 2);
        for (int a = 0; a < 4; ++a) ok = ok && p->delta[a] > 0;
        ok = ok && fabs(p->delta[1] - p->delta[3]) <= 1e-12 * p->delta[1] &&
             fabs(p->delta[0] - p->delta[2]) <= 1e-12 * p->delta[0];
        if (!ok) { free_plan(p); return WIG_ERR_UNSUPPORTED; }
        int s;
        if ((s = build_tc_bimg(p->delta[1], &p->tc_bimg[0])) || (s = build_tc_bimg(p->delta[0], &p->tc_bimg[1]))) {
            free_plan(p); return s;
        }
        const int npl_k = 64 * 64, npl_p = 64 * 64;
        if (!p->pingpong && cudaMalloc(&p->pingpong, (size_t)p->npts * esz) != cudaSuccess) { free_plan(p); return WIG_ERR_ALLOC; }
        if (!p->fold && cudaMalloc(&p->fold, FOLD_BLOCKS * NSUM * sizeof(double)) != cudaSuccess) { free_plan(p); return WIG_ERR_ALLOC; }
        if (cudaMalloc(&p->tc_pv, (size_t)(npl_k + npl_p) * 128 * sizeof(double2)) != cudaSuccess) {
            free_plan(p); return WIG_ERR_ALLOC;
        }
        // FP64 plane vectors from FP64 copies of the host tables (the plan
        // itself keeps the float32 tables of a complex64 state)
        long long n64 = 0;
        for (int i = 0; i < desc->n_kin; ++i) n64 += tab_elems(desc->kin[i]);
        for (int i = 0; i < desc->n_pot; ++i) n64 += tab_elems(desc->pot[i]);
        double2* t64 = nullptr;
        if (n64 > 0 && cudaMalloc(&t64, (size_t)n64 * sizeof(double2)) != cudaSuccess) { free_plan(p); return WIG_ERR_ALLOC; }
        FactorSet<double2> k64 = p->kin_d, p64 = p->pot_d;
        long long o64 = 0;
        bool up = true;
        for (int i = 0; i < desc->n_kin; ++i) {
            const long long n = tab_elems(desc->kin[i]);
            up = up && cudaMemcpy(t64 + o64, desc->kin[i].host_data, n * 16, cudaMemcpyHostToDevice) == cudaSuccess;
            k64.data[i] = t64 + o64; o64 += n;
        }
        for (int i = 0; i < desc->n_pot; ++i) {
            const long long n = tab_elems(desc->pot[i]);
            up = up && cudaMemcpy(t64 + o64, desc->pot[i].host_data, n * 16, cudaMemcpyHostToDevice) == cudaSuccess;
            p64.data[i] = t64 + o64; o64 += n;
        }
        double2* pv = (double2*)p->tc_pv;
        if (up) {
            k_plane_vectors<double2><<<(npl_k * 128 + 255) / 256, 256>>>(k64, 1, 3, 0, 2, 64, npl_k, pv, 0);
            k_plane_vectors<double2><<<(npl_p * 128 + 255) / 256, 256>>>(p64, 0, 2, 1, 3, 64, npl_p,
                                                                        pv + (size_t)npl_k * 128, 0);
            up = cudaDeviceSynchronize() == cudaSuccess;
        }
        cudaFree(t64);
        if (!up) { wig_set_cuda_error(cudaGetLastError(), "tc plane vectors"); free_plan(p); return WIG_ERR_CUDA; }
        if (cudaFuncSetAttribute(k_tc64<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc64::SMEM) != cudaSuccess ||
            cudaFuncSetAttribute(k_tc64<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc64::SMEM) != cudaSuccess) {
            wig_set_cuda_error(cudaGetLastError(), "k_tc64 attributes"); free_plan(p); return WIG_ERR_CUDA;
        }
        p->tc = desc->transform == 1;
        p->tc_ready = true;
    }
    // mixed form: complex64 state, FP64 transforms and factors (k_r4<double2, ., ., float2>)
    if (desc->transform == 3) {
        if (desc->dtype != WIG_C64 || !p->r4) { free_plan(p); return WIG_ERR_UNSUPPORTED; }
        if (cudaMalloc(&p->tw64d, 64 * sizeof(double2)) != cudaSuccess) { free_plan(p); return WIG_ERR_ALLOC; }
        k_make_r4_twiddles<double2><<<1, 64>>>((double2*)p->tw64d);
        const int rsm = (int)r4_smem_bytes<double2>();
        cudaFuncSetAttribute(k_r4<double2, true, false, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm);
        cudaFuncSetAttribute(k_r4<double2, false, false, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm);
        cudaFuncSetAttribute(k_r4<double2, true, true, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm);
        cudaFuncSetAttribute(k_r4<double2, false, true, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm);
        p->r4_mixed = true;
        // k_r4ring_mx by default; WIG_MIXED_KERNEL=r4 keeps k_r4<double2, ., ., float2>
        const char* mk = getenv("WIG_MIXED_KERNEL");
        if (!(mk && strcmp(mk, "r4") == 0)) {
            int r;
            if ((r = encode_unit_map_mx(&p->map_t_load_mx, p->pingpong))) { free_plan(p); return r; }
            cudaFuncSetAttribute(k_r4ring_mx<double2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)r4mx::SMEM);
            cudaFuncSetAttribute(k_r4ring_mx<double2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)r4mx::SMEM);
            p->mx_ring = true;
        }
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { wig_set_cuda_error(e, "wig4d_plan_create"); free_plan(p); return WIG_ERR_CUDA; }
    *out = p;
    return WIG_OK;
}

extern "C" int wig4d_plan_destroy(wig4d_plan* p) {
    if (!p) return WIG_ERR_INVALID_ARG;
    cudaDeviceSynchronize();
    free_plan(p);
    return WIG_OK;
}

extern "C" int wig4d_plan_info(const wig4d_plan* p, int info[4]) {
    if (!p || !info) return WIG_ERR_INVALID_ARG;
    info[0] = p->fused_kin; info[1] = p->fused_pot; info[2] = p->fast64;
    info[3] = p->tc ? 6 : (!p->fast64 ? 0 : (p->r4_mixed ? (p->mx_ring ? 11 : 7) : p->mx_f32 ? 12 : (p->r4ring ? (p->r4ring_pc ? 10 : 9) : 3)));
    return WIG_OK;
}

// ---- 64 x 64 component-plane transforms for the Wigner-Dirac plan ----------
// (dirac.cu calls these; the kernels share the k_r4 machinery in r4.cuh)
int wig_r4_twiddles(void* tw, int dtype, cudaStream_t st) {
    if (dtype == WIG_C128) k_make_r4_twiddles<double2><<<1, 64, 0, st>>>((double2*)tw);
    else k_make_r4_twiddles<float2><<<1, 64, 0, st>>>((float2*)tw);
    WIG_LAUNCHED("k_make_r4_twiddles");
    return WIG_OK;
}

template <class C, int KIND, bool FWD>
static int launch_dplane_r4(void* const* slots, int nslots, const void* tw, double scale, const double* d_norm,
                            cudaStream_t st) {
    PlaneSlots<C> S;
    for (int k = 0; k < 16; ++k) S.p[k] = k < nslots ? (C*)slots[k] : nullptr;
    auto kern = k_dplane_r4<C, KIND, FWD>;
    const size_t sm = sizeof(C) * (64 * 64 + 64);
    WIG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    kern<<<dim3(64 * 64, nslots), r4::NT, sm, st>>>(S, (const C*)tw, make_double2(scale, 0.0), d_norm);
    WIG_LAUNCHED("k_dplane_r4");
    return WIG_OK;
}

// 4-D view of one 64^4 component for k_dplane_r4t:
// (2 * 64 reals, i2, i1, i0); box (reals, 64, 1, rows) = (2 GP reals = 16
// bytes, 64, 1, 64).
template <class C>
static int encode_dplane_map(CUtensorMap* m, const void* base, int reals, int rows) {
    constexpr cuuint64_t E = sizeof(C);
    const cuuint64_t dims[4] = {128, 64, 64, 64};
    const cuuint64_t strides[3] = {64 * E, 64 * 64 * E, 64 * 64 * 64 * E};
    const cuuint32_t box[4] = {(cuuint32_t)reals, 64, 1, (cuuint32_t)rows};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    EncodeTiledFn enc = encode_tiled_fn();
    if (!enc) {
        snprintf(wig_last_error_buffer(), 256, "cuTensorMapEncodeTiled is not available from the driver");
        return WIG_ERR_CUDA;
    }
    const CUresult r = enc(m, E == 16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                           const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        snprintf(wig_last_error_buffer(), 256, "cuTensorMapEncodeTiled failed (%d)", (int)r);
        return WIG_ERR_CUDA;
    }
    return WIG_OK;
}

template <class C, bool FWD>
static int launch_dplane_r4t(void* const* slots, int nslots, const void* tw, double scale, const double* d_norm,
                             cudaStream_t st, const DEpi* epi = nullptr) {
    PlaneMaps<C> maps;
    PlaneSlots<C> S;
    memset(&maps, 0, sizeof(maps));
    for (int k = 0; k < 16; ++k) S.p[k] = k < nslots ? (C*)slots[k] : nullptr;
    for (int k = 0; k < nslots; ++k) {
        int r;
        if ((r = encode_dplane_map<C>(&maps.m[k], slots[k], 2 * dplane_gp<C>(), 64))) return r;
    }
    constexpr int GP = dplane_gp<C>();
    const size_t sm = dplane_r4t_smem_bytes<C>();
    if constexpr (!FWD) {
        if (epi) {
            if (nslots != 16) return WIG_ERR_INVALID_ARG;
            auto kern = k_dplane_r4t<C, FWD, true>;
            WIG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            kern<<<dim3(64 * 64 / GP, nslots), r4::NT * GP, sm, st>>>(maps, S, (const C*)tw,
                                                                      make_double2(scale, 0.0), d_norm, *epi);
            WIG_LAUNCHED("k_dplane_r4t<epi>");
            return WIG_OK;
        }
    }
    if (epi) return WIG_ERR_INVALID_ARG;
    auto kern = k_dplane_r4t<C, FWD, false>;
    WIG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    DEpi none;
    memset(&none, 0, sizeof(none));
    kern<<<dim3(64 * 64 / GP, nslots), r4::NT * GP, sm, st>>>(maps, S, (const C*)tw, make_double2(scale, 0.0),
                                                              d_norm, none);
    WIG_LAUNCHED("k_dplane_r4t");
    return WIG_OK;
}

// kind 0: axes (1, 3), kind 1: axes (0, 2) of a 64^4 component; fwd: exp(-i ...)
// epi (Theta -> P, kind 1, fwd 0, all 16 slots): fuse the next iteration's
// boundary_xp, Real and sums into the transform (k_dplane_r4t<EPI>)
int wig_dplane64(void* const* slots, int nslots, int dtype, int kind, int fwd, double scale, const double* d_norm,
                 const void* tw, cudaStream_t st, const DEpi* epi) {
    if (nslots < 1 || nslots > 16 || !tw) return WIG_ERR_INVALID_ARG;
    for (int k = 0; k < nslots; ++k)
        if (!slots[k] || (reinterpret_cast<uintptr_t>(slots[k]) & 15)) return WIG_ERR_INVALID_ARG;
    if (epi && (kind != 1 || fwd || getenv("WIG_NO_DPLANE_TMA"))) return WIG_ERR_UNSUPPORTED;
    if (kind == 1 && !getenv("WIG_NO_DPLANE_TMA")) {
        if (dtype == WIG_C128) return fwd ? launch_dplane_r4t<double2, true>(slots, nslots, tw, scale, d_norm, st)
                                          : launch_dplane_r4t<double2, false>(slots, nslots, tw, scale, d_norm, st, epi);
        return fwd ? launch_dplane_r4t<float2, true>(slots, nslots, tw, scale, d_norm, st)
                   : launch_dplane_r4t<float2, false>(slots, nslots, tw, scale, d_norm, st, epi);
    }
    if (dtype == WIG_C128) {
        if (kind == 0) return fwd ? launch_dplane_r4<double2, 0, true>(slots, nslots, tw, scale, d_norm, st)
                                  : launch_dplane_r4<double2, 0, false>(slots, nslots, tw, scale, d_norm, st);
        return fwd ? launch_dplane_r4<double2, 1, true>(slots, nslots, tw, scale, d_norm, st)
                   : launch_dplane_r4<double2, 1, false>(slots, nslots, tw, scale, d_norm, st);
    }
    if (kind == 0) return fwd ? launch_dplane_r4<float2, 0, true>(slots, nslots, tw, scale, d_norm, st)
                              : launch_dplane_r4<float2, 0, false>(slots, nslots, tw, scale, d_norm, st);
    return fwd ? launch_dplane_r4<float2, 1, true>(slots, nslots, tw, scale, d_norm, st)
               : launch_dplane_r4<float2, 1, false>(slots, nslots, tw, scale, d_norm, st);
}

extern "C" long long wig4d_plan_device_bytes(const wig4d_plan* p) {
    if (!p) return -1;
    const long long N0 = p->shape[0], N1 = p->shape[1], N2 = p->shape[2], N3 = p->shape[3];
    const long long esz = p->dtype == WIG_C128 ? 16 : 8;
    return p->tab_bytes + 8 * (N0 + N1 + N2 + N3 + N0 * N2 + N1 * N3) + 8LL * N1 * N3 * NPART + 32 +
           (p->pingpong ? p->npts * esz : 0);
}

extern "C" int wig4d_kinetic(wig4d_plan* p, void* W, const double* d_norm, void* stream) {
    if (!p || !W) return WIG_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    return p->dtype == WIG_C128 ? kinetic_impl<double2>(p, (double2*)W, d_norm, st)
                                : kinetic_impl<float2>(p, (float2*)W, d_norm, st);
}

extern "C" int wig4d_potential(wig4d_plan* p, void* W, void* stream) {
    if (!p || !W) return WIG_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    return p->dtype == WIG_C128 ? potential_impl<double2>(p, (double2*)W, nullptr, st)
                                : potential_impl<float2>(p, (float2*)W, nullptr, st);
}

extern "C" int wig4d_apply_factor(wig4d_plan* p, void* W, int which, void* stream) {
    if (!p || !W || (which != 0 && which != 1)) return WIG_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    // the factor alone, without the FAFT 2Nd factors or wrapper divisors
    const double2 one = make_double2(1.0, 0.0);
    if (p->dtype == WIG_C128) {
        k_apply_factor<double2><<<grid_for(p->npts), 256, 0, st>>>((double2*)W, p->shape[0], p->shape[1],
            p->shape[2], p->shape[3], which == 0 ? p->kin_d : p->pot_d, one);
    } else {
        k_apply_factor<float2><<<grid_for(p->npts), 256, 0, st>>>((float2*)W, p->shape[0], p->shape[1],
            p->shape[2], p->shape[3], which == 0 ? p->kin_f : p->pot_f, one);
    }
    WIG_LAUNCHED("k_apply_factor");
    return WIG_OK;
}

extern "C" int wig4d_reduce(wig4d_plan* p, const void* W, double* d_out, void* stream) {
    if (!p || !W || !d_out) return WIG_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    int s = p->dtype == WIG_C128 ? reduce_impl<double2>(p, (const double2*)W, st)
                                 : reduce_impl<float2>(p, (const float2*)W, st);
    if (s) return s;
    return finalize(p, d_out, nullptr, 0, st, d_out + WIG4D_NOBS);
}

// ---------------------------------------------------------------------------
// Observables without any device allocation.
//
// Some callers cannot allocate device memory: code running where cudaMalloc
// is not allowed or not wanted (an application with its own fixed memory
// pool or a memory budget that forbids the library from growing its
// footprint, or a host that only hands out pre-registered buffers).  They
// also cannot create a plan, since wig4d_plan_create allocates its tables.
// wig4d_observables_noalloc computes what wig4d_reduce computes from tables
// the caller already holds on the device, and keeps its per-column partial
// sums in the fixed array below instead of plan memory.
//
// The array is part of the library image: every GPU that loads the library
// holds it (WIG4D_NOALLOC_MAX_COLUMNS * NPART doubles, 1.5 MiB) until the
// process exits.  All calls share it, so two calls whose kernels overlap on
// the GPU (different streams, or different host threads on one device) race
// on it; calls on one stream are ordered and safe.  Every partial a call
// reads is first written by the same call, so nothing needs clearing.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_noalloc_partials[(size_t)WIG4D_NOALLOC_MAX_COLUMNS * NPART];

// Device address of g_noalloc_partials, looked up once per device with the
// device current (in host code the symbol is only a stand-in, not an address).
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
static CtxGetCurrentFn ctx_get_current_fn() {
    static CtxGetCurrentFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(f);
    });
    return fn;
}

// The array's device address for the current device, looked up at the first
// call on that device and again whenever the device's current context is not
// the one of the cached address (after a device reset the old address would
// point into freed memory).
static double* noalloc_scratch(int* status) {
    static std::mutex mu;
    static double* addr[64] = {nullptr};
    static CUcontext ctxs[64] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { wig_set_cuda_error(e, "cudaGetDevice"); *status = WIG_ERR_CUDA; return nullptr; }
    if (dev < 0 || dev >= 64) { *status = WIG_ERR_UNSUPPORTED; return nullptr; }
    CUcontext ctx = nullptr;
    const CtxGetCurrentFn get_ctx = ctx_get_current_fn();
    if (get_ctx) get_ctx(&ctx);
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev] || ctxs[dev] != ctx || !get_ctx) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_partials);
        if (e != cudaSuccess || !ptr) {
            wig_set_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_partials)");
            *status = WIG_ERR_CUDA;
            return nullptr;
        }
        addr[dev] = static_cast<double*>(ptr);
        ctxs[dev] = ctx;
    }
    *status = WIG_OK;
    return addr[dev];
}

extern "C" int wig4d_observables_noalloc(const void* W, const int shape[4], int dtype,
                                         const double* d_coord_py, const double* d_coord_y,
                                         const double* d_coord_px, const double* d_coord_x,
                                         const double* d_energy_p, const double* d_energy_x,
                                         double dv_norm, double dv_obs, double* d_out, void* stream) {
    if (!W || !shape || !d_coord_py || !d_coord_y || !d_coord_px || !d_coord_x || !d_energy_p ||
        !d_energy_x || !d_out)
        return WIG_ERR_INVALID_ARG;
    if (dtype != WIG_C128 && dtype != WIG_C64) return WIG_ERR_INVALID_ARG;
    for (int a = 0; a < 4; ++a)
        if (shape[a] < 1) return WIG_ERR_INVALID_ARG;
    const long long columns = (long long)shape[1] * shape[3];
    if (columns > WIG4D_NOALLOC_MAX_COLUMNS) {
        snprintf(wig_last_error_buffer(), 256,
                 "wig4d_observables_noalloc: N_y * N_x = %lld is above the fixed limit %d", columns,
                 WIG4D_NOALLOC_MAX_COLUMNS);
        return WIG_ERR_TOO_LARGE;
    }
    int status = WIG_OK;
    double* partials = noalloc_scratch(&status);
    if (!partials) return status;
    ObsTabs ob;
    ob.cpy = d_coord_py; ob.cy = d_coord_y; ob.cpx = d_coord_px; ob.cx = d_coord_x;
    ob.ep = d_energy_p; ob.ex = d_energy_x;
    cudaStream_t st = as_stream(stream);
    if (dtype == WIG_C128)
        k_reduce_xp<double2, 256><<<(unsigned)columns, 256, 0, st>>>((const double2*)W, shape[0], shape[1],
                                                                    shape[2], shape[3], ob, partials);
    else
        k_reduce_xp<float2, 256><<<(unsigned)columns, 256, 0, st>>>((const float2*)W, shape[0], shape[1],
                                                                   shape[2], shape[3], ob, partials);
    WIG_LAUNCHED("k_reduce_xp (noalloc)");
    k_finalize<<<1, 1024, 0, st>>>(partials, (int)columns, shape[3], ob, dv_norm, dv_obs, d_out, nullptr, 0,
                                   nullptr, nullptr, d_out + WIG4D_NOBS);
    WIG_LAUNCHED("k_finalize (noalloc)");
    return WIG_OK;
}

// One Run() iteration in three parts: kinetic (dividing by the current norm),
// potential with the partial sums of the new state, finalize into the history.
// Run() reduction of k_r4's per-column partial rows: fold into FOLD_BLOCKS
// rows, then k_finalize_sums (norm, observables row, current norm, counter).
static int fold_and_finalize(wig4d_plan* p, double* hist, int rows, cudaStream_t st) {
    const int ncols = p->shape[1] * p->shape[3];
    const int per = (ncols + FOLD_BLOCKS - 1) / FOLD_BLOCKS;
    k_fold_columns<<<FOLD_BLOCKS, 256, 0, st>>>(p->partials, ncols, p->shape[3], per, p->ob, p->fold);
    WIG_LAUNCHED("k_fold_columns");
    k_finalize_sums<<<1, 32 * NSUM, 0, st>>>(p->fold, FOLD_BLOCKS, p->dv_norm, p->dv_obs, hist, p->counter, rows,
                                             p->cur_norm, p->flag);
    WIG_LAUNCHED("k_finalize_sums");
    return WIG_OK;
}

// k_r4 launch: with clusters of IL CTAs (full-sector stores) or plain.
template <class C, bool KIN, class S = C>
static cudaError_t launch_r4(bool cluster, unsigned grid, size_t sm, cudaStream_t st, const S* src, S* dst,
                             const double2* pv, const C* tw, double2 scale, const double* d_norm, ObsTabs ob,
                             double* partials) {
    if (!cluster) {
        k_r4<C, KIN, false, S><<<grid, r4::NT, sm, st>>>(src, dst, pv, tw, scale, d_norm, ob, partials);
        return cudaGetLastError();
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(r4::NT);
    cfg.dynamicSmemBytes = sm;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = r4::Il<S>::v;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_r4<C, KIN, true, S>, src, dst, pv, tw, scale, d_norm, ob, partials);
}

template <class C>
static int iteration_part(wig4d_plan* p, C* W, double* hist, int rows, cudaStream_t st, int part) {
    if constexpr (std::is_same<C, float2>::value) {
        if (p->tc) {
            // W holds LP, the ping-pong buffer LK (converted around the loop)
            float2* P = reinterpret_cast<float2*>(p->pingpong);
            const double2* pv = reinterpret_cast<const double2*>(p->tc_pv);
            const unsigned grid = (unsigned)(wig_num_sms() < 1024 ? wig_num_sms() : 1024);
            if (part == 0) {
                k_tc64<true><<<grid, tc64::NT, tc64::SMEM, st>>>(P, W, pv, (const uint4*)p->tc_bimg[0],
                                                                 make_double2(p->kin_scale, 0.0), p->cur_norm, p->ob,
                                                                 nullptr, p->flag);
                WIG_LAUNCHED("k_tc64<kin>");
            } else if (part == 1) {
                k_tc64<false><<<grid, tc64::NT, tc64::SMEM, st>>>(W, P, pv + (size_t)p->shape[0] * p->shape[2] * 128,
                                                                  (const uint4*)p->tc_bimg[1],
                                                                  make_double2(p->pot_scale, 0.0), nullptr, p->ob,
                                                                  p->partials, p->flag);
                WIG_LAUNCHED("k_tc64<pot>");
            } else {
                return fold_and_finalize(p, hist, rows, st);
            }
            return WIG_OK;
        }
    }
    if constexpr (std::is_same<C, double2>::value) {
        if (p->r4ring) {
            int s;
            if ((s = ensure_w_maps(p, W))) return s;
            const double2* pv = reinterpret_cast<const double2*>(p->pv);
            typedef r4ring::Cfg<double2> K;
            const unsigned grid = (unsigned)(wig_num_sms() < 4096 / K::IL ? wig_num_sms() : 4096 / K::IL);
            // kinetic: LA (ping-pong) -> LB (W); potential: LB (W) -> LA (ping-pong)
            const double2* tw = (const double2*)p->tw64;
            const double2* pvp = pv + (size_t)p->shape[0] * p->shape[2] * 128;
            double2* P = reinterpret_cast<double2*>(p->pingpong);
            const double2 ks = make_double2(p->kin_scale, 0.0), ps = make_double2(p->pot_scale, 0.0);
            if (p->r4ring_pc) {
                // kinetic: LK (ping-pong) -> LP (W); potential: LP (W) -> LK (ping-pong)
                if (part == 0)
                    k_r4ring<double2, true, true><<<grid, K::NTH, K::SMEM, st>>>(
                        p->map_t_load_pc, p->map_w_store, W, pv, tw, ks, p->cur_norm, p->ob, nullptr);
                else if (part == 1)
                    k_r4ring<double2, false, true><<<grid, K::NTH, K::SMEM, st>>>(
                        p->map_w_load_pc, p->map_t_store, P, pvp, tw, ps, p->cur_norm, p->ob, p->partials);
                else
                    return fold_and_finalize(p, hist, rows, st);
                WIG_LAUNCHED(part == 0 ? "k_r4ring<kin, pc>" : "k_r4ring<pot, pc>");
                return WIG_OK;
            }
            if (part == 0) {
                k_r4ring<double2, true, false><<<grid, K::NTH, K::SMEM, st>>>(p->map_t_load, p->map_w_store, W, pv,
                                                                              tw, ks, p->cur_norm, p->ob, nullptr);
                WIG_LAUNCHED("k_r4ring<kin>");
            } else if (part == 1) {
                k_r4ring<double2, false, false><<<grid, K::NTH, K::SMEM, st>>>(p->map_w_load, p->map_t_store, P, pvp,
                                                                               tw, ps, p->cur_norm, p->ob, p->partials);
                WIG_LAUNCHED("k_r4ring<pot>");
            } else {
                return fold_and_finalize(p, hist, rows, st);
            }
            return WIG_OK;
        }
    }
    if constexpr (std::is_same<C, float2>::value) {
        if (p->r4 && p->mx_ring) {
            // complex64 LK / LP layouts, FP64 transforms: kinetic LK (ping-pong) -> LP (W),
            // potential LP (W) -> LK (ping-pong)
            if (p->map_w_mx_ptr != (const void*)W) {
                int s;
                if ((s = encode_unit_map_mx(&p->map_w_load_mx, W))) return s;
                p->map_w_mx_ptr = W;
            }
            float2* P = reinterpret_cast<float2*>(p->pingpong);
            const double2* pv = reinterpret_cast<const double2*>(p->pv);
            const double2* pvp = pv + (size_t)p->shape[0] * p->shape[2] * 128;
            const double2* tw = reinterpret_cast<const double2*>(p->tw64d);
            const float2* tw32 = reinterpret_cast<const float2*>(p->tw64);
            const double2 ks = make_double2(p->kin_scale, 0.0), ps = make_double2(p->pot_scale, 0.0);
            const unsigned grid = (unsigned)(wig_num_sms() < 2048 ? wig_num_sms() : 2048);
            if (part == 0) {
                if (p->mx_f32)
                    k_r4ring_mx<float2, true><<<grid, r4mx::NTH, r4mx::SMEM, st>>>(p->map_t_load_mx, W, pv, tw32, ks,
                                                                                   p->cur_norm, p->ob, nullptr);
                else
                    k_r4ring_mx<double2, true><<<grid, r4mx::NTH, r4mx::SMEM, st>>>(p->map_t_load_mx, W, pv, tw, ks,
                                                                                    p->cur_norm, p->ob, nullptr);
                WIG_LAUNCHED("k_r4ring_mx<kin>");
            } else if (part == 1) {
                if (p->mx_f32)
                    k_r4ring_mx<float2, false><<<grid, r4mx::NTH, r4mx::SMEM, st>>>(p->map_w_load_mx, P, pvp, tw32, ps,
                                                                                    p->cur_norm, p->ob, p->partials);
                else
                    k_r4ring_mx<double2, false><<<grid, r4mx::NTH, r4mx::SMEM, st>>>(p->map_w_load_mx, P, pvp, tw, ps,
                                                                                     p->cur_norm, p->ob, p->partials);
                WIG_LAUNCHED("k_r4ring_mx<pot>");
            } else {
                return fold_and_finalize(p, hist, rows, st);
            }
            return WIG_OK;
        }
        if (p->r4 && p->r4_mixed) {
            // complex64 LA / LB layouts, FP64 transforms
            float2* P = reinterpret_cast<float2*>(p->pingpong);
            const double2* pv = reinterpret_cast<const double2*>(p->pv);
            constexpr size_t sm = r4_smem_bytes<double2>();
            const double2* tw = reinterpret_cast<const double2*>(p->tw64d);
            if (part == 0) {
                WIG_CUDA((launch_r4<double2, true, float2>(p->r4_cluster, 64 * 64, sm, st, P, W, pv, tw,
                                                           make_double2(p->kin_scale, 0.0), p->cur_norm, p->ob,
                                                           nullptr)));
                WIG_LAUNCHED("k_r4<double2, kin, float2>");
            } else if (part == 1) {
                WIG_CUDA((launch_r4<double2, false, float2>(p->r4_cluster, 64 * 64, sm, st, W, P,
                                                            pv + (size_t)p->shape[0] * p->shape[2] * 128, tw,
                                                            make_double2(p->pot_scale, 0.0), nullptr, p->ob,
                                                            p->partials)));
                WIG_LAUNCHED("k_r4<double2, pot, float2>");
            } else {
                return fold_and_finalize(p, hist, rows, st);
            }
            return WIG_OK;
        }
    }
    if (p->r4) {
        // W holds LB, the ping-pong buffer LA (converted around the loop)
        C* P = reinterpret_cast<C*>(p->pingpong);
        const double2* pv = reinterpret_cast<const double2*>(p->pv);
        constexpr size_t sm = r4_smem_bytes<C>();
        const unsigned nplanes = 64 * 64;
        if (part == 0) {
            WIG_CUDA((launch_r4<C, true>(p->r4_cluster, nplanes, sm, st, P, W, pv, (const C*)p->tw64,
                                         make_double2(p->kin_scale, 0.0), p->cur_norm, p->ob, nullptr)));
            WIG_LAUNCHED("k_r4<kin>");
        } else if (part == 1) {
            WIG_CUDA((launch_r4<C, false>(p->r4_cluster, nplanes, sm, st, W, P,
                                          pv + (size_t)p->shape[0] * p->shape[2] * 128, (const C*)p->tw64,
                                          make_double2(p->pot_scale, 0.0), nullptr, p->ob, p->partials)));
            WIG_LAUNCHED("k_r4<pot>");
        } else {
            return fold_and_finalize(p, hist, rows, st);
        }
        return WIG_OK;
    }
    if (part == 0) return kinetic_impl<C>(p, W, p->cur_norm, st);
    if (part == 1) return potential_impl<C>(p, W, p->partials, st);
    return finalize(p, hist, p->counter, rows, st);
}

template <class C>
static int iteration(wig4d_plan* p, C* W, double* hist, int rows, cudaStream_t st) {
    for (int part = 0; part < 3; ++part) {
        int s = iteration_part<C>(p, W, hist, rows, st, part);
        if (s) return s;
    }
    return WIG_OK;
}

// Before the first iteration: the complex64 64^4 loop works on the LA / LB
// layouts (the state moves to the ping-pong buffer as LA).
static int enter_loop_layout(wig4d_plan* p, void* W, cudaStream_t st) {
    if (p->tc) {
        k_to_tc_layout<<<wig_num_sms() * 8, 256, 0, st>>>((const float2*)W, (float2*)p->pingpong, p->npts);
        WIG_LAUNCHED("k_to_tc_layout");
        return WIG_OK;
    }
    if (p->r4 && p->mx_ring) {
        k_pc_transpose<float2, true><<<dim3(2, 2, 4096), 256, 0, st>>>((const float2*)W, (float2*)p->pingpong,
                                                                        nullptr);
        WIG_LAUNCHED("k_pc_transpose<to>");
        return WIG_OK;
    }
    if (p->r4 && p->r4ring_pc) {
        k_pc_transpose<double2, true><<<dim3(2, 2, 4096), 256, 0, st>>>((const double2*)W, (double2*)p->pingpong,
                                                                         nullptr);
        WIG_LAUNCHED("k_pc_transpose<to>");
        return WIG_OK;
    }
    if (p->r4) {
        if (p->dtype == WIG_C128)
            k_to_r4_layout<double2><<<wig_num_sms() * 8, 256, 0, st>>>((const double2*)W, (double2*)p->pingpong, p->npts);
        else
            k_to_r4_layout<float2><<<wig_num_sms() * 8, 256, 0, st>>>((const float2*)W, (float2*)p->pingpong, p->npts);
        WIG_LAUNCHED("k_to_r4_layout");
        return WIG_OK;
    }
    return WIG_OK;
}

// After the last iteration: the state back in the reference layout, divided
// by its norm (the final renormalisation, GPU_Wigner4D.py:516-517).
static int leave_loop_layout(wig4d_plan* p, void* W, cudaStream_t st, bool divide = true) {
    if (p->tc) {
        k_from_tc_layout<<<wig_num_sms() * 8, 256, 0, st>>>((const float2*)p->pingpong, (float2*)W, p->npts,
                                                            divide ? p->cur_norm : nullptr);
        WIG_LAUNCHED("k_from_tc_layout");
        return WIG_OK;
    }
    if (p->r4 && p->mx_ring) {
        k_pc_transpose<float2, false><<<dim3(2, 2, 4096), 256, 0, st>>>((const float2*)p->pingpong, (float2*)W,
                                                                         divide ? p->cur_norm : nullptr);
        WIG_LAUNCHED("k_pc_transpose<from>");
        return WIG_OK;
    }
    if (p->r4 && p->r4ring_pc) {
        k_pc_transpose<double2, false><<<dim3(2, 2, 4096), 256, 0, st>>>((const double2*)p->pingpong, (double2*)W,
                                                                          divide ? p->cur_norm : nullptr);
        WIG_LAUNCHED("k_pc_transpose<from>");
        return WIG_OK;
    }
    if (p->r4) {
        const double* nrm = divide ? p->cur_norm : nullptr;
        if (p->dtype == WIG_C128)
            k_from_r4_layout<double2><<<wig_num_sms() * 8, 256, 0, st>>>((const double2*)p->pingpong, (double2*)W,
                                                                         p->npts, nrm);
        else
            k_from_r4_layout<float2><<<wig_num_sms() * 8, 256, 0, st>>>((const float2*)p->pingpong, (float2*)W,
                                                                        p->npts, nrm);
        WIG_LAUNCHED("k_from_r4_layout");
        return WIG_OK;
    }
    return divide ? wig_divide_by_device_scalar(W, p->npts, p->dtype, p->cur_norm, st) : WIG_OK;
}

template <class C>
static int run_impl(wig4d_plan* p, C* W, int iterations, double* hist, cudaStream_t st, bool divide = true) {
    int s;
    // counter = 0, flag = 0
    WIG_CUDA(cudaMemsetAsync(p->counter, 0, 2 * sizeof(int), st));
    // observables of the initial state are row 0; its norm divides iteration 0
    if ((s = reduce_impl<C>(p, W, st))) return s;
    if ((s = finalize(p, hist, p->counter, iterations, st))) return s;
    if (iterations <= 0) return WIG_OK;
    if ((s = enter_loop_layout(p, W, st))) return s;
    // iteration 0 runs eagerly (kernel attributes get set outside any capture);
    // the rest replay a CUDA graph of one iteration
    if ((s = iteration<C>(p, W, hist, iterations, st))) return s;
    if (iterations == 1) return leave_loop_layout(p, W, st, divide);
    if (!p->graph || p->graph_W != (void*)W || p->graph_hist != hist || p->graph_rows != iterations) {
        if (p->graph) { cudaGraphExecDestroy(p->graph); p->graph = nullptr; }
        cudaStream_t cap;
        WIG_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaGraph_t g;
        WIG_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        int r = iteration<C>(p, W, hist, iterations, cap);
        cudaError_t e = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (r) return r;
        if (e != cudaSuccess) { wig_set_cuda_error(e, "cudaStreamEndCapture"); return WIG_ERR_CUDA; }
        e = cudaGraphInstantiate(&p->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { wig_set_cuda_error(e, "cudaGraphInstantiate"); p->graph = nullptr; return WIG_ERR_CUDA; }
        p->graph_W = W; p->graph_hist = hist; p->graph_rows = iterations;
    }
    // iterations: the last row recorded is that of the final state
    for (int i = 1; i < iterations; ++i) WIG_CUDA(cudaGraphLaunch(p->graph, st));
    return leave_loop_layout(p, W, st, divide);
}

extern "C" int wig4d_run_ex(wig4d_plan* p, void* W, int iterations, double* d_history, int flags, void* stream) {
    if (!p || !W || !d_history || iterations < 0 || (flags & ~WIG_RUN_KEEP_NORM)) return WIG_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    const bool divide = !(flags & WIG_RUN_KEEP_NORM);
    return p->dtype == WIG_C128 ? run_impl<double2>(p, (double2*)W, iterations, d_history, st, divide)
                                : run_impl<float2>(p, (float2*)W, iterations, d_history, st, divide);
}

extern "C" int wig4d_run(wig4d_plan* p, void* W, int iterations, double* d_history, void* stream) {
    return wig4d_run_ex(p, W, iterations, d_history, 0, stream);
}

// ---------------------------------------------------------------------------
// Autotuner: the kernel choices of a plan, timed on a scratch state.
// ---------------------------------------------------------------------------
namespace {

struct TuneKey {
    int shape[4], dtype, fast64, dense_n, tc_ready;
    bool operator<(const TuneKey& o) const { return memcmp(this, &o, sizeof(*this)) < 0; }
};
struct TuneChoice { int engine, kin48, pot_gmax; };

// engine: 0 k_r4 plain stores, 1 k_r4 cluster stores, 3 k_tc64, 4 the
// CUDA-core path of a plan without the 64^4 radix kernels, 6 k_r4ring on
// LA / LB (TMA tensor stores), 7 k_r4ring on the plane-contiguous layouts
int apply_choice(wig4d_plan* p, const TuneChoice& c) {
    if (c.engine == 6 || c.engine == 7) {
        const int r = ensure_r4ring(p);
        if (r) return r;
    }
    p->tc = c.engine == 3;
    p->r4_cluster = c.engine == 1;
    p->r4ring = c.engine == 6 || c.engine == 7;
    p->r4ring_pc = c.engine == 7;
    p->kin48 = c.kin48 != 0;
    p->pot_gmax = c.pot_gmax;
    if (p->graph) { cudaGraphExecDestroy(p->graph); p->graph = nullptr; }
    return WIG_OK;
}

TuneChoice current_choice(const wig4d_plan* p) {
    TuneChoice c;
    c.engine = p->tc ? 3 : (p->r4 ? (p->r4ring ? (p->r4ring_pc ? 7 : 6) : (p->r4_cluster ? 1 : 0)) : 4);
    c.kin48 = p->kin48;
    c.pot_gmax = p->pot_gmax;
    return c;
}

std::mutex tune_mu;
std::map<TuneKey, TuneChoice> tune_cache;

}  // namespace

extern "C" int wig4d_autotune(wig4d_plan* p, int iterations, int flags, void* stream, int* choice_out) {
    if (!p || iterations < 1 || (flags & ~WIG_TUNE_FORCE)) return WIG_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    TuneKey key;
    memset(&key, 0, sizeof(key));
    memcpy(key.shape, p->shape, sizeof(key.shape));
    key.dtype = p->dtype; key.fast64 = p->fast64; key.dense_n = p->dense_n; key.tc_ready = p->tc_ready;
    {
        std::lock_guard<std::mutex> lk(tune_mu);
        auto it = tune_cache.find(key);
        if (it != tune_cache.end() && !(flags & WIG_TUNE_FORCE)) {
            const int r = apply_choice(p, it->second);
            if (r) return r;
            p->tuned = 1;
            if (choice_out) { choice_out[0] = it->second.engine; choice_out[1] = it->second.kin48;
                              choice_out[2] = it->second.pot_gmax; choice_out[3] = 0; }
            return WIG_OK;
        }
    }
    // candidates: the 64^4 engines, then (for the generic kernels) the 48 x 48
    // kinetic kernel and the potential kernel's columns per CTA
    std::vector<TuneChoice> engines;
    const TuneChoice base = current_choice(p);
    if (p->r4) {
        engines.push_back({1, base.kin48, base.pot_gmax});
        engines.push_back({0, base.kin48, base.pot_gmax});
        if (p->dtype == WIG_C128) engines.push_back({6, base.kin48, base.pot_gmax});
        if (p->dtype == WIG_C128) engines.push_back({7, base.kin48, base.pot_gmax});
    } else {
        engines.push_back({4, base.kin48, base.pot_gmax});
    }
    if (p->tc_ready) engines.push_back({3, base.kin48, base.pot_gmax});
    const size_t esz = p->dtype == WIG_C128 ? 16 : 8;
    void* scratch = nullptr;
    double* hist = nullptr;
    if (cudaMalloc(&scratch, (size_t)p->npts * esz) != cudaSuccess) return WIG_ERR_ALLOC;
    if (cudaMalloc(&hist, (size_t)(iterations + 2) * WIG4D_NOBS * sizeof(double)) != cudaSuccess) {
        cudaFree(scratch); return WIG_ERR_ALLOC;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const TuneChoice saved = base;
    int status = WIG_OK;
    float tried = 0;
    auto time_choice = [&](const TuneChoice& c, float* ms) -> int {
        int s = apply_choice(p, c);
        if (s) return s;
        s = wig4d_init_gaussian(p, scratch, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, 1.0, stream);
        if (s) return s;
        if ((s = wig4d_run(p, scratch, 2, hist, stream))) return s;   // warm-up: attributes, graph
        WIG_CUDA(cudaEventRecord(e0, st));
        if ((s = wig4d_run(p, scratch, iterations, hist, stream))) return s;
        WIG_CUDA(cudaEventRecord(e1, st));
        WIG_CUDA(cudaEventSynchronize(e1));
        WIG_CUDA(cudaEventElapsedTime(ms, e0, e1));
        tried += 1;
        return WIG_OK;
    };
    TuneChoice best = base;
    float best_ms = 3.4e38f;
    for (const TuneChoice& c : engines) {
        float ms;
        if ((status = time_choice(c, &ms))) break;
        if (ms < best_ms) { best_ms = ms; best = c; }
    }
    if (!status && best.engine == 4) {
        // generic kernels: the 48 x 48 kinetic kernel, then the potential's G
        if (p->shape[1] == 48 && p->shape[3] == 48) {
            TuneChoice c = best;
            c.kin48 = !best.kin48;
            float ms;
            if (!(status = time_choice(c, &ms)) && ms < best_ms) { best_ms = ms; best = c; }
        }
        for (int g : {8, 4, 2, 1}) {
            if (status || g == best.pot_gmax) continue;
            TuneChoice c = best;
            c.pot_gmax = g;
            float ms;
            if (!(status = time_choice(c, &ms)) && ms < best_ms) { best_ms = ms; best = c; }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(hist);
    cudaFree(scratch);
    if (status) { apply_choice(p, saved); return status; }
    if ((status = apply_choice(p, best))) return status;
    p->tuned = 1;
    {
        std::lock_guard<std::mutex> lk(tune_mu);
        tune_cache[key] = best;
    }
    if (choice_out) { choice_out[0] = best.engine; choice_out[1] = best.kin48; choice_out[2] = best.pot_gmax;
                      choice_out[3] = (int)tried; }
    return WIG_OK;
}

// ---------------------------------------------------------------------------
// Batched Run(): independent instances (own grid, dtype, factors, state and
// history) advanced together.  Each instance's first iteration runs eagerly;
// the others replay ONE CUDA graph per step whose branches are the
// instances' iterations (a child graph each, no edges between them), so the
// kernels of different instances run concurrently and a step costs one
// graph launch.
// ---------------------------------------------------------------------------
static int batch_prologue(wig4d_plan* p, void* W, double* hist, int iterations, cudaStream_t st) {
    int s;
    WIG_CUDA(cudaMemsetAsync(p->counter, 0, 2 * sizeof(int), st));
    if (p->dtype == WIG_C128) {
        if ((s = reduce_impl<double2>(p, (const double2*)W, st))) return s;
    } else {
        if ((s = reduce_impl<float2>(p, (const float2*)W, st))) return s;
    }
    if ((s = finalize(p, hist, p->counter, iterations, st))) return s;
    if (iterations <= 0) return WIG_OK;
    if ((s = enter_loop_layout(p, W, st))) return s;
    return p->dtype == WIG_C128 ? iteration<double2>(p, (double2*)W, hist, iterations, st)
                                : iteration<float2>(p, (float2*)W, hist, iterations, st);
}

extern "C" int wig4d_run_batch(wig4d_plan* const* plans, void* const* states, int n, int iterations,
                               double* const* d_histories, void* stream) {
    if (!plans || !states || !d_histories || n < 0 || iterations < 0) return WIG_ERR_INVALID_ARG;
    for (int i = 0; i < n; ++i) {
        if (!plans[i] || !states[i] || !d_histories[i]) return WIG_ERR_INVALID_ARG;
        for (int j = 0; j < i; ++j)
            if (plans[j] == plans[i] || states[j] == states[i]) return WIG_ERR_ALIAS;
    }
    cudaStream_t st = as_stream(stream);
    int s;
    for (int i = 0; i < n; ++i)
        if ((s = batch_prologue(plans[i], states[i], d_histories[i], iterations, st))) return s;
    if (iterations > 1 && n > 0) {
        cudaGraph_t parent = nullptr;
        WIG_CUDA(cudaGraphCreate(&parent, 0));
        cudaStream_t cap = nullptr;
        cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
        s = WIG_OK;
        for (int i = 0; i < n && e == cudaSuccess && s == WIG_OK; ++i) {
            wig4d_plan* p = plans[i];
            cudaGraph_t child = nullptr;
            e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) break;
            s = p->dtype == WIG_C128 ? iteration<double2>(p, (double2*)states[i], d_histories[i], iterations, cap)
                                     : iteration<float2>(p, (float2*)states[i], d_histories[i], iterations, cap);
            const cudaError_t e2 = cudaStreamEndCapture(cap, &child);
            if (s == WIG_OK) e = e2;
            if (child) {
                cudaGraphNode_t node;
                if (s == WIG_OK && e == cudaSuccess) e = cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, child);
                cudaGraphDestroy(child);
            }
        }
        if (cap) cudaStreamDestroy(cap);
        cudaGraphExec_t exec = nullptr;
        if (s == WIG_OK && e == cudaSuccess) e = cudaGraphInstantiate(&exec, parent, 0);
        cudaGraphDestroy(parent);
        if (s) return s;
        if (e != cudaSuccess) { wig_set_cuda_error(e, "batch graph"); return WIG_ERR_CUDA; }
        for (int it = 1; it < iterations && e == cudaSuccess; ++it) e = cudaGraphLaunch(exec, st);
        cudaGraphExecDestroy(exec);      // deferred by the driver until the launches finish
        if (e != cudaSuccess) { wig_set_cuda_error(e, "cudaGraphLaunch"); return WIG_ERR_CUDA; }
    }
    if (iterations > 0)
        for (int i = 0; i < n; ++i)
            if ((s = leave_loop_layout(plans[i], states[i], st))) return s;
    return WIG_OK;
}

// Run() with the kernels of every iteration bracketed by CUDA events: the
// same launches as run_impl, issued one by one instead of through the graph.
// Events of up to RING iterations are in flight; a slot is read back (its
// last event synchronised) before it is reused.
template <class C>
static int run_timed_impl(wig4d_plan* p, C* W, int iterations, double* hist, cudaStream_t st, double* ms) {
    constexpr int RING = 64;
    int s;
    ms[0] = ms[1] = ms[2] = 0.0;
    WIG_CUDA(cudaMemsetAsync(p->counter, 0, 2 * sizeof(int), st));
    if ((s = reduce_impl<C>(p, W, st))) return s;
    if ((s = finalize(p, hist, p->counter, iterations, st))) return s;
    if (iterations <= 0) return WIG_OK;
    if ((s = enter_loop_layout(p, W, st))) return s;
    cudaEvent_t ev[RING][4];
    cudaEvent_t* flat = &ev[0][0];
    int made = 0;
    cudaError_t e = cudaSuccess;
    while (made < RING * 4 && (e = cudaEventCreate(&flat[made])) == cudaSuccess) ++made;
    if (e != cudaSuccess) {
        for (int i = 0; i < made; ++i) cudaEventDestroy(flat[i]);
        wig_set_cuda_error(e, "cudaEventCreate");
        return WIG_ERR_CUDA;
    }
    auto collect = [&](int slot) -> cudaError_t {
        cudaError_t r = cudaEventSynchronize(ev[slot][3]);
        for (int k = 0; k < 3 && r == cudaSuccess; ++k) {
            float t = 0.f;
            r = cudaEventElapsedTime(&t, ev[slot][k], ev[slot][k + 1]);
            ms[k] += t;
        }
        return r;
    };
    s = WIG_OK;
    for (int i = 0; i < iterations && s == WIG_OK; ++i) {
        const int slot = i % RING;
        if (i >= RING && (e = collect(slot)) != cudaSuccess) { wig_set_cuda_error(e, "event readback"); s = WIG_ERR_CUDA; break; }
        for (int part = 0; part < 3 && s == WIG_OK; ++part) {
            if ((e = cudaEventRecord(ev[slot][part], st)) != cudaSuccess) { wig_set_cuda_error(e, "cudaEventRecord"); s = WIG_ERR_CUDA; break; }
            s = iteration_part<C>(p, W, hist, iterations, st, part);
        }
        if (s == WIG_OK && (e = cudaEventRecord(ev[slot][3], st)) != cudaSuccess) {
            wig_set_cuda_error(e, "cudaEventRecord"); s = WIG_ERR_CUDA;
        }
    }
    if (s == WIG_OK) {
        const int first = iterations > RING ? iterations - RING : 0;
        for (int i = first; i < iterations && s == WIG_OK; ++i)
            if ((e = collect(i % RING)) != cudaSuccess) { wig_set_cuda_error(e, "event readback"); s = WIG_ERR_CUDA; }
    }
    for (int i = 0; i < RING * 4; ++i) cudaEventDestroy(flat[i]);
    if (s) return s;
    return leave_loop_layout(p, W, st);
}

extern "C" int wig4d_run_timed(wig4d_plan* p, void* W, int iterations, double* d_history, void* stream,
                               double* ms_out) {
    if (!p || !W || !d_history || !ms_out || iterations < 0) return WIG_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    return p->dtype == WIG_C128 ? run_timed_impl<double2>(p, (double2*)W, iterations, d_history, st, ms_out)
                                : run_timed_impl<float2>(p, (float2*)W, iterations, d_history, st, ms_out);
}

extern "C" int wig4d_init_ho_ground(wig4d_plan* p, void* W, double x_mu, double y_mu, double px_mu,
                                    double py_mu, double wx, double wy, double mass, void* stream) {
    if (!p || !W) return WIG_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    if (p->dtype == WIG_C128)
        k_init_ho<double2><<<grid_for(p->npts), 256, 0, st>>>((double2*)W, p->shape[0], p->shape[1], p->shape[2],
                                                             p->shape[3], p->ob, x_mu, y_mu, px_mu, py_mu, wx, wy, mass);
    else
        k_init_ho<float2><<<grid_for(p->npts), 256, 0, st>>>((float2*)W, p->shape[0], p->shape[1], p->shape[2],
                                                            p->shape[3], p->ob, x_mu, y_mu, px_mu, py_mu, wx, wy, mass);
    WIG_LAUNCHED("k_init_ho");
    return WIG_OK;
}

extern "C" int wig4d_init_cat_xtheta(wig4d_plan* p, void* W, double dtheta_y, double dtheta_x, double x_mu,
                                    double y_mu, double p_x_mu, double p_y_mu, double a_x, double a_y,
                                    void* stream) {
    if (!p || !W) return WIG_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    if (p->dtype == WIG_C128)
        k_init_cat<double2><<<grid_for(p->npts), 256, 0, st>>>((double2*)W, p->shape[0], p->shape[1], p->shape[2],
                                                              p->shape[3], p->ob, dtheta_y, dtheta_x, x_mu, y_mu,
                                                              p_x_mu, p_y_mu, a_x, a_y);
    else
        k_init_cat<float2><<<grid_for(p->npts), 256, 0, st>>>((float2*)W, p->shape[0], p->shape[1], p->shape[2],
                                                             p->shape[3], p->ob, dtheta_y, dtheta_x, x_mu, y_mu,
                                                             p_x_mu, p_y_mu, a_x, a_y);
    WIG_LAUNCHED("k_init_cat");
    return WIG_OK;
}

extern "C" int wig4d_init_gaussian(wig4d_plan* p, void* W, double mpy, double my, double mpx, double mx,
                                   double spy, double sy, double spx, double sx, void* stream) {
    if (!p || !W) return WIG_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    if (p->dtype == WIG_C128)
        k_init_gauss<double2><<<grid_for(p->npts), 256, 0, st>>>((double2*)W, p->shape[0], p->shape[1], p->shape[2],
                                                                p->shape[3], p->ob, mpy, my, mpx, mx, spy, sy, spx, sx);
    else
        k_init_gauss<float2><<<grid_for(p->npts), 256, 0, st>>>((float2*)W, p->shape[0], p->shape[1], p->shape[2],
                                                               p->shape[3], p->ob, mpy, my, mpx, mx, spy, sy, spx, sx);
    WIG_LAUNCHED("k_init_gauss");
    return WIG_OK;
}
