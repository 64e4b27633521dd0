// dense_half.cuh -- fused half-steps for the general fractional transform
// (|delta| N != 1, e.g. the reference notebooks' windows).  Included by
// wigner4d.cu after FactorSet / ObsTabs / block_sum_partials.
//
// One CTA of 256 threads owns one N x N plane (N = 16, 32 or 64).  The plane
// and the two FAFT matrices of the half-step's axes,
//   M_a[k][n] = exp(-2 pi i |delta_a| (n - N/2)(k - N/2))      (faft.cu),
// sit in shared memory; a transform along an axis is the matrix product
//   rows:    OUT[r][k] = sum_n M_c[k][n] IN[r][n]
//   columns: OUT[k][c] = sum_n M_r[k][n] IN[n][c]
// with M conjugated for a negative delta.  Thread (tr, tc) accumulates the
// R x R outputs (tr + 16 i, tc + 16 j), R = N / 16, in registers over n.
// The forward pair (the delta signs of the plan), the factor with the
// half-step scale (which holds the 2 N d of every transform and the
// wrapper divisors), and the inverse pair (opposite signs) run in one
// kernel, so the state is read and written once per half-step instead of
// five times.
#pragma once

namespace dense_half {

constexpr int NT = 256;

// acc += (CONJ ? conj(m) : m) * x
template <class C, bool CONJ>
__device__ __forceinline__ void cmac(C& acc, C m, C x) {
    if (!CONJ) {
        acc.x = fma(m.x, x.x, fma(-m.y, x.y, acc.x));
        acc.y = fma(m.x, x.y, fma(m.y, x.x, acc.y));
    } else {
        acc.x = fma(m.x, x.x, fma(m.y, x.y, acc.x));
        acc.y = fma(m.x, x.y, fma(-m.y, x.x, acc.y));
    }
}

// In-place transform of the plane s (row stride LD) along its columns
// (ROWS = false: the slow axis r) or rows (ROWS = true: the fast axis c).
template <class C, int N, bool ROWS, bool CONJ>
__device__ __forceinline__ void transform(C* s, const C* M, int tr, int tc) {
    constexpr int R = N / 16, LD = N + 1;
    C acc[R][R];
#pragma unroll
    for (int i = 0; i < R; ++i)
#pragma unroll
        for (int j = 0; j < R; ++j) acc[i][j] = mk<C>(0, 0);
#pragma unroll 4
    for (int n = 0; n < N; ++n) {
        C a[R], b[R];
        if (ROWS) {
            // out (r, k) = (tr + 16 i, tc + 16 j): IN[r][n], M[k][n]
#pragma unroll
            for (int i = 0; i < R; ++i) a[i] = s[(tr + 16 * i) * LD + n];
#pragma unroll
            for (int j = 0; j < R; ++j) b[j] = M[(tc + 16 * j) * LD + n];
#pragma unroll
            for (int i = 0; i < R; ++i)
#pragma unroll
                for (int j = 0; j < R; ++j) cmac<C, CONJ>(acc[i][j], b[j], a[i]);
        } else {
            // out (k, c) = (tr + 16 i, tc + 16 j): M[k][n], IN[n][c]
#pragma unroll
            for (int i = 0; i < R; ++i) a[i] = M[(tr + 16 * i) * LD + n];
#pragma unroll
            for (int j = 0; j < R; ++j) b[j] = s[n * LD + tc + 16 * j];
#pragma unroll
            for (int i = 0; i < R; ++i)
#pragma unroll
                for (int j = 0; j < R; ++j) cmac<C, CONJ>(acc[i][j], a[i], b[j]);
        }
    }
    __syncthreads();                  // every thread has read the plane
#pragma unroll
    for (int i = 0; i < R; ++i)
#pragma unroll
        for (int j = 0; j < R; ++j) s[(tr + 16 * i) * LD + tc + 16 * j] = acc[i][j];
    __syncthreads();
}

template <class C, int N, bool ROWS>
__device__ __forceinline__ void transform_sign(C* s, const C* M, int tr, int tc, bool conj) {
    if (conj) transform<C, N, ROWS, true>(s, M, tr, tc);
    else transform<C, N, ROWS, false>(s, M, tr, tc);
}

}  // namespace dense_half

template <class C, int N>
constexpr size_t dense_half_smem_bytes(bool two_matrices) {
    return sizeof(C) * (size_t)(N * (N + 1)) * (two_matrices ? 3 : 2);
}

// KIN: plane (y, x) at fixed (p_y, p_x) = blockIdx (rows contiguous in W);
// POT: plane (p_y, p_x) at fixed (y, x), with one NPART partial row per plane.
// Mr / Mc: FAFT matrices of the row (slow) and column (fast) in-plane axes,
// the same pointer when they coincide; neg_r / neg_c: the forward deltas are
// negative (the forward then uses the conjugate matrix, the inverse the plain one).
template <class C, int N, bool KIN>
__global__ void __launch_bounds__(dense_half::NT, 1)
k_dense_half(C* __restrict__ W, int n_f1, const C* __restrict__ Mr, const C* __restrict__ Mc, int neg_r, int neg_c,
             const __grid_constant__ FactorSet<C> F, double2 scale, const double* __restrict__ d_norm, ObsTabs ob,
             double* __restrict__ partials, int nx_o) {
    using namespace dense_half;
    constexpr int LD = N + 1, PTS = N * N;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* s = reinterpret_cast<C*>(smraw);
    C* mc = s + N * LD;
    C* mr = (Mr == Mc) ? mc : mc + N * LD;
    const int t = threadIdx.x, tr = t >> 4, tc = t & 15;
    const int f1 = blockIdx.x % n_f1, f0 = blockIdx.x / n_f1;
    // plane addressing: KIN (rows y, cols x) in L0 = [p_y][y][p_x][x];
    //                   POT (rows p_y, cols p_x) at fixed (y, x)
    long long base, rs, cs;
    if (KIN) { base = ((long long)f0 * N * n_f1 + f1) * N; rs = (long long)n_f1 * N; cs = 1; }
    else     { base = (long long)f0 * N * nx_o + f1; rs = (long long)N * N * nx_o; cs = nx_o; }
    for (int e = t; e < PTS; e += NT) s[(e / N) * LD + e % N] = W[base + (e / N) * rs + (e % N) * cs];
    for (int e = t; e < PTS; e += NT) mc[(e / N) * LD + e % N] = __ldg(Mc + e);
    if (Mr != Mc)
        for (int e = t; e < PTS; e += NT) mr[(e / N) * LD + e % N] = __ldg(Mr + e);
    double2 c0 = scale;
    if (KIN && d_norm) c0 = zmul(c0, zinv(make_double2(d_norm[0], d_norm[1])));
    const C cc = to_c<C>(c0);
    __syncthreads();
    // forward: along the fast axis, then the slow axis
    transform_sign<C, N, true>(s, mc, tr, tc, neg_c != 0);
    transform_sign<C, N, false>(s, mr, tr, tc, neg_r != 0);
    // factor at (k_r, k_c) = (r, c), with the scale
    for (int e = t; e < PTS; e += NT) {
        const int r = e / N, c = e % N;
        C* q = s + r * LD + c;
        long long lin;
        C f;
        if (KIN) {
            lin = base + r * rs + c * cs;
            f = factor_at(F, f0, r, f1, c, lin, cc);
        } else {
            lin = base + r * rs + c * cs;
            f = factor_at(F, r, f0, c, f1, lin, cc);
        }
        *q = cmul(*q, f);
    }
    __syncthreads();
    // inverse: opposite signs, slow axis then fast axis
    transform_sign<C, N, false>(s, mr, tr, tc, neg_r == 0);
    transform_sign<C, N, true>(s, mc, tr, tc, neg_c == 0);
    double a[NPART];
#pragma unroll
    for (int i = 0; i < NPART; ++i) a[i] = 0.0;
    for (int e = t; e < PTS; e += NT) {
        const int r = e / N, c = e % N;
        const C v = s[r * LD + c];
        W[base + r * rs + c * cs] = v;
        if (!KIN && partials) {
            const double2 w = to_d2(v);
            const double qx = __ldg(ob.cpx + c), qy = __ldg(ob.cpy + r), k = __ldg(ob.ep + r * N + c);
            a[0] += w.x; a[1] += w.y;
            a[2] = fma(qx, w.x, a[2]); a[3] = fma(qx, w.y, a[3]);
            a[4] = fma(qx * qx, w.x, a[4]); a[5] = fma(qx * qx, w.y, a[5]);
            a[6] = fma(qy, w.x, a[6]); a[7] = fma(qy, w.y, a[7]);
            a[8] = fma(qy * qy, w.x, a[8]); a[9] = fma(qy * qy, w.y, a[9]);
            a[10] = fma(k, w.x, a[10]); a[11] = fma(k, w.y, a[11]);
        }
    }
    if (!KIN && partials) {
        __syncthreads();
        block_sum_partials<dense_half::NT>(a, reinterpret_cast<double*>(smraw),
                                           partials + (long long)blockIdx.x * NPART);
    }
}
