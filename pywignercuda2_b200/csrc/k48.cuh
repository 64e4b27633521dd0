// k48.cuh -- the fused kinetic half-step on 48 x 48 (y, x) planes with the
// plane in registers.  Included by wigner4d.cu after the generic kernels;
// same contract as k_kinetic<C, 48, 48, NT>: one CTA per (p_y, p_x) plane,
//   W <- S IDFT2( F * DFT2( S W ) ),  S = (-1)^(y + x),
// F the plane's kinetic factor at frequency (y, x) times the scale (and
// 1/norm), the inverse unnormalised (the scale carries 1/N^2).
//
// Each axis index is n = n2 + 16 n1 (n1 < 3, n2 < 16), each frequency
// k = k1 + 3 k2 (k1 < 3, k2 < 16), and
//   X[k1 + 3 k2] = sum_n2 w16^(n2 k2) w48^(n2 k1) sum_n1 w3^(n1 k1) x[n2 + 16 n1],
// with the 16-point part split again as n2 = a + 4 b, k2 = c + 4 d:
//   w16^((a + 4 b)(c + 4 d)) = w4^(b c) w16^(a c) w4^(a d).
// Both axes are split the same way at once:
//   A  thread (n2r, n2c) of 256 holds the 3 x 3 points (n2r + 16 n1r,
//      n2c + 16 n1c), takes the 3 x 3 DFT and the twiddle
//      w48^(n2r k1r + n2c k1c), and writes sub-plane (k1r, k1c) at (n2r, n2c);
//   B1 the nine 16 x 16 sub-planes go to teams of 16 threads (threads
//      0..143): thread a = (qr, qc) holds (qr + 4 i, qc + 4 j), takes the
//      4 x 4 DFT over b = (i, j), the twiddle w16^(a c), and writes [c][a];
//   B2 thread c = (qr, qc) reads a = (i, j), takes the 4 x 4 DFT over a and
//      holds the frequencies k2 = (qr + 4 i, qc + 4 j).
// The factor is applied at (k1r + 3 k2r, k1c + 3 k2c); the inverse runs the
// mirror image (conjugate kernels and twiddles).  The centring signs are
// one negation per thread: the parity of y + x is that of n2r + n2c.
#pragma once

namespace k48 {

constexpr int NT = 256;
constexpr int PS = 16 * 17;          // one 16 x 16 sub-plane, rows padded to 17

template <class C>
constexpr size_t smem_bytes() { return sizeof(C) * (9 * PS + 48); }

// 4 x 4 block: DFTs over j (each row i) then over i (each column j)
template <class C, bool FWD> __device__ __forceinline__ void dft4x4(C (&v)[16]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) dft4<C, FWD>(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
#pragma unroll
    for (int j = 0; j < 4; ++j) dft4<C, FWD>(v[j], v[4 + j], v[8 + j], v[12 + j]);
}

// v[i][j] *= w48^(3 (qr i + qc j)) = w16^(qr i + qc j), or its conjugate
template <class C, bool FWD> __device__ __forceinline__ void tw16(C (&v)[16], const C* tw, int qr, int qc) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (i == 0 && j == 0) continue;
            C w = tw[(3 * (qr * i + qc * j)) % 48];
            if (!FWD) w = cconj(w);
            v[4 * i + j] = cmul(v[4 * i + j], w);
        }
}

}  // namespace k48

namespace k48 {

// The transform of one 48 x 48 plane held by a group of 256 threads (thread
// t of the group), in place on the registers u: on entry u[3 a + b] is the
// point (n2r + 16 a, n2c + 16 b), n2r = t / 16, n2c = t % 16; on exit the
// same points of IDFT2(f * DFT2(u)) (unnormalised), with f(y, x) the factor
// at frequency (y, x).  s: the group's 9 * PS exchange elements, which must
// not be read by any thread of the CTA any more; tw: the 48 twiddles.  Every
// thread of the CTA calls this (it contains __syncthreads).
template <class C, class Factor>
__device__ __forceinline__ void transform(C (&u)[9], C* s, const C* tw, int t, Factor f) {
    const int n2r = t >> 4, n2c = t & 15;
    // ---- A: 3 x 3 DFTs, twiddle w48^(n2r k1r + n2c k1c)
#pragma unroll
    for (int a = 0; a < 3; ++a) dft3<C, true>(u[3 * a], u[3 * a + 1], u[3 * a + 2]);
#pragma unroll
    for (int b = 0; b < 3; ++b) dft3<C, true>(u[b], u[3 + b], u[6 + b]);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            if (a == 0 && b == 0) continue;
            u[3 * a + b] = cmul(u[3 * a + b], tw[(n2r * a + n2c * b) % 48]);
        }
#pragma unroll
    for (int k = 0; k < 9; ++k) s[k * PS + n2r * 17 + n2c] = u[k];
    __syncthreads();
    // ---- B: 16 x 16 DFTs of the nine sub-planes, factor, inverse
    const bool team = t < 144;
    const int sp = t >> 4, qr = (t >> 2) & 3, qc = t & 3;
    C v[16];
    if (team) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) v[4 * i + j] = s[sp * PS + (qr + 4 * i) * 17 + qc + 4 * j];
        dft4x4<C, true>(v);
        tw16<C, true>(v, tw, qr, qc);
    }
    __syncthreads();
    if (team) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) s[sp * PS + (4 * i + j) * 17 + 4 * qr + qc] = v[4 * i + j];
    }
    __syncthreads();
    if (team) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) v[4 * i + j] = s[sp * PS + (4 * qr + qc) * 17 + 4 * i + j];
        dft4x4<C, true>(v);
        // frequencies (k1r + 3 (qr + 4 i), k1c + 3 (qc + 4 j))
        const int k1r = sp / 3, k1c = sp % 3;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
                v[4 * i + j] = cmul(v[4 * i + j], f(k1r + 3 * (qr + 4 * i), k1c + 3 * (qc + 4 * j)));
        dft4x4<C, false>(v);
    }
    __syncthreads();                                   // every team has read [c][a]
    if (team) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) s[sp * PS + (4 * qr + qc) * 17 + 4 * i + j] = v[4 * i + j];
    }
    __syncthreads();
    if (team) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) v[4 * i + j] = s[sp * PS + (4 * i + j) * 17 + 4 * qr + qc];
        tw16<C, false>(v, tw, qr, qc);
        dft4x4<C, false>(v);
    }
    __syncthreads();                                   // every team has read [a][c]
    if (team) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) s[sp * PS + (qr + 4 * i) * 17 + qc + 4 * j] = v[4 * i + j];
    }
    __syncthreads();
    // ---- A inverse
#pragma unroll
    for (int k = 0; k < 9; ++k) u[k] = s[k * PS + n2r * 17 + n2c];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            if (a == 0 && b == 0) continue;
            u[3 * a + b] = cmul(u[3 * a + b], cconj(tw[(n2r * a + n2c * b) % 48]));
        }
#pragma unroll
    for (int a = 0; a < 3; ++a) dft3<C, false>(u[3 * a], u[3 * a + 1], u[3 * a + 2]);
#pragma unroll
    for (int b = 0; b < 3; ++b) dft3<C, false>(u[b], u[3 + b], u[6 + b]);
}

}  // namespace k48

template <class C>
__global__ void __launch_bounds__(k48::NT) k_kin48(C* __restrict__ W, int npy, int npx,
                                                   const __grid_constant__ FactorSet<C> F, double2 scale,
                                                   const double* __restrict__ d_norm) {
    using namespace k48;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* s = reinterpret_cast<C*>(smraw);
    C* tw = s + 9 * PS;
    const int t = threadIdx.x;
    const int ipx = blockIdx.x % npx, ipy = blockIdx.x / npx;
    const long long rowstride = (long long)npx * 48;
    const long long lin0 = ((long long)ipy * 48 * npx + ipx) * 48;
    C* g = W + lin0;
    const int n2r = t >> 4, n2c = t & 15;
    const bool neg = (n2r + n2c) & 1;
    C u[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) u[3 * a + b] = g[(n2r + 16 * a) * rowstride + n2c + 16 * b];
    make_twiddles(tw, 48);
    double2 c0 = scale;
    if (d_norm) c0 = zmul(c0, zinv(make_double2(d_norm[0], d_norm[1])));
    const C cc = to_c<C>(c0);
    if (neg) {
#pragma unroll
        for (int k = 0; k < 9; ++k) u[k] = cneg(u[k]);
    }
    __syncthreads();                                   // twiddles ready
    transform(u, s, tw, t, [&](int y, int x) { return factor_at(F, ipy, y, ipx, x, lin0 + y * rowstride + x, cc); });
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            g[(n2r + 16 * a) * rowstride + n2c + 16 * b] = neg ? cneg(u[3 * a + b]) : u[3 * a + b];
}
