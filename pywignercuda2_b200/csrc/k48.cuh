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

// k_pot48: the fused potential half-step on 48 x 48 (p_y, p_x) planes, the
// contract of k_potential_g<C, 48, 48, G>: a CTA takes the G columns x0 ..
// x0 + G - 1 at one y (G = 2 complex128, 4 complex64: 32-byte runs),
// gathered by cp.async into one 9 * PS-element buffer per column; group g of
// 256 threads transforms column g with k48::transform.  No centring signs:
// the factor is read at frequencies shifted by 24.  Each group then writes
// its column's NPART partial sums, as k_potential_g does.
template <class C>
constexpr int pot48_g() { return sizeof(C) == 16 ? 2 : 4; }
template <class C>
constexpr size_t pot48_smem_bytes() {
    return sizeof(C) * ((size_t)pot48_g<C>() * 9 * k48::PS + 48) + sizeof(double) * NPART * 8 * pot48_g<C>();
}

template <class C>
__global__ void __launch_bounds__(k48::NT * pot48_g<C>(), 1)
k_pot48(C* __restrict__ W, int ny, int nx, const __grid_constant__ FactorSet<C> F, double2 scale, ObsTabs ob,
        double* __restrict__ partials) {
    using namespace k48;
    constexpr int G = pot48_g<C>();
    constexpr int NTB = NT * G;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* s = reinterpret_cast<C*>(smraw);
    C* tw = s + G * 9 * PS;
    double* red = reinterpret_cast<double*>(tw + 48);
    const int grp = threadIdx.x >> 8, t = threadIdx.x & 255;
    const int nxg = nx / G;
    const int x0 = (blockIdx.x % nxg) * G, iy = blockIdx.x / nxg;
    const long long pys = (long long)ny * 48 * nx;      // stride of p_y
    C* gb = W + (long long)iy * 48 * nx + x0;           // element (p_y, p_x, g): gb[p_y*pys + p_x*nx + g]
    for (int e = threadIdx.x; e < G * 48 * 48; e += NTB) {
        const int g = e % G, px = (e / G) % 48, py = e / (G * 48);
        cp_async_elem(s + g * 9 * PS + py * 49 + px, gb + py * pys + (long long)px * nx + g);
    }
    make_twiddles(tw, 48);
    const C cc = to_c<C>(scale);
    cp_async_wait_all();
    __syncthreads();
    C* sg = s + grp * 9 * PS;
    const int n2r = t >> 4, n2c = t & 15;
    C u[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) u[3 * a + b] = sg[(n2r + 16 * a) * 49 + n2c + 16 * b];
    __syncthreads();                                   // the gathered planes have been read
    const int ix = x0 + grp;
    transform(u, sg, tw, t, [&](int y, int x) {
        const int ky = (y + 24) % 48, kx = (x + 24) % 48;
        const long long lin = ky * pys + (long long)iy * 48 * nx + (long long)kx * nx + ix;
        return factor_at_unrolled(F, ky, iy, kx, ix, lin, cc);
    });
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) gb[(n2r + 16 * a) * pys + (long long)(n2c + 16 * b) * nx + grp] = u[3 * a + b];
    if (!partials) return;
    double acc[NPART];
#pragma unroll
    for (int i = 0; i < NPART; ++i) acc[i] = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int py = n2r + 16 * a;
        const double qy = __ldg(ob.cpy + py);
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const int px = n2c + 16 * b;
            const double2 w = to_d2(u[3 * a + b]);
            const double qx = __ldg(ob.cpx + px), k = __ldg(ob.ep + py * 48 + px);
            acc[0] += w.x; acc[1] += w.y;
            acc[2] = fma(qx, w.x, acc[2]); acc[3] = fma(qx, w.y, acc[3]);
            acc[4] = fma(qx * qx, w.x, acc[4]); acc[5] = fma(qx * qx, w.y, acc[5]);
            acc[6] = fma(qy, w.x, acc[6]); acc[7] = fma(qy, w.y, acc[7]);
            acc[8] = fma(qy * qy, w.x, acc[8]); acc[9] = fma(qy * qy, w.y, acc[9]);
            acc[10] = fma(k, w.x, acc[10]); acc[11] = fma(k, w.y, acc[11]);
        }
    }
#pragma unroll
    for (int i = 0; i < NPART; ++i)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[i] += __shfl_down_sync(0xffffffffu, acc[i], o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
#pragma unroll
        for (int i = 0; i < NPART; ++i) red[w * NPART + i] = acc[i];
    __syncthreads();
    if (threadIdx.x < G * NPART) {
        const int gg = threadIdx.x / NPART, i = threadIdx.x % NPART;
        double sum = 0.0;
        for (int k = 0; k < 8; ++k) sum += red[(gg * 8 + k) * NPART + i];
        partials[((long long)iy * nx + x0 + gg) * NPART + i] = sum;
    }
}
