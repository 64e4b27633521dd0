// quad64.cuh -- complex64 half-steps of the 64^4 Run() with 64 points per
// thread.  Included by wigner4d.cu after ObsTabs / NSUM.
//
// Work split.  A CTA of 256 threads is four plane groups (PG) of 64 threads;
// a CTA step takes a QUAD of planes (f0, 4m .. 4m+3), PG g the plane
// f1 = 4m + g.  Thread (a, b) = (t >> 3, t & 7) of a PG holds the 64 points
// (r, c) = (a + 8i, b + 8j), i, j = 0..7, of its plane in registers.
//
// 2-D transform of a 64 x 64 plane, 64 = 8 x 8 in each axis:
//   layout A (space):  8-point DFTs over j and over i in registers, with the
//                      twiddles w^(b k1c) and w^(a k1r) between them;
//   one exchange through shared memory (thread (a, b) <-> register (k1r, k1c));
//   layout B (freq.):  8-point DFTs over the old thread digits; thread
//                      (k1r, k1c) then holds the frequencies
//                      (k1r + 8 k2r, k1c + 8 k2c).
// The inverse runs the same steps backwards (conjugate kernels), so a
// half-step costs two exchanges against six for eight-point lanes.
//
// Accuracy.  Everything that is applied identically at every step is kept
// free of a systematic float32 rounding error, since such an error would
// compound over the thousands of steps of a run:
//   * twiddles are float32 pairs chosen (among the neighbours of the rounded
//     cos/sin) so that |w|^2 is closest to 1; the inverse uses their exact
//     conjugates, so a forward/inverse pair restores every path;
//   * 1/sqrt(2) inside the 8-point DFT is applied as hi + lo;
//   * the factor of a plane is applied as (hi + lo) float pairs of its FP64
//     row and column vectors (row vector times the half-step scale in FP64).
// Rounding errors that depend on the state (products, sums) stay float32.
//
// Memory layouts during Run() (c64 only; the state is converted from and
// back to the reference layout L0 = [p_y][y][p_x][x] around the loop):
//   LA = [y][x/4][p_y][p_x][x%4]    (kinetic source, potential destination)
//   LB = [p_y][p_x/4][y][x][p_x%4]  (kinetic destination, potential source)
// With (f0, f1) the plane and (r, c) the in-plane point, both half-steps read
//   src[(((r*16 + c/4)*64 + f0)*64 + f1)*4 + c%4]
// (each 32-byte sector read whole by four lanes of one instruction) and write
//   dst[(((f0*16 + f1/4)*64 + r)*64 + c)*4 + f1%4],
// whose four planes of a quad are one 32-byte run per point: the quad's
// results are staged in shared memory and stored as contiguous 1 KB runs.
#pragma once

namespace quad64 {

constexpr int NT = 256;         // threads per CTA (4 plane groups)
constexpr int RS = 72;          // row stride (elements) of a staged plane
constexpr int EX = 64 * RS;     // elements of one PG's exchange / staging region
constexpr int KS = 72;          // row stride of the K(p_y, p_x) table

// 1/sqrt(2) = H_HI + H_LO to about 2^-48
constexpr float H_HI = 0.70710677f;
constexpr float H_LO = 1.21016175e-08f;

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// Packed two-lane float32 arithmetic (one f32x2 instruction for both parts).
__device__ __forceinline__ unsigned long long pk(float2 a) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 upk(unsigned long long r) {
    float2 a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
__device__ __forceinline__ float2 fadd(float2 a, float2 b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
    return upk(d);
}
__device__ __forceinline__ float2 fsub(float2 a, float2 b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
    return upk(d);
}
// a * h + a * l for a real pair per lane (h, l splat): the hi + lo product
__device__ __forceinline__ float2 fmul_h(float2 a) {
    unsigned long long t, d;
    const float2 hh = make_float2(H_HI, H_HI), hl = make_float2(H_LO, H_LO);
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(t) : "l"(pk(a)), "l"(pk(hh)));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(pk(a)), "l"(pk(hl)), "l"(t));
    return upk(d);
}
__device__ __forceinline__ float2 fmulc(float2 a, float2 w) {
    return f2(fmaf(a.x, w.x, -a.y * w.y), fmaf(a.x, w.y, a.y * w.x));
}
// a * (h + l) with (h, l) a float-float complex factor
__device__ __forceinline__ float2 fmul_hl(float2 a, float2 h, float2 l) {
    const float tx = fmaf(a.x, l.x, -a.y * l.y), ty = fmaf(a.x, l.y, a.y * l.x);
    return f2(fmaf(a.x, h.x, fmaf(-a.y, h.y, tx)), fmaf(a.x, h.y, fmaf(a.y, h.x, ty)));
}

// In-place forward 8-point DFT (kernel exp(-2 pi i / 8)) of v[O + S k],
// k = 0..7; the inverse is conj o dft8 o conj.
template <int O, int S>
__device__ __forceinline__ void dft8(float2* v) {
    const float2 x0 = v[O], x1 = v[O + S], x2 = v[O + 2 * S], x3 = v[O + 3 * S];
    const float2 x4 = v[O + 4 * S], x5 = v[O + 5 * S], x6 = v[O + 6 * S], x7 = v[O + 7 * S];
    const float2 a0 = fadd(x0, x4), a1 = fsub(x0, x4);
    const float2 b0 = fadd(x2, x6), b1 = fsub(x2, x6);
    const float2 c0 = fadd(x1, x5), c1 = fsub(x1, x5);
    const float2 d0 = fadd(x3, x7), d1 = fsub(x3, x7);
    // even outputs: 4-point DFT of (a0, c0, b0, d0)
    const float2 e0 = fadd(a0, b0), e2 = fsub(a0, b0), f0 = fadd(c0, d0), t = fsub(c0, d0);
    // odd outputs: z = (a1, c1 w8, -i b1, -i d1 w8); g = a1 -+ i b1, h = c1 -+ i d1
    const float2 g0 = f2(a1.x + b1.y, a1.y - b1.x), g2 = f2(a1.x - b1.y, a1.y + b1.x);
    const float2 h0 = f2(c1.x + d1.y, c1.y - d1.x), h2 = f2(c1.x - d1.y, c1.y + d1.x);
    // h0 * w8 = (h0.x + h0.y, h0.y - h0.x) / sqrt2, h2 * w8^3 = (h2.y - h2.x, -(h2.x + h2.y)) / sqrt2
    const float2 hw0 = fmul_h(f2(h0.x + h0.y, h0.y - h0.x));
    const float2 hw2 = fmul_h(f2(h2.y - h2.x, -(h2.x + h2.y)));
    v[O] = fadd(e0, f0);
    v[O + 4 * S] = fsub(e0, f0);
    v[O + 2 * S] = f2(e2.x + t.y, e2.y - t.x);     // e2 - i t
    v[O + 6 * S] = f2(e2.x - t.y, e2.y + t.x);     // e2 + i t
    v[O + 1 * S] = fadd(g0, hw0);
    v[O + 5 * S] = fsub(g0, hw0);
    v[O + 3 * S] = fadd(g2, hw2);
    v[O + 7 * S] = fsub(g2, hw2);
}

// DFT over j (stride 1) for all 8 rows, and over i (stride 8) for all 8 columns.
__device__ __forceinline__ void dft_rows(float2* v) {
    dft8<0, 1>(v);  dft8<8, 1>(v);  dft8<16, 1>(v); dft8<24, 1>(v);
    dft8<32, 1>(v); dft8<40, 1>(v); dft8<48, 1>(v); dft8<56, 1>(v);
}
__device__ __forceinline__ void dft_cols(float2* v) {
    dft8<0, 8>(v); dft8<1, 8>(v); dft8<2, 8>(v); dft8<3, 8>(v);
    dft8<4, 8>(v); dft8<5, 8>(v); dft8<6, 8>(v); dft8<7, 8>(v);
}

// Twiddle table w^m = exp(-2 pi i m / 64), m = 0..63: among the float pairs
// within two units in the last place of the rounded (cos, sin), the one
// whose squared modulus is closest to 1.
__device__ __forceinline__ void make_norm_twiddles(float2* tw) {
    for (int m = threadIdx.x; m < 64; m += blockDim.x) {
        double s, c;
        sincospi(-(double)m / 32.0, &s, &c);
        const float cf = (float)c, sf = (float)s;
        float bc = cf, bs = sf;
        double best = fabs((double)cf * cf + (double)sf * sf - 1.0);
        for (int dc = -2; dc <= 2; ++dc)
            for (int ds = -2; ds <= 2; ++ds) {
                if ((cf == 0.0f && dc) || (sf == 0.0f && ds)) continue;
                const float cc = __uint_as_float(__float_as_uint(cf) + dc);
                const float ss = __uint_as_float(__float_as_uint(sf) + ds);
                const double e = fabs((double)cc * cc + (double)ss * ss - 1.0);
                if (e < best) { best = e; bc = cc; bs = ss; }
            }
        tw[m] = make_float2(bc, bs);
    }
}

__device__ __forceinline__ void pg_sync(int g) {
    asm volatile("bar.sync %0, 64;" ::"r"(g + 1) : "memory");
}

// float-float split of a complex double
__device__ __forceinline__ void split_hl(double2 d, float2& h, float2& l) {
    h = make_float2((float)d.x, (float)d.y);
    l = make_float2((float)(d.x - (double)h.x), (float)(d.y - (double)h.y));
}

__device__ __forceinline__ void st_v4(float2* p, float2 a, float2 b) {
    asm volatile("st.global.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y)
                 : "memory");
}

}  // namespace quad64

// Shared memory of k_quad64 (bytes).
constexpr size_t quad64_smem_bytes() {
    return sizeof(float2) * (4 * quad64::EX + 64) + sizeof(float) * 64 * quad64::KS +
           sizeof(double) * NSUM * quad64::NT;
}

// One half-step over all planes of the quad layout (see the file comment).
//   KIN: src LA, dst LB, factor scale / norm;  POT: src LB, dst LA, factor
//   scale, and the NSUM observable sums of the new (x, p) state, one row per CTA.
// PV: FP64 per-plane vectors [plane][128] (row frequencies, then column
// frequencies, already shifted by N/2 as k_plane_vectors builds them).
template <bool KIN>
__global__ void __launch_bounds__(quad64::NT, 1) k_quad64(const float2* __restrict__ src, float2* __restrict__ dst,
                                                          int n_f0, const double2* __restrict__ PV, double2 scale,
                                                          const double* __restrict__ d_norm, ObsTabs ob,
                                                          double* __restrict__ partials) {
    using namespace quad64;
    extern __shared__ __align__(16) unsigned char smraw[];
    float2* E = reinterpret_cast<float2*>(smraw);            // [4][EX] exchange + staging
    float2* tw = E + 4 * EX;                                  // [64]
    float* Kt = reinterpret_cast<float*>(tw + 64);            // [64][KS] (POT)
    double* R = reinterpret_cast<double*>(Kt + 64 * KS);      // [NSUM][NT] running sums (POT)

    const int tid = threadIdx.x, g = tid >> 6, t = tid & 63, ta = t >> 3, tb = t & 7;
    float2* Eg = E + g * EX;
    make_norm_twiddles(tw);
    if (!KIN) {
        for (int k = tid; k < 64 * 64; k += NT) Kt[(k >> 6) * KS + (k & 63)] = (float)__ldg(ob.ep + k);
#pragma unroll
        for (int k = 0; k < NSUM; ++k) R[k * NT + tid] = 0.0;
    }
    __syncthreads();
    double2 cc = scale;
    if (KIN && d_norm) cc = zmul(cc, zinv(make_double2(d_norm[0], d_norm[1])));

    const int nquads = n_f0 * 16;
    for (int qd = blockIdx.x; qd < nquads; qd += gridDim.x) {
        const int f0 = qd >> 4, m = qd & 15, f1 = 4 * m + g, pl = f0 * 64 + f1;
        float2 v[64];
        {
            const float2* s = src + ((((long long)ta * 16 + (tb >> 2)) * 64 + f0) * 64 + f1) * 4 + (tb & 3);
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) v[i * 8 + j] = s[(long long)i * (8 * 16 * 64 * 64 * 4) + j * (2 * 64 * 64 * 4)];
        }
        // Four passes of one code body.  Forward: pass 0 (layout A, with
        // twiddles), exchange, pass 1 (layout B).  Inverse = conj o forward
        // o conj with the same passes in the same order (pass 2 = pass 0 in
        // layout B, pass 3 = pass 1 in layout A); the inner conjugations
        // cancel across the exchange, the outer ones are folded into the
        // factor (v <- conj(v F)) and into the output.
#pragma unroll 1
        for (int ps = 0; ps < 4; ++ps) {
            dft_rows(v);
            if (!(ps & 1)) {      // column twiddles w^(tb k)
#pragma unroll
                for (int k = 1; k < 8; ++k) {
                    const float2 w = tw[(tb * k) & 63];
#pragma unroll
                    for (int i = 0; i < 8; ++i) v[i * 8 + k] = fmulc(v[i * 8 + k], w);
                }
            }
            dft_cols(v);
            if (!(ps & 1)) {      // row twiddles w^(ta k)
#pragma unroll
                for (int k = 1; k < 8; ++k) {
                    const float2 w = tw[(ta * k) & 63];
#pragma unroll
                    for (int j = 0; j < 8; ++j) v[k * 8 + j] = fmulc(v[k * 8 + j], w);
                }
                // exchange: register k of thread s <-> register s of thread k
                __syncthreads();      // E is free: previous exchange / store phase done
#pragma unroll
                for (int k = 0; k < 64; ++k) Eg[k * 66 + t] = v[k];
                pg_sync(g);
#pragma unroll
                for (int k = 0; k < 64; k += 2) {
                    const float4 w = *reinterpret_cast<const float4*>(Eg + t * 66 + k);
                    v[k] = make_float2(w.x, w.y);
                    v[k + 1] = make_float2(w.z, w.w);
                }
            } else if (ps == 1) {
                // factor at row frequency ta + 8a, column frequency tb + 8b,
                // then the conjugation that starts the inverse
                const double2* pv = PV + (long long)pl * 128;
                float2 bh[8], bl[8];
#pragma unroll
                for (int b = 0; b < 8; ++b) split_hl(__ldg(pv + 64 + tb + 8 * b), bh[b], bl[b]);
#pragma unroll
                for (int a = 0; a < 8; ++a) {
                    float2 ah, al;
                    split_hl(zmul(__ldg(pv + ta + 8 * a), cc), ah, al);
#pragma unroll
                    for (int b = 0; b < 8; ++b) {
                        const float2 w = fmul_hl(fmul_hl(v[a * 8 + b], ah, al), bh[b], bl[b]);
                        v[a * 8 + b] = make_float2(w.x, -w.y);
                    }
                }
            }
        }
        // v now holds conj of the result (x, p) state, rows ta + 8i, columns tb + 8j
        // ---- observables of the new (x, p) state: rows p_y = ta + 8i, columns p_x = tb + 8j
        if (!KIN) {
            double s0x = 0, s0y = 0, s1x = 0, s1y = 0, s2x = 0, s2y = 0;   // W, p_y W, p_y^2 W
            double s3x = 0, s3y = 0, s4x = 0, s4y = 0, s5x = 0, s5y = 0;   // p_x W, p_x^2 W, K W
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                float a0x = 0.f, a0y = 0.f, a1x = 0.f, a1y = 0.f, a2x = 0.f, a2y = 0.f, a3x = 0.f, a3y = 0.f;
                const float* kr = Kt + (ta + 8 * i) * KS + tb;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float2 w = make_float2(v[i * 8 + j].x, -v[i * 8 + j].y);
                    const float kk = kr[8 * j], q = (float)__ldg(ob.cpx + tb + 8 * j), qw_x = q * w.x, qw_y = q * w.y;
                    a0x += w.x; a0y += w.y;
                    a1x += qw_x; a1y += qw_y;
                    a2x = fmaf(q, qw_x, a2x); a2y = fmaf(q, qw_y, a2y);
                    a3x = fmaf(kk, w.x, a3x); a3y = fmaf(kk, w.y, a3y);
                }
                const double py = __ldg(ob.cpy + ta + 8 * i);
                const double w0x = a0x, w0y = a0y;
                s0x += w0x; s0y += w0y;
                s1x = fma(py, w0x, s1x); s1y = fma(py, w0y, s1y);
                s2x = fma(py * py, w0x, s2x); s2y = fma(py * py, w0y, s2y);
                s3x += (double)a1x; s3y += (double)a1y;
                s4x += (double)a2x; s4y += (double)a2y;
                s5x += (double)a3x; s5y += (double)a3y;
            }
            const double x = __ldg(ob.cx + f1), y = __ldg(ob.cy + f0), V = __ldg(ob.ex + f0 * 64 + f1);
            double* r = R + tid;
            r[0 * NT] += s0x;          r[1 * NT] += s0y;            // W
            r[2 * NT] += x * s0x;      r[3 * NT] += x * s0y;        // x W
            r[4 * NT] += x * x * s0x;  r[5 * NT] += x * x * s0y;    // x^2 W
            r[6 * NT] += s3x;          r[7 * NT] += s3y;            // p_x W
            r[8 * NT] += s4x;          r[9 * NT] += s4y;            // p_x^2 W
            r[10 * NT] += y * s0x;     r[11 * NT] += y * s0y;       // y W
            r[12 * NT] += y * y * s0x; r[13 * NT] += y * y * s0y;   // y^2 W
            r[14 * NT] += s1x;         r[15 * NT] += s1y;           // p_y W
            r[16 * NT] += s2x;         r[17 * NT] += s2y;           // p_y^2 W
            r[18 * NT] += s5x;         r[19 * NT] += s5y;           // K W
            r[20 * NT] += V * s0x;     r[21 * NT] += V * s0y;       // V W
        }
        // ---- stage the plane: S_g[r * RS + c], r = ta + 8i, c = tb + 8j
        pg_sync(g);                            // every lane has read its B -> A slots
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j) Eg[(ta + 8 * i) * RS + tb + 8 * j] = make_float2(v[i * 8 + j].x, -v[i * 8 + j].y);
        __syncthreads();
        // ---- store: point p = tid + NT k, the quad's four planes as one 32-byte run
        float2* d = dst + (((long long)f0 * 16 + m) * 64 * 64) * 4;
#pragma unroll 4
        for (int k = 0; k < 16; ++k) {
            const int p = tid + NT * k, r = p >> 6, c = p & 63, o = r * RS + c;
            float2* q = d + (long long)p * 4;
            st_v4(q, E[o], E[EX + o]);
            st_v4(q + 2, E[2 * EX + o], E[3 * EX + o]);
        }
    }
    if (!KIN) {
        __syncthreads();
        if (tid < NSUM) {
            double s = 0.0;
            for (int k = 0; k < NT; ++k) s += R[tid * NT + k];
            partials[(long long)blockIdx.x * NSUM + tid] = s;
        }
    }
}

// L0 = [p_y][y][p_x][x] -> LA = [y][x/4][p_y][p_x][x%4]; one thread per LA element.
__global__ void k_to_quad_layout(const float2* __restrict__ W, float2* __restrict__ P, long long n) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int xr = (int)(e & 3), px = (int)((e >> 2) & 63), py = (int)((e >> 8) & 63);
        const int xq = (int)((e >> 14) & 15), y = (int)(e >> 18);
        const int x = 4 * xq + xr;
        P[e] = W[(((long long)py * 64 + y) * 64 + px) * 64 + x];
    }
}

// LA -> L0 with the final division by the complex norm (none when d_norm is
// null); one thread per L0 element.
__global__ void k_from_quad_layout(const float2* __restrict__ P, float2* __restrict__ W, long long n,
                                   const double* __restrict__ d_norm) {
    const double2 inv = d_norm ? zinv(make_double2(d_norm[0], d_norm[1])) : make_double2(1.0, 0.0);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(e & 63), px = (int)((e >> 6) & 63), y = (int)((e >> 12) & 63), py = (int)(e >> 18);
        const float2 a = P[((((long long)y * 16 + (x >> 2)) * 64 + py) * 64 + px) * 4 + (x & 3)];
        const double2 r = zmul(make_double2(a.x, a.y), inv);
        W[e] = make_float2((float)r.x, (float)r.y);
    }
}
