// dirac.cu -- 4 x 4 spinor Wigner-Dirac (and KvN) split-operator kernels, sm_100a.
//
// Replaces the Dirac/KvN JIT kernels and wrappers of the reference:
//   boundary_p_GPU / boundary_xp_GPU ...... GPU_WignerDirac4D.py:292-366
//   Real_GPU ............................. GPU_WignerDirac4D.py:240-244
//   exp_p_lambda_GPU (kinetic sandwich) ... GPU_WignerDirac4D.py:377-481 (KvN:388-476)
//   Potential_Propagator_Kernel ........... GPU_WignerDirac4D.py:492-708 (KvN:~486-690)
//   ParticleProjector_GPU ................. GPU_WignerDirac4D.py:1040-1148 (KvN:853-945)
//   initial states ........................ GPU_WignerDirac4D.py:908-1032 (KvN:776-795)
//   reductions, Normalize_4x4_GPU ......... GPU_WignerDirac4D.py:1156-1388
//   Fourier_*_64_64_4x4_GPU ............... GPU_WignerDirac4D.py:1428-1596
//
// The sixteen components W11..W44 are passed as sixteen slot pointers.  The
// elementwise kernels keep the reference's per-thread order -- read all
// slots, compute, write slots in order (sandwiches), or read-modify-write
// slot by slot (mask, divide) -- so a caller passing the same pointer in
// two slots (the reference's Run() binds W21 to W22) gets the reference's
// result; the C ABI accepts that only for the elementwise entry points.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "fft_smem.cuh"

void* wig_dense_matrix(int n, double delta, int dtype, cudaStream_t st);
int wig_r4_twiddles(void* tw, int dtype, cudaStream_t st);
int wig_dplane64(void* const* slots, int nslots, int dtype, int kind, int fwd, double scale, const double* d_norm,
                 const void* tw, cudaStream_t st, const DEpi* epi = nullptr);

#define NSLOT 16

template <class C>
struct Slots {
    C* p[NSLOT];
};

// factor tables (same convention as the scalar plan)
template <class C>
struct DFactors {
    int n;
    const C* data[WIG_MAX_FACTORS];
    int ia[WIG_MAX_FACTORS], ib[WIG_MAX_FACTORS], nb[WIG_MAX_FACTORS];
};

__device__ __forceinline__ int dsel4(int a, int i0, int i1, int i2, int i3) {
    return a == 0 ? i0 : (a == 1 ? i1 : (a == 2 ? i2 : i3));
}

template <class C>
__device__ __forceinline__ double2 dfactor_at(const DFactors<C>& F, int i0, int i1, int i2, int i3, long long lin) {
    double2 acc = make_double2(1.0, 0.0);
    for (int t = 0; t < F.n; ++t) {
        long long idx;
        if (F.ia[t] < 0) idx = lin;
        else if (F.ib[t] < 0) idx = dsel4(F.ia[t], i0, i1, i2, i3);
        else idx = (long long)dsel4(F.ia[t], i0, i1, i2, i3) * F.nb[t] + dsel4(F.ib[t], i0, i1, i2, i3);
        acc = zmul(acc, to_d2(F.data[t][idx]));
    }
    return acc;
}

// Device-side parameters of a plan (all coordinates float64).
struct DParams {
    int n0, n1, n2, n3;          // N_py, N_y, N_px, N_x
    int kvn;
    double c, hbar, mass, dt, m_pot;
    const double* cpy; const double* cy; const double* cpx; const double* cx;     // (x, p) grid
    const double* ty; const double* ly; const double* tx; const double* lx;       // theta_y, lambda_y, theta_x, lambda_x
    const double* mxp[4];                          // boundary_xp factors per axis
    const double* mp[4];                           // boundary_p factors per axis
    int arank;                                     // rank of the A1..A3 tables
    const double* atab;                            // [3][2][R][N2*N3 + N1*N0], u part [itx][ix]
    const double* obs_xy;                          // [7][N1][N3]
    int pow2, s3, s32, s321;                       // all sizes powers of two: shifts of axes 2, 1, 0
    int a3zero;                                    // A3 vanishes on both Bopp sides (rank tables)
    const double* afull;                           // or full tables [3][2][points] in the state layout
};

// Point index -> (i0, i1, i2, i3) in 32-bit arithmetic (plans hold fewer
// than 2^31 points): shifts and masks for power-of-two sizes, else three
// unsigned divisions.
__device__ __forceinline__ void decode(long long li, const DParams& P, int& i0, int& i1, int& i2, int& i3) {
    const unsigned i = (unsigned)li;
    if (P.pow2) {
        i3 = (int)(i & (unsigned)(P.n3 - 1));
        i2 = (int)((i >> P.s3) & (unsigned)(P.n2 - 1));
        i1 = (int)((i >> P.s32) & (unsigned)(P.n1 - 1));
        i0 = (int)(i >> P.s321);
        return;
    }
    const unsigned q3 = i / (unsigned)P.n3, q2 = q3 / (unsigned)P.n2, q1 = q2 / (unsigned)P.n1;
    i3 = (int)(i - q3 * (unsigned)P.n3);
    i2 = (int)(q3 - q2 * (unsigned)P.n2);
    i1 = (int)(q2 - q1 * (unsigned)P.n1);
    i0 = (int)q1;
}

// ---------------------------------------------------------------------------
// 4 x 4 complex matrices: dense arrays, entries that are structurally zero in
// the reference's expansions are zero here and cost a few extra FMAs.
// ---------------------------------------------------------------------------
struct M4 { double2 a[4][4]; };

__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 zscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// [[a,0,0,b],[0,a,s*conj(b),0],[0,b,a33,0],[s*conj(b),0,0,a33]]
__device__ __forceinline__ M4 spin_matrix(double2 a, double2 b, double s, double2 a33) {
    M4 m;
    const double2 z = make_double2(0.0, 0.0);
    const double2 cb = zscale(zconj(b), s);
    m.a[0][0] = a; m.a[0][1] = z; m.a[0][2] = z; m.a[0][3] = b;
    m.a[1][0] = z; m.a[1][1] = a; m.a[1][2] = cb; m.a[1][3] = z;
    m.a[2][0] = z; m.a[2][1] = b; m.a[2][2] = a33; m.a[2][3] = z;
    m.a[3][0] = cb; m.a[3][1] = z; m.a[3][2] = z; m.a[3][3] = a33;
    return m;
}

// Structural non-zeros of the matrices (bit 4 r + c set for entry (r, c)):
// spin_matrix and the KvN potential propagator have two per row, the Dirac
// potential propagator three (no (0,1), (1,0), (2,3), (3,2)).
constexpr unsigned SPIN_NZ = (1u << 0) | (1u << 3) | (1u << 5) | (1u << 6) | (1u << 9) | (1u << 10) |
                             (1u << 12) | (1u << 15);
constexpr unsigned DPOT_NZ = 0xffffu & ~((1u << 1) | (1u << 4) | (1u << 11) | (1u << 14));

// w <- L * w * R (4 x 4), w row-major w[4*a + b]; entries outside NZ are
// zero and their products are skipped (each sum runs over the non-zero
// entries in increasing k, as the dense product adds them).
template <unsigned NZL, unsigned NZR>
__device__ __forceinline__ void sandwich(const M4& L, double2 (&w)[16], const M4& R) {
    double2 t[16];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            double2 s = make_double2(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if ((NZL >> (4 * a + k)) & 1u) s = zadd(s, zmul(L.a[a][k], w[4 * k + b]));
            t[4 * a + b] = s;
        }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            double2 s = make_double2(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if ((NZR >> (4 * k + b)) & 1u) s = zadd(s, zmul(t[4 * a + k], R.a[k][b]));
            w[4 * a + b] = s;
        }
}

// The two halves of sandwich() in place, with the same sums in the same order:
// w <- L w one column at a time, w <- w R one row at a time (four temporaries
// each), so that a kernel can build R only after L has been applied.
template <unsigned NZL>
__device__ __forceinline__ void left_apply(const M4& L, double2 (&w)[16]) {
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        double2 col[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            double2 s = make_double2(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if ((NZL >> (4 * a + k)) & 1u) s = zadd(s, zmul(L.a[a][k], w[4 * k + b]));
            col[a] = s;
        }
#pragma unroll
        for (int a = 0; a < 4; ++a) w[4 * a + b] = col[a];
    }
}
template <unsigned NZR>
__device__ __forceinline__ void right_apply(double2 (&w)[16], const M4& R) {
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        double2 row[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            double2 s = make_double2(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if ((NZR >> (4 * k + b)) & 1u) s = zadd(s, zmul(w[4 * a + k], R.a[k][b]));
            row[b] = s;
        }
#pragma unroll
        for (int b = 0; b < 4; ++b) w[4 * a + b] = row[b];
    }
}

// K11, K14 of the free Dirac propagator (GPU_WignerDirac4D.py:377-388)
__device__ __forceinline__ void kin_entries(double px, double py, double m, double dt, const DParams& P,
                                            double2& k11, double2& k14) {
    const double c = P.c, hb = P.hbar;
    const double om = c / hb * sqrt(m * c * m * c + px * px + py * py);
    double s, co;
    sincos(dt * om, &s, &co);
    k11 = make_double2(co, -(c * c * m * s) / (om * hb));
    k14 = make_double2(-(c * py * s) / (om * hb), -(c * px * s) / (om * hb));
}

// U of the potential propagator at field (A1, A2, A3) (WD4D:580-604; KvN:584-597).
__device__ __forceinline__ M4 pot_matrix(double A1, double A2, double A3, double dt, bool right, const DParams& P) {
    const double c = P.c, hb = P.hbar, m = P.m_pot;
    M4 u;
    const double2 z = make_double2(0.0, 0.0);
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) u.a[i][j] = z;
    if (P.kvn) {
        const double F = sqrt(m * c * m * c + A1 * A1 + A2 * A2);
        double s, co;
        sincos(c * dt * F / hb, &s, &co);          // dt > 0 on both sides for KvN
        if (!right) {
            const double sm = -s / F;              // sin(-c dt F / hbar) / F
            u.a[0][0] = u.a[1][1] = make_double2(co, -m * c * (-s) / F);
            u.a[2][2] = u.a[3][3] = make_double2(co, m * c * (-s) / F);
            u.a[0][3] = make_double2(-A2 * sm, -A1 * sm);
            u.a[3][0] = make_double2(A2 * sm, -A1 * sm);
            u.a[1][2] = make_double2(A2 * sm, -A1 * sm);
            u.a[2][1] = make_double2(-A2 * sm, -A1 * sm);
        } else {
            const double sp = s / F;
            u.a[0][0] = u.a[1][1] = make_double2(co, m * c * (-s) / F);
            u.a[2][2] = u.a[3][3] = make_double2(co, -m * c * (-s) / F);
            u.a[0][3] = make_double2(-A2 * sp, -A1 * sp);
            u.a[3][0] = make_double2(A2 * sp, -A1 * sp);
            u.a[1][2] = make_double2(A2 * sp, -A1 * sp);
            u.a[2][1] = make_double2(-A2 * sp, -A1 * sp);
        }
        return u;
    }
    const double F = sqrt(m * c * m * c + A1 * A1 + A2 * A2 + A3 * A3);
    double s, co;
    sincos(c * dt * F / hb, &s, &co);
    const double sf = s / F;
    u.a[0][0] = u.a[1][1] = make_double2(co, m * c * sf);
    u.a[2][2] = u.a[3][3] = make_double2(co, -m * c * sf);
    u.a[0][3] = make_double2(A2 * sf, A1 * sf);
    u.a[1][2] = make_double2(A2 * sf, -A1 * sf);
    u.a[2][1] = make_double2(-A2 * sf, -A1 * sf);
    u.a[3][0] = make_double2(-A2 * sf, A1 * sf);
    if (P.a3zero) return u;                        // sin(A3 c dt) = 0: the four entries below vanish
    const double s3 = sin(A3 * c * dt);
    u.a[0][2] = make_double2(0.0, s3);
    u.a[1][3] = make_double2(0.0, -s3);
    u.a[2][0] = make_double2(0.0, s3);
    u.a[3][1] = make_double2(0.0, -s3);
    (void)right;
    return u;
}

// A_k at the Bopp-shifted point from the rank tables: side 0 = (x - theta/2),
// side 1 = (x + theta/2); indices ix (axis 3), itx (axis 2), iy (axis 1), ity (axis 0).
__device__ __forceinline__ double a_field(const DParams& P, int k, int side, int ix, int itx, int iy, int ity) {
    const long long nu = (long long)P.n3 * P.n2, nv = (long long)P.n1 * P.n0;
    if (P.afull)
        return P.afull[(long long)(k * 2 + side) * nu * nv + (((long long)ity * P.n1 + iy) * P.n2 + itx) * P.n3 + ix];
    const double* base = P.atab + ((long long)(k * 2 + side) * P.arank) * (nu + nv);
    double acc = 0.0;
    for (int r = 0; r < P.arank; ++r) {
        const double* f = base + r * (nu + nv);
        acc = fma(f[(long long)itx * P.n3 + ix], f[nu + (long long)iy * P.n0 + ity], acc);
    }
    return acc;
}

template <class C>
__device__ __forceinline__ void load16(const Slots<C>& S, long long i, double2 (&w)[16]) {
#pragma unroll
    for (int k = 0; k < 16; ++k) w[k] = to_d2(S.p[k][i]);
}
template <class C>
__device__ __forceinline__ void store16(const Slots<C>& S, long long i, const double2 (&w)[16]) {
#pragma unroll
    for (int k = 0; k < 16; ++k) S.p[k][i] = to_c<C>(w[k]);
}

// ---------------------------------------------------------------------------
// Elementwise kernels
// ---------------------------------------------------------------------------
// The distinct component pointers of a slot list with how often each occurs
// (the reference's Run() binds W21 to W22, so a pointer can occur twice).
template <class C>
struct USlots {
    C* p[NSLOT];
    int mult[NSLOT];
    int n;
};

// kind 1: boundary_xp (mxp), kind 2: boundary_p (mp).  The reference's
// statements W11[i] = r*W11[i]; ... run slot by slot, so a pointer that
// occurs m times is scaled m times; here each distinct pointer is loaded
// once, scaled m times with the storage rounding between, and stored once.
template <class C>
__global__ void __launch_bounds__(256) k_dmask(USlots<C> U, DParams P, int kind) {
    const long long n = (long long)P.n0 * P.n1 * P.n2 * P.n3;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int i0, i1, i2, i3;
        decode(i, P, i0, i1, i2, i3);
        const double r = kind == 1 ? P.mxp[2][i2] * P.mxp[0][i0] * P.mxp[3][i3] * P.mxp[1][i1]
                                   : P.mp[2][i2] * P.mp[0][i0] * P.mp[3][i3] * P.mp[1][i1];
        C w[NSLOT];
#pragma unroll
        for (int u = 0; u < NSLOT; ++u)
            if (u < U.n) w[u] = U.p[u][i];
#pragma unroll
        for (int u = 0; u < NSLOT; ++u)
            if (u < U.n) {
                C v = w[u];
                for (int k = 0; k < U.mult[u]; ++k) v = to_c<C>(zscale(to_d2(v), r));
                U.p[u][i] = v;
            }
    }
}

// W[slot] /= *d_norm slot by slot (Normalize_4x4_GPU, WD4D:1366-1388), over
// the distinct pointers as k_dmask does
template <class C>
__global__ void __launch_bounds__(256) k_ddivide(USlots<C> U, long long n, const double* d_norm) {
    const double2 inv = zinv(make_double2(d_norm[0], d_norm[1]));
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        C w[NSLOT];
#pragma unroll
        for (int u = 0; u < NSLOT; ++u)
            if (u < U.n) w[u] = U.p[u][i];
#pragma unroll
        for (int u = 0; u < NSLOT; ++u)
            if (u < U.n) {
                C v = w[u];
                for (int k = 0; k < U.mult[u]; ++k) v = to_c<C>(zmul(to_d2(v), inv));
                U.p[u][i] = v;
            }
    }
}

template <class C>
__global__ void k_dreal(Slots<C> S, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        S.p[0][i].y = 0; S.p[5][i].y = 0; S.p[10][i].y = 0; S.p[15][i].y = 0;
    }
}

// projector (sign != 0, first) and kinetic sandwich (kin != 0) on the
// (lambda, p) grid: axis 0 p_y, 1 lambda_y, 2 p_x, 3 lambda_x
template <class C>
__global__ void __launch_bounds__(256, 2) k_dkinetic(Slots<C> S, DParams P, int sign, int kin, double dlx, double dly) {
    const long long n = (long long)P.n0 * P.n1 * P.n2 * P.n3;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int i0, i1, i2, i3;
        decode(i, P, i0, i1, i2, i3);
        const double py = P.cpy[i0], ly = P.ly[i1], px = P.cpx[i2], lx = P.lx[i3];
        double2 w[16];
        load16(S, i, w);
        if (sign != 0) {   // WD4D:1040-1148: W <- P(p+) W P(p-) / 4
            double pxp, pyp, pxm, pym;
            if (P.kvn) { pxp = pxm = px; pyp = pym = py; }
            else {
                pxp = px + 0.5 * P.hbar * lx; pyp = py + 0.5 * P.hbar * ly;
                pxm = px - 0.5 * P.hbar * lx; pym = py - 0.5 * P.hbar * ly;
            }
            const double c = P.c, m = P.mass, s = (double)sign;
            auto proj = [&](double qx, double qy) {
                const double K = c * sqrt(m * c * m * c + qx * qx + qy * qy);
                const double2 p11 = make_double2(1.0 + (c * c * m * s) / K, 0.0);
                const double2 p33 = make_double2(1.0 - (c * c * m * s) / K, 0.0);
                const double2 p14 = make_double2(s * (c * qx) / K, s * (-c * qy) / K);
                return spin_matrix(p11, p14, 1.0, p33);
            };
            const M4 L = proj(pxp, pyp), R = proj(pxm, pym);
#pragma unroll
            for (int k = 0; k < 16; ++k) w[k] = zscale(w[k], 0.25);
            sandwich<SPIN_NZ, SPIN_NZ>(L, w, R);
        }
        if (kin) {          // WD4D:392-481
            double pxp, pyp, pxm, pym;
            if (P.kvn) { pxp = 0.5 * lx; pyp = 0.5 * ly; pxm = -0.5 * lx; pym = -0.5 * ly; }
            else {
                pxp = px + 0.5 * P.hbar * lx; pyp = py + 0.5 * P.hbar * ly;
                pxm = px - 0.5 * P.hbar * lx; pym = py - 0.5 * P.hbar * ly;
            }
            double2 a, b, cc, d;
            kin_entries(pxp, pyp, P.mass, P.dt, P, a, b);
            kin_entries(pxm, pym, P.mass, -P.dt, P, cc, d);
            const M4 L = spin_matrix(a, b, -1.0, zconj(a)), R = spin_matrix(cc, d, -1.0, zconj(cc));
            sandwich<SPIN_NZ, SPIN_NZ>(L, w, R);
            const double r = exp(-P.dt * dlx * lx * lx - P.dt * dly * ly * ly);
#pragma unroll
            for (int k = 0; k < 16; ++k) w[k] = zscale(w[k], r);
        }
        store16(S, i, w);
    }
}

// potential sandwich on the (x, theta) grid: axis 0 theta_y, 1 y, 2 theta_x, 3 x
template <class C>
__global__ void __launch_bounds__(128, 4) k_dpotential(Slots<C> S, DParams P, DFactors<C> phase) {
    const long long n = (long long)P.n0 * P.n1 * P.n2 * P.n3;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int i0, i1, i2, i3;
        decode(i, P, i0, i1, i2, i3);
        double2 w[16];
        load16(S, i, w);
        // UL W UR, UR built only after UL has been applied (fewer live registers)
        const bool spin = P.kvn || P.a3zero;
        {
            const double A1m = a_field(P, 0, 0, i3, i2, i1, i0), A2m = a_field(P, 1, 0, i3, i2, i1, i0);
            const double A3m = P.a3zero ? 0.0 : a_field(P, 2, 0, i3, i2, i1, i0);
            const M4 UL = pot_matrix(A1m, A2m, A3m, P.dt, false, P);
            if (spin) left_apply<SPIN_NZ>(UL, w);
            else left_apply<DPOT_NZ>(UL, w);
        }
        {
            const double A1p = a_field(P, 0, 1, i3, i2, i1, i0), A2p = a_field(P, 1, 1, i3, i2, i1, i0);
            const double A3p = P.a3zero ? 0.0 : a_field(P, 2, 1, i3, i2, i1, i0);
            const M4 UR = pot_matrix(A1p, A2p, A3p, P.kvn ? P.dt : -P.dt, true, P);
            if (spin) right_apply<SPIN_NZ>(w, UR);
            else right_apply<DPOT_NZ>(w, UR);
        }
        const double2 ev = dfactor_at(phase, i0, i1, i2, i3, i);
#pragma unroll
        for (int k = 0; k < 16; ++k) w[k] = zmul(w[k], ev);
        store16(S, i, w);
    }
}

// ---- initial states on the (x, theta) grid (WD4D:908-1032) ----------------
__device__ __forceinline__ void psi14(double x, double y, double ux, double uy, double sx, double sy,
                                      const DParams& P, double2& p1, double2& p4) {
    const double c = P.c, m = P.mass;
    const double u0 = sqrt(ux * ux + uy * uy + c * c);
    const double ph = m * (x * ux + y * uy);
    double s, co;
    sincos(ph, &s, &co);
    const double g = exp(-0.5 * (x / sx) * (x / sx) - 0.5 * (y / sy) * (y / sy));
    p1 = make_double2(g * (c + u0) * co, g * (c + u0) * s);
    p4 = make_double2(g * (co * ux - s * uy), g * (s * ux + co * uy));
}

template <class C>
__global__ void k_dinit(Slots<C> S, DParams P, int kind, double a0, double a1, double a2, double a3, double a4,
                        double a5) {
    const long long n = (long long)P.n0 * P.n1 * P.n2 * P.n3;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int i0, i1, i2, i3;
        decode(i, P, i0, i1, i2, i3);
        const double x = P.cx[i3], tx = P.tx[i2], y = P.cy[i1], ty = P.ty[i0];
        const double hb = P.hbar;
        if (kind == 2) {   // Landau ground, W11 only
            const double xm = x - 0.5 * hb * tx - a1, ym = y - 0.5 * hb * ty - a2;
            const double xp = x + 0.5 * hb * tx - a1, yp = y + 0.5 * hb * ty - a2;
            const double f = exp(-a0 * 0.25 * xm * xm - a0 * 0.25 * ym * ym) *
                             exp(-a0 * 0.25 * xp * xp - a0 * 0.25 * yp * yp);
            S.p[0][i] = to_c<C>(make_double2(f, 0.0));
            continue;
        }
        // ParticleUp (kind 0) / Majorana (kind 1): a0 = u_x, a1 = u_y, a2 = x_mu, a3 = y_mu, a4 = sx, a5 = sy
        const double xm = x - 0.5 * hb * tx - a2, ym = y - 0.5 * hb * ty - a3;
        const double xp = x + 0.5 * hb * tx - a2, yp = y + 0.5 * hb * ty - a3;
        double2 p1m, p4m, p1p, p4p;
        psi14(xm, ym, a0, a1, a4, a5, P, p1m, p4m);
        psi14(xp, yp, a0, a1, a4, a5, P, p1p, p4p);
        if (kind == 1) {
            const double2 am = zadd(p1m, zscale(zconj(p4m), -1.0)), bm = zadd(p4m, zscale(zconj(p1m), -1.0));
            const double2 ap = zadd(p1p, zscale(zconj(p4p), -1.0)), bp = zadd(p4p, zscale(zconj(p1p), -1.0));
            p1m = am; p4m = bm; p1p = ap; p4p = bp;
        }
        S.p[0][i] = to_c<C>(zmul(p1m, zconj(p1p)));
        S.p[3][i] = to_c<C>(zmul(p1m, zconj(p4p)));
        S.p[12][i] = to_c<C>(zmul(p4m, zconj(p1p)));
        S.p[15][i] = to_c<C>(zmul(p4m, zconj(p4p)));
    }
}

// ---- reductions (WD4D:1156-1342, KvN:955-1140) ------------------------------
#define DSUM 20
// Sums, on the (x, p) grid:
//  0,1 sum trace (complex)   2 x tr  3 p_x tr  4 x^2 tr  5 p_x^2 tr  6 y tr  7 p_y tr
//  8 y^2 tr  9 p_y^2 tr  10 alpha1  11 alpha2  12 x alpha1  13 y alpha2  14 kinetic energy
//  15 potential energy  16 D1A0  17 D1A1  18 D1A2  19 unused
// Components the sums read (W11 W13 W14 W22 W23 W24 W31 W32 W33 W41 W42 W44).
constexpr unsigned RED_SLOTS = 0xffffu & ~((1u << 1) | (1u << 4) | (1u << 11) | (1u << 14));

// One point's contributions to the DSUM sums; w row-major W11..W44.
__device__ __forceinline__ void dreduce_point(const DParams& P, int i0, int i1, int i2, int i3,
                                              const double2 (&w)[16], double (&a)[DSUM]) {
    const long long nxy = (long long)P.n1 * P.n3;
    const double x = P.cx[i3], px = P.cpx[i2], y = P.cy[i1], py = P.cpy[i0];
    const double2 W11 = w[0], W22 = w[5], W33 = w[10], W44 = w[15];
    const double2 W14 = w[3], W41 = w[12], W23 = w[6], W32 = w[9];
    const double2 W13 = w[2], W24 = w[7], W31 = w[8], W42 = w[13];
    const double trr = W11.x + W22.x + W33.x + W44.x, tri = W11.y + W22.y + W33.y + W44.y;
    const double a1 = W14.x + W41.x + W23.x + W32.x;           // Re(W14+W41+W23+W32)
    const double a2 = -(W14.y - W41.y + W32.y - W23.y);        // -Im(W14-W41+W32-W23)
    const double mterm = W11.x + W22.x - W33.x - W44.x;
    const long long ixy = (long long)i1 * P.n3 + i3;
    const double A0 = P.obs_xy[ixy], A1 = P.obs_xy[nxy + ixy], A2 = P.obs_xy[2 * nxy + ixy];
    const double A3 = P.obs_xy[3 * nxy + ixy], D10 = P.obs_xy[4 * nxy + ixy];
    const double D11 = P.obs_xy[5 * nxy + ixy], D12 = P.obs_xy[6 * nxy + ixy];
    const double c = P.c;
    a[0] += trr; a[1] += tri;
    a[2] = fma(x, trr, a[2]); a[3] = fma(px, trr, a[3]);
    a[4] = fma(x * x, trr, a[4]); a[5] = fma(px * px, trr, a[5]);
    a[6] = fma(y, trr, a[6]); a[7] = fma(py, trr, a[7]);
    a[8] = fma(y * y, trr, a[8]); a[9] = fma(py * py, trr, a[9]);
    a[10] += a1; a[11] += a2;
    a[12] = fma(x, a1, a[12]); a[13] = fma(y, a2, a[13]);
    // c p_x Re(W14+W41+W32+W23) - c p_y Im(W14-W41+W32-W23) + m c^2 Re(W11+W22-W33-W44)
    a[14] += c * px * a1 + c * py * a2 + P.mass * c * c * mterm;
    if (P.kvn) {   // KvN:1107-1109, 1137
        const double k2 = W14.y - W41.y - W23.y + W32.y;
        a[15] += A1 * c * a1 - A2 * c * k2 + c * A0 * trr;
        a[18] += c * D12 * (W14.x - W41.x - W23.x + W32.x);
    } else {       // WD4D:1309-1312, 1340
        const double e2 = -W14.y + W23.y - W32.y + W41.y;
        const double e3 = -W13.x + W24.x - W31.x + W42.x;
        a[15] += A1 * c * (-a1) - A2 * c * e2 + A3 * c * e3 + c * A0 * trr;
        a[18] += -D12 * c * e2;
    }
    a[16] += c * D10 * trr;
    a[17] += c * D11 * a1;
}

// The block's sums -> one partial row (256 threads).
__device__ __forceinline__ void dreduce_block(double (&a)[DSUM], double* __restrict__ partials) {
    __shared__ double sm[DSUM * 8];
#pragma unroll
    for (int k = 0; k < DSUM; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_down_sync(0xffffffffu, a[k], o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
        for (int k = 0; k < DSUM; ++k) sm[w * DSUM + k] = a[k];
    __syncthreads();
    if (threadIdx.x < DSUM) {
        double t = 0.0;
        for (int k = 0; k < 8; ++k) t += sm[k * DSUM + threadIdx.x];
        partials[(long long)blockIdx.x * DSUM + threadIdx.x] = t;
    }
}

template <class C>
__global__ void __launch_bounds__(256) k_dreduce(Slots<C> S, DParams P, double* __restrict__ partials) {
    double a[DSUM];
#pragma unroll
    for (int k = 0; k < DSUM; ++k) a[k] = 0.0;
    const long long n = (long long)P.n0 * P.n1 * P.n2 * P.n3;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int i0, i1, i2, i3;
        decode(i, P, i0, i1, i2, i3);
        double2 w[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) w[k] = ((RED_SLOTS >> k) & 1u) ? to_d2(S.p[k][i]) : make_double2(0.0, 0.0);
        dreduce_point(P, i0, i1, i2, i3, w, a);
    }
    dreduce_block(a, partials);
}

// The Run() loop's first three passes in one: boundary_xp (k_dmask kind 1),
// Real_GPU of the diagonal (k_dreal) and the sums (k_dreduce) of the result.
// Needs distinct component pointers; the sums see the stored (rounded)
// values, as k_dreduce would.
template <class C>
__global__ void __launch_bounds__(256, 2) k_dmask_real_reduce(Slots<C> S, DParams P, double* __restrict__ partials) {
    double a[DSUM];
#pragma unroll
    for (int k = 0; k < DSUM; ++k) a[k] = 0.0;
    const long long n = (long long)P.n0 * P.n1 * P.n2 * P.n3;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int i0, i1, i2, i3;
        decode(i, P, i0, i1, i2, i3);
        const double r = P.mxp[2][i2] * P.mxp[0][i0] * P.mxp[3][i3] * P.mxp[1][i1];
        double2 w[16];
        load16(S, i, w);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            C v = to_c<C>(zscale(w[k], r));
            if (k == 0 || k == 5 || k == 10 || k == 15) v.y = 0;
            S.p[k][i] = v;
            w[k] = to_d2(v);
        }
        dreduce_point(P, i0, i1, i2, i3, w, a);
    }
    dreduce_block(a, partials);
}

// The fused Theta -> P epilogue's per-plane rows -> EPI_FOLD rows: block b
// adds its contiguous share of the rows, one warp per column (a fixed order).
#define EPI_FOLD 256
static_assert(DSUM == DEPI_SUMS, "the epilogue rows have the layout of the reductions");
__global__ void k_dfold(const double* __restrict__ rows, int nrows, double* __restrict__ out) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int per = (nrows + gridDim.x - 1) / gridDim.x, r0 = blockIdx.x * per;
    const int r1 = r0 + per < nrows ? r0 + per : nrows;
    double t = 0.0;
    for (int r = r0 + l; r < r1; r += 32) t += rows[(long long)r * DSUM + w];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (l == 0) out[(long long)blockIdx.x * DSUM + w] = t;
}

// out: [norm_re, norm_im, 17 observables] = WIGD_NOBS values.  When divide,
// observables are divided by the trace norm as Run() sees them after
// Normalize (the real part of 1/norm: the sums are of real parts); else they
// are the sums of the state as given.
__global__ void k_dfinalize(const double* __restrict__ part, int nblk, double dv_norm, double dv_obs, int divide,
                            double* out, int* counter, int max_rows, double* cur_norm, int* flag) {
    __shared__ double S[DSUM];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (w < DSUM) {
        double t = 0.0;
        for (int r = l; r < nblk; r += 32) t += part[(long long)r * DSUM + w];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (l == 0) S[w] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double2 n = make_double2(S[0] * dv_norm, S[1] * dv_norm);
        const double2 inv = divide ? zinv(n) : make_double2(1.0, 0.0);
        double row[WIGD_NOBS];
        row[0] = n.x; row[1] = n.y;
        for (int k = 2; k < 19; ++k) row[k] = dv_obs * S[k] * inv.x;
        double* dst = out;
        if (counter) {
            const int r = *counter;
            dst = (r < max_rows) ? out + (long long)r * WIGD_NOBS : nullptr;
            *counter = r + 1;
        }
        bool bad = false;
        for (int k = 0; k < WIGD_NOBS; ++k) bad |= !isfinite(row[k]);
        if (bad && flag) *flag = WIG_ERR_NONFINITE;
        if (dst)
            for (int k = 0; k < WIGD_NOBS; ++k) dst[k] = row[k];
        if (cur_norm) { cur_norm[0] = n.x; cur_norm[1] = n.y; }
    }
}

// ---- 2-D transforms of one component plane (forward or inverse) ------------
// KIND 0: plane (axis 1 rows, axis 3 columns) at fixed (axis 0, axis 2)
// KIND 1: plane (axis 0 rows, axis 2 columns) at fixed (axis 1, axis 3)
// value_out = scale * S * DFT2(S * value_in), S = (-1)^(row+col), which is
// the pair of FAFT calls for |delta| N = 1 with N/2 even.
template <class C, int NA, int NB, int NT, int KIND, bool FWD>
__global__ void __launch_bounds__(NT) k_dplane(const __grid_constant__ Slots<C> S, int n0, int n1, int n2, int n3, double2 scale,
                                               const double* __restrict__ d_norm) {
    extern __shared__ __align__(16) unsigned char smraw[];
    C* s = reinterpret_cast<C*>(smraw);
    constexpr int LD = NB + 1;
    C* twb = s + NA * LD;
    C* twa = twb + NB;
    make_twiddles(twb, NB);
    if (NA != NB) make_twiddles(twa, NA);
    const C* ta = (NA != NB) ? twa : twb;
    C* base = S.p[blockIdx.y];
    long long off, rs, cs;
    if (KIND == 0) {   // fixed (i0, i2); rows i1 (stride n2*n3), columns i3 (stride 1)
        const int i2 = blockIdx.x % n2, i0 = blockIdx.x / n2;
        off = ((long long)i0 * n1 * n2 + i2) * n3; rs = (long long)n2 * n3; cs = 1;
    } else {           // fixed (i1, i3); rows i0 (stride n1*n2*n3), columns i2 (stride n3)
        const int i3 = blockIdx.x % n3, i1 = blockIdx.x / n3;
        off = (long long)i1 * n2 * n3 + i3; rs = (long long)n1 * n2 * n3; cs = n3;
    }
    C* g = base + off;
    double2 sc = scale;
    if (d_norm) sc = zmul(sc, zinv(make_double2(d_norm[0], d_norm[1])));
    const C cc = to_c<C>(sc);
    for (int e = threadIdx.x; e < NA * NB; e += NT) {
        const int a = e / NB, b = e % NB;
        C v = g[a * rs + b * cs];
        if ((a + b) & 1) v = cneg(v);
        s[a * LD + b] = v;
    }
    __syncthreads();
    const LineMap rows{1, LD, 0, 1}, cols{1, 1, 0, LD};
    fft_lines<C, NB, NA, NT, FWD, true>(s, rows, twb);
    fft_lines<C, NA, NB, NT, FWD, true>(s, cols, ta);
    for (int e = threadIdx.x; e < NA * NB; e += NT) {
        const int a = e / NB, b = e % NB;
        C v = cmul(s[a * LD + b], cc);
        if ((a + b) & 1) v = cneg(v);
        g[a * rs + b * cs] = v;
    }
}

// KIND 1 over G neighbouring columns i3 per CTA.  A (axis 0, axis 2) plane at
// fixed (i1, i3) is a gather at stride N_3; G = 32 bytes / element makes every
// access one whole 32-byte sector, copied by cp.async straight into shared
// memory.  The centring signs are folded into the store:
//   S DFT2(S v)[k] = (-1)^(ka + kb) DFT2(v)[k + N/2],
// so the transform reads its plane unsigned and the store reads the result
// at frequencies shifted by N/2.
template <int NA, int LD>
struct DPlaneG {
    static constexpr int PSP = ((NA * LD + 13) / 16) * 16 + 2;   // plane stride, = 2 (mod 16)
};
template <class C, int NA, int NB, int NT, bool FWD, int G>
__global__ void __launch_bounds__(NT) k_dplane_g(const __grid_constant__ Slots<C> S, int n0, int n1, int n2, int n3, double2 scale,
                                                 const double* __restrict__ d_norm) {
    extern __shared__ __align__(16) unsigned char smraw[];
    constexpr int LD = NB + 1, PSP = DPlaneG<NA, LD>::PSP;
    C* s = reinterpret_cast<C*>(smraw);
    C* twb = s + G * PSP;
    C* twa = twb + NB;
    const int n3g = n3 / G;
    const int i3 = (blockIdx.x % n3g) * G, i1 = blockIdx.x / n3g;
    const long long rs = (long long)n1 * n2 * n3, cs = n3;
    C* g0 = S.p[blockIdx.y] + (long long)i1 * n2 * n3 + i3;
    for (int e = threadIdx.x; e < G * NA * NB; e += NT) {
        const int g = e % G, b = (e / G) % NB, a = e / (G * NB);
        cp_async_elem(s + g * PSP + a * LD + b, g0 + a * rs + b * cs + g);
    }
    make_twiddles(twb, NB);
    if (NA != NB) make_twiddles(twa, NA);
    const C* ta = (NA != NB) ? twa : twb;
    double2 sc = scale;
    if (d_norm) sc = zmul(sc, zinv(make_double2(d_norm[0], d_norm[1])));
    const C cc = to_c<C>(sc);
    cp_async_wait_all();
    __syncthreads();
    const LineMap rows{1, LD, 0, 1}, cols{1, 1, 0, LD};
    for (int g = 0; g < G; ++g) {
        fft_lines<C, NB, NA, NT, FWD, true>(s + g * PSP, rows, twb);
        fft_lines<C, NA, NB, NT, FWD, true>(s + g * PSP, cols, ta);
    }
    for (int e = threadIdx.x; e < G * NA * NB; e += NT) {
        const int g = e % G, b = (e / G) % NB, a = e / (G * NB);
        const int sa = (a + NA / 2) % NA, sb = (b + NB / 2) % NB;
        C v = cmul(s[g * PSP + sa * LD + sb], cc);
        if ((a + b) & 1) v = cneg(v);
        g0[a * rs + b * cs + g] = v;
    }
}

// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------
struct wigd_plan {
    wigd_desc d;
    long long npts;
    int esz;
    double* dmem;            // coordinates, masks, rank tables, observable tables
    void* tabs;              // A0 phase factor tables
    DFactors<double2> ph_d;
    DFactors<float2> ph_f;
    DParams P;
    double* partials;
    double* cur_norm;        // 2 doubles + counter/flag ints
    int* counter;
    int* flag;
    int nblk;
    void* tw64;              // twiddles of k_dplane_r4 (64^4 grids only)
    double* afull;           // full A1..A3 tables (fields that are not of low rank)
    double* epi_rows;        // 64^4: per-plane sums of the fused Theta -> P epilogue [16][4096][DSUM]
    double* epi_fold;        // and their EPI_FOLD folded rows
};

static unsigned dgrid(long long n, int threads = 256, int per_sm = 8) {
    long long b = (n + threads - 1) / threads, cap = (long long)wig_num_sms() * per_sm;
    return (unsigned)(b < cap ? (b > 0 ? b : 1) : cap);
}

static void free_dplan(wigd_plan* p) {
    if (!p) return;
    cudaFree(p->dmem);
    cudaFree(p->tabs);
    cudaFree(p->partials);
    cudaFree(p->cur_norm);
    cudaFree(p->tw64);
    cudaFree(p->epi_rows);
    cudaFree(p->epi_fold);
    cudaFree(p->afull);
    delete p;
}

extern "C" int wigd_plan_create(const wigd_desc* desc, wigd_plan** out) {
    if (!desc || !out) return WIG_ERR_INVALID_ARG;
    *out = nullptr;
    if (desc->dtype != WIG_C128 && desc->dtype != WIG_C64) return WIG_ERR_INVALID_ARG;
    for (int a = 0; a < 4; ++a) {
        if (desc->shape[a] < 2 || desc->shape[a] > 1024 || (desc->shape[a] & 1)) return WIG_ERR_UNSUPPORTED;
        if (!desc->coord[a] || !desc->acoord[a] || !desc->mask_xp[a] || !desc->mask_p[a]) return WIG_ERR_INVALID_ARG;
    }
    if (desc->a_rank < 0 || desc->a_rank > 16 || (desc->a_rank > 0 && !desc->a_tabs) || !desc->obs_xy ||
        (desc->a_full && desc->a_rank != 0) ||
        desc->n_phase < 0 || desc->n_phase > WIG_MAX_FACTORS)
        return WIG_ERR_INVALID_ARG;
    wigd_plan* p = new wigd_plan();
    memset(p, 0, sizeof(*p));
    p->d = *desc;
    const int N0 = desc->shape[0], N1 = desc->shape[1], N2 = desc->shape[2], N3 = desc->shape[3];
    p->npts = (long long)N0 * N1 * N2 * N3;
    if (p->npts >= (1LL << 31)) { delete p; return WIG_ERR_UNSUPPORTED; }   // 32-bit point indices
    p->esz = desc->dtype == WIG_C128 ? 16 : 8;
    const int ns[4] = {N0, N1, N2, N3};
    // ---- float64 tables in one allocation ----
    const long long nu = (long long)N3 * N2, nv = (long long)N1 * N0;
    std::vector<double> h;
    long long offs[4][4];
    for (int a = 0; a < 4; ++a) {
        const double* srcs[4] = {desc->coord[a], desc->acoord[a], desc->mask_xp[a], desc->mask_p[a]};
        for (int t = 0; t < 4; ++t) {
            offs[a][t] = (long long)h.size();
            h.insert(h.end(), srcs[t], srcs[t] + ns[a]);
        }
    }
    const long long off_a = h.size();
    if (desc->a_rank > 0) {
        // the u part of each table, given as [ix][itx], is stored as [itx][ix] so
        // that neighbouring x points read neighbouring words
        h.insert(h.end(), desc->a_tabs, desc->a_tabs + 6LL * desc->a_rank * (nu + nv));
        for (long long b = 0; b < 6LL * desc->a_rank; ++b) {
            const double* src = desc->a_tabs + b * (nu + nv);
            double* dst = h.data() + off_a + b * (nu + nv);
            for (int ix = 0; ix < N3; ++ix)
                for (int itx = 0; itx < N2; ++itx) dst[(long long)itx * N3 + ix] = src[(long long)ix * N2 + itx];
        }
    }
    const long long off_o = h.size();
    h.insert(h.end(), desc->obs_xy, desc->obs_xy + 7LL * N1 * N3);
    if (cudaMalloc(&p->dmem, h.size() * sizeof(double)) != cudaSuccess) { free_dplan(p); return WIG_ERR_ALLOC; }
    cudaMemcpy(p->dmem, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
    double* D = p->dmem;
    DParams& P = p->P;
    P.n0 = N0; P.n1 = N1; P.n2 = N2; P.n3 = N3;
    auto lg = [](int n) { int l = 0; while ((1 << l) < n) ++l; return (1 << l) == n ? l : -1; };
    P.pow2 = lg(N0) >= 0 && lg(N1) >= 0 && lg(N2) >= 0 && lg(N3) >= 0;
    if (P.pow2) { P.s3 = lg(N3); P.s32 = P.s3 + lg(N2); P.s321 = P.s32 + lg(N1); }
    P.kvn = desc->kvn;
    P.c = desc->c; P.hbar = desc->hbar; P.mass = desc->mass; P.dt = desc->dt; P.m_pot = desc->m_pot;
    P.cpy = D + offs[0][0]; P.cy = D + offs[1][0]; P.cpx = D + offs[2][0]; P.cx = D + offs[3][0];
    P.ty = D + offs[0][1]; P.ly = D + offs[1][1]; P.tx = D + offs[2][1]; P.lx = D + offs[3][1];
    for (int a = 0; a < 4; ++a) { P.mxp[a] = D + offs[a][2]; P.mp[a] = D + offs[a][3]; }
    P.arank = desc->a_rank;
    P.atab = D + off_a;
    // A3 = sum_r u_r(x, theta_x) v_r(y, theta_y) on both sides: zero when every
    // rank term has an all-zero factor (or there is no rank term)
    P.a3zero = 1;
    for (int side = 0; side < 2 && P.a3zero; ++side)
        for (int r = 0; r < desc->a_rank; ++r) {
            const double* f = desc->a_tabs + ((long long)(2 * 2 + side) * desc->a_rank + r) * (nu + nv);
            bool uz = true, vz = true;
            for (long long e = 0; e < nu && uz; ++e) uz = f[e] == 0.0;
            for (long long e = 0; e < nv && vz; ++e) vz = f[nu + e] == 0.0;
            if (!uz && !vz) { P.a3zero = 0; break; }
        }
    if (desc->a_full) {
        // fields without a low-rank form: A_k at both Bopp sides on every point
        const size_t nb = 6 * (size_t)p->npts * sizeof(double);
        if (cudaMalloc(&p->afull, nb) != cudaSuccess) { free_dplan(p); return WIG_ERR_ALLOC; }
        cudaMemcpy(p->afull, desc->a_full, nb, cudaMemcpyHostToDevice);
        P.afull = p->afull;
        P.a3zero = 1;
        for (long long e = 4 * p->npts; e < 6 * p->npts && P.a3zero; ++e) P.a3zero = desc->a_full[e] == 0.0;
    }
    P.obs_xy = D + off_o;
    // ---- A0 phase factor tables ----
    auto tab_elems = [&](const wig_factor& f) -> long long {
        if (f.axis_a < 0) return p->npts;
        if (f.axis_b < 0) return ns[f.axis_a];
        return (long long)ns[f.axis_a] * ns[f.axis_b];
    };
    long long te = 0;
    for (int i = 0; i < desc->n_phase; ++i) {
        if (!desc->phase[i].host_data) { free_dplan(p); return WIG_ERR_INVALID_ARG; }
        te += tab_elems(desc->phase[i]);
    }
    if (te > 0 && cudaMalloc(&p->tabs, te * p->esz) != cudaSuccess) { free_dplan(p); return WIG_ERR_ALLOC; }
    long long off = 0;
    p->ph_d.n = p->ph_f.n = desc->n_phase;
    for (int i = 0; i < desc->n_phase; ++i) {
        const wig_factor& f = desc->phase[i];
        const long long n = tab_elems(f);
        char* base = reinterpret_cast<char*>(p->tabs) + off * p->esz;
        if (desc->dtype == WIG_C128) cudaMemcpy(base, f.host_data, n * 16, cudaMemcpyHostToDevice);
        else {
            std::vector<float> tmp(2 * n);
            for (long long k = 0; k < 2 * n; ++k) tmp[k] = (float)f.host_data[k];
            cudaMemcpy(base, tmp.data(), n * 8, cudaMemcpyHostToDevice);
        }
        p->ph_d.data[i] = (const double2*)base; p->ph_f.data[i] = (const float2*)base;
        p->ph_d.ia[i] = p->ph_f.ia[i] = f.axis_a;
        p->ph_d.ib[i] = p->ph_f.ib[i] = f.axis_b;
        p->ph_d.nb[i] = p->ph_f.nb[i] = f.axis_b >= 0 ? ns[f.axis_b] : 1;
        off += n;
    }
    p->nblk = wig_num_sms() * 4;
    if (cudaMalloc(&p->partials, (size_t)p->nblk * DSUM * sizeof(double)) != cudaSuccess) { free_dplan(p); return WIG_ERR_ALLOC; }
    if (cudaMalloc(&p->cur_norm, 4 * sizeof(double)) != cudaSuccess) { free_dplan(p); return WIG_ERR_ALLOC; }
    p->counter = reinterpret_cast<int*>(p->cur_norm + 2);
    p->flag = p->counter + 1;
    cudaMemset(p->cur_norm, 0, 4 * sizeof(double));
    for (int a = 0; a < 4; ++a) {
        const bool fast = (ns[a] == 16 || ns[a] == 32 || ns[a] == 64 || ns[a] == 128) &&
                          fabs(fabs(desc->delta[a]) * ns[a] - 1.0) < 1e-12;
        if (!fast && !wig_dense_matrix(ns[a], fabs(desc->delta[a]), desc->dtype, 0)) { free_dplan(p); return WIG_ERR_ALLOC; }
    }
    if (N0 == 64 && N1 == 64 && N2 == 64 && N3 == 64) {
        if (cudaMalloc(&p->tw64, 64 * sizeof(double2)) != cudaSuccess) { free_dplan(p); return WIG_ERR_ALLOC; }
        if (wig_r4_twiddles(p->tw64, desc->dtype, 0) != WIG_OK) { free_dplan(p); return WIG_ERR_CUDA; }
        if (cudaMalloc(&p->epi_rows, (size_t)NSLOT * 4096 * DSUM * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&p->epi_fold, (size_t)EPI_FOLD * DSUM * sizeof(double)) != cudaSuccess) {
            free_dplan(p); return WIG_ERR_ALLOC;
        }
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { wig_set_cuda_error(e, "wigd_plan_create"); free_dplan(p); return WIG_ERR_CUDA; }
    *out = p;
    return WIG_OK;
}

extern "C" int wigd_plan_destroy(wigd_plan* p) {
    if (!p) return WIG_ERR_INVALID_ARG;
    cudaDeviceSynchronize();
    free_dplan(p);
    return WIG_OK;
}

template <class C>
static int make_slots(void* const* slots, Slots<C>& S, bool allow_alias) {
    if (!slots) return WIG_ERR_INVALID_ARG;
    for (int k = 0; k < NSLOT; ++k) {
        if (!slots[k]) return WIG_ERR_INVALID_ARG;
        S.p[k] = reinterpret_cast<C*>(slots[k]);
    }
    if (!allow_alias)
        for (int a = 0; a < NSLOT; ++a)
            for (int b = a + 1; b < NSLOT; ++b)
                if (slots[a] == slots[b]) return WIG_ERR_ALIAS;
    return WIG_OK;
}

template <class C>
static USlots<C> unique_slots(const Slots<C>& S) {
    USlots<C> U;
    U.n = 0;
    for (int k = 0; k < NSLOT; ++k) {
        U.p[k] = nullptr;
        U.mult[k] = 0;
    }
    for (int k = 0; k < NSLOT; ++k) {
        int u = 0;
        while (u < U.n && U.p[u] != S.p[k]) ++u;
        if (u == U.n) U.p[U.n++] = S.p[k];
        ++U.mult[u];
    }
    return U;
}

#define DISPATCH(p, body_c128, body_c64) \
    ((p)->d.dtype == WIG_C128 ? (body_c128) : (body_c64))

template <class C>
static int mask_impl(wigd_plan* p, void* const* slots, int kind, cudaStream_t st) {
    Slots<C> S;
    int r = make_slots(slots, S, true);
    if (r) return r;
    k_dmask<C><<<dgrid(p->npts), 256, 0, st>>>(unique_slots(S), p->P, kind);
    WIG_LAUNCHED("k_dmask");
    return WIG_OK;
}

// Replace the plan's mask factors (host float64, one vector per axis).
extern "C" int wigd_set_mask(wigd_plan* p, int kind, const double* const* factors) {
    if (!p || !factors || (kind != 1 && kind != 2)) return WIG_ERR_INVALID_ARG;
    const int ns[4] = {p->P.n0, p->P.n1, p->P.n2, p->P.n3};
    for (int a = 0; a < 4; ++a) {
        if (!factors[a]) return WIG_ERR_INVALID_ARG;
        double* dst = const_cast<double*>(kind == 1 ? p->P.mxp[a] : p->P.mp[a]);
        WIG_CUDA(cudaMemcpy(dst, factors[a], ns[a] * sizeof(double), cudaMemcpyHostToDevice));
    }
    return WIG_OK;
}

extern "C" int wigd_mask(wigd_plan* p, void* const* slots, int kind, void* stream) {
    if (!p || (kind != 1 && kind != 2)) return WIG_ERR_INVALID_ARG;
    return DISPATCH(p, mask_impl<double2>(p, slots, kind, as_stream(stream)),
                    mask_impl<float2>(p, slots, kind, as_stream(stream)));
}

template <class C>
static int real_impl(wigd_plan* p, void* const* slots, cudaStream_t st) {
    Slots<C> S;
    int r = make_slots(slots, S, true);
    if (r) return r;
    k_dreal<C><<<dgrid(p->npts), 256, 0, st>>>(S, p->npts);
    WIG_LAUNCHED("k_dreal");
    return WIG_OK;
}
extern "C" int wigd_real_diag(wigd_plan* p, void* const* slots, void* stream) {
    if (!p) return WIG_ERR_INVALID_ARG;
    return DISPATCH(p, real_impl<double2>(p, slots, as_stream(stream)), real_impl<float2>(p, slots, as_stream(stream)));
}

template <class C>
static int divide_impl(wigd_plan* p, void* const* slots, const double* d_norm, cudaStream_t st) {
    Slots<C> S;
    int r = make_slots(slots, S, true);
    if (r) return r;
    k_ddivide<C><<<dgrid(p->npts), 256, 0, st>>>(unique_slots(S), p->npts, d_norm);
    WIG_LAUNCHED("k_ddivide");
    return WIG_OK;
}
extern "C" int wigd_divide(wigd_plan* p, void* const* slots, const double* d_norm, void* stream) {
    if (!p || !d_norm) return WIG_ERR_INVALID_ARG;
    return DISPATCH(p, divide_impl<double2>(p, slots, d_norm, as_stream(stream)),
                    divide_impl<float2>(p, slots, d_norm, as_stream(stream)));
}

template <class C>
static int reduce_impl(wigd_plan* p, void* const* slots, double* d_out, int divide, int* counter, int rows,
                       cudaStream_t st) {
    Slots<C> S;
    int r = make_slots(slots, S, true);
    if (r) return r;
    k_dreduce<C><<<p->nblk, 256, 0, st>>>(S, p->P, p->partials);
    WIG_LAUNCHED("k_dreduce");
    k_dfinalize<<<1, 32 * DSUM, 0, st>>>(p->partials, p->nblk, p->d.dv_norm, p->d.dv_obs, divide, d_out, counter,
                                         rows, p->cur_norm, p->flag);
    WIG_LAUNCHED("k_dfinalize");
    return WIG_OK;
}
extern "C" int wigd_reduce(wigd_plan* p, void* const* slots, double* d_out, int divide, void* stream) {
    if (!p || !d_out) return WIG_ERR_INVALID_ARG;
    return DISPATCH(p, reduce_impl<double2>(p, slots, d_out, divide, nullptr, 0, as_stream(stream)),
                    reduce_impl<float2>(p, slots, d_out, divide, nullptr, 0, as_stream(stream)));
}
extern "C" const double* wigd_norm_ptr(wigd_plan* p) { return p ? p->cur_norm : nullptr; }

template <class C>
static int kinetic_impl(wigd_plan* p, void* const* slots, int sign, int kin, cudaStream_t st) {
    Slots<C> S;
    int r = make_slots(slots, S, true);
    if (r) return r;
    k_dkinetic<C><<<dgrid(p->npts), 256, 0, st>>>(S, p->P, sign, kin, p->d.d_lambda_x, p->d.d_lambda_y);
    WIG_LAUNCHED("k_dkinetic");
    return WIG_OK;
}
extern "C" int wigd_kinetic(wigd_plan* p, void* const* slots, int projector_sign, int kinetic, void* stream) {
    if (!p) return WIG_ERR_INVALID_ARG;
    return DISPATCH(p, kinetic_impl<double2>(p, slots, projector_sign, kinetic, as_stream(stream)),
                    kinetic_impl<float2>(p, slots, projector_sign, kinetic, as_stream(stream)));
}

template <class C> static const DFactors<C>& phase_set(wigd_plan* p);
template <> const DFactors<double2>& phase_set<double2>(wigd_plan* p) { return p->ph_d; }
template <> const DFactors<float2>& phase_set<float2>(wigd_plan* p) { return p->ph_f; }

template <class C>
static int potential_impl(wigd_plan* p, void* const* slots, cudaStream_t st) {
    Slots<C> S;
    int r = make_slots(slots, S, true);
    if (r) return r;
    k_dpotential<C><<<dgrid(p->npts, 128, 16), 128, 0, st>>>(S, p->P, phase_set<C>(p));
    WIG_LAUNCHED("k_dpotential");
    return WIG_OK;
}
extern "C" int wigd_potential(wigd_plan* p, void* const* slots, void* stream) {
    if (!p) return WIG_ERR_INVALID_ARG;
    return DISPATCH(p, potential_impl<double2>(p, slots, as_stream(stream)),
                    potential_impl<float2>(p, slots, as_stream(stream)));
}

template <class C>
static int init_impl(wigd_plan* p, void* const* slots, int kind, const double* a, cudaStream_t st) {
    Slots<C> S;
    int r = make_slots(slots, S, true);
    if (r) return r;
    k_dinit<C><<<dgrid(p->npts), 256, 0, st>>>(S, p->P, kind, a[0], a[1], a[2], a[3], a[4], a[5]);
    WIG_LAUNCHED("k_dinit");
    return WIG_OK;
}
extern "C" int wigd_init_particle_up(wigd_plan* p, void* const* slots, double ux, double uy, double x_mu,
                                     double y_mu, double sx, double sy, void* stream) {
    if (!p) return WIG_ERR_INVALID_ARG;
    const double a[6] = {ux, uy, x_mu, y_mu, sx, sy};
    return DISPATCH(p, init_impl<double2>(p, slots, 0, a, as_stream(stream)), init_impl<float2>(p, slots, 0, a, as_stream(stream)));
}
extern "C" int wigd_init_majorana(wigd_plan* p, void* const* slots, double ux, double uy, double x_mu,
                                  double y_mu, double sx, double sy, void* stream) {
    if (!p) return WIG_ERR_INVALID_ARG;
    const double a[6] = {ux, uy, x_mu, y_mu, sx, sy};
    return DISPATCH(p, init_impl<double2>(p, slots, 1, a, as_stream(stream)), init_impl<float2>(p, slots, 1, a, as_stream(stream)));
}
extern "C" int wigd_init_landau(wigd_plan* p, void* const* slots, double B, double x_off, double y_off, void* stream) {
    if (!p) return WIG_ERR_INVALID_ARG;
    const double a[6] = {B, x_off, y_off, 0, 0, 0};
    return DISPATCH(p, init_impl<double2>(p, slots, 2, a, as_stream(stream)), init_impl<float2>(p, slots, 2, a, as_stream(stream)));
}

// ---- transforms ----
#define DPLANE_CASES(X) X(16, 16) X(32, 32) X(64, 64) X(128, 128) X(64, 128) X(128, 64)

template <class C, int KIND, bool FWD>
static int launch_dplane(wigd_plan* p, const Slots<C>& S, int nslots, double2 sc, const double* d_norm, cudaStream_t st,
                         const DEpi* epi = nullptr) {
    const int NA = KIND == 0 ? p->d.shape[1] : p->d.shape[0];
    const int NB = KIND == 0 ? p->d.shape[3] : p->d.shape[2];
    const unsigned planes = KIND == 0 ? (unsigned)(p->d.shape[0] * p->d.shape[2]) : (unsigned)(p->d.shape[1] * p->d.shape[3]);
    dim3 grid(planes, nslots);
    if (p->tw64 && !getenv("WIG_NO_DPLANE_R4")) {   // 64^4: radix-4 register transform
        void* ptrs[NSLOT];
        for (int k = 0; k < nslots; ++k) ptrs[k] = S.p[k];
        return wig_dplane64(ptrs, nslots, p->d.dtype, KIND, FWD ? 1 : 0, sc.x, d_norm, p->tw64, st, epi);
    }
    if (epi) return WIG_ERR_UNSUPPORTED;
    constexpr int G = 32 / (int)sizeof(C);
#define DCASE(a, b)                                                                              \
    if (NA == a && NB == b) {                                                                    \
        constexpr int NT = (a * b / 8 >= 512) ? 512 : 256;                                       \
        if (KIND == 1 && p->d.shape[3] % G == 0 && !getenv("WIG_NO_DPLANE_G")) {                 \
            auto kg = k_dplane_g<C, a, b, NT, FWD, G>;                                           \
            const size_t smg = sizeof(C) * ((size_t)G * DPlaneG<a, b + 1>::PSP + a + b);         \
            if (smg <= 227 * 1024) {                                                             \
                WIG_CUDA(cudaFuncSetAttribute(kg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smg)); \
                kg<<<dim3(planes / G, nslots), NT, smg, st>>>(S, p->d.shape[0], p->d.shape[1],   \
                                                              p->d.shape[2], p->d.shape[3], sc, d_norm); \
                WIG_LAUNCHED("k_dplane_g");                                                      \
                return WIG_OK;                                                                   \
            }                                                                                    \
        }                                                                                        \
        auto kern = k_dplane<C, a, b, NT, KIND, FWD>;                                            \
        const size_t sm = sizeof(C) * ((size_t)a * (b + 1) + a + b);                             \
        if (sm > 227 * 1024) return WIG_ERR_UNSUPPORTED;                                        \
        WIG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)); \
        kern<<<grid, NT, sm, st>>>(S, p->d.shape[0], p->d.shape[1], p->d.shape[2], p->d.shape[3], sc, d_norm); \
        WIG_LAUNCHED("k_dplane");                                                                \
        return WIG_OK;                                                                           \
    }
    DPLANE_CASES(DCASE)
#undef DCASE
    return WIG_ERR_UNSUPPORTED;
}

// which: 0 X->Lambda, 1 Lambda->X, 2 P->Theta, 3 Theta->P.
template <class C>
static int transform_impl(wigd_plan* p, void* const* slots, int nslots, int which, const double* d_norm, cudaStream_t st,
                          const DEpi* epi = nullptr) {
    if (nslots < 1 || nslots > NSLOT) return WIG_ERR_INVALID_ARG;
    Slots<C> S;
    for (int k = 0; k < NSLOT; ++k) S.p[k] = nullptr;
    for (int k = 0; k < nslots; ++k) {
        if (!slots[k]) return WIG_ERR_INVALID_ARG;
        S.p[k] = reinterpret_cast<C*>(slots[k]);
        for (int j = 0; j < k; ++j)
            if (slots[j] == slots[k]) return WIG_ERR_ALIAS;   // one launch transforms the slots concurrently
    }
    const int kind = which < 2 ? 0 : 1;
    const int ax_a = kind == 0 ? 1 : 0, ax_b = kind == 0 ? 3 : 2;
    const double sgn = (which == 0 || which == 2) ? 1.0 : -1.0;
    const int* ns = p->d.shape;
    auto fast = [&](int a) {
        return (ns[a] == 16 || ns[a] == 32 || ns[a] == 64 || ns[a] == 128) &&
               fabs(fabs(p->d.delta[a]) * ns[a] - 1.0) < 1e-12;
    };
    const double post = p->d.post[which];
    if (fast(ax_a) && fast(ax_b)) {
        const double sc = post * (2.0 * ns[ax_a] * p->d.d[ax_a]) * (2.0 * ns[ax_b] * p->d.d[ax_b]);
        int r;
        if (kind == 0) r = sgn > 0 ? launch_dplane<C, 0, true>(p, S, nslots, make_double2(sc, 0.0), d_norm, st)
                                   : launch_dplane<C, 0, false>(p, S, nslots, make_double2(sc, 0.0), d_norm, st);
        else r = sgn > 0 ? launch_dplane<C, 1, true>(p, S, nslots, make_double2(sc, 0.0), d_norm, st)
                         : launch_dplane<C, 1, false>(p, S, nslots, make_double2(sc, 0.0), d_norm, st, epi);
        if (r != WIG_ERR_UNSUPPORTED || epi) return r;
    }
    if (epi) return WIG_ERR_UNSUPPORTED;
    // general delta or size: two standalone FAFTs per slot (in slot order)
    for (int k = 0; k < nslots; ++k) {
        int r = wig_faft(slots[k], ns, p->d.dtype, ax_b, p->d.d[ax_b], sgn * p->d.delta[ax_b], 1.0, st);
        if (r) return r;
        r = wig_faft(slots[k], ns, p->d.dtype, ax_a, p->d.d[ax_a], sgn * p->d.delta[ax_a], post, st);
        if (r) return r;
        if (d_norm) {
            if ((r = wig_divide_by_device_scalar(slots[k], p->npts, p->d.dtype, d_norm, st))) return r;
        }
    }
    return WIG_OK;
}
extern "C" int wigd_transform(wigd_plan* p, void* const* slots, int nslots, int which, const double* d_norm,
                              void* stream) {
    if (!p || !slots || which < 0 || which > 3) return WIG_ERR_INVALID_ARG;
    return DISPATCH(p, transform_impl<double2>(p, slots, nslots, which, d_norm, as_stream(stream)),
                    transform_impl<float2>(p, slots, nslots, which, d_norm, as_stream(stream)));
}

// ---- the whole Run() loop for distinct component pointers -------------------
template <class C>
static int run_impl(wigd_plan* p, void* const* slots, int iterations, int filter, double* hist, cudaStream_t st) {
    int r;
    Slots<C> S;
    if ((r = make_slots(slots, S, false))) return r;
    const bool fused_mrr = getenv("WIG_NO_DFUSE") == nullptr;
    // 64^4 with |delta| N = 1 on the P <-> Theta axes: the Theta -> P transform
    // of iteration it also runs iteration it + 1's boundary_xp, Real and sums
    auto fast = [&](int a) { return fabs(fabs(p->d.delta[a]) * p->d.shape[a] - 1.0) < 1e-12; };
    const bool fuse_tp = fused_mrr && p->epi_rows && fast(0) && fast(2) && !getenv("WIG_NO_DTP_FUSE") &&
                         !getenv("WIG_NO_DPLANE_R4") && !getenv("WIG_NO_DPLANE_TMA");
    DEpi E;
    memset(&E, 0, sizeof(E));
    for (int a = 0; a < 4; ++a) E.mxp[a] = p->P.mxp[a];
    E.cx = p->P.cx; E.cy = p->P.cy; E.cpx = p->P.cpx; E.cpy = p->P.cpy;
    E.obs_xy = p->P.obs_xy; E.c = p->P.c; E.mass = p->P.mass; E.kvn = p->P.kvn; E.rows = p->epi_rows;
    WIG_CUDA(cudaMemsetAsync(p->counter, 0, 2 * sizeof(int), st));
    for (int it = 0; it < iterations; ++it) {
        // boundary_xp, Real, trace norm + observables of the normalised state
        if (fuse_tp && it > 0) {
            // done by the previous Theta -> P: fold its per-plane sums
            k_dfold<<<EPI_FOLD, 32 * DSUM, 0, st>>>(p->epi_rows, NSLOT * 4096, p->epi_fold);
            WIG_LAUNCHED("k_dfold");
            k_dfinalize<<<1, 32 * DSUM, 0, st>>>(p->epi_fold, EPI_FOLD, p->d.dv_norm, p->d.dv_obs, 1, hist,
                                                 p->counter, iterations, p->cur_norm, p->flag);
            WIG_LAUNCHED("k_dfinalize");
        } else if (fused_mrr) {
            k_dmask_real_reduce<C><<<p->nblk, 256, 0, st>>>(S, p->P, p->partials);
            WIG_LAUNCHED("k_dmask_real_reduce");
            k_dfinalize<<<1, 32 * DSUM, 0, st>>>(p->partials, p->nblk, p->d.dv_norm, p->d.dv_obs, 1, hist,
                                                 p->counter, iterations, p->cur_norm, p->flag);
            WIG_LAUNCHED("k_dfinalize");
        } else {
            if ((r = mask_impl<C>(p, slots, 1, st))) return r;
            if ((r = real_impl<C>(p, slots, st))) return r;
            if ((r = reduce_impl<C>(p, slots, hist, 1, p->counter, iterations, st))) return r;
        }
        // X -> Lambda with the 1/norm folded in
        if ((r = transform_impl<C>(p, slots, NSLOT, 0, p->cur_norm, st))) return r;
        if ((r = kinetic_impl<C>(p, slots, filter ? 1 : 0, 1, st))) return r;
        if ((r = transform_impl<C>(p, slots, NSLOT, 1, nullptr, st))) return r;
        if ((r = transform_impl<C>(p, slots, NSLOT, 2, nullptr, st))) return r;
        if ((r = potential_impl<C>(p, slots, st))) return r;
        if ((r = transform_impl<C>(p, slots, NSLOT, 3, nullptr, st, fuse_tp && it + 1 < iterations ? &E : nullptr)))
            return r;
    }
    return WIG_OK;
}
extern "C" int wigd_run(wigd_plan* p, void* const* slots, int iterations, int filter, double* d_history,
                        void* stream) {
    if (!p || !slots || !d_history || iterations < 0) return WIG_ERR_INVALID_ARG;
    for (int a = 0; a < NSLOT; ++a) {
        if (!slots[a]) return WIG_ERR_INVALID_ARG;
        for (int b = a + 1; b < NSLOT; ++b)
            if (slots[a] == slots[b]) return WIG_ERR_ALIAS;
    }
    return DISPATCH(p, run_impl<double2>(p, slots, iterations, filter, d_history, as_stream(stream)),
                    run_impl<float2>(p, slots, iterations, filter, d_history, as_stream(stream)));
}
