// r4.cuh -- 64^4 Run() half-steps with 16 points per thread (radix-4 digit
// pairs), for both complex128 and complex64.  Included by wigner4d.cu.
//
// A CTA of 256 threads transforms one 64 x 64 plane; two (complex128) or
// four (complex64) CTAs share an SM and overlap each other's memory waits.
//
// 2-D transform.  Each in-plane index is three radix-4 digits, c = c0 + 4 c1
// + 16 c2 (same for r).  A thread holds a 4 x 4 block of registers
// v[i][j] -- one digit of each axis -- and the plane moves through three
// thread layouts (T = thread index, (R, C) the point in shared memory):
//   L1: T = (c0 + 4 c1) + 16 (r0 + 4 r1),  (R, C) = (r0 + 4 r1 + 16 i, c0 + 4 c1 + 16 j)
//   L2: T = (c0 + 4 c2) + 16 (r0 + 4 r2),  (R, C) = (r0 + 4 i + 16 r2, c0 + 4 j + 16 c2)
//   L3: T = (c1 + 4 c2) + 16 (r1 + 4 r2),  (R, C) = (i + 4 r1 + 16 r2, j + 4 c1 + 16 c2)
// Forward (decimation in time, stride-16 digit first):
//   L1: 4-point DFTs over j and i, twiddle w64^((c0 + 4 c1) j + (r0 + 4 r1) i);
//   L2: 4-point DFTs, twiddle w64^(4 (c0 j + r0 i));
//   L3: 4-point DFTs; thread (c1, c2, r1, r2) then holds the frequencies
//       kc = c2 + 4 c1 + 16 j, kr = r2 + 4 r1 + 16 i (its own digits reused).
// The inverse runs the mirror image from L3 back to L1 (conjugate kernels,
// twiddles w64^-((c2 + 4 c1) j + ...) in L3 and w64^-(4 (c2 j + r2 i)) in L2)
// and ends in L1 in natural order.  A half-step is four exchanges through
// one 64 x 64 shared-memory plane, whose columns are XOR-swizzled so that
// every exchange is free of bank conflicts.
//
// Memory layouts during Run() (IL planes share each 32-byte sector,
// IL = 2 for complex128, 4 for complex64; the state is converted from and
// back to the reference layout around the loop):
//   LA = [y][x/IL][p_y][p_x][x%IL]    kinetic source, potential destination
//   LB = [p_y][p_x/IL][y][x][p_x%IL]  kinetic destination, potential source
// With (f0, f1) the plane and (r, c) the in-plane point, both half-steps read
//   src[(((r*(64/IL) + c/IL)*64 + f0)*64 + f1)*IL + c%IL]
// (whole sectors per warp instruction) and write
//   dst[(((f0*(64/IL) + f1/IL)*64 + r)*64 + c)*IL + f1%IL]
// (each sector completed in L2 by the CTAs of the IL neighbouring planes).
#pragma once

namespace r4 {

constexpr int NT = 256;

template <class C> struct Il { static constexpr int v = 32 / (int)sizeof(C); };

// swizzled column of a shared-memory row (element units; see the file comment)
template <class C> __device__ __forceinline__ int swz(int c) {
    if (sizeof(C) == 16) return c ^ ((c >> 3) & 1) ^ (((c >> 4) & 1) * 6);
    return c ^ (((c >> 4) & 1) * 5) ^ (((c >> 5) & 1) * 10);
}

// 4-point DFTs over j (each row i), then over i (each column j)
template <class C, bool FWD> __device__ __forceinline__ void pass(C (&v)[16]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) dft4<C, FWD>(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
#pragma unroll
    for (int j = 0; j < 4; ++j) dft4<C, FWD>(v[j], v[4 + j], v[8 + j], v[12 + j]);
}

// Slot of w^k (k < 16) in the complex128 shared table: with k's bits b0..b3,
// slot = b0 + 2 b2 + 4 (b1 ^ b3) + 8 b3, so that every quarter-warp of the
// four twiddle calls (a = t & 15, 4 (t & 3), (t >> 2 & 3) + 4 (t & 3),
// 4 (t >> 2 & 3) and the warp-uniform b) reads distinct 16-byte bank groups.
__device__ __forceinline__ int tw_slot(int k) {
    return (k & 1) | ((k >> 1) & 2) | ((((k >> 1) ^ (k >> 3)) & 1) << 2) | (k & 8);
}
// fill the shared twiddle table from the plan's table gtw[k] = w^k
__device__ __forceinline__ void load_tw(double2* tw, const double2* gtw, int t) {
    if (t < 16) tw[tw_slot(t)] = gtw[t];
}
__device__ __forceinline__ void load_tw(float2* tw, const float2* gtw, int t) {
    if (t < 64) tw[t] = gtw[t];
}
// w^a, w^2a, w^3a (a <= 15).  complex128: one table load, the square and the
// cube in FP64 (a few units in the last place); a 128-bit shared load is
// served per quarter-warp, so three loads of scattered entries cost several
// times the wavefronts of one.  complex64: the table's normalised entries
// (|w|^2 closest to 1), which a float32 recurrence would not keep.
__device__ __forceinline__ void tw_powers(const double2* tw, int a, double2 (&w)[3]) {
    w[0] = tw[tw_slot(a)];
    w[1] = make_double2(fma(w[0].x, w[0].x, -w[0].y * w[0].y), (2.0 * w[0].x) * w[0].y);
    w[2] = zmul(w[1], w[0]);
}
__device__ __forceinline__ void tw_powers(const float2* tw, int a, float2 (&w)[3]) {
    w[0] = tw[a];
    w[1] = tw[2 * a];
    w[2] = tw[3 * a];
}

// v[i][j] *= w^(a j + b i) (FWD) or its conjugate, w = exp(-2 pi i / 64)
template <class C, bool FWD> __device__ __forceinline__ void twiddle(C (&v)[16], const C* tw, int a, int b) {
    C wa[3], wb[3];
    tw_powers(tw, a, wa);
    tw_powers(tw, b, wb);
#pragma unroll
    for (int j = 1; j < 4; ++j) {
        const C w = FWD ? wa[j - 1] : cconj(wa[j - 1]);
#pragma unroll
        for (int i = 0; i < 4; ++i) v[4 * i + j] = cmul(v[4 * i + j], w);
    }
#pragma unroll
    for (int i = 1; i < 4; ++i) {
        const C w = FWD ? wb[i - 1] : cconj(wb[i - 1]);
#pragma unroll
        for (int j = 0; j < 4; ++j) v[4 * i + j] = cmul(v[4 * i + j], w);
    }
}

// shared-memory point of register (i, j) in each layout
struct Lay {
    int r0, c0;     // the thread's contribution to R and C
    int ri, cj;     // stride of register i in R, of register j in C
};
__device__ __forceinline__ Lay lay1(int t) { return {(t >> 4), (t & 15), 16, 16}; }
__device__ __forceinline__ Lay lay2(int t) {
    return {((t >> 4) & 3) + 16 * (t >> 6), (t & 3) + 16 * ((t >> 2) & 3), 4, 4};
}
__device__ __forceinline__ Lay lay3(int t) {
    return {4 * ((t >> 4) & 3) + 16 * (t >> 6), 4 * (t & 3) + 16 * ((t >> 2) & 3), 1, 1};
}

template <class C> __device__ __forceinline__ void put(C* s, const Lay& L, const C (&v)[16]) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) s[(L.r0 + L.ri * i) * 64 + swz<C>(L.c0 + L.cj * j)] = v[4 * i + j];
}
template <class C> __device__ __forceinline__ void get(const C* s, const Lay& L, C (&v)[16]) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) v[4 * i + j] = s[(L.r0 + L.ri * i) * 64 + swz<C>(L.c0 + L.cj * j)];
}

// v *= (row factor a) * (column factor b); complex128 in FP64, complex64 as
// float-float products of the FP64 factors (no systematic float32 rounding)
__device__ __forceinline__ void factor_mul(double2& v, double2 a, double2 b) { v = zmul(zmul(v, a), b); }
__device__ __forceinline__ void factor_mul(float2& v, double2 a, double2 b) {
    float2 ah, al, bh, bl;
    ff::split_hl(a, ah, al);
    ff::split_hl(b, bh, bl);
    v = ff::fmul_hl(ff::fmul_hl(v, ah, al), bh, bl);
}

// one 32-byte sector: IL neighbouring planes' values of one point
__device__ __forceinline__ void st_sector(double2* p, const double2 (&v)[2]) {
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(v[0].x), "d"(v[0].y), "d"(v[1].x),
                 "d"(v[1].y)
                 : "memory");
}
__device__ __forceinline__ void st_sector(float2* p, const float2 (&v)[4]) {
    asm volatile("st.global.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v[0].x), "f"(v[0].y), "f"(v[1].x),
                 "f"(v[1].y)
                 : "memory");
    asm volatile("st.global.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p + 2), "f"(v[2].x), "f"(v[2].y), "f"(v[3].x),
                 "f"(v[3].y)
                 : "memory");
}

// storage <-> arithmetic types (the mixed form: complex64 in memory, FP64
// transforms)
template <class C> __device__ __forceinline__ C widen(double2 v) { return v; }
template <class C> __device__ __forceinline__ C widen(float2 v);
template <> __device__ __forceinline__ double2 widen<double2>(float2 v) { return make_double2(v.x, v.y); }
template <> __device__ __forceinline__ float2 widen<float2>(float2 v) { return v; }
template <class S> __device__ __forceinline__ S narrow(double2 v);
template <> __device__ __forceinline__ double2 narrow<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 narrow<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }
template <class S> __device__ __forceinline__ S narrow(float2 v) { return v; }

template <class C> __device__ __forceinline__ void make_tw(C* tw);
template <> __device__ __forceinline__ void make_tw<double2>(double2* tw) { make_twiddles(tw, 64); }
template <> __device__ __forceinline__ void make_tw<float2>(float2* tw) { ff::make_norm_twiddles(tw); }

}  // namespace r4

template <class C>
constexpr size_t r4_smem_bytes() { return sizeof(C) * (64 * 64 + 64) + sizeof(double2) * 128; }

// One half-step, one plane per CTA (blockIdx = f0 * 64 + f1).
//   KIN: src LA -> dst LB, factor scale / norm;
//   POT: src LB -> dst LA, factor scale, and one NPART partial row per plane.
// PV: FP64 per-plane vectors [plane][128] (row then column frequencies,
// shifted by N/2 as k_plane_vectors builds them).
// CL: launched as clusters of the IL planes f1 = IL m .. IL m + IL - 1 that
// share each destination sector; the stores then go through distributed
// shared memory so that every 32-byte sector is written whole (see the end).
// S: the state's type in memory (C by default); S = float2 with C = double2
// is the mixed form, complex64 storage with FP64 transforms and factors.
template <class C, bool KIN, bool CL, class S = C>
__global__ void __launch_bounds__(r4::NT, (sizeof(C) == 16 ? 2 : 4))
k_r4(const S* __restrict__ src, S* __restrict__ dst, const double2* __restrict__ PV, const C* __restrict__ gtw,
     double2 scale, const double* __restrict__ d_norm, ObsTabs ob, double* __restrict__ partials) {
    using namespace r4;
    constexpr int IL = Il<S>::v, NQ = 64 / IL;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* s = reinterpret_cast<C*>(smraw);
    C* tw = s + 64 * 64;
    double2* pvs = reinterpret_cast<double2*>(tw + 64);         // this plane's factor vectors
    const int t = threadIdx.x, pl = blockIdx.x, f0 = pl >> 6, f1 = pl & 63;
    const int ac = t & 15, ar = t >> 4;
    C v[16];
    {
        const S* g = src + ((((long long)ar * NQ + ac / IL) * 64 + f0) * 64 + f1) * IL + (ac % IL);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
                v[4 * i + j] = widen<C>(g[(long long)i * (16LL * 64 * 64 * 64) + (long long)j * (16LL * 64 * 64)]);
    }
    load_tw(tw, gtw, t);
    // row vector as is; column entry kc at 64 + (kc & 48) + 4 (kc & 3) + (kc >> 2 & 3),
    // so that each quarter-warp's column factors lie in distinct bank groups
    if (t < 128) pvs[t < 64 ? t : 64 + (t & 48) + ((t & 3) << 2) + ((t >> 2) & 3)] = __ldg(PV + (long long)pl * 128 + t);
    double2 cc = scale;
    if (KIN && d_norm) cc = zmul(cc, zinv(make_double2(d_norm[0], d_norm[1])));
    const Lay L1 = lay1(t), L2 = lay2(t), L3 = lay3(t);
    __syncthreads();                                           // twiddles and factor vectors ready
    // ---- forward
    pass<C, true>(v);
    twiddle<C, true>(v, tw, ac, ar);
    put(s, L1, v);
    __syncthreads();
    get(s, L2, v);
    pass<C, true>(v);
    twiddle<C, true>(v, tw, 4 * (t & 3), 4 * ((t >> 4) & 3));
    __syncthreads();
    put(s, L2, v);
    __syncthreads();
    get(s, L3, v);
    pass<C, true>(v);
    // ---- factor at kc = c2 + 4 c1 + 16 j, kr = r2 + 4 r1 + 16 i
    {
        const int c1 = t & 3, c2 = (t >> 2) & 3, r1 = (t >> 4) & 3, r2 = t >> 6;
        double2 b[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = pvs[64 + 16 * j + 4 * c2 + c1];     // column kc = c2 + 4 c1 + 16 j
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const double2 a = zmul(pvs[r2 + 4 * r1 + 16 * i], cc);
#pragma unroll
            for (int j = 0; j < 4; ++j) factor_mul(v[4 * i + j], a, b[j]);
        }
    }
    // ---- inverse
    pass<C, false>(v);
    twiddle<C, false>(v, tw, ((t >> 2) & 3) + 4 * (t & 3), (t >> 6) + 4 * ((t >> 4) & 3));
    __syncthreads();
    put(s, L3, v);
    __syncthreads();
    get(s, L2, v);
    pass<C, false>(v);
    twiddle<C, false>(v, tw, 4 * ((t >> 2) & 3), 4 * (t >> 6));
    __syncthreads();
    put(s, L2, v);
    __syncthreads();
    get(s, L1, v);
    pass<C, false>(v);
    // ---- store: point (r, c) = (ar + 16 i, ac + 16 j)
    if (!CL) {
        S* g = dst + (((long long)f0 * NQ + f1 / IL) * 64 * 64 + ar * 64 + ac) * IL + (f1 % IL);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) g[(i * 16 * 64 + j * 16) * IL] = narrow<S>(v[4 * i + j]);
    }
    if (!KIN) {
        // observables of the new (x, p) state: p_y = ar + 16 i, p_x = ac + 16 j
        typedef typename real_of<C>::type R;
        R a[NPART];
#pragma unroll
        for (int k = 0; k < NPART; ++k) a[k] = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const R qy = (R)__ldg(ob.cpy + ar + 16 * i);
            R w0x = 0, w0y = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const C w = v[4 * i + j];
                const R qx = (R)__ldg(ob.cpx + ac + 16 * j), k = (R)__ldg(ob.ep + (ar + 16 * i) * 64 + ac + 16 * j);
                w0x += w.x; w0y += w.y;
                a[2] += qx * w.x; a[3] += qx * w.y;
                a[4] += qx * qx * w.x; a[5] += qx * qx * w.y;
                a[10] += k * w.x; a[11] += k * w.y;
            }
            a[0] += w0x; a[1] += w0y;
            a[6] += qy * w0x; a[7] += qy * w0y;
            a[8] += qy * qy * w0x; a[9] += qy * qy * w0y;
        }
        double* red = reinterpret_cast<double*>(smraw);
        __syncthreads();                                        // plane buffer free
#pragma unroll
        for (int k = 0; k < NPART; ++k) red[k * NT + t] = (double)a[k];
        __syncthreads();
        const int w = t >> 5, l = t & 31;
        for (int k = w; k < NPART; k += NT / 32) {
            double sum = 0.0;
#pragma unroll
            for (int m = 0; m < NT / 32; ++m) sum += red[k * NT + m * 32 + l];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
            if (l == 0) partials[(long long)pl * NPART + k] = sum;
        }
    }
    if (CL) {
        // Stage the plane as [r][c]; cluster CTA q then writes the points
        // q * 4096/IL .. of all IL planes of its cluster, reading the other
        // planes from the partner CTAs' shared memory: each point's IL values
        // form one whole 32-byte sector, and a warp writes a contiguous run.
        namespace cg = cooperative_groups;
        cg::cluster_group cl = cg::this_cluster();
        __syncthreads();                                 // last exchange / reduction reads done
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) s[(ar + 16 * i) * 64 + ac + 16 * j] = v[4 * i + j];
        cl.sync();
        const int q = (int)cl.block_rank();              // = f1 % IL
        const C* part[IL];
#pragma unroll
        for (int g = 0; g < IL; ++g) part[g] = cl.map_shared_rank(s, g);
        S* gb = dst + ((long long)f0 * NQ + f1 / IL) * 64 * 64 * IL;
        constexpr int PER = 4096 / IL / NT;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int pt = q * (4096 / IL) + k * NT + t;
            S val[IL];
#pragma unroll
            for (int g = 0; g < IL; ++g) val[g] = narrow<S>(part[g][pt]);
            st_sector(gb + (long long)pt * IL, val);
        }
        cl.sync();                                       // partners done reading this CTA's plane
    }
}

// L0 = [p_y][y][p_x][x] -> LA = [y][x/IL][p_y][p_x][x%IL]; one thread per LA element.
template <class C>
__global__ void k_to_r4_layout(const C* __restrict__ W, C* __restrict__ P, long long n) {
    constexpr int IL = r4::Il<C>::v, LG = IL == 2 ? 1 : 2, NQ = 64 / IL;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int xr = (int)(e & (IL - 1)), px = (int)((e >> LG) & 63), py = (int)((e >> (LG + 6)) & 63);
        const int xq = (int)((e >> (LG + 12)) % NQ), y = (int)((e >> (LG + 12)) / NQ);
        P[e] = W[(((long long)py * 64 + y) * 64 + px) * 64 + xq * IL + xr];
    }
}

// LA -> L0, divided by the complex norm (none when d_norm is null); one thread per L0 element.
template <class C>
__global__ void k_from_r4_layout(const C* __restrict__ P, C* __restrict__ W, long long n,
                                 const double* __restrict__ d_norm) {
    constexpr int IL = r4::Il<C>::v, NQ = 64 / IL;
    const double2 inv = d_norm ? zinv(make_double2(d_norm[0], d_norm[1])) : make_double2(1.0, 0.0);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(e & 63), px = (int)((e >> 6) & 63), y = (int)((e >> 12) & 63), py = (int)(e >> 18);
        const C a = P[((((long long)y * NQ + x / IL) * 64 + py) * 64 + px) * IL + x % IL];
        const double2 r = zmul(to_d2(a), inv);
        W[e] = to_c<C>(r);
    }
}

// ---------------------------------------------------------------------------
// TMA and mbarrier helpers of the persistent ring kernels and the Dirac plane
// kernels: shared-memory addresses, mbarrier init / expect-tx / bounded waits,
// and the 5-D tensor box load (cp.async.bulk.tensor, no multicast).
// ---------------------------------------------------------------------------
namespace r4t {

__device__ __forceinline__ uint32_t sa(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sa(bar)) : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sa(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(sa(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait for phase 0 of the barrier
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar) {
    for (int it = 0; it < (1 << 22); ++it)
        if (mbar_try_wait(bar, 0)) return true;
    return false;
}
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            int c4, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
        ::"r"(sa(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(sa(bar))
        : "memory");
}

}  // namespace r4t

// ---------------------------------------------------------------------------
// k_r4ring: the 64^4 half-steps of k_r4 as a persistent kernel whose planes
// stream through a ring of shared-memory buffers filled by TMA.
//
// One CTA per SM holds NG = IL plane groups of 256 threads (2 for
// complex128, 4 for complex64) and NB = NG + 1 plane buffers.  The CTA
// walks the units u = blockIdx.x, blockIdx.x + gridDim.x, ...; a unit is the
// IL planes f1 = IL m .. IL m + IL - 1 of one f0 that share every
// destination sector, so the IL groups store the halves (quarters) of the
// same sectors at about the same time.  Local plane k (plane k % IL of the
// CTA's unit k / IL) belongs to group k % NG and lives in buffer k % NB.
//
// A buffer is refilled with local plane k + NB by one thread of the group
// that used it for plane k, as soon as that group has read its last
// exchange out of it; the group then runs its last inverse pass, the
// observables and the stores from registers while the copy is in flight.
// Every group's next plane has therefore been loading since the group
// before it released a buffer, and no thread issues a global load of the
// state.  A plane lands in natural [r][c] order, is read
// straight into layout L1, and its buffer then serves as the exchange plane.
// Exchanges and arithmetic are k_r4's, on one named barrier per group.
//
// Each copy completes on its buffer's mbarrier (bytes counted).  Waits are
// bounded and the group decides together (bar.red.and) whether its plane
// arrived; if not, it poisons the norm (kinetic) or the plane's partial row
// (potential) with NaN, raises the CTA's abort word (other groups stop at
// their next wait), and before the CTA exits one thread waits, bounded
// again, for every copy it issued.
// ---------------------------------------------------------------------------
namespace r4ring {

template <class C> struct Cfg {
    static constexpr int IL = r4::Il<C>::v, NG = IL, NB = NG + 1, NTH = NG * r4::NT;
    static constexpr size_t PLANE = 64 * 64 * sizeof(C);
    static constexpr size_t TW_OFF = NB * PLANE;                           // 64 twiddles
    static constexpr size_t PV_OFF = TW_OFF + 64 * sizeof(C);              // per group: 128 FP64 factors
    static constexpr size_t RED_OFF = PV_OFF + NG * 128 * sizeof(double2); // per group: 8 warps x 16 slots
    static constexpr size_t BAR_OFF = RED_OFF + NG * 8 * 16 * sizeof(double);
    static constexpr size_t CNT_OFF = BAR_OFF + NB * sizeof(uint64_t);     // copies issued per buffer, abort
    static constexpr size_t SMEM = CNT_OFF + 16 * sizeof(int) + 128;       // + alignment of the base
    static_assert(SMEM <= 232448, "k_r4ring shared memory");
};

__device__ __forceinline__ void group_sync(int g) { asm volatile("bar.sync %0, 256;" ::"r"(1 + g) : "memory"); }

// true on every thread of group g iff p holds on all of them
__device__ __forceinline__ bool group_all(bool p, int g) {
    uint32_t r;
    asm volatile(
        "{\n .reg .pred q, d;\n setp.ne.u32 q, %1, 0;\n bar.red.and.pred d, %2, 256, q;\n selp.u32 %0, 1, 0, d;\n}\n"
        : "=r"(r)
        : "r"((uint32_t)p), "r"(1 + g)
        : "memory");
    return r != 0;
}

// Bounded wait for use n of a buffer (its (n+1)-th copy).  A parity wait
// alone cannot tell phase n from phase n - 2: a group may reach use n while
// the buffer still holds (or awaits) use n - 1 of another group.  So first
// wait until the copy of use n has been issued (issued > n), which happens
// only after use n - 1 has landed and been consumed; then the parity of
// phase n is unambiguous.  Gives up early once the CTA's abort word is set.
__device__ __forceinline__ bool wait_plane(uint64_t* bar, const volatile int* issued, int n,
                                           const volatile int* abort_word) {
    int it = 0;
    for (; it < (1 << 22); ++it) {
        if (*issued > n) break;
        if ((it & 1023) == 1023 && *abort_word) return false;
    }
    for (; it < (1 << 22); ++it) {
        if (r4t::mbar_try_wait(bar, (uint32_t)(n & 1))) return true;
        if ((it & 1023) == 1023 && *abort_word) return false;
    }
    return false;
}

// TMA tensor store of one plane from shared memory (bulk group of the
// issuing thread), and the waits for its reads of shared memory / for all of it
__device__ __forceinline__ void tma_store_5d(const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                             const void* src) {
    asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];"
                 ::"l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(r4t::sa(src))
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// one contiguous block from shared to global memory (bulk group of the issuing
// thread); both addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_store_1d(void* gdst, const void* ssrc, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(r4t::sa(ssrc)),
                 "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Sum of 16 per-lane values over the warp, transposed: after the call a[0]
// on lane l holds the warp's total of slot (l >> 1) & 15 (4 halving levels
// of xor-shuffles that each move half of the remaining slots, then one of
// plain addition), 32 shuffles of doubles in all.
__device__ __forceinline__ double warp_slot_sums(double (&a)[16], int lane) {
#pragma unroll
    for (int lv = 0; lv < 4; ++lv) {
        const int h = 8 >> lv, m = 16 >> lv;
        const bool up = (lane & m) != 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            if (q < h) {
                const double send = up ? a[q] : a[q + h];
                const double keep = up ? a[q + h] : a[q];
                a[q] = keep + __shfl_xor_sync(0xffffffffu, send, m);
            }
        }
    }
    return a[0] + __shfl_xor_sync(0xffffffffu, a[0], 1);
}

}  // namespace r4ring

// The result leaves by one copy per plane from the plane's buffer, written
// there in natural [r][c] order; the buffer's refill then waits until the
// copy has read it, which the group's thread 0 checks at the group's next
// plane (after reading its input) or after its last plane.  On LA / LB the
// copy is a TMA tensor store (dst_map, box (2 reals, 1, 64, 64, 1) at
// (0, f1 % IL, 0, 0, unit)).
// PC: the plane-contiguous layouts LK = [y][x][p_y][p_x] (kinetic
// source, potential destination) and LP = [p_y][p_x][y][x] (the reverse).
// Both half-steps then read point (r, c) of plane (f0, f1) at
// src[((r * 64 + c) * 64 + f0) * 64 + f1] -- a box of one-point rows whose
// sectors the other group's plane (f1 ^ 1) reads at the same time -- and
// write the plane as one contiguous 64 KB block at dst + (f0 * 64 + f1) *
// 4096 with a single bulk copy: whole lines, no partial-sector writes.
template <class C, bool KIN, bool PC>
__global__ void __launch_bounds__(r4ring::Cfg<C>::NTH, 1)
k_r4ring(const __grid_constant__ CUtensorMap src_map, const __grid_constant__ CUtensorMap dst_map,
         C* __restrict__ dst, const double2* __restrict__ PV, const C* __restrict__ gtw, double2 scale,
         double* __restrict__ d_norm, ObsTabs ob, double* __restrict__ partials) {
    using namespace r4;
    using namespace r4t;
    using namespace r4ring;
    typedef Cfg<C> K;
    constexpr int IL = K::IL, NG = K::NG, NB = K::NB, NQ = 64 / IL;
    extern __shared__ __align__(16) unsigned char smraw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
    C* tw = reinterpret_cast<C*>(base + K::TW_OFF);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + K::BAR_OFF);
    volatile int* issued = reinterpret_cast<int*>(base + K::CNT_OFF);  // [NB] copies per buffer, [NB] abort word
    volatile int* abort_word = issued + NB;
    const int tid = threadIdx.x, g = tid >> 8, t = tid & (NT - 1), lane = t & 31, wp = t >> 5;
    double2* pvs = reinterpret_cast<double2*>(base + K::PV_OFF) + g * 128;
    double* red = reinterpret_cast<double*>(base + K::RED_OFF) + g * 128;
    const int nunits = 4096 / IL;
    const int nloc = (int)blockIdx.x < nunits ? ((nunits - 1 - (int)blockIdx.x) / (int)gridDim.x + 1) * IL : 0;
    auto plane_of = [&](int k) { return ((int)blockIdx.x + (k / IL) * (int)gridDim.x) * IL + k % IL; };
    if (tid == 0) {
        for (int b = 0; b < NB; ++b) {
            mbar_init(bars + b);
            issued[b] = 0;
        }
        issued[NB] = 0;
        issued[NB + 1] = 0;                            // stays 0: the final drain never gives up early
        fence_async_smem();
        for (int k = 0; k < NB && k < nloc; ++k) {
            const int pl = plane_of(k);
            mbar_expect_tx(bars + k, (uint32_t)K::PLANE);
            tma_load_5d(base + k * K::PLANE, &src_map, 0, pl & 63, pl >> 6, 0, 0, bars + k);
            issued[k] = 1;
        }
    }
    if (tid < 64) load_tw(tw, gtw, tid);
    double2 cc = scale;
    if (KIN) cc = zmul(cc, zinv(make_double2(d_norm[0], d_norm[1])));
    const int ac = t & 15, ar = t >> 4;
    const Lay L1 = lay1(t), L2 = lay2(t), L3 = lay3(t);
    // thread 0 of a group: refill buffer (k + NB) % NB with local plane k + NB
    auto refill = [&](int kk) {
        if (kk + NB < nloc) {
            const int b = kk % NB, pn = plane_of(kk + NB);
            fence_async_smem();
            mbar_expect_tx(bars + b, (uint32_t)K::PLANE);
            tma_load_5d(base + b * K::PLANE, &src_map, 0, pn & 63, pn >> 6, 0, 0, bars + b);
            issued[b] += 1;
        }
    };
    int pend = -1;                                     // thread 0: plane whose buffer awaits its refill
    __syncthreads();                                   // barriers, counters and twiddles ready
    for (int k = g; k < nloc; k += NG) {
        const int bf = k % NB, pl = plane_of(k), f0 = pl >> 6, f1 = pl & 63;
        C* s = reinterpret_cast<C*>(base + bf * K::PLANE);
        // this plane's factor vectors (first read after the exchanges' barriers;
        // column entry kc at 64 + (kc & 48) + 4 (kc & 3) + (kc >> 2 & 3))
        if (t < 128) pvs[t < 64 ? t : 64 + (t & 48) + ((t & 3) << 2) + ((t >> 2) & 3)] = __ldg(PV + (long long)pl * 128 + t);
        const bool arrived = wait_plane(bars + bf, issued + bf, k / NB, abort_word);
        if (!group_all(arrived, g)) {
            if (t == 0) {
                if (KIN) d_norm[0] = __longlong_as_double(0x7ff8000000000000LL);
                else partials[(long long)pl * NPART] = __longlong_as_double(0x7ff8000000000000LL);
                *abort_word = 1;
            }
            break;
        }
        C v[16];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) v[4 * i + j] = s[(ar + 16 * i) * 64 + ac + 16 * j];
        // ---- forward
        pass<C, true>(v);
        twiddle<C, true>(v, tw, ac, ar);
        group_sync(g);                                 // the landed plane has been read
        if (t == 0 && pend >= 0) {
            bulk_wait_read();                          // the previous plane's store has left its buffer
            refill(pend);
            pend = -1;
        }
        put(s, L1, v);
        group_sync(g);
        get(s, L2, v);
        pass<C, true>(v);
        twiddle<C, true>(v, tw, 4 * (t & 3), 4 * ((t >> 4) & 3));
        group_sync(g);
        put(s, L2, v);
        group_sync(g);
        get(s, L3, v);
        pass<C, true>(v);
        {
            const int c1 = t & 3, c2 = (t >> 2) & 3, r1 = (t >> 4) & 3, r2 = t >> 6;
            double2 b[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = pvs[64 + 16 * j + 4 * c2 + c1];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const double2 a = zmul(pvs[r2 + 4 * r1 + 16 * i], cc);
#pragma unroll
                for (int j = 0; j < 4; ++j) factor_mul(v[4 * i + j], a, b[j]);
            }
        }
        // ---- inverse
        pass<C, false>(v);
        twiddle<C, false>(v, tw, ((t >> 2) & 3) + 4 * (t & 3), (t >> 6) + 4 * ((t >> 4) & 3));
        group_sync(g);
        put(s, L3, v);
        group_sync(g);
        get(s, L2, v);
        pass<C, false>(v);
        twiddle<C, false>(v, tw, 4 * ((t >> 2) & 3), 4 * (t >> 6));
        group_sync(g);
        put(s, L2, v);
        group_sync(g);
        get(s, L1, v);
        group_sync(g);                                 // the group's last exchange has been read
        pass<C, false>(v);
        {
            // ---- stage the plane as [r][c] and store it with one copy
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) s[(ar + 16 * i) * 64 + ac + 16 * j] = v[4 * i + j];
            fence_async_smem();                        // generic-proxy writes visible to the copy engine
            group_sync(g);
            if (t == 0) {
                if (PC) bulk_store_1d(dst + (long long)pl * 4096, s, (uint32_t)K::PLANE);
                else tma_store_5d(&dst_map, 0, f1 % IL, 0, 0, f0 * NQ + f1 / IL, s);
                pend = k;
            }
        }
        if (!KIN) {
            // observables of the new (x, p) state: p_y = ar + 16 i, p_x = ac + 16 j
            typedef typename real_of<C>::type R;
            R a[NPART];
#pragma unroll
            for (int q = 0; q < NPART; ++q) a[q] = 0;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const R qy = (R)__ldg(ob.cpy + ar + 16 * i);
                R w0x = 0, w0y = 0;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const C w = v[4 * i + j];
                    const R qx = (R)__ldg(ob.cpx + ac + 16 * j), kk = (R)__ldg(ob.ep + (ar + 16 * i) * 64 + ac + 16 * j);
                    w0x += w.x; w0y += w.y;
                    a[2] += qx * w.x; a[3] += qx * w.y;
                    a[4] += qx * qx * w.x; a[5] += qx * qx * w.y;
                    a[10] += kk * w.x; a[11] += kk * w.y;
                }
                a[0] += w0x; a[1] += w0y;
                a[6] += qy * w0x; a[7] += qy * w0y;
                a[8] += qy * qy * w0x; a[9] += qy * qy * w0y;
            }
            double d[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) d[q] = q < NPART ? (double)a[q] : 0.0;
            const double sum = warp_slot_sums(d, lane);
            if (!(lane & 1)) red[wp * 16 + (lane >> 1)] = sum;
            group_sync(g);
            if (t < NPART) {
                double tot = 0.0;
#pragma unroll
                for (int w = 0; w < NT / 32; ++w) tot += red[w * 16 + t];
                partials[(long long)pl * NPART + t] = tot;
            }
        }
    }
    if (t == 0) {
        if (pend >= 0) {
            bulk_wait_read();
            if (!*abort_word) refill(pend);            // another group may still need that plane
        }
        bulk_wait_all();                               // every store of this group has completed
    }
    __syncthreads();
    if (tid == 0 && *abort_word) {
        // no copy may still target this CTA's shared memory when it exits
        for (int b = 0; b < NB; ++b)
            if (issued[b] > 0) wait_plane(bars + b, issued + b, issued[b] - 1, issued + NB + 1);
    }
}

// Conversions between the reference layout [p_y][y][p_x][x] and k_r4ring's
// LK = [y][x][p_y][p_x]: for each (p_y, y) a 64 x 64 transpose of (p_x, x)
// through a shared tile (both sides move whole 1 KB rows).  TO: W -> LK;
// else LK -> W divided by the complex norm (none when d_norm is null).
// Grid (2, 2, 4096) of 32 x 8 threads; blockIdx.z = p_y * 64 + y.
template <class C, bool TO>
__global__ void __launch_bounds__(256) k_pc_transpose(const C* __restrict__ src, C* __restrict__ dst,
                                                      const double* __restrict__ d_norm) {
    __shared__ C tile[32][33];
    const int py = blockIdx.z >> 6, y = blockIdx.z & 63;
    // u: the source's contiguous index, v: the destination's
    const long long sbase = TO ? ((long long)py * 64 + y) * 4096 : (long long)y * 262144 + py * 64;
    const long long dbase = TO ? (long long)y * 262144 + py * 64 : ((long long)py * 64 + y) * 4096;
    const long long sstride = TO ? 64 : 4096, dstride = TO ? 4096 : 64;
    const int u0 = blockIdx.x * 32, v0 = blockIdx.y * 32, tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 32; k += 8) tile[ty + k][tx] = src[sbase + (long long)(v0 + ty + k) * sstride + u0 + tx];
    __syncthreads();
    double2 inv = make_double2(1.0, 0.0);
    if (!TO && d_norm) inv = zinv(make_double2(d_norm[0], d_norm[1]));
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const C a = tile[tx][ty + k];
        dst[dbase + (long long)(u0 + ty + k) * dstride + v0 + tx] = TO ? a : to_c<C>(zmul(to_d2(a), inv));
    }
}

// ---------------------------------------------------------------------------
// k_r4ring_mx: the mixed form (complex64 state in memory, complex128
// arithmetic) on the plane-contiguous layouts LK / LP.
//
// A complex64 point is 8 bytes, less than the 16 bytes a tensor box row
// needs, so the unit's two planes (f1 = 2m, 2m + 1: neighbours in memory) come
// in one box of two-point rows, 64 KB laid out [r][c][plane].  One CTA per SM,
// two groups of 256 threads, group g on plane g of every unit; each group has
// its own 64 KB complex128 exchange plane.  Both groups read their plane out
// of the landing box, then (one CTA barrier) thread 0 refills the box with
// the CTA's next unit, which lands while both planes are transformed.  Each
// result is staged as complex64 [r][c] in the group's exchange plane and
// written by one 32 KB bulk copy (the plane is contiguous); the group's next
// first exchange waits until that copy has read the plane.
// The box's wait is bounded and decided by the whole CTA (__syncthreads_and):
// on a timeout the CTA poisons the norm or the partial row with NaN and
// stops; before it exits, thread 0 waits (bounded) for a copy still in flight.
// ---------------------------------------------------------------------------
namespace r4mx {
constexpr int NTH = 2 * r4::NT;
constexpr size_t BOX = 2 * 4096 * sizeof(float2);                     // 64 KB
constexpr size_t EX_OFF = BOX;                                         // 2 x 64 KB complex128
constexpr size_t TW_OFF = EX_OFF + 2 * 4096 * sizeof(double2);
constexpr size_t PV_OFF = TW_OFF + 64 * sizeof(double2);
constexpr size_t RED_OFF = PV_OFF + 2 * 128 * sizeof(double2);
constexpr size_t BAR_OFF = RED_OFF + 2 * 8 * 16 * sizeof(double);
constexpr size_t SMEM = BAR_OFF + 64 + 128;
static_assert(SMEM <= 232448, "k_r4ring_mx shared memory");
}  // namespace r4mx

// C: the arithmetic type, double2 (the mixed form) or float2 (the complex64
// radix form on the same layouts; exchanges in the first 32 KB of each
// group's plane, twiddles from the normalised float32 table).
template <class C, bool KIN>
__global__ void __launch_bounds__(r4mx::NTH, 1)
k_r4ring_mx(const __grid_constant__ CUtensorMap src_map, float2* __restrict__ dst, const double2* __restrict__ PV,
            const C* __restrict__ gtw, double2 scale, double* __restrict__ d_norm, ObsTabs ob,
            double* __restrict__ partials) {
    using namespace r4;
    using namespace r4t;
    using namespace r4ring;
    extern __shared__ __align__(16) unsigned char smraw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
    const float2* box = reinterpret_cast<const float2*>(base);
    C* tw = reinterpret_cast<C*>(base + r4mx::TW_OFF);
    uint64_t* bar = reinterpret_cast<uint64_t*>(base + r4mx::BAR_OFF);
    const int tid = threadIdx.x, g = tid >> 8, t = tid & (NT - 1), lane = t & 31, wp = t >> 5;
    C* s = reinterpret_cast<C*>(base + r4mx::EX_OFF + (size_t)g * 4096 * sizeof(double2));
    double2* pvs = reinterpret_cast<double2*>(base + r4mx::PV_OFF) + g * 128;
    double* red = reinterpret_cast<double*>(base + r4mx::RED_OFF) + g * 128;
    const int nunits = 2048;
    const int nloc = (int)blockIdx.x < nunits ? (nunits - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    auto unit_of = [&](int n) { return (int)blockIdx.x + n * (int)gridDim.x; };
    auto load_unit = [&](int n) {
        const int u = unit_of(n), f0 = u >> 5, m = u & 31;      // planes (f0, 2m) and (f0, 2m + 1)
        fence_async_smem();
        mbar_expect_tx(bar, (uint32_t)r4mx::BOX);
        tma_load_5d(base, &src_map, 0, m, f0, 0, 0, bar);
    };
    if (tid == 0) {
        mbar_init(bar);
        fence_async_smem();
        if (nloc > 0) load_unit(0);
    }
    if (tid < 64) load_tw(tw, gtw, tid);
    double2 cc = scale;
    if (KIN) cc = zmul(cc, zinv(make_double2(d_norm[0], d_norm[1])));
    const int ac = t & 15, ar = t >> 4;
    const Lay L1 = lay1(t), L2 = lay2(t), L3 = lay3(t);
    bool stored = false;                               // thread 0 of a group: a bulk copy may be reading s
    int aborted_at = -1;                               // the unit whose box did not arrive
    __syncthreads();                                   // barrier initialised, twiddles ready
    for (int n = 0; n < nloc; ++n) {
        const int pl = 2 * unit_of(n) + g;             // plane (f0, f1) = (pl >> 6, pl & 63)
        if (t < 128) pvs[t < 64 ? t : 64 + (t & 48) + ((t & 3) << 2) + ((t >> 2) & 3)] = __ldg(PV + (long long)pl * 128 + t);
        bool arrived = false;
        for (int it = 0; it < (1 << 22) && !arrived; ++it) arrived = mbar_try_wait(bar, (uint32_t)(n & 1));
        if (!__syncthreads_and(arrived ? 1 : 0)) {
            if (t == 0) {
                if (KIN) d_norm[0] = __longlong_as_double(0x7ff8000000000000LL);
                else partials[(long long)pl * NPART] = __longlong_as_double(0x7ff8000000000000LL);
            }
            aborted_at = n;
            break;
        }
        C v[16];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) v[4 * i + j] = widen<C>(box[((ar + 16 * i) * 64 + ac + 16 * j) * 2 + g]);
        __syncthreads();                               // both planes have been read out of the box
        if (tid == 0 && n + 1 < nloc) load_unit(n + 1);
        // ---- forward
        pass<C, true>(v);
        twiddle<C, true>(v, tw, ac, ar);
        if (t == 0 && stored) {
            bulk_wait_read();                          // the previous plane's copy has left s
            stored = false;
        }
        group_sync(g);
        put(s, L1, v);
        group_sync(g);
        get(s, L2, v);
        pass<C, true>(v);
        twiddle<C, true>(v, tw, 4 * (t & 3), 4 * ((t >> 4) & 3));
        group_sync(g);
        put(s, L2, v);
        group_sync(g);
        get(s, L3, v);
        pass<C, true>(v);
        {
            const int c1 = t & 3, c2 = (t >> 2) & 3, r1 = (t >> 4) & 3, r2 = t >> 6;
            double2 b[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = pvs[64 + 16 * j + 4 * c2 + c1];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const double2 a = zmul(pvs[r2 + 4 * r1 + 16 * i], cc);
#pragma unroll
                for (int j = 0; j < 4; ++j) factor_mul(v[4 * i + j], a, b[j]);
            }
        }
        // ---- inverse
        pass<C, false>(v);
        twiddle<C, false>(v, tw, ((t >> 2) & 3) + 4 * (t & 3), (t >> 6) + 4 * ((t >> 4) & 3));
        group_sync(g);
        put(s, L3, v);
        group_sync(g);
        get(s, L2, v);
        pass<C, false>(v);
        twiddle<C, false>(v, tw, 4 * ((t >> 2) & 3), 4 * (t >> 6));
        group_sync(g);
        put(s, L2, v);
        group_sync(g);
        get(s, L1, v);
        pass<C, false>(v);
        group_sync(g);                                 // the last exchange has been read
        {
            float2* sf = reinterpret_cast<float2*>(s);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) sf[(ar + 16 * i) * 64 + ac + 16 * j] = narrow<float2>(v[4 * i + j]);
            fence_async_smem();
            group_sync(g);
            if (t == 0) {
                bulk_store_1d(dst + (long long)pl * 4096, sf, (uint32_t)(4096 * sizeof(float2)));
                stored = true;
            }
        }
        if (!KIN) {
            // observables of the new (x, p) state: p_y = ar + 16 i, p_x = ac + 16 j
            // (the values before rounding to the storage type, as k_r4 sums them)
            double a[NPART];
#pragma unroll
            for (int q = 0; q < NPART; ++q) a[q] = 0;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const double qy = __ldg(ob.cpy + ar + 16 * i);
                double w0x = 0, w0y = 0;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const C w = v[4 * i + j];
                    const double qx = __ldg(ob.cpx + ac + 16 * j), kk = __ldg(ob.ep + (ar + 16 * i) * 64 + ac + 16 * j);
                    w0x += w.x; w0y += w.y;
                    a[2] += qx * w.x; a[3] += qx * w.y;
                    a[4] += qx * qx * w.x; a[5] += qx * qx * w.y;
                    a[10] += kk * w.x; a[11] += kk * w.y;
                }
                a[0] += w0x; a[1] += w0y;
                a[6] += qy * w0x; a[7] += qy * w0y;
                a[8] += qy * qy * w0x; a[9] += qy * qy * w0y;
            }
            double d[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) d[q] = q < NPART ? a[q] : 0.0;
            const double sum = warp_slot_sums(d, lane);
            if (!(lane & 1)) red[wp * 16 + (lane >> 1)] = sum;
            group_sync(g);
            if (t < NPART) {
                double tot = 0.0;
#pragma unroll
                for (int w = 0; w < NT / 32; ++w) tot += red[w * 16 + t];
                partials[(long long)pl * NPART + t] = tot;
            }
        }
    }
    if (t == 0) bulk_wait_all();                       // every copy of this group has completed
    if (tid == 0 && aborted_at >= 0) {
        // the timed-out unit's copy (the last one issued) may still be in flight
        for (int it = 0; it < (1 << 22); ++it)
            if (mbar_try_wait(bar, (uint32_t)(aborted_at & 1))) break;
    }
}

// The 64-entry twiddle table of k_r4 and the ring kernels, built once per plan.
template <class C>
__global__ void k_make_r4_twiddles(C* tw) { r4::make_tw<C>(tw); }

// ---------------------------------------------------------------------------
// k_dplane_r4: the Wigner-Dirac component-plane transforms on 64^4 grids,
//   value_out = scale * S * DFT2(S * value_in),  S = (-1)^(row + col),
// the pair of centred FAFT calls for |delta| N = 1 that the reference's
// Fourier_*_64_64_4x4_GPU wrappers make per component
// (GPU_WignerDirac4D.py:1428-1596).
//
// One plane per CTA (blockIdx.x the plane, blockIdx.y the component slot),
// in place.  The plane is read in natural order straight into layout L1 and
// goes L1 -> L2 -> L3 like the forward half of k_r4 (conjugate kernels and
// twiddles for the inverse direction: the same digit order with w^-1).
// Each thread then holds the frequencies (kr, kc) = (r2 + 4 r1 + 16 i,
// c2 + 4 c1 + 16 j) and stores them from registers: two exchanges per
// transform and no staging.  S is constant over a thread's 16 points in L1
// (parity of ar + ac) and in L3 (parity of r2 + c2), since the register
// digits enter with weight 16.
//   KIND 0: plane (i0, i2), rows axis 1 (stride 64^2), columns axis 3 (stride 1)
//   KIND 1: plane (i1, i3), rows axis 0 (stride 64^3), columns axis 2 (stride 64);
//           consecutive blocks are neighbouring i3, so the two (complex128)
//           or four (complex64) planes of each 32-byte sector are read and
//           written together and the sector is completed in L2.
template <class C> struct PlaneSlots { C* p[16]; };

template <class C, int KIND, bool FWD>
__global__ void __launch_bounds__(r4::NT, (sizeof(C) == 16 ? 2 : 4))
k_dplane_r4(const __grid_constant__ PlaneSlots<C> S, const C* __restrict__ gtw, double2 scale, const double* __restrict__ d_norm) {
    using namespace r4;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* s = reinterpret_cast<C*>(smraw);
    C* tw = s + 64 * 64;
    const int t = threadIdx.x, ac = t & 15, ar = t >> 4, pl = blockIdx.x;
    const long long rs = KIND == 0 ? 64LL * 64 : 64LL * 64 * 64;
    const long long cs = KIND == 0 ? 1 : 64;
    const long long off = KIND == 0 ? (long long)(pl >> 6) * (64 * 64 * 64) + (long long)(pl & 63) * 64
                                    : (long long)(pl >> 6) * (64 * 64) + (pl & 63);
    C* g = S.p[blockIdx.y] + off;
    C v[16];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) v[4 * i + j] = g[(ar + 16 * i) * rs + (ac + 16 * j) * cs];
    load_tw(tw, gtw, t);
    double2 sc = scale;
    if (d_norm) sc = zmul(sc, zinv(make_double2(d_norm[0], d_norm[1])));
    const C cc = to_c<C>(sc);
    if ((ar + ac) & 1) {
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = cneg(v[k]);
    }
    const Lay L1 = lay1(t), L2 = lay2(t), L3 = lay3(t);
    __syncthreads();                                   // twiddles ready
    pass<C, FWD>(v);
    twiddle<C, FWD>(v, tw, ac, ar);
    put(s, L1, v);
    __syncthreads();
    get(s, L2, v);
    pass<C, FWD>(v);
    twiddle<C, FWD>(v, tw, 4 * (t & 3), 4 * ((t >> 4) & 3));
    __syncthreads();
    put(s, L2, v);
    __syncthreads();
    get(s, L3, v);
    pass<C, FWD>(v);
    const int c1 = t & 3, c2 = (t >> 2) & 3, r1 = (t >> 4) & 3, r2 = t >> 6;
    const C ccs = ((r2 + c2) & 1) ? cneg(cc) : cc;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
            g[(r2 + 4 * r1 + 16 * i) * rs + (c2 + 4 * c1 + 16 * j) * cs] = cmul(v[4 * i + j], ccs);
}

// k_dplane_r4t: the KIND 1 transform of k_dplane_r4 with the plane moved by
// the tensor memory accelerator.  A (axis 0, axis 2) plane at fixed (i1, i3)
// is 4096 points at a 1 KB stride, so per-thread loads and stores touch one
// cache line per point.  Here one cp.async.bulk.tensor box per CTA brings
// GP = 16 B / sizeof(C) neighbouring planes (i3 = GP m .. GP m + GP - 1: one
// 16-byte piece of every row) into shared memory as [i0][i2][g], and one
// tensor store writes the result back from the same buffer.  Thread group
// g = t / 256 transforms plane g exactly as k_dplane_r4 does.
// Map (innermost first, reals): (2 * 64, i2, i1, i0), box (2 GP, 64, 1, 64),
// 64 KB per box for both dtypes; the box's x coordinate is 16 m bytes.
// The load completes on an mbarrier whose wait is bounded: after the limit
// the CTA writes NaN into its first plane (the next reduction reports a
// non-finite norm), waits once more (bounded) and returns.
template <class C> struct PlaneMaps { CUtensorMap m[16]; };

namespace dpt {
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(r4t::sa(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(r4t::sa(bar))
        : "memory");
}
// issue and commit only (the issuing thread waits later, cp.async.bulk.wait_group.read)
__device__ __forceinline__ void tma_store_4d_issue(const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                                   const void* src) {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];"
                 ::"l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(r4t::sa(src))
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void tma_store_4d(const CUtensorMap* map, int c0, int c1, int c2, int c3, const void* src) {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];"
                 ::"l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(r4t::sa(src))
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
}  // namespace dpt

template <class C>
constexpr int dplane_gp() { return 16 / (int)sizeof(C); }
template <class C>
constexpr size_t dplane_r4t_smem_bytes() {
    return 128 + 65536 + 64 * sizeof(C) + 16 + 2 * 8 * 8 * sizeof(double) + 2 * 16 * sizeof(double);
}

// EPI (Theta -> P only): boundary_xp and Real_GPU of the diagonal on the
// transformed values before they are stored (the same rounding as the
// separate passes: the stored transform value, scaled in FP64 by the
// product of the four factors in the order k_dmask_real_reduce uses), and
// one row of DEPI_SUMS sums per plane of the stored result.  In a plane
// (i1, i3) only p_x = cpx[i2] and p_y = cpy[i0] vary, so each thread keeps
// seven moments (sum Re w * {1, p_x, p_x^2, p_y, p_y^2}, sum Im w * {1, p_y});
// one thread per plane turns the plane's moments into its component's share
// of the sums (depi_row).
namespace depi {
constexpr int NM = 7;
// the 20 sums of one component k from its plane's moments m at (x, y) with
// the field tables of the plane (A0..A3, D1A0..D1A2)
__device__ __forceinline__ void row(const DEpi& E, int k, double x, double y, const double (&A)[7],
                                    const double (&m)[NM], double* out) {
    double a[DEPI_SUMS];
#pragma unroll
    for (int q = 0; q < DEPI_SUMS; ++q) a[q] = 0.0;
    const double R0 = m[0], Rpx = m[1], Rpx2 = m[2], Rpy = m[3], Rpy2 = m[4], I0 = m[5], Ipy = m[6];
    const double c = E.c;
    if (k == 0 || k == 5 || k == 10 || k == 15) {          // the trace W11 + W22 + W33 + W44
        const double sg = k < 10 ? 1.0 : -1.0;             // mass term Re(W11 + W22 - W33 - W44)
        a[0] = R0; a[1] = I0;
        a[2] = x * R0; a[3] = Rpx; a[4] = x * x * R0; a[5] = Rpx2;
        a[6] = y * R0; a[7] = Rpy; a[8] = y * y * R0; a[9] = Rpy2;
        a[14] = sg * E.mass * c * c * R0;
        a[15] = c * A[0] * R0;
        a[16] = c * A[4] * R0;
    } else if (k == 3 || k == 12 || k == 6 || k == 9) {    // W14, W41, W23, W32
        // alpha1 = Re(W14 + W41 + W23 + W32); alpha2 = -Im(W14 - W41 + W32 - W23)
        const double tau = (k == 3 || k == 9) ? -1.0 : 1.0;
        a[10] = R0; a[12] = x * R0;
        a[11] = tau * I0; a[13] = tau * y * I0;
        a[14] = c * Rpx + tau * c * Ipy;
        a[17] = c * A[5] * R0;
        if (E.kvn) {   // k2 = Im(W14 - W41 - W23 + W32), and Re of the same combination
            const double kap = (k == 3 || k == 9) ? 1.0 : -1.0;
            a[15] = A[1] * c * R0 - A[2] * c * kap * I0;
            a[18] = c * A[6] * kap * R0;
        } else {       // e2 = Im(-W14 + W23 - W32 + W41) = alpha2
            a[15] = -A[1] * c * R0 - A[2] * c * tau * I0;
            a[18] = -A[6] * c * tau * I0;
        }
    } else if (!E.kvn && (k == 2 || k == 7 || k == 8 || k == 13)) {   // e3 = Re(-W13 + W24 - W31 + W42)
        const double eps = (k == 2 || k == 8) ? -1.0 : 1.0;
        a[15] = A[3] * c * eps * R0;
    }
#pragma unroll
    for (int q = 0; q < DEPI_SUMS; ++q) out[q] = a[q];
}
}  // namespace depi

template <class C, bool FWD, bool EPI = false>
__global__ void __launch_bounds__(r4::NT * dplane_gp<C>(), 2)
k_dplane_r4t(const __grid_constant__ PlaneMaps<C> maps, const __grid_constant__ PlaneSlots<C> S,
             const C* __restrict__ gtw, double2 scale, const double* __restrict__ d_norm,
             const __grid_constant__ DEpi E) {
    using namespace r4;
    constexpr int GP = dplane_gp<C>();
    extern __shared__ __align__(16) unsigned char smraw[];
    C* s = reinterpret_cast<C*>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
    C* tw = s + 4096 * GP;
    uint64_t* bar = reinterpret_cast<uint64_t*>(tw + 64);
    const int t = threadIdx.x & 255, grp = threadIdx.x >> 8, ac = t & 15, ar = t >> 4;
    const int i1 = blockIdx.x / (64 / GP), m = blockIdx.x % (64 / GP);
    const CUtensorMap* map = &maps.m[blockIdx.y];
    if (threadIdx.x == 0) {
        r4t::mbar_init(bar);
        r4t::fence_async_smem();
        r4t::mbar_expect_tx(bar, 65536);
        dpt::tma_load_4d(s, map, 2 * GP * m, 0, i1, 0, bar);
    }
    load_tw(tw, gtw, threadIdx.x);
    // EPI: the plane's constants (A0..A3, D1A0..D1A2 at (i1, i3), then x, y), read
    // now so that their latency hides behind the copy and the transform
    double* pconst = reinterpret_cast<double*>(bar + 2) + 2 * 64;
    if (EPI && t < 9) {
        const int i3c = GP * m + grp;
        pconst[grp * 16 + t] = t < 7 ? E.obs_xy[t * 4096 + i1 * 64 + i3c] : (t == 7 ? E.cx[i3c] : E.cy[i1]);
    }
    double2 sc = scale;
    if (d_norm) sc = zmul(sc, zinv(make_double2(d_norm[0], d_norm[1])));
    const C cc = to_c<C>(sc);
    __syncthreads();                                   // barrier initialised, twiddles ready
    if (!r4t::mbar_wait_bounded(bar)) {
        if (threadIdx.x == 0) {
            typedef typename real_of<C>::type R;
            S.p[blockIdx.y][(long long)i1 * 64 * 64 + GP * m].x = (R)__longlong_as_double(0x7ff8000000000000LL);
        }
        r4t::mbar_wait_bounded(bar);
        return;
    }
    C v[16];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) v[4 * i + j] = s[((ar + 16 * i) * 64 + ac + 16 * j) * GP + grp];
    if ((ar + ac) & 1) {
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = cneg(v[k]);
    }
    C* sg = s + 4096 * grp;                            // this group's exchange plane
    const Lay L1 = lay1(t), L2 = lay2(t), L3 = lay3(t);
    __syncthreads();                                   // the box has been read
    pass<C, FWD>(v);
    twiddle<C, FWD>(v, tw, ac, ar);
    put(sg, L1, v);
    __syncthreads();
    get(sg, L2, v);
    pass<C, FWD>(v);
    twiddle<C, FWD>(v, tw, 4 * (t & 3), 4 * ((t >> 4) & 3));
    __syncthreads();
    put(sg, L2, v);
    __syncthreads();
    get(sg, L3, v);
    pass<C, FWD>(v);
    const int c1 = t & 3, c2 = (t >> 2) & 3, r1 = (t >> 4) & 3, r2 = t >> 6;
    const C ccs = ((r2 + c2) & 1) ? cneg(cc) : cc;
    __syncthreads();                                   // every group's last exchange has been read
    if (!EPI) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
                s[((r2 + 4 * r1 + 16 * i) * 64 + c2 + 4 * c1 + 16 * j) * GP + grp] = cmul(v[4 * i + j], ccs);
    } else {
        // output point (i0, i2) = (r2 + 4 r1 + 16 i, c2 + 4 c1 + 16 j) of plane (i1, i3)
        const int slot = blockIdx.y, i3 = GP * m + grp;
        const bool diag = slot == 0 || slot == 5 || slot == 10 || slot == 15;
        const double m13 = E.mxp[3][i3], m11 = E.mxp[1][i1];
        // this thread's four columns i2: held in registers for complex128; the
        // complex64 kernel (64 registers) reads them per point
        constexpr bool HOLD = sizeof(C) == 16;
        double m2[4], pxj[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            m2[j] = HOLD ? E.mxp[2][c2 + 4 * c1 + 16 * j] : 0.0;
            pxj[j] = HOLD ? E.cpx[c2 + 4 * c1 + 16 * j] : 0.0;
        }
        double mo[depi::NM];
#pragma unroll
        for (int q = 0; q < depi::NM; ++q) mo[q] = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int i0 = r2 + 4 * r1 + 16 * i;
            const double m0 = E.mxp[0][i0], py = E.cpy[i0];
            double sr = 0.0, sx = 0.0, sx2 = 0.0, si = 0.0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int i2 = c2 + 4 * c1 + 16 * j;
                const double r = (HOLD ? m2[j] : E.mxp[2][i2]) * m0 * m13 * m11;
                const double2 d = to_d2(cmul(v[4 * i + j], ccs));   // the value a plain transform stores
                C w = to_c<C>(make_double2(d.x * r, d.y * r));
                if (diag) w.y = 0;
                s[(i0 * 64 + i2) * GP + grp] = w;
                const double px = HOLD ? pxj[j] : E.cpx[i2], wr = (double)w.x, wi = (double)w.y;
                sr += wr; sx = fma(px, wr, sx); sx2 = fma(px * px, wr, sx2); si += wi;
            }
            mo[0] += sr; mo[1] += sx; mo[2] += sx2;
            mo[3] = fma(py, sr, mo[3]); mo[4] = fma(py * py, sr, mo[4]);
            mo[5] += si; mo[6] = fma(py, si, mo[6]);
        }
        // plane sums: warps, then the group's 8 warps in shared memory
#pragma unroll
        for (int q = 0; q < depi::NM; ++q)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) mo[q] += __shfl_down_sync(0xffffffffu, mo[q], o);
        double* red = reinterpret_cast<double*>(bar + 2) + grp * 64;
        const int w = t >> 5, l = t & 31;
        if (l == 0)
#pragma unroll
            for (int q = 0; q < depi::NM; ++q) red[w * 8 + q] = mo[q];
        r4t::fence_async_smem();                       // generic-proxy writes visible to the tensor store
        __syncthreads();
        // the store leaves first; each group's thread 0 then turns its plane's
        // moments into the plane's row while the copy reads shared memory
        if (threadIdx.x == 0) dpt::tma_store_4d_issue(map, 2 * GP * m, 0, i1, 0, s);
        if (t == 0) {
            double tot[depi::NM];
#pragma unroll
            for (int q = 0; q < depi::NM; ++q) {
                tot[q] = 0.0;
                for (int ww = 0; ww < 8; ++ww) tot[q] += red[ww * 8 + q];
            }
            const double* pc = pconst + grp * 16;
            double A[7];
#pragma unroll
            for (int q = 0; q < 7; ++q) A[q] = pc[q];
            const long long ixy = (long long)i1 * 64 + i3;
            depi::row(E, slot, pc[7], pc[8], A, tot, E.rows + ((long long)slot * 4096 + ixy) * DEPI_SUMS);
        }
        if (threadIdx.x == 0) r4ring::bulk_wait_read();    // the copy has read the box before the CTA exits
        return;
    }
    r4t::fence_async_smem();                           // generic-proxy writes visible to the tensor store
    __syncthreads();
    if (threadIdx.x == 0) dpt::tma_store_4d(map, 2 * GP * m, 0, i1, 0, s);
}

