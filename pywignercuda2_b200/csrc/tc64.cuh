// tc64.cuh -- complex64 64^4 Run() half-steps with the 64-point transforms
// on the tensor cores (tcgen05.mma, kind::f16, FP32 accumulation in tensor
// memory).  Included by wigner4d.cu after r4.cuh.
//
// Work unit: a quad of four planes (f0, 4m .. 4m+3), two plane pairs.  A
// pair is one M = 128 tile: row m = p * 64 + i (p the plane of the pair, i
// the in-plane index the stage keeps).  The 2-D transform of a plane and its
// inverse are four dense complex GEMMs per pair, each written as a real GEMM
// with the complex matrix embedded as [[Fr, Fi], [-Fi, Fr]] (K = N = 128):
//   stage 1  Z  = X F^T      A1[(p, r), (ri, c)]  = X[r][c]       (K-major)
//   stage 2  Y  = F Z        A2[(p, kc), (ri, r)] = Z[r][kc]      (MN-major)
//   factor   Y' = Y * a(kr) b(kc), then conjugated
//   stage 3  Z3 = conj(F conj(Y'))  A3[(p, kc), (ri, kr)]         (K-major)
//   stage 4  X' = conj(conj(Z3) F^T) A4[(p, r), (ri, kc)]         (MN-major)
// F[k][n] = exp(-2 pi i k n / 64) (the plain DFT; the centring signs are in
// the per-plane factor vectors, read at frequencies shifted by N/2, exactly
// as k_r4 uses them).  The thread that owns TMEM lane m of a stage's result
// holds a whole row of it (128 FP32 columns: 64 real, 64 imaginary parts)
// and writes it into the next stage's operand: its own row (K-major) or one
// K-row of the transposed operand (MN-major, 16-byte chunks).  Every write
// is free of shared-memory bank conflicts.
//
// Precision: each operand is a pair of fp16 values, hi = fp16(v) and
// lo = fp16(v - hi), and each GEMM is three products, A_hi B_hi + A_lo B_hi +
// A_hi B_lo (about 22 significant bits, FP32 accumulation).  Before each
// split the pair's values are scaled by a power of two so that their
// largest magnitude lies in [2^14, 2^15), and the DFT matrix is stored
// times 2^14: lo stays a normal fp16 number down to 2^-18 of the largest
// value (below that it is subnormal, absolute error 2^-40 of the largest).
// The scales are undone exactly at the end.  The factor multiply uses
// float-float products of the FP64 factor vectors; the observable sums are
// in FP64 above the row level (a row's 64 terms are
// summed in float32, with the K(p) table and the p_x coordinates held in
// shared memory rounded to float32).
//
// Global layouts during Run() (both symmetric under (y, x) <-> (p_y, p_x)):
//   LK = [y][x/4][p_y][p_x/4][x%4][p_x%4]   kinetic source, potential destination
//   LP = [p_y][p_x/4][y][x/4][p_x%4][x%4]   kinetic destination, potential source
// For plane (f0, f1 = 4 m + q) and in-plane point (r, c) a half-step reads
//   src[((((r*16 + c/4)*64 + f0)*16 + m)*4 + c%4)*4 + q]
// (the quad's four planes at four c form a 128-byte line) and writes
//   dst[((((f0*16 + m)*64 + r)*16 + c/4)*4 + q)*4 + c%4]
// (each thread writes 32 contiguous bytes per four c).
//
// Waits on the MMA completion barrier are bounded (about a second of clock
// cycles); a wait that gives up sets *flag = WIG_ERR_TIMEOUT and the
// kernel writes NaN instead of its results, so Run()'s history is
// non-finite and the host raises.
#pragma once

#include <cuda_fp16.h>

namespace tc64 {

constexpr int NT = 512;                          // two pairs of eight warps
constexpr int PT = 256;                          // threads of a pair
constexpr int OP_BYTES = 32768;                  // one 128 x 128 fp16 operand
constexpr int A_OFF = 0;                         // pair g: hi at g * 64K, lo at + 32K
constexpr int B_OFF = 4 * OP_BYTES;              // B hi, then B lo
constexpr int PV_OFF = B_OFF + 2 * OP_BYTES;     // pair g: 2 planes x 64 (row factor hi, lo) float2 pairs
constexpr int RED_OFF = PV_OFF + 2 * 2 * 64 * 16;  // 16 warps x NPART doubles
constexpr int EP_LD = 65;                       // padded row of the K(p) table
constexpr int EP_OFF = RED_OFF + 16 * NPART * 8; // K(p_y, p_x) as float32 [64][EP_LD]
constexpr int QX_OFF = EP_OFF + 64 * EP_LD * 4;  // p_x coordinate as float32 [64]
constexpr int MX_OFF = QX_OFF + 64 * 4;          // 16 floats (pair max per warp)
constexpr int BAR_OFF = MX_OFF + 64;             // 2 mbarriers
constexpr int TM_OFF = BAR_OFF + 16;             // TMEM base address
constexpr int SMEM = TM_OFF + 16;
static_assert(SMEM <= 232448, "k_tc64 shared memory above the per-CTA limit");
constexpr long long TIMEOUT_CYCLES = 2000000000LL;
constexpr int OP_EXP = 15;                       // operands scaled to [2^14, 2^15)
constexpr int B_EXP = 14;                        // the DFT matrix is stored times 2^14

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: no swizzle, LBO = 2048 B between the two
// K-chunks of one MMA, SBO = 128 B between 8-row core-matrix groups.
__device__ __forceinline__ uint64_t desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(2048 >> 4) << 16) | ((uint64_t)(128 >> 4) << 32) |
           ((uint64_t)1 << 46);
}

// kind::f16 instruction descriptor: fp16 A and B, FP32 D, M = N = 128,
// B K-major, A K-major (mn = 0) or MN-major (mn = 1).
__device__ __forceinline__ uint32_t idesc(int mn) {
    return (1u << 4) | ((uint32_t)mn << 15) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
}

// One stage of a pair: D = A_hi B_hi + A_lo B_hi + A_hi B_lo over K = 128,
// then a commit that arrives on mbar when the products are done.
__device__ __forceinline__ void issue_stage(uint32_t dtm, uint32_t a_hi, uint32_t b_hi, int mn, uint32_t mbar) {
    const uint32_t id = idesc(mn);
#pragma unroll
    for (int pass = 0; pass < 3; ++pass) {
        const uint32_t a = a_hi + (pass == 1 ? OP_BYTES : 0), b = b_hi + (pass == 2 ? OP_BYTES : 0);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint64_t ad = desc(a + j * 4096), bd = desc(b + j * 4096);
            const uint32_t acc = (pass | j) != 0;
            asm volatile("{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                         "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                         ::"r"(dtm), "l"(ad), "l"(bd), "r"(id), "r"(acc));
        }
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

// Bounded wait for the phase with the given parity; false if it gave up.
__device__ __forceinline__ bool wait_phase(uint32_t mbar, uint32_t parity) {
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile("{\n.reg .pred P1;\nmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n"
                     "selp.b32 %0, 1, 0, P1;\n}\n"
                     : "=r"(done) : "r"(mbar), "r"(parity) : "memory");
        if (done) return true;
        if (clock64() - t0 > TIMEOUT_CYCLES) return false;
    }
}

__device__ __forceinline__ void pair_sync(int g) {
    asm volatile("bar.sync %0, 256;" ::"r"(1 + g) : "memory");
}

// 32 consecutive FP32 columns of this warp's TMEM lanes.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                   "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                   "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t h2u(__half2 h) { return *reinterpret_cast<uint32_t*>(&h); }

// v rounded to 11 significant bits (Veltkamp's split with 2^13 + 1; the
// intrinsics keep the compiler from contracting it into an FMA)
__device__ __forceinline__ float round11(float v) {
    const float t = __fmul_rn(v, 8193.0f);
    return __fsub_rn(t, __fsub_rn(t, v));
}

// hi = fp16(a), lo = fp16(a - hi) for two values, packed (first in the low
// half).  hi is formed in float32 (exact in fp16 for |a| >= 2^-14), so only
// the two packing conversions remain.
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
    const float ah = round11(a), bh = round11(b);
    hi = h2u(__floats2half2_rn(ah, bh));
    lo = h2u(__floats2half2_rn(__fsub_rn(a, ah), __fsub_rn(b, bh)));
}

// Largest |value| of the pair (256 threads): each thread passes its own
// maximum (non-negative); returns the power-of-two exponent e with
// max * 2^-e in [2^14, 2^15) (-OP_EXP for an all-zero pair).
__device__ __forceinline__ int pair_exponent(float mx, int g, int wp, int lane, float* slots) {
    const unsigned m = __reduce_max_sync(0xffffffffu, __float_as_uint(mx));
    if (lane == 0) slots[8 * g + wp] = __uint_as_float(m);
    pair_sync(g);
    float M = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) M = fmaxf(M, slots[8 * g + k]);
    int e = (M > 0.0f) ? (int)((__float_as_uint(M) >> 23) & 0xff) - 126 : 0;
    e = e < -110 ? -110 : (e > 110 ? 110 : e);
    return e - OP_EXP;
}

__device__ __forceinline__ float pow2f(int e) { return __uint_as_float((uint32_t)(127 + e) << 23); }

}  // namespace tc64

// One half-step, persistent (one CTA of two independent plane pairs per SM).
// A pair's work unit is half a quad: unit u covers planes (f0, 4m + 2h + p),
// p = 0, 1, with (f0, m) = quad u/2 and h = u%2; pair g of CTA b takes the
// units 2b + g, 2b + g + 2 gridDim, ...
//   KIN: src LK -> dst LP, the plane vectors of the kinetic half-step, and
//        the state divided by *d_norm;
//   POT: src LP -> dst LK, the potential plane vectors, and one NPART
//        partial row per plane (observables of the new state).
// bimg: the 64 KB shared-memory image of the embedded DFT matrix (hi, lo).
// Thread roles within a pair: warp wp = 0..7 reads TMEM lanes 32 (wp % 4) ..
// (its row m = 32 (wp % 4) + lane, plane p = m / 64, row index ii = m % 64)
// and the half hf = wp / 4 of the row's 64 complex values.
template <bool KIN>
__global__ void __launch_bounds__(tc64::NT, 1)
k_tc64(const float2* __restrict__ src, float2* __restrict__ dst, const double2* __restrict__ PV,
       const uint4* __restrict__ bimg, double2 scale, const double* __restrict__ d_norm, ObsTabs ob,
       double* __restrict__ partials, int* __restrict__ flag) {
    using namespace tc64;
    extern __shared__ __align__(1024) unsigned char sm[];
    const int t = threadIdx.x, g = t >> 8, tp = t & 255, wp = tp >> 5, lane = t & 31;
    const int quarter = wp & 3, hf = wp >> 2;
    const int m = 32 * quarter + lane, p = m >> 6, ii = m & 63;
    float4* pvs = reinterpret_cast<float4*>(sm + PV_OFF) + g * 128;   // [plane][kr]: (hi, lo) of a(kr)
    double* red = reinterpret_cast<double*>(sm + RED_OFF);
    float* slots = reinterpret_cast<float*>(sm + MX_OFF);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + BAR_OFF);
    uint32_t* tmp = reinterpret_cast<uint32_t*>(sm + TM_OFF);
    const uint32_t a_hi = su32(sm + A_OFF + g * 2 * OP_BYTES), b_hi = su32(sm + B_OFF);
    const uint32_t mbar = su32(bars + g);
    unsigned char* Ahi = sm + A_OFF + g * 2 * OP_BYTES;
    unsigned char* Alo = Ahi + OP_BYTES;

    // ---- set-up: B image, tables, barriers, tensor memory (128 columns per pair)
    for (int e = t; e < 2 * OP_BYTES / 16; e += NT) reinterpret_cast<uint4*>(sm + B_OFF)[e] = __ldg(bimg + e);
    float* eps = reinterpret_cast<float*>(sm + EP_OFF);
    float* qxs = reinterpret_cast<float*>(sm + QX_OFF);
    if (!KIN) {
        for (int e = t; e < 64 * 64; e += NT) eps[(e >> 6) * EP_LD + (e & 63)] = (float)__ldg(ob.ep + e);
        if (t < 64) qxs[t] = (float)__ldg(ob.cpx + t);
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(bars)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(bars + 1)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (t < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(su32(tmp)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t dtm = *tmp + 128u * g;                        // this pair's accumulator
    const uint32_t tl = dtm + ((uint32_t)(32 * quarter) << 16);  // this warp's lanes
    double2 cc = scale;
    if (KIN && d_norm) cc = zmul(cc, zinv(make_double2(d_norm[0], d_norm[1])));
    uint32_t phase = 0;
    bool ok = true;

    for (int u = 2 * blockIdx.x + g; u < 2048; u += 2 * gridDim.x) {
        const int quad = u >> 1, half = u & 1, f0 = quad >> 4, m4 = quad & 15;
        const int plane0 = f0 * 64 + 4 * m4 + 2 * half;           // first plane of this unit
        // row factor vectors of the unit as float-float (used after stage 2)
        if (tp < 128) {
            float2 h, l;
            ff::split_hl(__ldg(PV + (long long)(plane0 + (tp >> 6)) * 128 + (tp & 63)), h, l);
            pvs[tp] = make_float4(h.x, h.y, l.x, l.y);
        }
        int E;
        // ---- load: 4 runs per thread, each 4 c of both planes of the unit
        {
            float4 x[4][4];
            float mx = 0.0f;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = (lane & 7) + 8 * (4 * hf + i), c4 = ((lane >> 3) & 3) + 4 * quarter;
                const float4* s4 = reinterpret_cast<const float4*>(
                    src + ((long long)(r * 16 + c4) * 64 + f0) * 256 + m4 * 16 + 2 * half);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    x[i][j] = __ldg(s4 + 2 * j);
                    mx = fmaxf(mx, fmaxf(fmaxf(fabsf(x[i][j].x), fabsf(x[i][j].y)),
                                         fmaxf(fabsf(x[i][j].z), fabsf(x[i][j].w))));
                }
            }
            E = pair_exponent(mx, g, wp, lane, slots);
            const float s = pow2f(-E);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = (lane & 7) + 8 * (4 * hf + i), c4 = ((lane >> 3) & 3) + 4 * quarter;
#pragma unroll
                for (int pp = 0; pp < 2; ++pp)
#pragma unroll
                    for (int ri = 0; ri < 2; ++ri) {
                        float v[4];
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            v[j] = s * (pp == 0 ? (ri ? x[i][j].y : x[i][j].x) : (ri ? x[i][j].w : x[i][j].z));
                        uint2 h, lo;
                        split2(v[0], v[1], h.x, lo.x);
                        split2(v[2], v[3], h.y, lo.y);
                        const int mrow = pp * 64 + r, k0 = ri * 64 + 4 * c4;
                        const int off = (k0 >> 3) * 2048 + (mrow >> 3) * 128 + (mrow & 7) * 16 + (k0 & 7) * 2;
                        *reinterpret_cast<uint2*>(Ahi + off) = h;
                        *reinterpret_cast<uint2*>(Alo + off) = lo;
                    }
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        pair_sync(g);
        if (tp == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            issue_stage(dtm, a_hi, b_hi, 0, mbar);
        }
        // ---- stages 1..3: result -> next operand.  This thread's 64 values:
        // v[j] = Re, v[32 + j] = Im of index 32 hf + j of its row.
#pragma unroll 1
        for (int st = 1; st <= 3; ++st) {
            ok = wait_phase(mbar, phase) && ok;
            phase ^= 1u;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            float v[64];
            tmem_ld32(tl + 32 * hf, v);
            tmem_ld32(tl + 64 + 32 * hf, v + 32);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (st == 2) {
                // factor a(kr) b(kc) as float-float products; this thread's kc = ii
                float2 bh, bl;
                ff::split_hl(__ldg(PV + (long long)(plane0 + p) * 128 + 64 + ii), bh, bl);
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const float4 a = pvs[p * 64 + 32 * hf + j];
                    float2 w = ff::fmul_hl(make_float2(v[j], v[32 + j]), bh, bl);
                    w = ff::fmul_hl(w, make_float2(a.x, a.y), make_float2(a.z, a.w));
                    v[j] = w.x;
                    v[32 + j] = w.y;
                }
            }
            float mx = 0.0f;
#pragma unroll
            for (int k = 0; k < 64; ++k) mx = fmaxf(mx, fabsf(v[k]));
            const int e = pair_exponent(mx, g, wp, lane, slots);
            E += e - B_EXP;
            const float s = pow2f(-e), si = (st == 2) ? -s : s;     // conjugate the stage-3 operand
#pragma unroll
            for (int ri = 0; ri < 2; ++ri)
#pragma unroll
                for (int j4 = 0; j4 < 4; ++j4) {
                    uint4 h, lo;
                    const float* w = v + ri * 32 + j4 * 8;
                    const float sc = ri ? si : s;
                    split2(sc * w[0], sc * w[1], h.x, lo.x);
                    split2(sc * w[2], sc * w[3], h.y, lo.y);
                    split2(sc * w[4], sc * w[5], h.z, lo.z);
                    split2(sc * w[6], sc * w[7], h.w, lo.w);
                    const int j8 = 4 * hf + j4;              // chunk of 8 along the row
                    int off;
                    if (st == 2) {
                        // K-major: this thread's own row, K = (ri, kr)
                        off = (ri * 8 + j8) * 2048 + (m >> 3) * 128 + (m & 7) * 16;
                    } else {
                        // MN-major: K-row (ri, ii), M = (p, j)
                        const int kk = ri * 64 + ii;
                        off = (kk >> 3) * 2048 + (p * 8 + j8) * 128 + (kk & 7) * 16;
                    }
                    *reinterpret_cast<uint4*>(Ahi + off) = h;
                    *reinterpret_cast<uint4*>(Alo + off) = lo;
                }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            pair_sync(g);
            if (tp == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                issue_stage(dtm, a_hi, b_hi, st == 2 ? 0 : 1, mbar);
            }
        }
        // ---- stage 4 result: row ii of plane p, X'[ii][c] = conj(D4) 2^E cc
        ok = wait_phase(mbar, phase) && ok;
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        float v[64];
        tmem_ld32(tl + 32 * hf, v);
        tmem_ld32(tl + 64 + 32 * hf, v + 32);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        const int Et = E - B_EXP;                                   // stage 4's product
        const double2 ce = make_double2(ldexp(cc.x, Et), ldexp(cc.y, Et));
        const float2 cf = make_float2((float)ce.x, (float)ce.y);
        const float nan = __int_as_float(0x7fc00000);
        const int q = 2 * half + p;
        float2* d = dst + (((long long)(f0 * 16 + m4) * 64 + ii) * 16) * 16 + q * 4;
        // row sums of the new state in float32 (two interleaved accumulators
        // of 16 terms each), combined in FP64 below
        float sa[2][8];
#pragma unroll
        for (int h2 = 0; h2 < 2; ++h2)
#pragma unroll
            for (int k = 0; k < 8; ++k) sa[h2][k] = 0.0f;
#pragma unroll
        for (int c4l = 0; c4l < 8; ++c4l) {
            const int c4 = 8 * hf + c4l;
            float2 o[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int jl = 4 * c4l + j, c = 4 * c4 + j;
                const float re = v[jl], im = -v[32 + jl];           // conj(D4)
                o[j] = ok ? make_float2(re * cf.x - im * cf.y, re * cf.y + im * cf.x) : make_float2(nan, nan);
                if (!KIN) {
                    float* s = sa[c4l & 1];
                    const float qx = qxs[c], kk = eps[ii * EP_LD + c], wx = o[j].x, wy = o[j].y;
                    s[0] += wx; s[1] += wy;
                    s[2] = fmaf(qx, wx, s[2]); s[3] = fmaf(qx, wy, s[3]);
                    s[4] = fmaf(qx * qx, wx, s[4]); s[5] = fmaf(qx * qx, wy, s[5]);
                    s[6] = fmaf(kk, wx, s[6]); s[7] = fmaf(kk, wy, s[7]);
                }
            }
            float4* d4 = reinterpret_cast<float4*>(d + c4 * 16);
            d4[0] = make_float4(o[0].x, o[0].y, o[1].x, o[1].y);
            d4[1] = make_float4(o[2].x, o[2].y, o[3].x, o[3].y);
        }
        if (!KIN) {
            double a[NPART];
            a[0] = (double)sa[0][0] + sa[1][0]; a[1] = (double)sa[0][1] + sa[1][1];
            a[2] = (double)sa[0][2] + sa[1][2]; a[3] = (double)sa[0][3] + sa[1][3];
            a[4] = (double)sa[0][4] + sa[1][4]; a[5] = (double)sa[0][5] + sa[1][5];
            a[10] = (double)sa[0][6] + sa[1][6]; a[11] = (double)sa[0][7] + sa[1][7];
            const double qy = __ldg(ob.cpy + ii);
            a[6] = qy * a[0]; a[7] = qy * a[1];
            a[8] = qy * qy * a[0]; a[9] = qy * qy * a[1];
#pragma unroll
            for (int k = 0; k < NPART; ++k) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_down_sync(0xffffffffu, a[k], o);
            }
            if (lane == 0) {
#pragma unroll
                for (int k = 0; k < NPART; ++k) red[(8 * g + wp) * NPART + k] = a[k];
            }
            pair_sync(g);
            if (tp < 2 * NPART) {
                // plane pq of the unit: warps with quarter 2 pq, 2 pq + 1 and both halves
                const int pq = tp / NPART, k = tp % NPART;
                const double sum = red[(8 * g + 2 * pq) * NPART + k] + red[(8 * g + 2 * pq + 1) * NPART + k] +
                                   red[(8 * g + 2 * pq + 4) * NPART + k] + red[(8 * g + 2 * pq + 5) * NPART + k];
                partials[(long long)(plane0 + pq) * NPART + k] = ok ? sum : (double)nan;
            }
        }
    }
    if (!ok && tp == 0) atomicExch(flag, WIG_ERR_TIMEOUT);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (t < 32) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(*tmp));
    }
}

// L0 = [p_y][y][p_x][x] -> LK; one thread per LK element.
__global__ void k_to_tc_layout(const float2* __restrict__ W, float2* __restrict__ P, long long n) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int pxr = (int)(e & 3), xr = (int)((e >> 2) & 3), px4 = (int)((e >> 4) & 15);
        const int py = (int)((e >> 8) & 63), x4 = (int)((e >> 14) & 15), y = (int)(e >> 18);
        P[e] = W[(((long long)py * 64 + y) * 64 + 4 * px4 + pxr) * 64 + 4 * x4 + xr];
    }
}

// LK -> L0, divided by the complex norm (none when d_norm is null).
__global__ void k_from_tc_layout(const float2* __restrict__ P, float2* __restrict__ W, long long n,
                                 const double* __restrict__ d_norm) {
    const double2 inv = d_norm ? zinv(make_double2(d_norm[0], d_norm[1])) : make_double2(1.0, 0.0);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(e & 63), px = (int)((e >> 6) & 63), y = (int)((e >> 12) & 63), py = (int)(e >> 18);
        const float2 a = P[((((long long)y * 16 + x / 4) * 64 + py) * 16 + px / 4) * 16 + (x % 4) * 4 + px % 4];
        const double2 r = zmul(make_double2(a.x, a.y), inv);
        W[e] = make_float2((float)r.x, (float)r.y);
    }
}
