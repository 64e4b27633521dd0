// fft_smem.cuh -- batched 1-D transforms over lines held in shared memory.
//
// A "line" is N complex values at s[base(line) + n * es].  Two engines:
//  * radix (N = 16, 32, 64, 128): Stockham autosort passes of radix 8/4/2,
//    natural order in and out, computed in place with a read -> sync -> write
//    pattern (every thread keeps its butterflies in registers across the
//    barrier, so no second buffer is needed);
//  * dense (any N): out[k] = sum_n M[k][n] in[n] with M in global memory,
//    for the fractional transform with |delta| N != 1.
// Twiddles are generated in FP64 (sincospi) and rounded once to the line's
// precision.
#pragma once
#include "common.cuh"

struct LineMap {
    int nB;       // line = a * nB + b
    int sA, sB;   // base(line) = a * sA + b * sB
    int es;       // element stride within a line
    __device__ __forceinline__ int base(int line) const {
        return (nB == 1) ? line * sA : (line / nB) * sA + (line % nB) * sB;
    }
};

// tw[m] = exp(-2 pi i m / N), m in [0, N)
template <class C>
__device__ __forceinline__ void make_twiddles(C* tw, int n) {
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
        double s, c;
        sincospi(-2.0 * (double)m / (double)n, &s, &c);
        tw[m] = mk<C>((typename real_of<C>::type)c, (typename real_of<C>::type)s);
    }
}

// ---- radix butterflies (FWD: exp(-2 pi i / R) kernel; inverse: conjugate) ----
template <class C, bool FWD> __device__ __forceinline__ void dft2(C& a, C& b) {
    C t = a; a = cadd(t, b); b = csub(t, b);
}
template <class C, bool FWD> __device__ __forceinline__ void dft4(C& v0, C& v1, C& v2, C& v3) {
    C t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3);
    C t3 = mul_mi<C, FWD>(csub(v1, v3));
    v0 = cadd(t0, t2); v2 = csub(t0, t2); v1 = cadd(t1, t3); v3 = csub(t1, t3);
}
template <class C, bool FWD> __device__ __forceinline__ void dft8(C* v) {
    typedef typename real_of<C>::type R;
    const R h = (R)0.70710678118654752440;
    C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<C, FWD>(e0, e1, e2, e3);
    dft4<C, FWD>(o0, o1, o2, o3);
    // o_k *= w8^k
    C w1, w3;
    if (FWD) {
        w1 = mk<C>((o1.x + o1.y) * h, (o1.y - o1.x) * h);
        w3 = mk<C>((o3.y - o3.x) * h, -(o3.x + o3.y) * h);
    } else {
        w1 = mk<C>((o1.x - o1.y) * h, (o1.x + o1.y) * h);
        w3 = mk<C>(-(o3.x + o3.y) * h, (o3.x - o3.y) * h);
    }
    C w2 = mul_mi<C, FWD>(o2);
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, w1); v[5] = csub(e1, w1);
    v[2] = cadd(e2, w2); v[6] = csub(e2, w2);
    v[3] = cadd(e3, w3); v[7] = csub(e3, w3);
}
// 3-point DFT: y1,2 = x0 - (x1 + x2)/2 -+ i (sqrt3/2)(x1 - x2) (FWD), signs of i swapped otherwise
template <class C, bool FWD> __device__ __forceinline__ void dft3(C& v0, C& v1, C& v2) {
    typedef typename real_of<C>::type R;
    const R h = (R)0.86602540378443864676;
    const C t1 = cadd(v1, v2), t2 = csub(v1, v2);
    const C m = mk<C>(v0.x - (R)0.5 * t1.x, v0.y - (R)0.5 * t1.y);
    const C s = FWD ? mk<C>(h * t2.y, -h * t2.x) : mk<C>(-h * t2.y, h * t2.x);   // -+ i h t2
    v0 = cadd(v0, t1);
    v1 = cadd(m, s);
    v2 = csub(m, s);
}
template <class C, int R, bool FWD> __device__ __forceinline__ void dft_r(C* v) {
    if (R == 2) dft2<C, FWD>(v[0], v[1]);
    else if (R == 3) dft3<C, FWD>(v[0], v[1], v[2]);
    else if (R == 4) dft4<C, FWD>(v[0], v[1], v[2], v[3]);
    else dft8<C, FWD>(v);
}

// One Stockham pass of radix R over L lines of length N, with NT threads.
// LINE_FAST: consecutive threads take consecutive lines (strided element
// axis); otherwise consecutive butterflies of one line (contiguous axis).
template <class C, int N, int R, int L, int NT, bool FWD, bool LINE_FAST>
__device__ __forceinline__ void stockham_pass(C* s, const LineMap& m, int Ns, const C* tw) {
    constexpr int B = N / R;
    constexpr int TOT = L * B;
    constexpr int PER = (TOT + NT - 1) / NT;
    C v[PER][R];
    const int tid = threadIdx.x;
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int t = tid + i * NT;
        if ((TOT % NT) == 0 || t < TOT) {
            const int line = LINE_FAST ? (t % L) : (t / B);
            const int j = LINE_FAST ? (t / L) : (t % B);
            const C* p = s + m.base(line);
#pragma unroll
            for (int r = 0; r < R; ++r) v[i][r] = p[(j + r * B) * m.es];
            if (Ns > 1) {
                const int k = j & (Ns - 1);
                const int step = N / (Ns * R);
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    C w = tw[r * k * step];          // r k step < N
                    if (!FWD) w = cconj(w);
                    v[i][r] = cmul(v[i][r], w);
                }
            }
            dft_r<C, R, FWD>(v[i]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int t = tid + i * NT;
        if ((TOT % NT) == 0 || t < TOT) {
            const int line = LINE_FAST ? (t % L) : (t / B);
            const int j = LINE_FAST ? (t / L) : (t % B);
            const int k = j & (Ns - 1);
            C* p = s + m.base(line);
            const int o = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) p[(o + r * Ns) * m.es] = v[i][r];
        }
    }
    __syncthreads();
}

// Full length-N transform of L lines (N in {16, 32, 48, 64, 128}).
template <class C, int N, int L, int NT, bool FWD, bool LINE_FAST>
__device__ __forceinline__ void fft_lines(C* s, const LineMap& m, const C* tw) {
    if (N == 16) {
        stockham_pass<C, N, 4, L, NT, FWD, LINE_FAST>(s, m, 1, tw);
        stockham_pass<C, N, 4, L, NT, FWD, LINE_FAST>(s, m, 4, tw);
    } else if (N == 32) {
        stockham_pass<C, N, 8, L, NT, FWD, LINE_FAST>(s, m, 1, tw);
        stockham_pass<C, N, 4, L, NT, FWD, LINE_FAST>(s, m, 8, tw);
    } else if (N == 48) {
        stockham_pass<C, N, 4, L, NT, FWD, LINE_FAST>(s, m, 1, tw);
        stockham_pass<C, N, 4, L, NT, FWD, LINE_FAST>(s, m, 4, tw);
        stockham_pass<C, N, 3, L, NT, FWD, LINE_FAST>(s, m, 16, tw);
    } else if (N == 64) {
        stockham_pass<C, N, 8, L, NT, FWD, LINE_FAST>(s, m, 1, tw);
        stockham_pass<C, N, 8, L, NT, FWD, LINE_FAST>(s, m, 8, tw);
    } else if (N == 128) {
        stockham_pass<C, N, 8, L, NT, FWD, LINE_FAST>(s, m, 1, tw);
        stockham_pass<C, N, 8, L, NT, FWD, LINE_FAST>(s, m, 8, tw);
        stockham_pass<C, N, 2, L, NT, FWD, LINE_FAST>(s, m, 64, tw);
    }
}

// Dense transform of L lines of runtime length n with matrix M[k * n + j]
// (global memory, read through the read-only path).  CONJ uses conj(M).
template <class C, bool CONJ>
__device__ __forceinline__ void dense_lines(C* s, const LineMap& m, int L, int n,
                                            const C* __restrict__ M, bool line_fast) {
    // Lines are independent, so they are transformed in groups small enough
    // that every output of a group (at most 16 per thread) is held in
    // registers until the whole group has been read.
    int lc = (16 * (int)blockDim.x) / n;
    if (lc < 1) lc = 1;
    if (lc > L) lc = L;
    for (int l0 = 0; l0 < L; l0 += lc) {
        const int nl = (L - l0 < lc) ? (L - l0) : lc;
        const int tot = nl * n;
        C acc[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int t = threadIdx.x + i * blockDim.x;
            acc[i] = mk<C>(0, 0);
            if (t < tot) {
                const int line = l0 + (line_fast ? (t % nl) : (t / n));
                const int k = line_fast ? (t / nl) : (t % n);
                const C* p = s + m.base(line);
                const C* row = M + (size_t)k * n;
                C a = mk<C>(0, 0);
                for (int j = 0; j < n; ++j) {
                    C w = __ldg(row + j);
                    if (CONJ) w = cconj(w);
                    C x = p[j * m.es];
                    a.x = fma(w.x, x.x, a.x); a.x = fma(-w.y, x.y, a.x);
                    a.y = fma(w.x, x.y, a.y); a.y = fma(w.y, x.x, a.y);
                }
                acc[i] = a;
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int t = threadIdx.x + i * blockDim.x;
            if (t < tot) {
                const int line = l0 + (line_fast ? (t % nl) : (t / n));
                const int k = line_fast ? (t / nl) : (t % n);
                s[m.base(line) + k * m.es] = acc[i];
            }
        }
        __syncthreads();
    }
}
