// common.cuh -- complex arithmetic, status handling and launch helpers shared
// by the sm_100a kernels of the Wigner propagator.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "wigner_b200.h"

// ---------------------------------------------------------------------------
// Complex types: double2 (complex128 state) and float2 (complex64 state).
// ---------------------------------------------------------------------------
template <class R> struct cplx_of;
template <> struct cplx_of<double> { typedef double2 type; };
template <> struct cplx_of<float>  { typedef float2 type; };
template <class C> struct real_of;
template <> struct real_of<double2> { typedef double type; };
template <> struct real_of<float2>  { typedef float type; };

template <class C> __host__ __device__ __forceinline__ C mk(typename real_of<C>::type a,
                                                            typename real_of<C>::type b) {
    C r; r.x = a; r.y = b; return r;
}
template <class C> __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <class C> __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <class C> __device__ __forceinline__ C cmul(C a, C b) {
    return mk<C>(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
template <class C> __device__ __forceinline__ C cconj(C a) { return mk<C>(a.x, -a.y); }
template <class C> __device__ __forceinline__ C cneg(C a) { return mk<C>(-a.x, -a.y); }
template <class C> __device__ __forceinline__ C cscale(C a, typename real_of<C>::type s) {
    return mk<C>(a.x * s, a.y * s);
}
// multiply by -i (fwd) or +i (inverse)
template <class C, bool FWD> __device__ __forceinline__ C mul_mi(C a) {
    return FWD ? mk<C>(a.y, -a.x) : mk<C>(-a.y, a.x);
}
template <class C> __device__ __forceinline__ C to_c(double2 v) {
    return mk<C>((typename real_of<C>::type)v.x, (typename real_of<C>::type)v.y);
}
__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 zinv(double2 a) {
    double d = a.x * a.x + a.y * a.y;
    return make_double2(a.x / d, -a.y / d);
}

// ---------------------------------------------------------------------------
// Status handling.  Entry points return WIG_* codes; the text of the last CUDA
// error is kept per host thread for wig_last_error().
// ---------------------------------------------------------------------------
void wig_set_cuda_error(cudaError_t e, const char* where);
// the per-thread buffer wig_last_error() returns (256 bytes)
char* wig_last_error_buffer();

#define WIG_CUDA(call)                                                      \
    do {                                                                    \
        cudaError_t _e = (call);                                            \
        if (_e != cudaSuccess) { wig_set_cuda_error(_e, #call); return WIG_ERR_CUDA; } \
    } while (0)

#define WIG_LAUNCHED(where)                                                 \
    do {                                                                    \
        cudaError_t _e = cudaGetLastError();                                \
        if (_e != cudaSuccess) { wig_set_cuda_error(_e, where); return WIG_ERR_CUDA; } \
    } while (0)

static inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Number of SMs of the current device (148 on B200), cached per process.
int wig_num_sms();

// Line lengths with a radix transform (Stockham passes of radix 8/4/3/2).
static inline bool wig_radix_size(int n) { return n == 16 || n == 32 || n == 48 || n == 64 || n == 128; }

// Asynchronous global -> shared copies of one complex element (cp.async).
__device__ __forceinline__ void cp_async_elem(double2* dst, const double2* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_elem(float2* dst, const float2* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ---------------------------------------------------------------------------
// Epilogue of the Wigner-Dirac Theta -> P plane transform on 64^4 grids that
// also runs the next Run() iteration's first three passes: boundary_xp (the
// product of the four per-axis factors), Real_GPU of the diagonal components
// and the observable sums of the result.  Each plane writes one row of
// DEPI_SUMS partial sums (the layout of the Dirac reductions:
// 0,1 trace, 2..9 x/p_x/y/p_y moments of the trace, 10,11 alpha, 12,13 x
// alpha1 / y alpha2, 14 kinetic, 15 potential energy, 16..18 D1A0..D1A2).
// ---------------------------------------------------------------------------
#define DEPI_SUMS 20
struct DEpi {
    const double* mxp[4];                   // boundary_xp factors per axis (i0 .. i3)
    const double* cx; const double* cy;     // x[N_x], y[N_y]
    const double* cpx; const double* cpy;   // p_x[N_px], p_y[N_py]
    const double* obs_xy;                   // [7][N_y][N_x]: A0, A1, A2, A3, D1A0, D1A1, D1A2
    double c, mass;
    int kvn;
    double* rows;                           // [slot][i1 * 64 + i3][DEPI_SUMS]
};
