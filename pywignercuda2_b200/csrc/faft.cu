// faft.cu -- the fractional centred transform along one axis of a 4-D array
// (the replacement of the reference's external FAFT library,
// GPU_Wigner4D.py:29-58) and small elementwise helpers.
//
// Contract (restated from the call sites GPU_Wigner4D.py:409-427,
// GPU_WignerDirac4D.py:1428-1458):
//   F[k] = post * 2 N d * sum_n f[n] exp(-2 pi i delta (n - N/2)(k - N/2))
// When |delta| N == 1 this is (-1)^(N/2) (-1)^k DFT_N((-1)^n f) and runs as a
// radix transform in shared memory; otherwise a dense N x N product.
//
// Tiling: the array is viewed as [outer][N][inner] around the transformed
// axis.  A CTA owns TL whole lines: TL consecutive rows when the axis is the
// contiguous one (inner == 1), else TL consecutive inner indices of one outer
// slab, so every global access is a contiguous run of TL or N elements.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <unordered_map>

#include "common.cuh"
#include "fft_smem.cuh"

static thread_local char g_last_err[256] = "";

void wig_set_cuda_error(cudaError_t e, const char* where) {
    snprintf(g_last_err, sizeof(g_last_err), "%s: %s", where, cudaGetErrorString(e));
}

int wig_num_sms() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

extern "C" const char* wig_last_error(void) { return g_last_err; }

char* wig_last_error_buffer() { return g_last_err; }

extern "C" const char* wig_status_string(int s) {
    switch (s) {
        case WIG_OK: return "ok";
        case WIG_ERR_INVALID_ARG: return "invalid argument";
        case WIG_ERR_UNSUPPORTED: return "unsupported shape or parameter";
        case WIG_ERR_CUDA: return "CUDA error";
        case WIG_ERR_ALLOC: return "device allocation failed";
        case WIG_ERR_NONFINITE: return "non-finite value in a reduction";
        case WIG_ERR_ALIAS: return "component pointers alias";
        case WIG_ERR_TOO_LARGE: return "size above the limit of this call";
        case WIG_ERR_TIMEOUT: return "a bounded device wait gave up";
        default: return "unknown status";
    }
}

extern "C" int wig_version(void) { return 100; }

// ---------------------------------------------------------------------------
// Dense transform matrices, cached per (N, delta, dtype) on the device.
// M[k][n] = exp(-2 pi i delta (n - N/2)(k - N/2)), generated in FP64.
// ---------------------------------------------------------------------------
__global__ void k_make_dense(double2* M, int n, double delta) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * n) return;
    int k = t / n, j = t % n;
    double a = (double)(j - n / 2) * (double)(k - n / 2) * delta;
    // reduce the argument modulo 1 before sincospi to keep full precision
    a = a - rint(a);
    double s, c;
    sincospi(-2.0 * a, &s, &c);
    M[t] = make_double2(c, s);
}
__global__ void k_d2f(const double2* a, float2* b, int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) b[t] = make_float2((float)a[t].x, (float)a[t].y);
}

struct DenseKey {
    int n, dtype, dev; double delta;
    bool operator==(const DenseKey& o) const {
        return n == o.n && dtype == o.dtype && dev == o.dev && delta == o.delta;
    }
};
struct DenseKeyHash {
    size_t operator()(const DenseKey& k) const {
        size_t h; memcpy(&h, &k.delta, sizeof(h));
        return h ^ ((size_t)k.n << 1) ^ ((size_t)k.dtype << 20) ^ ((size_t)k.dev << 24);
    }
};
static std::mutex g_dense_mu;
static std::unordered_map<DenseKey, void*, DenseKeyHash> g_dense;

// Returns a device pointer to the dense matrix (complex of dtype), or null.
void* wig_dense_matrix(int n, double delta, int dtype, cudaStream_t st) {
    int dev = 0;
    cudaGetDevice(&dev);
    DenseKey key{n, dtype, dev, delta};
    std::lock_guard<std::mutex> lk(g_dense_mu);
    auto it = g_dense.find(key);
    if (it != g_dense.end()) return it->second;
    double2* M = nullptr;
    if (cudaMalloc(&M, sizeof(double2) * n * n) != cudaSuccess) return nullptr;
    k_make_dense<<<(n * n + 255) / 256, 256, 0, st>>>(M, n, delta);
    void* out = M;
    if (dtype == WIG_C64) {
        float2* F = nullptr;
        if (cudaMalloc(&F, sizeof(float2) * n * n) != cudaSuccess) return nullptr;
        k_d2f<<<(n * n + 255) / 256, 256, 0, st>>>(M, F, n * n);
        cudaStreamSynchronize(st);
        cudaFree(M);
        out = F;
    }
    cudaStreamSynchronize(st);
    g_dense[key] = out;
    return out;
}

// ---------------------------------------------------------------------------
// Standalone transform kernels.
// ---------------------------------------------------------------------------
template <class C>
struct AxisView {
    long long outer;   // product of dims before the axis
    int n;             // length of the axis
    long long inner;   // product of dims after the axis (stride of the axis)
};

// Load/store TL lines of a tile into smem.  Layout in smem:
//   contiguous axis (inner == 1): s[l * N + k]   (rows)
//   strided axis:                 s[k * TL + l]  (inner index fastest)
template <class C, int NT>
__device__ __forceinline__ void tile_io(C* s, C* g, const AxisView<C>& v, int TL, long long tile,
                                        bool store, bool sign_in, C scale_out, bool sign_out) {
    const int n = v.n;
    if (v.inner == 1) {
        C* base = g + tile * (long long)TL * n;
        for (int e = threadIdx.x; e < TL * n; e += NT) {
            int k = e % n;
            if (!store) {
                C x = base[e];
                if (sign_in && (k & 1)) x = cneg(x);
                s[e] = x;
            } else {
                C x = cmul(s[e], scale_out);
                if (sign_out && (k & 1)) x = cneg(x);
                base[e] = x;
            }
        }
    } else {
        const long long tiles_per_outer = v.inner / TL;
        const long long o = tile / tiles_per_outer;
        const long long i0 = (tile % tiles_per_outer) * TL;
        C* base = g + o * (long long)n * v.inner + i0;
        for (int e = threadIdx.x; e < TL * n; e += NT) {
            int k = e / TL, l = e % TL;
            C* p = base + (long long)k * v.inner + l;
            if (!store) {
                C x = *p;
                if (sign_in && (k & 1)) x = cneg(x);
                s[e] = x;
            } else {
                C x = cmul(s[e], scale_out);
                if (sign_out && (k & 1)) x = cneg(x);
                *p = x;
            }
        }
    }
}

template <class C, int N, int TL, int NT, bool FWD>
__global__ void __launch_bounds__(NT) k_faft_fast(C* g, AxisView<C> v, C scale) {
    extern __shared__ __align__(16) unsigned char smraw[];
    C* s = reinterpret_cast<C*>(smraw);
    C* tw = s + TL * N;
    make_twiddles(tw, N);
    tile_io<C, NT>(s, g, v, TL, blockIdx.x, false, true, scale, false);
    __syncthreads();
    LineMap m;
    if (v.inner == 1) { m.nB = 1; m.sA = N; m.sB = 0; m.es = 1; fft_lines<C, N, TL, NT, FWD, false>(s, m, tw); }
    else              { m.nB = 1; m.sA = 1; m.sB = 0; m.es = TL; fft_lines<C, N, TL, NT, FWD, true>(s, m, tw); }
    tile_io<C, NT>(s, g, v, TL, blockIdx.x, true, false, scale, true);
}

template <class C, int NT, bool CONJ>
__global__ void __launch_bounds__(NT) k_faft_dense(C* g, AxisView<C> v, int TL, C scale, const C* M) {
    extern __shared__ __align__(16) unsigned char smraw[];
    C* s = reinterpret_cast<C*>(smraw);
    tile_io<C, NT>(s, g, v, TL, blockIdx.x, false, false, scale, false);
    __syncthreads();
    LineMap m;
    if (v.inner == 1) { m.nB = 1; m.sA = v.n; m.sB = 0; m.es = 1; dense_lines<C, CONJ>(s, m, TL, v.n, M, false); }
    else              { m.nB = 1; m.sA = 1; m.sB = 0; m.es = TL; dense_lines<C, CONJ>(s, m, TL, v.n, M, true); }
    tile_io<C, NT>(s, g, v, TL, blockIdx.x, true, false, scale, false);
}

template <class C, int N, bool FWD>
static int launch_fast(C* g, const AxisView<C>& v, int TL, C scale, cudaStream_t st) {
    constexpr int NT = 256;
    const long long tiles = v.outer * v.inner / TL;
    size_t smem = sizeof(C) * (16 * N + N);
    auto kern = k_faft_fast<C, N, 16, NT, FWD>;
    WIG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<(unsigned)tiles, NT, smem, st>>>(g, v, scale);
    WIG_LAUNCHED("k_faft_fast");
    return WIG_OK;
}

template <class C>
static int faft_impl(C* g, const int shape[4], int axis, double d, double delta, double post,
                     int dtype, cudaStream_t st) {
    AxisView<C> v;
    v.n = shape[axis];
    v.outer = 1; v.inner = 1;
    for (int a = 0; a < axis; ++a) v.outer *= shape[a];
    for (int a = axis + 1; a < 4; ++a) v.inner *= shape[a];
    const int n = v.n;
    const int TL = 16;
    if (v.inner != 1 && v.inner % TL != 0) return WIG_ERR_UNSUPPORTED;
    if ((v.outer * v.inner) % TL != 0) return WIG_ERR_UNSUPPORTED;
    const bool fast = wig_radix_size(n) && fabs(fabs(delta) * n - 1.0) < 1e-12;
    double sc = post * 2.0 * n * d;
    if (fast && (n / 2) % 2 == 1) sc = -sc;   // (-1)^(N/2)
    C scale = mk<C>((typename real_of<C>::type)sc, 0);
    if (fast) {
        const bool fwd = delta > 0;
        switch (n) {
            case 16: return fwd ? launch_fast<C, 16, true>(g, v, TL, scale, st) : launch_fast<C, 16, false>(g, v, TL, scale, st);
            case 32: return fwd ? launch_fast<C, 32, true>(g, v, TL, scale, st) : launch_fast<C, 32, false>(g, v, TL, scale, st);
            case 48: return fwd ? launch_fast<C, 48, true>(g, v, TL, scale, st) : launch_fast<C, 48, false>(g, v, TL, scale, st);
            case 64: return fwd ? launch_fast<C, 64, true>(g, v, TL, scale, st) : launch_fast<C, 64, false>(g, v, TL, scale, st);
            default: return fwd ? launch_fast<C, 128, true>(g, v, TL, scale, st) : launch_fast<C, 128, false>(g, v, TL, scale, st);
        }
    }
    if (n > 1024) return WIG_ERR_UNSUPPORTED;
    const C* M = reinterpret_cast<const C*>(wig_dense_matrix(n, fabs(delta), dtype, st));
    if (!M) return WIG_ERR_ALLOC;
    constexpr int NT = 256;
    const long long tiles = v.outer * v.inner / TL;
    size_t smem = sizeof(C) * TL * n;
    if (delta > 0) {
        auto kern = k_faft_dense<C, NT, false>;
        WIG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<(unsigned)tiles, NT, smem, st>>>(g, v, TL, scale, M);
    } else {
        auto kern = k_faft_dense<C, NT, true>;
        WIG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<(unsigned)tiles, NT, smem, st>>>(g, v, TL, scale, M);
    }
    WIG_LAUNCHED("k_faft_dense");
    return WIG_OK;
}

extern "C" int wig_faft(void* data, const int shape[4], int dtype, int axis, double d, double delta,
                        double post_scale, void* stream) {
    if (!data || !shape || axis < 0 || axis > 3) return WIG_ERR_INVALID_ARG;
    for (int a = 0; a < 4; ++a)
        if (shape[a] <= 0) return WIG_ERR_INVALID_ARG;
    if (delta == 0.0) return WIG_ERR_INVALID_ARG;
    if (dtype == WIG_C128)
        return faft_impl<double2>(reinterpret_cast<double2*>(data), shape, axis, d, delta, post_scale, dtype, as_stream(stream));
    if (dtype == WIG_C64)
        return faft_impl<float2>(reinterpret_cast<float2*>(data), shape, axis, d, delta, post_scale, dtype, as_stream(stream));
    return WIG_ERR_INVALID_ARG;
}

// Reference-signature shims (GPU_Wigner4D.py:32-58).
static int faft_shim(void* p, const int* shape, double d, double delta, int segment, int axes, double NF) {
    if (segment != 0 || NF != 1.0) return WIG_ERR_UNSUPPORTED;
    return wig_faft(p, shape, WIG_C128, axes, d, delta, 1.0, nullptr);
}
extern "C" int FAFT64_4D_Z2Z(void* p, double d, double delta, int segment, int axes, double NF) {
    static const int shape[4] = {64, 64, 64, 64};
    return faft_shim(p, shape, d, delta, segment, axes, NF);
}
extern "C" int IFAFT64_4D_Z2Z(void* p, double d, double delta, int segment, int axes, double NF) {
    static const int shape[4] = {64, 64, 64, 64};
    return faft_shim(p, shape, d, -delta, segment, axes, NF);
}
extern "C" int FAFT128_4D_Z2Z(void* p, double d, double delta, int segment, int axes, double NF) {
    static const int shape[4] = {64, 64, 128, 128};
    return faft_shim(p, shape, d, delta, segment, axes, NF);
}
extern "C" int FAFT256_4D_Z2Z(void* p, double d, double delta, int segment, int axes, double NF) {
    static const int shape[4] = {64, 64, 128, 128};
    return faft_shim(p, shape, d, delta, segment, axes, NF);
}

// ---------------------------------------------------------------------------
// Elementwise helpers.
// ---------------------------------------------------------------------------
template <class C>
__global__ void k_scale(C* a, long long n, double2 s) {
    const C sc = to_c<C>(s);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        a[i] = cmul(a[i], sc);
}
template <class C>
__global__ void k_divide_dev(C* a, long long n, const double* dn) {
    const double2 inv = zinv(make_double2(dn[0], dn[1]));
    const C sc = to_c<C>(inv);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        a[i] = cmul(a[i], sc);
}
template <class C>
__global__ void k_real(C* a, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        a[i].y = 0;
}

static unsigned ew_blocks(long long n) {
    long long b = (n + 255) / 256;
    long long cap = (long long)wig_num_sms() * 8;
    return (unsigned)(b < cap ? (b > 0 ? b : 1) : cap);
}

extern "C" int wig_scale(void* data, long long n, int dtype, double s_re, double s_im, void* stream) {
    if (!data || n < 0) return WIG_ERR_INVALID_ARG;
    if (n == 0) return WIG_OK;
    cudaStream_t st = as_stream(stream);
    double2 s = make_double2(s_re, s_im);
    if (dtype == WIG_C128) k_scale<double2><<<ew_blocks(n), 256, 0, st>>>((double2*)data, n, s);
    else if (dtype == WIG_C64) k_scale<float2><<<ew_blocks(n), 256, 0, st>>>((float2*)data, n, s);
    else return WIG_ERR_INVALID_ARG;
    WIG_LAUNCHED("k_scale");
    return WIG_OK;
}

extern "C" int wig_divide_by_device_scalar(void* data, long long n, int dtype, const double* d_norm,
                                           void* stream) {
    if (!data || !d_norm || n < 0) return WIG_ERR_INVALID_ARG;
    if (n == 0) return WIG_OK;
    cudaStream_t st = as_stream(stream);
    if (dtype == WIG_C128) k_divide_dev<double2><<<ew_blocks(n), 256, 0, st>>>((double2*)data, n, d_norm);
    else if (dtype == WIG_C64) k_divide_dev<float2><<<ew_blocks(n), 256, 0, st>>>((float2*)data, n, d_norm);
    else return WIG_ERR_INVALID_ARG;
    WIG_LAUNCHED("k_divide_dev");
    return WIG_OK;
}

extern "C" int wig_real(void* data, long long n, int dtype, void* stream) {
    if (!data || n < 0) return WIG_ERR_INVALID_ARG;
    if (n == 0) return WIG_OK;
    cudaStream_t st = as_stream(stream);
    if (dtype == WIG_C128) k_real<double2><<<ew_blocks(n), 256, 0, st>>>((double2*)data, n);
    else if (dtype == WIG_C64) k_real<float2><<<ew_blocks(n), 256, 0, st>>>((float2*)data, n);
    else return WIG_ERR_INVALID_ARG;
    WIG_LAUNCHED("k_real");
    return WIG_OK;
}
