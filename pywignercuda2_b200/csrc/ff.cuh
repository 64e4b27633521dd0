// ff.cuh -- float-float helpers of the complex64 kernels: a complex64 value
// times an FP64 factor held as a float pair (hi + lo), and a 64-entry
// twiddle table free of a systematic float32 rounding of |w|.
#pragma once

namespace ff {

// a * (h + l) with (h, l) a float-float complex factor
__device__ __forceinline__ float2 fmul_hl(float2 a, float2 h, float2 l) {
    const float tx = fmaf(a.x, l.x, -a.y * l.y), ty = fmaf(a.x, l.y, a.y * l.x);
    return make_float2(fmaf(a.x, h.x, fmaf(-a.y, h.y, tx)), fmaf(a.x, h.y, fmaf(a.y, h.x, ty)));
}

// float-float split of a complex double
__device__ __forceinline__ void split_hl(double2 d, float2& h, float2& l) {
    h = make_float2((float)d.x, (float)d.y);
    l = make_float2((float)(d.x - (double)h.x), (float)(d.y - (double)h.y));
}

// Twiddle table w^m = exp(-2 pi i m / 64), m = 0..63: among the float pairs
// within two units in the last place of the rounded (cos, sin), the one
// whose squared modulus is closest to 1, so that a forward and an inverse
// transform with conjugate twiddles do not drift in modulus.
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

}  // namespace ff
