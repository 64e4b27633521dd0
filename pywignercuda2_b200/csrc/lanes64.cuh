// lanes64.cuh -- register-resident 64-point transforms for 64 x 64 planes.
//
// A CTA of 512 threads (16 warps) owns one 64 x 64 plane.  A line of 64
// points is held by a group of 8 consecutive lanes, 8 points per lane:
// lane q of the group holds the points q + 8 r, r = 0..7.  A length-64
// transform is 64 = 8 x 8 decimation in time:
//
//   1. 8-point DFT over r in registers (points q + 8 r),
//   2. twiddle w64^(q k1),
//   3. 8 x 8 transpose across the group's lanes, through a warp-private
//      swizzled scratch in shared memory (only __syncwarp),
//   4. 8-point DFT in registers,
//
// after which lane q holds the outputs k = q + 8 k2: the same layout as the
// input, so an inverse transform runs on it directly.  A 2-D transform
// needs the plane to pass through shared memory once (rows -> columns),
// which is the only CTA-wide exchange: a half-step costs two plane
// transposes plus four warp-local lane transposes, against ten full
// read/write passes for radix passes over a shared-memory plane.
#pragma once
#include "fft_smem.cuh"

namespace lanes64 {

constexpr int NT = 512;       // threads per CTA
constexpr int LD = 65;        // padded row stride of the plane (elements)

// 8 x 8 transpose among the 8 lanes of a group.  ws: this warp's scratch of
// 4 groups x 64 elements; element (row = source lane, col = r) of group gi is
// stored at gi*64 + row*8 + (col ^ row), which keeps every 16-byte access
// of a warp on distinct bank quads.
template <class C>
__device__ __forceinline__ void lane_transpose(C (&v)[8], C* ws, int gi, int q) {
    C* g = ws + gi * 64;
    __syncwarp();
#pragma unroll
    for (int r = 0; r < 8; ++r) g[q * 8 + (r ^ q)] = v[r];
    __syncwarp();
#pragma unroll
    for (int s = 0; s < 8; ++s) v[s] = g[s * 8 + (q ^ s)];
    __syncwarp();
}

// Length-64 transform of the group's line (see the file comment).
template <class C, bool FWD>
__device__ __forceinline__ void fft64(C (&v)[8], C* ws, int gi, int q, const C* tw) {
    dft8<C, FWD>(v);
    // v[k1] *= w64^(q k1): w1 = w^q, w2 = w^2q, w4 = w^4q from the table,
    // the rest by at most two products.
    if (q != 0) {
        C w1 = tw[q], w2 = tw[2 * q], w4 = tw[(4 * q) & 63];
        if (!FWD) { w1 = cconj(w1); w2 = cconj(w2); w4 = cconj(w4); }
        const C w3 = cmul(w1, w2), w5 = cmul(w1, w4), w6 = cmul(w2, w4), w7 = cmul(w3, w4);
        v[1] = cmul(v[1], w1); v[2] = cmul(v[2], w2); v[3] = cmul(v[3], w3);
        v[4] = cmul(v[4], w4); v[5] = cmul(v[5], w5); v[6] = cmul(v[6], w6);
        v[7] = cmul(v[7], w7);
    }
    lane_transpose(v, ws, gi, q);
    dft8<C, FWD>(v);
}

}  // namespace lanes64
