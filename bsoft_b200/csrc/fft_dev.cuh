// fft_dev.cuh - warp-level shared-memory FFT used by the 2-D particle
// transforms and the 3-D map transform.
//
// One warp transforms one length-L line held in shared memory: the caller
// stores the input at bit-reversed positions, the radix-2 decimation-in-time
// stages run in place, and the result comes out in natural order.  Twiddles
// exp(-2 pi i j / L), j < L/2, are evaluated on the host in double precision
// and staged in shared memory by the caller.  FFTW's sign convention: the
// forward transform has the negative exponent, no normalisation.
#pragma once

#include <cuda_runtime.h>

namespace bsg {

__device__ __forceinline__ unsigned bitrev(unsigned i, int logL) {
    return logL ? (__brev(i) >> (32 - logL)) : 0u;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {   // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// In-place radix-2 DIT over x[0..L) by the calling warp.  Radix-4 fusion:
// two radix-2 stages per shared-memory round trip where possible.
template <bool INVERSE>
__device__ __forceinline__ void warp_fft(float2* x, int L, int logL, const float2* tw) {
    const int lane = threadIdx.x & 31;
    int s = 1;
    // pairs of stages (s, s+1) as radix-4 butterflies
    for (; s + 1 <= logL; s += 2) {
        const int half = 1 << (s - 1);          // butterfly span of stage s
        const int quads = L >> 2;
        const int tstride1 = L >> s;            // twiddle stride of stage s
        const int tstride2 = L >> (s + 1);      // twiddle stride of stage s+1
        for (int b = lane; b < quads; b += 32) {
            const int j = b & (half - 1);
            const int grp = b >> (s - 1);
            const int i0 = (grp << (s + 1)) + j;
            const int i1 = i0 + half, i2 = i0 + 2 * half, i3 = i0 + 3 * half;
            float2 w1 = tw[j * tstride1];
            float2 w2a = tw[j * tstride2];
            float2 w2b = tw[(j + half) * tstride2];
            if (INVERSE) { w1.y = -w1.y; w2a.y = -w2a.y; w2b.y = -w2b.y; }
            float2 a0 = x[i0], a1 = x[i1], a2 = x[i2], a3 = x[i3];
            // stage s: (a0,a1) and (a2,a3) with twiddle w1
            float2 t1 = cmul(a1, w1), t3 = cmul(a3, w1);
            float2 b0 = make_float2(a0.x + t1.x, a0.y + t1.y);
            float2 b1 = make_float2(a0.x - t1.x, a0.y - t1.y);
            float2 b2 = make_float2(a2.x + t3.x, a2.y + t3.y);
            float2 b3 = make_float2(a2.x - t3.x, a2.y - t3.y);
            // stage s+1: (b0,b2) with w2a, (b1,b3) with w2b
            float2 u2 = cmul(b2, w2a), u3 = cmul(b3, w2b);
            x[i0] = make_float2(b0.x + u2.x, b0.y + u2.y);
            x[i2] = make_float2(b0.x - u2.x, b0.y - u2.y);
            x[i1] = make_float2(b1.x + u3.x, b1.y + u3.y);
            x[i3] = make_float2(b1.x - u3.x, b1.y - u3.y);
        }
        __syncwarp();
    }
    if (s == logL) {   // odd number of stages: one radix-2 stage left
        const int half = 1 << (s - 1);
        const int tstride = L >> s;
        for (int b = lane; b < (L >> 1); b += 32) {
            const int j = b & (half - 1);
            const int grp = b >> (s - 1);
            const int i0 = (grp << s) + j, i1 = i0 + half;
            float2 w = tw[j * tstride];
            if (INVERSE) w.y = -w.y;
            float2 u = x[i0], t = cmul(x[i1], w);
            x[i0] = make_float2(u.x + t.x, u.y + t.y);
            x[i1] = make_float2(u.x - t.x, u.y - t.y);
        }
        __syncwarp();
    }
}

}  // namespace bsg
