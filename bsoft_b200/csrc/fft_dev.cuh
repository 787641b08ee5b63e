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

// Bank swizzle of a line in shared memory: element i moves within its
// aligned block of 16 (one 128-byte row of the 32 banks) by XOR with a
// function of the block number, so a power-of-two line of L >= 16 maps onto
// itself.  Unswizzled, the radix-4 stages of span 1 and 4 put 8 lanes on the
// same banks, and the bit-reversed stores of 32 consecutive inputs all land
// in one bank pair; swizzled, both spread over all 16 slots (the minimum of
// two wavefronts for 32 eight-byte accesses).
__device__ __forceinline__ int swz(int i) {
    const int row = i >> 4;
    return i ^ (((row & 3) * 5) ^ ((row >> 2) & 3));
}

template <bool SWZ>
__device__ __forceinline__ int line_at(int i) {
    return SWZ ? swz(i) : i;
}

// In-place radix-2 DIT over x[0..L) by the calling warp.  Radix-4 fusion:
// two radix-2 stages per shared-memory round trip where possible.  With SWZ
// the line is stored swizzled (element i at x[swz(i)]), inputs and outputs
// included.
template <bool INVERSE, bool SWZ = false>
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
            const int p0 = line_at<SWZ>(i0), p1 = line_at<SWZ>(i1), p2 = line_at<SWZ>(i2),
                      p3 = line_at<SWZ>(i3);
            float2 a0 = x[p0], a1 = x[p1], a2 = x[p2], a3 = x[p3];
            // stage s: (a0,a1) and (a2,a3) with twiddle w1
            float2 t1 = cmul(a1, w1), t3 = cmul(a3, w1);
            float2 b0 = make_float2(a0.x + t1.x, a0.y + t1.y);
            float2 b1 = make_float2(a0.x - t1.x, a0.y - t1.y);
            float2 b2 = make_float2(a2.x + t3.x, a2.y + t3.y);
            float2 b3 = make_float2(a2.x - t3.x, a2.y - t3.y);
            // stage s+1: (b0,b2) with w2a, (b1,b3) with w2b
            float2 u2 = cmul(b2, w2a), u3 = cmul(b3, w2b);
            x[p0] = make_float2(b0.x + u2.x, b0.y + u2.y);
            x[p2] = make_float2(b0.x - u2.x, b0.y - u2.y);
            x[p1] = make_float2(b1.x + u3.x, b1.y + u3.y);
            x[p3] = make_float2(b1.x - u3.x, b1.y - u3.y);
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
            const int p0 = line_at<SWZ>(i0), p1 = line_at<SWZ>(i1);
            float2 u = x[p0], t = cmul(x[p1], w);
            x[p0] = make_float2(u.x + t.x, u.y + t.y);
            x[p1] = make_float2(u.x - t.x, u.y - t.y);
        }
        __syncwarp();
    }
}

}  // namespace bsg

namespace bsg {

// Mixed-radix Stockham autosort transform by one warp, for lengths that are
// not powers of two (maps such as 24^3 or 384^3).  Stage with radix R and
// running product Ns (Ns = 1 at the start): element j in [0, N/R) loads R
// values strided N/R, twiddles them by exp(-+2 pi i r (j mod Ns)/(Ns R)),
// does an R-point DFT and stores them at (j / Ns) Ns R + (j mod Ns) + r Ns.
// `roots` holds exp(-2 pi i t / N), t < N.  x and y are ping-pong buffers of
// N values; the result is left in x.
constexpr int MAXRADIX = 8;

template <bool INVERSE>
__device__ __forceinline__ float2 root_at(const float2* roots, int t, int N) {
    t %= N;
    float2 w = roots[t];
    if (INVERSE) w.y = -w.y;
    return w;
}

template <bool INVERSE>
__device__ void warp_fft_mixed(float2* x, float2* y, int N, const int* radix, int nstage, const float2* roots) {
    const int lane = threadIdx.x & 31;
    float2* src = x;
    float2* dst = y;
    int Ns = 1;
    for (int st = 0; st < nstage; ++st) {
        const int R = radix[st];
        const int NR = N / R;
        for (int j = lane; j < NR; j += 32) {
            const int k = j % Ns;
            float2 v[MAXRADIX];
            const int tstep = (N / (Ns * R)) * k;       // twiddle exponent per r
            for (int r = 0; r < R; ++r) {
                float2 a = src[j + r * NR];
                if (r && k) a = cmul(a, root_at<INVERSE>(roots, r * tstep, N));
                v[r] = a;
            }
            // R-point DFT: out[q] = sum_r v[r] exp(-+2 pi i r q / R)
            float2 o[MAXRADIX];
            const int rs = N / R;                       // root index step for exp(-2 pi i / R)
            for (int q = 0; q < R; ++q) {
                float2 acc = v[0];
                for (int r = 1; r < R; ++r) {
                    const float2 w = root_at<INVERSE>(roots, ((r * q) % R) * rs, N);
                    const float2 t = cmul(v[r], w);
                    acc.x += t.x;
                    acc.y += t.y;
                }
                o[q] = acc;
            }
            const int base = (j / Ns) * Ns * R + k;
            for (int r = 0; r < R; ++r) dst[base + r * Ns] = o[r];
        }
        __syncwarp();
        Ns *= R;
        float2* t = src; src = dst; dst = t;
    }
    if (src != x) {
        for (int i = lane; i < N; i += 32) x[i] = src[i];
        __syncwarp();
    }
}

// Factor n into radices (4 first, then 2, 3, 5, 7).  Returns the number of
// stages, or -1 if n has a prime factor above 7.
__host__ __device__ inline int factor_radices(int n, int* radix) {
    int ns = 0;
    while (n % 4 == 0) { radix[ns++] = 4; n /= 4; }
    const int primes[4] = {2, 3, 5, 7};
    for (int i = 0; i < 4; ++i)
        while (n % primes[i] == 0) { radix[ns++] = primes[i]; n /= primes[i]; }
    return n == 1 ? ns : -1;
}

}  // namespace bsg
