// fft2d.cu - the 2-D half of particle_reconstruct on the GPU: background,
// padding, forward FFT (1/ft scale), origin phase shift and CTF, for a batch
// of particles.  Reference steps (bsoft/src):
//   calculate_background  img/Bimage_background.cpp:27-80
//   pad(ft, FILL_BACKGROUND)  img/Bimage_resize.cpp:28-110, 347-357
//   fft(plan, 1)          img/Bimage_fft.cpp:176-234
//   phase_shift_to_origin img/Bimage_complex.cpp:490-534
//   img_ctf_apply_complex mg/mg_ctf.cpp:661-676 with img_ctf_calculate :46-122
//
// Three kernels per batch:
//   background_kernel  one CTA per image: background mean (FP64 sum) and the
//                      separable phase-shift tables exp(i h shx), exp(i k shy)
//                      evaluated in double;
//   rows_kernel        one warp per pair of image rows: the pair is packed as
//                      one complex line (row a + i row b), padded with the
//                      background, transformed, and split into the two
//                      real-input half spectra (h = 0..ft/2);
//   cols_kernel        16 columns per CTA: column transforms of the row
//                      spectra (rows >= n are the constant background rows,
//                      whose transform is ft*bkg at h = 0 and 0 elsewhere),
//                      then the fused epilogue 1/ft * shift * CTF, written for
//                      the stored column h and its mirror -h (conjugate
//                      symmetry of a real image's transform), i.e. the full
//                      ft x ft spectrum, stored centred and padded as
//                      [k + ft/2][h + ft/2] with row pitch ft + 2 and ft + 1
//                      rows (the extra row/columns stay zero) so that the
//                      gridding kernel can fetch pixel tiles with TMA.
#include "context.cuh"
#include "fft_dev.cuh"

#include <math.h>

namespace bsg {

// ------------------------------------------------------------------ background
__global__ void background_kernel(const float* __restrict__ img, const DevParticle* __restrict__ part,
                                  int n, int ft, double* __restrict__ bkg, float2* __restrict__ phase) {
    const int b = blockIdx.x;
    const float* im = img + (size_t)b * n * n;
    const DevParticle& P = part[b];
    const int hn = n / 2;
    const double h = (double)hn;
    // dividing by a power of two is multiplying by its exact reciprocal:
    // the same doubles without the division sequence
    const bool pow2 = (hn & (hn - 1)) == 0;
    const double ih = 1.0 / h;
    double sum = 0.0;
    int cnt = 0;
    // pixel i = y n + x, stepped by blockDim.x without a division per pixel
    int y = threadIdx.x / n, x = threadIdx.x - y * n;
    const int dy = blockDim.x / n, dx = blockDim.x - dy * n;
    for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
        double x2, y2;
        if (pow2) { x2 = (x - P.bx) * ih; y2 = (y - P.by) * ih; }
        else { x2 = (x - P.bx) / h; y2 = (y - P.by) / h; }
        if (x2 * x2 + y2 * y2 - 1 > 0) { sum += (float)(im[i] * P.na + P.nb); ++cnt; }
        x += dx;
        y += dy;
        if (x >= n) { x -= n; ++y; }
    }
    // deterministic block reduction (fixed tree)
    __shared__ double ssum[256];
    __shared__ int scnt[256];
    ssum[threadIdx.x] = sum;
    scnt[threadIdx.x] = cnt;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            ssum[threadIdx.x] += ssum[threadIdx.x + o];
            scnt[threadIdx.x] += scnt[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) bkg[b] = scnt[0] ? ssum[0] / scnt[0] : 0.0;
    // separable origin shift factors, phi = h*shx + k*shy (double)
    float2* ex = phase + (size_t)b * 2 * ft;
    float2* ey = ex + ft;
    for (int i = threadIdx.x; i < ft; i += blockDim.x) {
        double f = (double)sfreq(i, ft);
        double s, c;
        sincos(f * P.shx, &s, &c);
        ex[i] = make_float2((float)c, (float)s);
        sincos(f * P.shy, &s, &c);
        ey[i] = make_float2((float)c, (float)s);
    }
}

// ------------------------------------------------------------------ rows
constexpr int ROW_WARPS = 8;

__global__ void __launch_bounds__(ROW_WARPS * 32)
rows_kernel(const float* __restrict__ img, const double* __restrict__ bkg, const float2* __restrict__ tw,
            const DevParticle* __restrict__ part, int n, int ft, int logft, float2* __restrict__ rows) {
    extern __shared__ float2 smem[];
    float2* stw = smem;                          // ft/2 twiddles
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float2* buf = smem + ft / 2 + warp * ft;
    for (int i = threadIdx.x; i < ft / 2; i += blockDim.x) stw[i] = tw[i];
    __syncthreads();
    const int b = blockIdx.y;
    const int pair = blockIdx.x * ROW_WARPS + warp;
    const int npairs = (n + 1) / 2;
    if (pair >= npairs) return;
    const int y0 = 2 * pair, y1 = y0 + 1;
    const float fill = (float)bkg[b];
    const float* r0 = img + ((size_t)b * n + y0) * n;
    const float* r1 = r0 + n;
    // the particle's normalisation (rescale_to_avg_std, stored as float)
    const double na = part[b].na, nb = part[b].nb;
    for (int x = lane; x < ft; x += 32) {
        float re = (x < n) ? (float)(r0[x] * na + nb) : fill;
        float im = (y1 < n && x < n) ? (float)(r1[x] * na + nb) : fill;
        buf[swz(bitrev(x, logft))] = make_float2(re, im);
    }
    __syncwarp();
    warp_fft<false, true>(buf, ft, logft, stw);
    const int hw = ft / 2 + 1;
    float2* o0 = rows + ((size_t)b * n + y0) * hw;
    float2* o1 = o0 + hw;
    for (int h = lane; h < hw; h += 32) {
        float2 z = buf[swz(h)], zm = buf[swz((ft - h) & (ft - 1))];
        o0[h] = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
        if (y1 < n) o1[h] = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
    }
}

// ------------------------------------------------------------------ columns + epilogue
constexpr int COL_W = 16;   // columns per CTA, one warp each

// Column buffers are ft + 1 apart, so the 16 columns' copies of one row fall
// in 16 different bank slots; within a column the line is swizzled (swz).
__host__ __device__ constexpr int col_stride(int ft) { return ft + 1; }

struct ColArgs {
    const float2* rows;
    const double* bkg;
    const float2* phase;
    const DevParticle* part;
    const float2* tw;
    float2* spec;
    int n, ft, logft;
    int ctf_action;
    double wiener;
    double shi2;
};

// The particle's CTF terms, held in registers for the epilogue: read through
// the record in global memory they would be loaded again after every store
// of the spectrum (the compiler cannot tell that the stores leave them alone).
struct CtfTerms {
    double fs, c00, c20, c22, c2m2, c40, c11, c1m1;
};

__device__ __forceinline__ CtfTerms ctf_terms(const DevParticle& P) {
    CtfTerms t;
    t.fs = P.fs; t.c00 = P.c00; t.c20 = P.c20; t.c22 = P.c22; t.c2m2 = P.c2m2; t.c40 = P.c40;
    t.c11 = P.c11; t.c1m1 = P.c1m1;
    return t;
}

// CTF weight of one pixel from its reduced even aberration r in (-pi, pi].
__device__ __forceinline__ float ctf_weight(const ColArgs& a, double r) {
    if (a.ctf_action == 1) return (r < 0.0) ? -1.f : 1.f;
    float w = sinf((float)r);
    if (a.wiener != 0.0) w = (float)((a.wiener + 1.0) * w / ((double)w * w + a.wiener));
    return w;
}

// Factors 1/ft * exp(i phi) * CTF of pixel (h, k) and, with MIRROR, of its
// mirror (-h, k).  exh = exp(i h shx) and eyk = exp(i k shy); the mirror's
// phase is conj(exh) * eyk.  img_ctf_calculate: s = (h, k) * fs, inside
// [0, shi2]; even aberration chi = c00 + s2 (c20 + c22 cos2a + c2m2 sin2a) +
// c40 s2^2 with s2 cos2a = sx^2 - sy^2, s2 sin2a = 2 sx sy (ctf.h:321-334),
// in double.  Mirroring h changes only the sign of the 2 sx sy term (and of
// sx in the odd, beam-tilt aberration psi = c1m1 sy + c11 sx).
template <bool MIRROR>
__device__ __forceinline__ void pixel_factors(const ColArgs& a, const CtfTerms& P, float2 exh, float2 eyk,
                                              int h, int k, float2& f, float2& fm) {
    const float sc = 1.0f / (float)a.ft;
    const float2 ph = cmul(exh, eyk);
    const float2 phm = cmulc(eyk, exh);
    f = make_float2(ph.x * sc, ph.y * sc);
    if (MIRROR) fm = make_float2(phm.x * sc, phm.y * sc);
    if (!a.ctf_action) return;
    const double sx = (double)h * P.fs, sy = (double)k * P.fs;
    const double s2 = sx * sx + sy * sy;
    if (!(s2 <= a.shi2)) {
        f = make_float2(0.f, 0.f);
        if (MIRROR) fm = f;
        return;
    }
    const double even = P.c00 + P.c20 * s2 + P.c22 * (sx * sx - sy * sy) + P.c40 * s2 * s2;
    const double cross = P.c2m2 * (2.0 * sx * sy);
    // reduce to (-pi, pi] in double so the sign of sin(chi) is exact
    const double chi = even + cross;
    const float w = ctf_weight(a, chi - 6.283185307179586 * rint(chi * 0.15915494309189535));
    f.x *= w; f.y *= w;
    float wm = 0.f;
    if (MIRROR) {
        const double chim = even - cross;
        wm = ctf_weight(a, chim - 6.283185307179586 * rint(chim * 0.15915494309189535));
        fm.x *= wm; fm.y *= wm;
    }
    if (P.c11 != 0.0 || P.c1m1 != 0.0) {
        float sp, cp;
        sincosf((float)(P.c1m1 * sy + P.c11 * sx), &sp, &cp);
        f = cmulc(f, make_float2(cp, sp));
        if (MIRROR) {
            sincosf((float)(P.c1m1 * sy - P.c11 * sx), &sp, &cp);
            fm = cmulc(fm, make_float2(cp, sp));
        }
    }
}

__global__ void __launch_bounds__(COL_W * 32, 2) cols_kernel(ColArgs a) {
    extern __shared__ float2 smem[];
    const int ft = a.ft, n = a.n, logft = a.logft;
    float2* stw = smem;
    float2* cols = smem + ft / 2;                // COL_W x col_stride(ft)
    const int cs = col_stride(ft);
    const int b = blockIdx.y;
    const int h0 = blockIdx.x * COL_W;
    const int hw = ft / 2 + 1;
    for (int i = threadIdx.x; i < ft / 2; i += blockDim.x) stw[i] = a.tw[i];
    const float dc = (float)(a.bkg[b] * ft);
    const float2* rows = a.rows + (size_t)b * n * hw;
    // coalesced load: c fastest
    for (int i = threadIdx.x; i < COL_W * ft; i += blockDim.x) {
        const int c = i % COL_W, y = i / COL_W;
        const int h = h0 + c;
        float2 v = make_float2(0.f, 0.f);
        if (h < hw) {
            if (y < n) v = rows[(size_t)y * hw + h];
            else if (h == 0) v = make_float2(dc, 0.f);
        }
        cols[c * cs + swz(bitrev(y, logft))] = v;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    if (h0 + warp < hw) warp_fft<false, true>(cols + warp * cs, ft, logft, stw);
    __syncthreads();
    const CtfTerms P = ctf_terms(a.part[b]);
    const float2* ex = a.phase + (size_t)b * 2 * ft;
    const float2* ey = ex + ft;
    // centred, padded layout: [k + ft/2][h + ft/2], row pitch ft + 2
    const int pitch = ft + 2, hf = ft / 2;
    float2* out = a.spec + (size_t)b * (ft + 1) * pitch;
    const int fm = ft - 1;
    for (int i = threadIdx.x; i < COL_W * ft; i += blockDim.x) {
        const int c = i % COL_W, kk = i / COL_W;
        const int hidx = h0 + c;
        if (hidx >= hw) continue;
        const int k = sfreq(kk, ft);
        const int h = sfreq(hidx, ft);            // hidx == ft/2 -> -ft/2
        float2 g = cols[c * cs + swz(kk)];
        float2* row = out + (size_t)(k + hf) * pitch + hf;
        float2 f, fmr;
        if (hidx >= 1 && hidx < ft / 2) {
            pixel_factors<true>(a, P, ex[hidx], ey[kk], h, k, f, fmr);
            // F(-h, k) = conj(G(h, -k)) * factor(-h, k)
            float2 gm = cols[c * cs + swz((-kk) & fm)];
            gm.y = -gm.y;
            const float2 vm = cmul(gm, fmr);
            row[-h] = vm;
        } else {
            pixel_factors<false>(a, P, ex[hidx], ey[kk], h, k, f, fmr);
        }
        row[h] = cmul(g, f);
    }
}

cudaError_t launch_background(const Context& c, const float* img, int nimg, cudaStream_t s) {
    background_kernel<<<nimg, 256, 0, s>>>(img, c.d_part, c.g.n, c.g.ft, c.d_bkg, c.d_phase);
    return cudaGetLastError();
}

cudaError_t launch_rows(const Context& c, const float* img, int nimg, cudaStream_t s) {
    const int npairs = (c.g.n + 1) / 2;
    dim3 grid((npairs + ROW_WARPS - 1) / ROW_WARPS, nimg);
    size_t smem = sizeof(float2) * ((size_t)c.g.ft / 2 + (size_t)ROW_WARPS * c.g.ft);
    rows_kernel<<<grid, ROW_WARPS * 32, smem, s>>>(img, c.d_bkg, c.d_tw, c.d_part, c.g.n, c.g.ft, c.g.logft, c.d_rows);
    return cudaGetLastError();
}

cudaError_t launch_cols(const Context& c, int nimg, float2* spectra, cudaStream_t s) {
    ColArgs a;
    a.rows = c.d_rows; a.bkg = c.d_bkg; a.phase = c.d_phase; a.part = c.d_part; a.tw = c.d_tw;
    a.spec = spectra; a.n = c.g.n; a.ft = c.g.ft; a.logft = c.g.logft;
    a.ctf_action = c.g.ctf_action; a.wiener = c.g.wiener; a.shi2 = c.g.ctf_shi2;
    const int hw = c.g.ft / 2 + 1;
    dim3 grid((hw + COL_W - 1) / COL_W, nimg);
    size_t smem = sizeof(float2) * ((size_t)c.g.ft / 2 + (size_t)COL_W * col_stride(c.g.ft));
    cols_kernel<<<grid, COL_W * 32, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t prepare_fft2d_attributes() {
    cudaError_t e = cudaFuncSetAttribute(rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(sizeof(float2) * (512 + ROW_WARPS * 1024)));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(cols_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(float2) * (512 + COL_W * col_stride(1024))));
}

}  // namespace bsg
