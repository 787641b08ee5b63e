// match.cu - projection matching on sm_100a (brefine's scoring path):
// the reference-map transform, particle transforms, central sections with
// the reference's FSI interpolation kernel and the FRC figure of merit of
// (image, view, origin) hypotheses.
//
// Reference steps (bsoft/src/mg/mg_refine.cpp):
//   map      :279-365  fft (1/sqrt(N^3)), cut to diam = even(2.2 N u / res),
//                      clear the zero-frequency term, phase shift to origin
//   particle :509-563  rescale_to_avg_std(0, 1), fft without scaling, clear
//                      the zero-frequency term, cut to diam
//   section  Bimage::central_section (Bimage_project.cpp:288-338) with
//            Bimage::fspace_interpolate (Bimage_fspace.cpp:85-147) and
//            FSI_Kernel (FSI_Kernel.h:28-68)
//   score    img_recip_space_fom (:660-781), FRC form, unit shell weights
//
// Device layout: the cut reference transform is a diam^3 float2 array in the
// reference's index order (L2-resident at the sizes brefine uses: 114^3 is
// 11.8 MB).  Particle transforms are kept cut (diam^2 float2 each).  The
// pixels that enter a figure of merit (min_rad <= |(h,k)| <= 1.1 max_rad)
// form one list sorted by shell, then angle; per image the CTF at those
// pixels and the per-shell image power are computed once.
//
// Transforms: FP64 (see the note at warp_fft64).
//
// Section gather: one warp per section pixel, lane = (x tap, row group);
// each of the 16 load rounds reads 4 rows of 8 consecutive x taps, so a
// pixel costs ~160 L1 sectors instead of 512 scattered loads, and a warp
// moves along a shell so successive pixels reuse most of their 8^3 taps.
#include "match.cuh"
#include "fft_dev.cuh"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <new>
#include <vector>

namespace bsg {

void set_error(const char* fmt, ...);

namespace {

// ---- transforms ---------------------------------------------------------

// The transforms run in FP64 and round to float once, as the reference's
// single-precision FFTW output does per value: an FP32 transform carries
// absolute errors of ~1e-7 of the total power into every coefficient, which
// is ~1e-3 relative at the outer shells of a smooth map.

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// in-place radix-2 DIT over bit-reversed input by one warp, forward
// (twiddles exp(-2 pi i j / L), j < L/2)
__device__ void warp_fft64(double2* x, int L, int logL, const double2* tw) {
    const int lane = threadIdx.x & 31;
    for (int s = 1; s <= logL; ++s) {
        const int half = 1 << (s - 1), tstride = L >> s;
        for (int b = lane; b < (L >> 1); b += 32) {
            const int j = b & (half - 1), grp = b >> (s - 1);
            const int i0 = (grp << s) + j, i1 = i0 + half;
            const double2 u = x[i0], t = zmul(x[i1], tw[j * tstride]);
            x[i0] = make_double2(u.x + t.x, u.y + t.y);
            x[i1] = make_double2(u.x - t.x, u.y - t.y);
        }
        __syncwarp();
    }
}

// one warp per contiguous line of L (power of two) values, 4 warps per CTA
constexpr int LW = 4;
__global__ void __launch_bounds__(LW * 32) lines64_kernel(double2* data, long nlines, int L, int logL,
                                                          const double2* tw) {
    extern __shared__ double2 zsm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double2* stw = zsm;
    double2* buf = zsm + L / 2 + warp * L;
    for (int i = threadIdx.x; i < L / 2; i += blockDim.x) stw[i] = tw[i];
    __syncthreads();
    const long line = (long)blockIdx.x * LW + warp;
    if (line >= nlines) return;
    double2* p = data + line * L;
    for (int i = lane; i < L; i += 32) buf[bitrev(i, logL)] = p[i];
    __syncwarp();
    warp_fft64(buf, L, logL, stw);
    for (int i = lane; i < L; i += 32) p[i] = buf[i];
}

// lines of L values with element stride S; a CTA takes 8 lines whose starts
// are consecutive (x0 .. x0+7 of `inner`), blockIdx.y the outer index
constexpr int SWL = 8;
__global__ void __launch_bounds__(SWL * 32) strided64_kernel(double2* data, int L, int logL, long S, long inner,
                                                             long ostride, const double2* tw) {
    extern __shared__ double2 zsm[];
    double2* stw = zsm;
    double2* tile = zsm + L / 2;
    for (int i = threadIdx.x; i < L / 2; i += blockDim.x) stw[i] = tw[i];
    const long x0 = (long)blockIdx.x * SWL;
    const long base = (long)blockIdx.y * ostride;
    for (int i = threadIdx.x; i < SWL * L; i += blockDim.x) {
        const int c = i % SWL, j = i / SWL;
        const long x = x0 + c;
        double2 v = make_double2(0.0, 0.0);
        if (x < inner) v = data[base + j * S + x];
        tile[c * L + bitrev(j, logL)] = v;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    if (x0 + warp < inner) warp_fft64(tile + warp * L, L, logL, stw);
    __syncthreads();
    for (int i = threadIdx.x; i < SWL * L; i += blockDim.x) {
        const int c = i % SWL, j = i / SWL;
        const long x = x0 + c;
        if (x < inner) data[base + j * S + x] = tile[c * L + j];
    }
}

// real values -> complex (float)(v * scale[b] + shift[b]) (the rescaled
// image is stored as float, Bimage_rescale.cpp:41-44); scale/shift per image
// b of `per` values (NULL: 1 and 0)
__global__ void to_complex_kernel(const float* __restrict__ in, double2* __restrict__ out, long count, long per,
                                  const double* __restrict__ scale, const double* __restrict__ shift) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
        double v = in[i];
        if (scale) { const long b = i / per; v = v * scale[b] + shift[b]; }
        out[i] = make_double2((double)(float)v, 0.0);
    }
}

// per-image population statistics (Bimage::statistics(long)) -> the
// rescale_to_avg_std(0, 1) factors; fixed-order FP64 reduction
__global__ void __launch_bounds__(256) image_stats_kernel(const float* __restrict__ img, int n2, double* scale,
                                                          double* shift) {
    __shared__ double s1[256], s2[256];
    const float* p = img + (size_t)blockIdx.x * n2;
    double a = 0, b = 0;
    for (int i = threadIdx.x; i < n2; i += 256) { const double v = p[i]; a += v; b += v * v; }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if (threadIdx.x < o) { s1[threadIdx.x] += s1[threadIdx.x + o]; s2[threadIdx.x] += s2[threadIdx.x + o]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double avg = s1[0] / n2;
        double sd = s2[0] / n2 - avg * avg;
        sd = sd > 0 ? sqrt(sd) : 0;
        const double sc = sd > 1e-30 ? 1.0 / sd : 1.0;
        scale[blockIdx.x] = sc;
        shift[blockIdx.x] = -avg * sc;
    }
}

__device__ __forceinline__ int crop_src(int xx, int nu, int size) { return xx > (nu - 1) / 2 ? xx + size - nu : xx; }

// full N^3 transform -> cut diam^3, x norm, zero-frequency term cleared,
// phase shift exp(i (h sx + k sy + l sz)) in FP64 (Bimage_complex.cpp:490-534)
__global__ void map_cut_kernel(const double2* __restrict__ full, int N, int D, double norm, double sx, double sy,
                               double sz, float2* __restrict__ out) {
    const long total = (long)D * D * D;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % D), y = (int)((i / D) % D), z = (int)(i / ((long)D * D));
        const size_t src = ((size_t)crop_src(z, D, N) * N + crop_src(y, D, N)) * N + crop_src(x, D, N);
        const double2 f = full[src];
        // fft(): the transform is scaled and stored as float (Bimage_fft.cpp:141-146)
        double re = (float)(f.x * norm), im = (float)(f.y * norm);
        if (i == 0) re = im = 0;
        const double phi = sfreq(x, D) * sx + sfreq(y, D) * sy + sfreq(z, D) * sz;
        double s, c;
        sincos(phi, &s, &c);
        out[i] = make_float2((float)(re * c - im * s), (float)(re * s + im * c));
    }
}

// the uncut transform for the projector (Bimage::project: fft with
// 1/sqrt(N^3), phase shift to the map origin, nothing cleared)
__global__ void map_full_kernel(const double2* __restrict__ full, int N, double norm, double sx, double sy, double sz,
                                float2* __restrict__ out) {
    const long total = (long)N * N * N;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % N), y = (int)((i / N) % N), z = (int)(i / ((long)N * N));
        const double2 f = full[i];
        const double re = (float)(f.x * norm), im = (float)(f.y * norm);
        const double phi = sfreq(x, N) * sx + sfreq(y, N) * sy + sfreq(z, N) * sz;
        double sn, cs;
        sincos(phi, &sn, &cs);
        out[i] = make_float2((float)(re * cs - im * sn), (float)(re * sn + im * cs));
    }
}

// projections (Bimage::project, Bimage_project.cpp:362-443): one CTA per
// view gathers the section pixels within the resolution limit from the
// uncut transform, optionally multiplies by a CTF (data synthesis), shifts
// the phases to the image origin (phase_shift_to_center when the origin is
// N/2: exp(-2 pi i (h ox + k oy) / N), Bimage_complex.cpp:443-478) and
// stores the conjugate, so that the forward transform that follows yields the
// inverse transform's real part
struct ProjArgs {
    const float2* vol;
    int N, wd;
    const double* lut;
    const MPix* pix;
    int npix;
    const MHyp* views;          // m, sx/sy = -2 pi origin / N
    const ImgCtf* ctf;          // per view or NULL
    double inv, real, fs;       // fs: CTF frequency step 1/(N pixel)
    double2* out;               // per view N^2
};

__global__ void __launch_bounds__(256) project_kernel(ProjArgs a) {
    __shared__ double lut[(NDIV + 1) * MAXW];
    for (int i = threadIdx.x; i < (NDIV + 1) * a.wd; i += blockDim.x) lut[i] = a.lut[i];
    __syncthreads();
    const MHyp& V = a.views[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double2* o = a.out + (size_t)blockIdx.x * a.N * a.N;
    for (int p = warp; p < a.npix; p += 8) {
        const MPix q = a.pix[p];
        const double ix = q.h * a.inv, iy = q.k * a.inv;
        const double mx = (V.m[0] * ix + V.m[1] * iy) * a.real;
        const double my = (V.m[3] * ix + V.m[4] * iy) * a.real;
        const double mz = (V.m[6] * ix + V.m[7] * iy) * a.real;
        double vr, vi;
        fsi_gather<double>(PtrSrc{a.vol, a.N}, a.N, mx, my, mz, lut, a.wd, lane, vr, vi);
        if (lane == 0) {
            // the section is stored as float (Complex<float>)
            vr = (float)vr;
            vi = (float)vi;
            if (a.ctf && a.ctf[blockIdx.x].apply) {
                const ImgCtf& C = a.ctf[blockIdx.x];
                double sx2 = a.fs * q.h; sx2 *= sx2;
                double sy2 = a.fs * q.k; sy2 *= sy2;
                const double s2 = sx2 + sy2, ang = atan2((double)q.k, (double)q.h);
                const double chi = C.c[0] + s2 * (C.c[3] * sin(2 * ang) + C.c[1] + C.c[2] * cos(2 * ang)) + s2 * s2 * C.c[4];
                double c = sin(chi);
                if (C.invert) c = -c;
                vr *= c;
                vi *= c;
            }
            const double phi = q.h * V.sx + q.k * V.sy;
            double sn, cs;
            sincos(phi, &sn, &cs);
            const double rr = vr * cs - vi * sn, ri = vr * sn + vi * cs;
            o[q.idx] = make_double2(rr, -ri);
        }
    }
}

// real part of the inverse transform: (forward transform of the conjugate)
// real part x 1/N (norm 1 of fft(FFTW_BACKWARD, 1), Bimage_fft.cpp:141-146)
__global__ void proj_real_kernel(const double2* __restrict__ in, long count, double norm, float* __restrict__ out) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x)
        out[i] = (float)(in[i].x * norm);
}

// full n^2 transforms -> cut diam^2 with the zero-frequency term cleared
__global__ void img_cut_kernel(const double2* __restrict__ full, int n, int D, long nimg, float2* __restrict__ out) {
    const long per = (long)D * D, total = per * nimg;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long b = i / per;
        const int x = (int)(i % D), y = (int)((i % per) / D);
        const double2 f = full[(size_t)b * n * n + (size_t)crop_src(y, D, n) * n + crop_src(x, D, n)];
        float2 v = make_float2((float)f.x, (float)f.y);
        if (x == 0 && y == 0) v = make_float2(0.f, 0.f);
        out[i] = v;
    }
}


// per image: CTF at the figure-of-merit pixels (ctf.h:321-365 with
// s = index / (n * pixel)) and the image power per shell (fixed order)
__global__ void __launch_bounds__(256) img_shells_kernel(const float2* __restrict__ spec, int D,
                                                         const MPix* __restrict__ pix, int npix,
                                                         const int* __restrict__ shell_start, int nshell,
                                                         const ImgCtf* __restrict__ ctf, double fs,
                                                         float* __restrict__ ctf_out, double* __restrict__ dsum) {
    const long b = blockIdx.x;
    const float2* X = spec + b * (long)D * D;
    const ImgCtf C = ctf[b];
    for (int p = threadIdx.x; p < npix; p += blockDim.x) ctf_out[b * npix + p] = ctf_factor(C, pix[p], fs);
    for (int j = threadIdx.x; j < nshell; j += blockDim.x) {
        double d = 0;
        for (int p = shell_start[j]; p < shell_start[j + 1]; ++p) {
            const float2 x = X[pix[p].idx];
            d += (double)x.x * x.x + (double)x.y * x.y;
        }
        dsum[b * nshell + j] = d;
    }
}

// CTF rows for arbitrary records (the refinement's defocus trials)
__global__ void __launch_bounds__(256) ctf_rows_kernel(const ImgCtf* __restrict__ rec, const MPix* __restrict__ pix,
                                                       int npix, double fs, float* __restrict__ out) {
    const long b = blockIdx.x;
    const ImgCtf C = rec[b];
    for (int p = threadIdx.x; p < npix; p += blockDim.x) out[b * npix + p] = ctf_factor(C, pix[p], fs);
}

// central sections for output: one CTA per view over the pixel list of the
// section (every pixel with s^2 <= 1/res^2)
__global__ void __launch_bounds__(256) section_kernel(const float2* __restrict__ vol, int D,
                                                      const double* __restrict__ lut_g, int wd,
                                                      const MPix* __restrict__ pix, int npix,
                                                      const MHyp* __restrict__ views, double inv, double real,
                                                      float2* __restrict__ out) {
    __shared__ double lut[(NDIV + 1) * MAXW];
    for (int i = threadIdx.x; i < (NDIV + 1) * wd; i += blockDim.x) lut[i] = lut_g[i];
    __syncthreads();
    const MHyp& V = views[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float2* o = out + (size_t)blockIdx.x * D * D;
    for (int p = warp; p < npix; p += 8) {
        const MPix q = pix[p];
        const double ix = q.h * inv, iy = q.k * inv;
        const double mx = (V.m[0] * ix + V.m[1] * iy) * real;
        const double my = (V.m[3] * ix + V.m[4] * iy) * real;
        const double mz = (V.m[6] * ix + V.m[7] * iy) * real;
        double vr, vi;
        fsi_gather<double>(PtrSrc{vol, D}, D, mx, my, mz, lut, wd, lane, vr, vi);
        if (lane == 0) o[q.idx] = make_float2((float)vr, (float)vi);
    }
}

// Figure of merit of one hypothesis group per CTA (img_recip_space_fom,
// unit weights; the FRC, fom_type 0, or with a.dpr the DPR form, fom_type 1,
// mg_refine.cpp:725-772: per shell the sums of (|X| + |R c|) dphi^2 and of
// |X| + |R c|, dphi the phase difference wrapped to [-pi, pi], and the mean
// over shells of cos(sqrt(ratio))): one image, one view, up to MAXORG trial
// origins.  Warps take 32 consecutive pixels of the shell-sorted list: the
// section value of each is gathered once by the whole warp, then every lane
// scores its own pixel at every origin (only the image phase depends on the
// origin) and the lanes of one shell are summed by a fixed shuffle tree into
// the warp's shell slots.  The shell totals are folded over the warps in
// FP64, in order, so results do not depend on the grouping.
struct FomArgs {
    cudaTextureObject_t tex;
    int D, wd;
    const float* lut;        // FSI table, FP32 (T = float)
    const double* lutd;      // the same, FP64 (T = double)
    const MPix* pix;
    int npix;
    const MHypG* hyps;
    const float2* spec;      // prepared images, diam^2 each
    const float* ctf;        // per image x npix
    const double* dsum;      // per image x nshell
    int nshell;
    double inv, real;        // section frequency step and real size
    int nf;                  // shells j < max_rad
    int cv0, cv1;            // cross-validation shells [cv0, cv1)
    const double* wshell;    // per-shell weights
    double wf, wc;           // their sums over [0, nf) and [cv0, cv1)
    double* fom;             // per group x MAXORG
    double* cv;
    const double2* sec;      // gathered sections (npix per view, FP64), or null: gather here
    const float2* psec;      // FP32 panel sections (npix per panel view, row H.sec; T = float), or null
    int dpr;                 // 1: the DPR form (fom_type 1) instead of the FRC
};

// T = float: the search's rescoring (agrees with the reference's figure of
// merit to ~1e-7); T = double: gather, products and shell sums in FP64, as
// the reference accumulates (~1e-8), for refinement whose decisions compare
// figures of merit against a 1e-6 threshold.
template <typename T>
__global__ void __launch_bounds__(FOM_WARPS * 32) fom_kernel(FomArgs a) {
    extern __shared__ __align__(16) unsigned char fom_smem[];
    T* lut = reinterpret_cast<T*>(fom_smem);                                // (NDIV+1)*wd
    T* wsum = lut + (NDIV + 1) * MAXW;                                      // FOM_WARPS x nshell x (1+MAXORG)
    constexpr int NV = 1 + MAXORG;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const T* glut;
    if constexpr (sizeof(T) == 8) glut = a.lutd; else glut = a.lut;
    for (int i = threadIdx.x; i < (NDIV + 1) * a.wd; i += blockDim.x) lut[i] = glut[i];
    for (int i = threadIdx.x; i < FOM_WARPS * a.nshell * NV; i += blockDim.x) wsum[i] = (T)0;
    __syncthreads();
    const MHypG& H = a.hyps[blockIdx.x];
    const int norg = H.norg;
    const long img = H.img;
    const float2* X = a.spec + img * (long)a.D * a.D;
    const float* C = a.ctf + (long)H.ctf * a.npix;
    T* my = wsum + warp * a.nshell * NV;
    for (int base = warp * 32; base < a.npix; base += FOM_WARPS * 32) {
        T Rx = 0, Ry = 0;
        const int cnt = min(32, a.npix - base);
        if (a.psec) {                                     // the panel's FP32 section, gathered once
            if (lane < cnt) {
                const float2 r = a.psec[(long)H.sec * a.npix + base + lane];
                Rx = (T)r.x;
                Ry = (T)r.y;
            }
        } else if (a.sec) {                               // section gathered once per view
            if (lane < cnt) {
                const double2 r = a.sec[(long)H.sec * a.npix + base + lane];
                Rx = (T)r.x;
                Ry = (T)r.y;
            }
        } else
        for (int q = 0; q < cnt; ++q) {
            const MPix pq = a.pix[base + q];
            if (!pq.insec) continue;                      // warp-uniform
            const double ix = pq.h * a.inv, iy = pq.k * a.inv;
            const double mx = (H.m[0] * ix + H.m[1] * iy) * a.real;
            const double myy = (H.m[3] * ix + H.m[4] * iy) * a.real;
            const double mz = (H.m[6] * ix + H.m[7] * iy) * a.real;
            T vr, vi;
            fsi_gather<T>(TexSrc{a.tex}, a.D, mx, myy, mz, lut, a.wd, lane, vr, vi);
            if (lane == q) {
                Rx = vr;
                Ry = vi;
            }
        }
        const int p = base + lane;
        T v[NV];
#pragma unroll
        for (int o = 0; o < NV; ++o) v[o] = 0;
        int shell = -1;
        if (lane < cnt) {
            const MPix pq = a.pix[p];
            shell = pq.shell;
            const float2 x = X[pq.idx];
            const T c = C[p];
            const T rr = Rx * c, ri = Ry * c;
            T amp = 0, pr = 0;
            if (a.dpr) {
                amp = sqrt((T)x.x * (T)x.x + (T)x.y * (T)x.y) + sqrt(rr * rr + ri * ri);
                pr = atan2(ri, rr);
                v[0] = amp;
            } else {
                v[0] = rr * rr + ri * ri;
            }
#pragma unroll
            for (int o = 0; o < MAXORG; ++o) {
                if (o < norg) {
                    double phi = pq.h * H.sx[o] + pq.k * H.sy[o];
                    T sn, cs;
                    if constexpr (sizeof(T) == 8) {
                        sincos(phi, &sn, &cs);
                    } else {
                        phi -= 6.283185307179586 * rint(phi * 0.15915494309189535);
                        sincosf((float)phi, &sn, &cs);
                    }
                    const T xr = (T)x.x * cs - (T)x.y * sn, xi = (T)x.x * sn + (T)x.y * cs;
                    if (a.dpr) {
                        T d = atan2(xi, xr) - pr;
                        if (d < (T)-3.14159265358979323846) d += (T)6.28318530717958647692;
                        else if (d > (T)3.14159265358979323846) d -= (T)6.28318530717958647692;
                        v[1 + o] = amp * d * d;
                    } else {
                        v[1 + o] = xr * rr + xi * ri;
                    }
                }
            }
        }
        // segmented sums over the lanes of each shell present in this group
        unsigned left = __ballot_sync(0xffffffffu, shell >= 0);
        while (left) {
            const int lead = __ffs(left) - 1;
            const int s = __shfl_sync(0xffffffffu, shell, lead);
            const bool in = shell == s;
#pragma unroll
            for (int o = 0; o < NV; ++o) {
                if (o > norg) break;
                T t = in ? v[o] : (T)0;
#pragma unroll
                for (int k = 16; k; k >>= 1) t += __shfl_xor_sync(0xffffffffu, t, k);
                if (lane == 0) my[s * NV + o] += t;
            }
            left &= ~__ballot_sync(0xffffffffu, in);
        }
    }
    __syncthreads();
    // one warp per origin: shells j (lane-strided), folded over warps in
    // order, then summed over j by a fixed shuffle tree
    // (MAXORG may exceed the warp count: warps take origins in turn)
    for (int o = warp; o < norg; o += FOM_WARPS) {
        const double* ds = a.dsum + img * (long)a.nshell;
        double tf = 0, tc = 0;
        for (int j = lane; j < a.nshell; j += 32) {
            double fj = 0, mj = 0;
            for (int w = 0; w < FOM_WARPS; ++w) {
                mj += wsum[(w * a.nshell + j) * NV];
                fj += wsum[(w * a.nshell + j) * NV + 1 + o];
            }
            double t;
            const double wj = a.wshell[j];
            if (a.dpr) {
                t = mj != 0.0 ? wj * cos(sqrt(fj / mj)) : 0.0;
            } else {
                const double den = ds[j] * mj;
                t = den > 0 ? wj * fj / sqrt(den) : 0.0;
            }
            if (j < a.nf) tf += t;
            if (j >= a.cv0 && j < a.cv1) tc += t;
        }
#pragma unroll
        for (int k = 16; k; k >>= 1) {
            tf += __shfl_xor_sync(0xffffffffu, tf, k);
            tc += __shfl_xor_sync(0xffffffffu, tc, k);
        }
        if (lane == 0) {
            a.fom[(long)blockIdx.x * MAXORG + o] = a.nf > 0 ? tf / a.wf : 0.0;
            a.cv[(long)blockIdx.x * MAXORG + o] = (a.cv1 > a.cv0) ? tc / a.wc : 0.0;
        }
    }
}

void twiddles(int L, std::vector<double2>& out) {
    out.assign(std::max(1, L / 2), make_double2(1.0, 0.0));
    for (int j = 0; j < L / 2; ++j) {
        const double a = -2.0 * M_PI * j / L;
        out[j] = make_double2(cos(a), sin(a));
    }
}

double electron_lambda(double volt) {
    // relativistic electron wavelength in angstrom (ctf.h:309-317)
    if (volt <= 0) return 0;
    const double h = 6.626070e-34, me = 9.109384e-31, e = 1.602177e-19, c = 299792458.0;
    return h * 1e10 / sqrt(2.0 * me * e * volt * (1.0 + e * volt / (2.0 * me * c * c)));
}

}  // namespace

}  // namespace bsg

using namespace bsg;

namespace {

int mfail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    set_error("%s", buf);
    return code;
}

#define MCK(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return mfail(BSG_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

bool pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

std::once_flag g_attr_once;
cudaError_t g_attr_err = cudaSuccess;

void set_attributes() {
    const int big = 100 * 1024;
    cudaError_t e = cudaFuncSetAttribute(strided64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fom_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fom_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    g_attr_err = e;
}

cudaError_t fft2_forward(double2* data, int L, long count, const double2* tw, cudaStream_t s) {
    // rows then columns of `count` L x L transforms
    const int logL = ilog2i(L);
    const long lines = (long)L * count;
    lines64_kernel<<<(unsigned)((lines + LW - 1) / LW), LW * 32, sizeof(double2) * (L / 2 + LW * L), s>>>(
        data, lines, L, logL, tw);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dim3 g((L + SWL - 1) / SWL, (unsigned)count);
    strided64_kernel<<<g, SWL * 32, sizeof(double2) * (L / 2 + SWL * L), s>>>(data, L, logL, L, L, (long)L * L, tw);
    return cudaGetLastError();
}

int ensure_work(Match& M, size_t elems) {
    if (elems <= M.work_elems) return BSG_OK;
    cudaFree(M.d_work);
    cudaFree(M.d_real);
    M.d_work = nullptr;
    M.d_real = nullptr;
    M.work_elems = 0;
    MCK(cudaMalloc(&M.d_work, sizeof(double2) * elems));
    MCK(cudaMalloc(&M.d_real, sizeof(float) * elems));
    M.work_elems = elems;
    return BSG_OK;
}

int ensure_pinned(Match& M, size_t bytes) {
    if (bytes <= M.pin_bytes) return BSG_OK;
    if (M.h_pin) cudaFreeHost(M.h_pin);
    M.h_pin = nullptr;
    M.pin_bytes = 0;
    MCK(cudaMallocHost(&M.h_pin, bytes));
    M.pin_bytes = bytes;
    return BSG_OK;
}

}  // namespace

extern "C" int bsg_match_create(const bsg_match_config* cfg, bsg_match** out) {
    if (!cfg || !out) return mfail(BSG_ERR_ARG, "bsg_match_create: null argument");
    *out = nullptr;
    const int N = cfg->map, n = cfg->n;
    if (!pow2(N) || N < 8 || N > 512 || !pow2(n) || n < 32 || n > 512)
        return mfail(BSG_ERR_ARG, "bsg_match_create: map %d and box %d must be powers of two (map 8..512, box 32..512)",
                     N, n);
    if (!(cfg->map_sampling > 0) || !(cfg->pixel > 0) || !(cfg->hi_res > 0))
        return mfail(BSG_ERR_ARG, "bsg_match_create: sampling, pixel size and resolution must be > 0");
    const int wd = cfg->kernel_power < 0 ? 1 : cfg->kernel_width;
    if (wd < 1 || wd > MAXW) return mfail(BSG_ERR_ARG, "bsg_match_create: kernel width %d outside 1..%d", wd, MAXW);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev)
        return mfail(BSG_ERR_NODEV, "bsg_match_create: no CUDA device %d", cfg->device);
    MCK(cudaSetDevice(cfg->device));
    std::call_once(g_attr_once, set_attributes);
    if (g_attr_err != cudaSuccess) return mfail(BSG_ERR_CUDA, "bsg_match_create: %s", cudaGetErrorString(g_attr_err));

    Match* M = new (std::nothrow) Match();
    if (!M) return mfail(BSG_ERR_NOMEM, "bsg_match_create: out of host memory");
    M->cfg = *cfg;
    M->device = cfg->device;
    M->N = N;
    M->n = n;
    M->wd = wd;
    // project_refine_orientations (mg_refine.cpp:290-316): check_resolution
    // on the map, the cut edge, check_resolution on the cut map
    double hr = cfg->hi_res;
    const double u = cfg->map_sampling;
    if (hr > N * u) hr = N * u;
    else hr = std::max(hr, 2.0 / sqrt(3.0 / (u * u)));
    int D = (int)(2.2 * N * u / hr + 0.5);
    if (D % 2) D += 1;
    if (D > N) D = N;
    const double us = u * N / D;
    if (hr > D * us) hr = D * us;
    else hr = std::max(hr, 2.0 / sqrt(3.0 / (us * us)));
    if (D > n) {
        delete M;
        return mfail(BSG_ERR_ARG, "bsg_match_create: the reference transform edge %d exceeds the particle box %d", D, n);
    }
    M->D = D;
    M->map_samp_cut = us;
    M->img_samp_cut = cfg->pixel * n / D;
    M->real_map = D * us;
    M->real_img = n * cfg->pixel;
    M->scx = M->scy = us / M->img_samp_cut;
    M->cut_scale = (double)((long double)D / n);
    M->sec_res = hr / 1.11;
    // img_recip_space_fom (mg_refine.cpp:666-687): check_resolution on the
    // 2-D section (sampling us), radii in pixels of the section
    if (hr > M->real_map) hr = M->real_map;
    else hr = std::max(hr, 2.0 / sqrt(2.0 / (us * us)));
    double lo = cfg->lo_res;
    if (lo > 0 && hr > lo) std::swap(hr, lo);
    M->hi_res = hr;
    M->max_rad = M->real_map / hr;
    M->max_rad_cv = 1.1 * M->max_rad;
    if (M->max_rad_cv <= M->max_rad) M->max_rad_cv = M->max_rad + 1;
    const double max_cv_sq = M->max_rad_cv * M->max_rad_cv;
    double min_sq = 0;
    if (lo > 0) { min_sq = M->real_map / lo; min_sq *= min_sq; }
    // figure-of-merit pixels, in reference order first
    const double inv = 1.0 / M->real_map, maxs2 = 1.0 / (M->sec_res * M->sec_res);
    std::vector<std::pair<double, MPix>> tmp;
    for (int yy = 0; yy < D; ++yy)
        for (int xx = 0; xx < D; ++xx) {
            const int h = sfreq(xx, D), k = sfreq(yy, D);
            const double ix = h * inv, iy = k * inv;
            const bool insec = ix * ix + iy * iy <= maxs2;
            MPix q{};
            q.h = (short)h;
            q.k = (short)k;
            q.idx = yy * D + xx;
            q.insec = insec ? 1 : 0;
            if (insec) M->h_secpix.push_back(q);
            const double d2 = (double)(h * h + k * k);
            if (d2 < min_sq || d2 > max_cv_sq) continue;
            const long j = (long)sqrt(d2);
            if (j >= D) continue;
            q.shell = (short)j;
            tmp.push_back({j * 10.0 + atan2((double)k, (double)h), q});
        }
    std::stable_sort(tmp.begin(), tmp.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    int maxshell = 0;
    for (auto& t : tmp) { M->h_pix.push_back(t.second); maxshell = std::max(maxshell, (int)t.second.shell); }
    M->nshell = std::max((int)ceil(M->max_rad_cv), maxshell + 1);
    M->h_shell_start.assign(M->nshell + 1, 0);
    for (auto& q : M->h_pix) M->h_shell_start[q.shell + 1]++;
    for (int j = 0; j < M->nshell; ++j) M->h_shell_start[j + 1] += M->h_shell_start[j];
    M->nf = 0;
    for (long j = 0; j < M->max_rad; ++j) M->nf++;
    M->cv0 = (int)(long)M->max_rad;
    M->cv1 = M->cv0;
    for (long j = (long)M->max_rad; j < M->max_rad_cv; ++j) M->cv1 = (int)j + 1;
    if (M->nf > M->nshell || M->cv1 > M->nshell) M->nshell = std::max(M->nf, M->cv1);
    // unit shell weights until the caller sets a curve
    M->h_wshell.assign(M->nshell, 1.0);
    M->wf = (double)M->nf;
    M->wc = (double)(M->cv1 - M->cv0);
    M->h_shell_start.resize(M->nshell + 1, M->h_shell_start.back());

    // FSI kernel table (FSI_Kernel.h:28-68): row r = fraction r/512, tap j
    // at distance d = r/512 + (w-1)/2 - j, sin(pi d) / (w sin(pi d/w)) *
    // cos(pi d/w)^power; rows 0 and 512 are the identity at taps (w-1)/2, +1
    std::vector<double> lut((size_t)(NDIV + 1) * wd, cfg->kernel_power < 0 ? 1.0 : 0.0);
    if (cfg->kernel_power >= 0) {
        const int h2 = (wd - 1) / 2;
        lut[h2] = 1.0;
        for (int r = 1; r < NDIV; ++r)
            for (int j = 0; j < wd; ++j) {
                const double d = (double)r / NDIV + h2 - j, a = M_PI * d / wd;
                lut[(size_t)r * wd + j] = sin(M_PI * d) / (wd * sin(a)) * pow(cos(a), cfg->kernel_power);
            }
        lut[(size_t)NDIV * wd + h2 + 1] = 1.0;
    }
    std::vector<double2> twm, twi;
    twiddles(N, twm);
    twiddles(n, twi);
    cudaError_t e = cudaStreamCreateWithFlags(&M->stream, cudaStreamNonBlocking);
#define ALLOC(p, bytes) if (e == cudaSuccess) e = cudaMalloc((void**)&(p), (bytes))
    ALLOC(M->d_pix, sizeof(MPix) * std::max<size_t>(1, M->h_pix.size()));
    ALLOC(M->d_shell_start, sizeof(int) * M->h_shell_start.size());
    ALLOC(M->d_secpix, sizeof(MPix) * std::max<size_t>(1, M->h_secpix.size()));
    ALLOC(M->d_lut, sizeof(double) * lut.size());
    ALLOC(M->d_lutf, sizeof(float) * lut.size());
    ALLOC(M->d_tw_map, sizeof(double2) * twm.size());
    ALLOC(M->d_tw_img, sizeof(double2) * twi.size());
    ALLOC(M->d_ref, sizeof(float2) * (size_t)D * D * D);
    ALLOC(M->d_wshell, sizeof(double) * std::max<size_t>(1, M->h_wshell.size()));
#undef ALLOC
    if (e == cudaSuccess)
        e = cudaMemcpy(M->d_wshell, M->h_wshell.data(), sizeof(double) * M->h_wshell.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(M->d_pix, M->h_pix.data(), sizeof(MPix) * M->h_pix.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(M->d_shell_start, M->h_shell_start.data(), sizeof(int) * M->h_shell_start.size(),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(M->d_secpix, M->h_secpix.data(), sizeof(MPix) * M->h_secpix.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(M->d_lut, lut.data(), sizeof(double) * lut.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        std::vector<float> lf(lut.begin(), lut.end());
        e = cudaMemcpy(M->d_lutf, lf.data(), sizeof(float) * lf.size(), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemcpy(M->d_tw_map, twm.data(), sizeof(double2) * twm.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(M->d_tw_img, twi.data(), sizeof(double2) * twi.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        bsg_match_destroy(reinterpret_cast<bsg_match*>(M));
        return mfail(BSG_ERR_CUDA, "bsg_match_create: %s", cudaGetErrorString(e));
    }
    *out = reinterpret_cast<bsg_match*>(M);
    return BSG_OK;
}

extern "C" void bsg_match_destroy(bsg_match* h) {
    Match* M = reinterpret_cast<Match*>(h);
    if (!M) return;
    cudaSetDevice(M->device);
    if (M->stream) cudaStreamSynchronize(M->stream);
    void* ptrs[] = {M->d_pix, M->d_shell_start, M->d_secpix, M->d_lut, M->d_lutf, M->d_tw_map, M->d_tw_img, M->d_ref,
                    M->d_spec, M->d_ctf, M->d_dsum, M->d_real, M->d_work, M->d_scale, M->d_shift, M->d_ictf,
                    M->d_hyp, M->d_out, M->d_full, M->d_grp, M->d_gout, M->d_cpix, M->d_cstart, M->d_secs, M->d_panel, M->d_A, M->d_pscore,
                    M->d_pidx, M->d_csec, M->d_corg, M->d_cscore, M->d_rots, M->d_gA, M->d_slopes,
                    M->d_lprop, M->d_lorg, M->d_nlorg, M->d_lcand, M->d_lcount,
                    M->d_status, M->d_pexact, M->d_wshell};
    for (void* p : ptrs) if (p) cudaFree(p);
    if (M->h_pin) cudaFreeHost(M->h_pin);
    if (M->ref_tex) cudaDestroyTextureObject(M->ref_tex);
    if (M->ref_array) cudaFreeArray(M->ref_array);
    if (M->stream) cudaStreamDestroy(M->stream);
    delete M;
}

extern "C" int bsg_match_info(const bsg_match* h, bsg_match_info_t* info) {
    const Match* M = reinterpret_cast<const Match*>(h);
    if (!M || !info) return mfail(BSG_ERR_ARG, "bsg_match_info: null argument");
    info->diam = M->D;
    info->npix = (int)M->h_pix.size();
    info->nshell = M->nshell;
    info->hi_res = M->hi_res;
    info->max_rad = M->max_rad;
    info->section_res = M->sec_res;
    info->map_sampling_cut = M->map_samp_cut;
    info->pixel_cut = M->img_samp_cut;
    return BSG_OK;
}

extern "C" int bsg_match_set_reference(bsg_match* h, const float* map, const double* origin, int flags) {
    Match* M = reinterpret_cast<Match*>(h);
    if (!M || !map || !origin) return mfail(BSG_ERR_ARG, "bsg_match_set_reference: null argument");
    MCK(cudaSetDevice(M->device));
    // the panel's exact sections belong to the previous map
    if (M->d_pexact) {
        cudaStreamSynchronize(M->stream);
        cudaFree(M->d_pexact);
        M->d_pexact = nullptr;
    }
    const int N = M->N, D = M->D;
    const size_t n3 = (size_t)N * N * N;
    int rc = ensure_work(*M, n3);
    if (rc) return rc;
    cudaStream_t s = M->stream;
    const float* src = map;
    if (!(flags & BSG_DEVICE_PTR)) {
        MCK(cudaMemcpyAsync(M->d_real, map, sizeof(float) * n3, cudaMemcpyHostToDevice, s));
        src = M->d_real;
    }
    to_complex_kernel<<<148 * 8, 256, 0, s>>>(src, M->d_work, (long)n3, (long)n3, nullptr, nullptr);
    MCK(cudaGetLastError());
    // 3-D forward transform: x lines, then y and z as strided lines
    const int logN = ilog2i(N);
    lines64_kernel<<<(unsigned)(((long)N * N + LW - 1) / LW), LW * 32, sizeof(double2) * (N / 2 + LW * N), s>>>(
        M->d_work, (long)N * N, N, logN, M->d_tw_map);
    MCK(cudaGetLastError());
    {
        dim3 g((N + SWL - 1) / SWL, N);
        strided64_kernel<<<g, SWL * 32, sizeof(double2) * (N / 2 + SWL * N), s>>>(
            M->d_work, N, logN, N, N, (long)N * N, M->d_tw_map);
        MCK(cudaGetLastError());
        dim3 g2((unsigned)(((long)N * N + SWL - 1) / SWL), 1);
        strided64_kernel<<<g2, SWL * 32, sizeof(double2) * (N / 2 + SWL * N), s>>>(
            M->d_work, N, logN, (long)N * N, (long)N * N, 0, M->d_tw_map);
        MCK(cudaGetLastError());
    }
    // cut, clear the zero-frequency term, shift to the origin scaled to the
    // cut edge (change_transform_size scales origins, Bimage_fft.cpp:433)
    const double sc = (double)D / N;
    const double sx = origin[0] * sc / D * 2 * M_PI, sy = origin[1] * sc / D * 2 * M_PI, sz = origin[2] * sc / D * 2 * M_PI;
    map_cut_kernel<<<148 * 8, 256, 0, s>>>(M->d_work, N, D, 1.0 / sqrt((double)n3), sx, sy, sz, M->d_ref);
    MCK(cudaGetLastError());
    if (!M->d_full) MCK(cudaMalloc(&M->d_full, sizeof(float2) * n3));
    {
        const double fx = origin[0] / N * 2 * M_PI, fy = origin[1] / N * 2 * M_PI, fz = origin[2] / N * 2 * M_PI;
        map_full_kernel<<<148 * 8, 256, 0, s>>>(M->d_work, N, 1.0 / sqrt((double)n3), fx, fy, fz, M->d_full);
        MCK(cudaGetLastError());
    }
    MCK(cudaStreamSynchronize(s));
    // the same transform behind a 3-D texture (point sampling, integer
    // coordinates: every fetch returns a stored value unchanged)
    if (!M->ref_array) {
        const cudaChannelFormatDesc ch = cudaCreateChannelDesc<float2>();
        MCK(cudaMalloc3DArray(&M->ref_array, &ch, make_cudaExtent(D, D, D)));
        cudaResourceDesc rd;
        memset(&rd, 0, sizeof(rd));
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = M->ref_array;
        cudaTextureDesc td;
        memset(&td, 0, sizeof(td));
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModePoint;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        MCK(cudaCreateTextureObject(&M->ref_tex, &rd, &td, nullptr));
    }
    cudaMemcpy3DParms cp;
    memset(&cp, 0, sizeof(cp));
    cp.srcPtr = make_cudaPitchedPtr(M->d_ref, sizeof(float2) * D, D, D);
    cp.dstArray = M->ref_array;
    cp.extent = make_cudaExtent(D, D, D);
    cp.kind = cudaMemcpyDeviceToDevice;
    MCK(cudaMemcpy3DAsync(&cp, s));
    MCK(cudaStreamSynchronize(s));
    M->have_ref = true;
    return BSG_OK;
}

extern "C" int bsg_match_reference_transform(bsg_match* h, float* out, int flags) {
    Match* M = reinterpret_cast<Match*>(h);
    if (!M || !out) return mfail(BSG_ERR_ARG, "bsg_match_reference_transform: null argument");
    if (!M->have_ref) return mfail(BSG_ERR_STATE, "bsg_match_reference_transform: no reference set");
    MCK(cudaSetDevice(M->device));
    const size_t bytes = sizeof(float2) * (size_t)M->D * M->D * M->D;
    MCK(cudaMemcpyAsync(out, M->d_ref, bytes, (flags & BSG_DEVICE_PTR) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                        M->stream));
    MCK(cudaStreamSynchronize(M->stream));
    return BSG_OK;
}

namespace bsg {
void match_view_rows(const Match& M, const double* mat, double* m) {
    // img_fit_in_recip_space_grid: rows 0 and 1 multiplied componentwise by
    // (pref sampling / particle sampling) per axis, z component by 1
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double v = mat[3 * r + c];
            if (r < 2) v *= (c == 0 ? M.scx : (c == 1 ? M.scy : 1.0));
            m[3 * r + c] = v;
        }
}

int match_fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    set_error("%s", buf);
    return code;
}

// The FP64 section values of nv views (9 doubles each, rows 0 and 1
// scaled as in MHyp) at the figure-of-merit pixels: the same gather, in the
// same order, as fom_kernel<double> performs for one group, so scores from
// these values equal the gathering kernel's.
__global__ void __launch_bounds__(FOM_WARPS * 32) secgather_kernel(cudaTextureObject_t tex, int D, int wd,
                                                                   const double* __restrict__ lut_g,
                                                                   const MPix* __restrict__ pix, int npix,
                                                                   const double* __restrict__ mats, double inv,
                                                                   double real, double2* __restrict__ out) {
    __shared__ double lut[(NDIV + 1) * MAXW];
    for (int i = threadIdx.x; i < (NDIV + 1) * wd; i += blockDim.x) lut[i] = lut_g[i];
    __syncthreads();
    const double* m = mats + 9 * (long)blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double2* o = out + (long)blockIdx.x * npix;
    for (int base = warp * 32; base < npix; base += FOM_WARPS * 32) {
        double Rx = 0, Ry = 0;
        const int cnt = min(32, npix - base);
        for (int q = 0; q < cnt; ++q) {
            const MPix pq = pix[base + q];
            if (!pq.insec) continue;                      // warp-uniform
            const double ix = pq.h * inv, iy = pq.k * inv;
            const double mx = (m[0] * ix + m[1] * iy) * real;
            const double myy = (m[3] * ix + m[4] * iy) * real;
            const double mz = (m[6] * ix + m[7] * iy) * real;
            double vr, vi;
            fsi_gather<double>(TexSrc{tex}, D, mx, myy, mz, lut, wd, lane, vr, vi);
            if (lane == q) {
                Rx = vr;
                Ry = vi;
            }
        }
        if (lane < cnt) o[base + lane] = make_double2(Rx, Ry);
    }
}

cudaError_t launch_secgather(const Match& M, const double* d_mats, long nv, double2* d_out, cudaStream_t s) {
    if (nv > 0)
        secgather_kernel<<<(unsigned)nv, FOM_WARPS * 32, 0, s>>>(M.ref_tex, M.D, M.wd, M.d_lut, M.d_pix,
                                                                 (int)M.h_pix.size(), d_mats, 1.0 / M.real_map,
                                                                 M.real_map, d_out);
    return cudaGetLastError();
}

// The panel's FP32 sections at the figure-of-merit pixels: one CTA per view,
// the pixels in the warp-strided blocks of 32 that fom_kernel<float> walks,
// each gathered by the whole warp with the same coordinates and the same
// FP32 FSI gather, so the stored values are the ones fom_kernel<float> would
// compute for that view.
__global__ void __launch_bounds__(FOM_WARPS * 32) panel_exact_kernel(cudaTextureObject_t tex, int D,
                                                                   const float* __restrict__ lut_g, int wd,
                                                                   const MPix* __restrict__ pix, int npix,
                                                                   const MHyp* __restrict__ secs, double inv,
                                                                   double real, float2* __restrict__ out) {
    __shared__ float lut[(NDIV + 1) * MAXW];
    for (int i = threadIdx.x; i < (NDIV + 1) * wd; i += blockDim.x) lut[i] = lut_g[i];
    __syncthreads();
    const MHyp& H = secs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float2* o = out + (size_t)blockIdx.x * npix;
    for (int base = warp * 32; base < npix; base += FOM_WARPS * 32) {
        float Rx = 0, Ry = 0;
        const int cnt = min(32, npix - base);
        for (int q = 0; q < cnt; ++q) {
            const MPix pq = pix[base + q];
            if (!pq.insec) continue;                      // warp-uniform
            const double ix = pq.h * inv, iy = pq.k * inv;
            const double mx = (H.m[0] * ix + H.m[1] * iy) * real;
            const double myy = (H.m[3] * ix + H.m[4] * iy) * real;
            const double mz = (H.m[6] * ix + H.m[7] * iy) * real;
            float vr, vi;
            fsi_gather<float>(TexSrc{tex}, D, mx, myy, mz, lut, wd, lane, vr, vi);
            if (lane == q) {
                Rx = vr;
                Ry = vi;
            }
        }
        if (lane < cnt) o[base + lane] = make_float2(Rx, Ry);
    }
}

cudaError_t launch_panel_exact(const Match& M, const MHyp* d_secs, long nsec, float2* d_out, cudaStream_t s) {
    const long npix = (long)M.h_pix.size();
    for (long v0 = 0; v0 < nsec; v0 += 1L << 20) {
        const long cnt = std::min(nsec - v0, 1L << 20);
        panel_exact_kernel<<<(unsigned)cnt, FOM_WARPS * 32, 0, s>>>(M.ref_tex, M.D, M.d_lutf, M.wd, M.d_pix, (int)npix,
                                                                   d_secs + v0, 1.0 / M.real_map, M.real_map,
                                                                   d_out + (size_t)v0 * npix);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_ctf_rows(const Match& M, const ImgCtf* d_rec, long nrec, float* d_out, cudaStream_t s) {
    if (nrec > 0)
        ctf_rows_kernel<<<(unsigned)nrec, 256, 0, s>>>(d_rec, M.d_pix, (int)M.h_pix.size(), 1.0 / M.real_img, d_out);
    return cudaGetLastError();
}

cudaError_t launch_fom(const Match& M, const MHypG* d_groups, long ng, double* d_fom, double* d_cv, cudaStream_t s,
                       bool fp64, const float* ctf_table, const double2* sec, bool dpr, const float2* psec) {
    FomArgs a{};
    a.dpr = dpr ? 1 : 0;
    a.psec = fp64 ? nullptr : psec;
    a.tex = M.ref_tex; a.D = M.D; a.wd = M.wd; a.lut = M.d_lutf; a.lutd = M.d_lut;
    a.pix = M.d_pix; a.npix = (int)M.h_pix.size(); a.hyps = d_groups;
    a.spec = M.d_spec; a.ctf = ctf_table ? ctf_table : M.d_ctf; a.dsum = M.d_dsum; a.nshell = M.nshell;
    a.inv = 1.0 / M.real_map; a.real = M.real_map;
    a.nf = M.nf; a.cv0 = M.cv0; a.cv1 = M.cv1;
    a.wshell = M.d_wshell; a.wf = M.wf; a.wc = M.wc;
    a.fom = d_fom; a.cv = d_cv; a.sec = sec;
    const size_t words = (NDIV + 1) * MAXW + FOM_WARPS * M.nshell * (1 + MAXORG);
    if (fp64 && sizeof(double) * words > 220 * 1024) return cudaErrorInvalidValue;
    if (ng > 0) {
        if (fp64) fom_kernel<double><<<(unsigned)ng, FOM_WARPS * 32, sizeof(double) * words, s>>>(a);
        else fom_kernel<float><<<(unsigned)ng, FOM_WARPS * 32, sizeof(float) * words, s>>>(a);
    }
    return cudaGetLastError();
}

// hypotheses (image, view, origin) -> groups of one image and view with up
// to MAXORG origins; slot[i] = group * MAXORG + position of hypothesis i
void group_hypotheses(const std::vector<MHyp>& hyps, std::vector<MHypG>& groups, std::vector<long>& slot) {
    std::vector<long> order(hyps.size());
    for (size_t i = 0; i < hyps.size(); ++i) order[i] = (long)i;
    auto key_less = [&](long x, long y) {
        const MHyp &a = hyps[x], &b = hyps[y];
        if (a.img != b.img) return a.img < b.img;
        const int c = memcmp(a.m, b.m, sizeof(a.m));
        if (c) return c < 0;
        return x < y;
    };
    std::stable_sort(order.begin(), order.end(), key_less);
    groups.clear();
    slot.assign(hyps.size(), 0);
    for (size_t k = 0; k < order.size(); ++k) {
        const MHyp& h = hyps[order[k]];
        bool same = !groups.empty() && groups.back().img == h.img && groups.back().norg < MAXORG &&
                    memcmp(groups.back().m, h.m, sizeof(h.m)) == 0;
        if (!same) {
            MHypG g;
            memset(&g, 0, sizeof(g));
            memcpy(g.m, h.m, sizeof(g.m));
            g.img = h.img;
            g.ctf = h.img;
            groups.push_back(g);
        }
        MHypG& g = groups.back();
        g.sx[g.norg] = h.sx;
        g.sy[g.norg] = h.sy;
        slot[order[k]] = (long)(groups.size() - 1) * MAXORG + g.norg;
        g.norg++;
    }
}
}  // namespace bsg

static int ensure_hyps(Match& M, long nh) {
    if (nh <= M.hyp_cap) return BSG_OK;
    cudaFree(M.d_hyp);
    cudaFree(M.d_out);
    M.d_hyp = nullptr;
    M.d_out = nullptr;
    M.hyp_cap = 0;
    MCK(cudaMalloc(&M.d_hyp, sizeof(MHyp) * nh));
    MCK(cudaMalloc(&M.d_out, sizeof(double) * 2 * nh));
    M.hyp_cap = nh;
    return BSG_OK;
}

namespace bsg {
int ensure_groups(Match& M, long ng) {
    if (ng <= M.grp_cap) return BSG_OK;
    cudaFree(M.d_grp);
    cudaFree(M.d_gout);
    M.d_grp = nullptr;
    M.d_gout = nullptr;
    M.grp_cap = 0;
    MCK(cudaMalloc(&M.d_grp, sizeof(MHypG) * ng));
    MCK(cudaMalloc(&M.d_gout, sizeof(double) * 2 * MAXORG * ng));
    M.grp_cap = ng;
    return BSG_OK;
}
}  // namespace bsg

extern "C" int bsg_match_sections(bsg_match* h, const double* mats, long nviews, float* out, int flags) {
    Match* M = reinterpret_cast<Match*>(h);
    if (!M || !mats || !out || nviews < 1) return mfail(BSG_ERR_ARG, "bsg_match_sections: bad argument");
    if (!M->have_ref) return mfail(BSG_ERR_STATE, "bsg_match_sections: no reference set");
    MCK(cudaSetDevice(M->device));
    const int D = M->D;
    const size_t per = (size_t)D * D;
    int rc = ensure_hyps(*M, nviews);
    if (rc) return rc;
    std::vector<MHyp> hv(nviews);
    for (long v = 0; v < nviews; ++v) {
        memset(&hv[v], 0, sizeof(MHyp));
        match_view_rows(*M, mats + 9 * v, hv[v].m);
    }
    cudaStream_t s = M->stream;
    MCK(cudaMemcpyAsync(M->d_hyp, hv.data(), sizeof(MHyp) * nviews, cudaMemcpyHostToDevice, s));
    float2* dst = reinterpret_cast<float2*>(out);
    float2* tmp = nullptr;
    if (!(flags & BSG_DEVICE_PTR)) {
        MCK(cudaMalloc(&tmp, sizeof(float2) * per * nviews));
        dst = tmp;
    }
    cudaError_t e = cudaMemsetAsync(dst, 0, sizeof(float2) * per * nviews, s);
    if (e == cudaSuccess) {
        section_kernel<<<(unsigned)nviews, 256, 0, s>>>(M->d_ref, D, M->d_lut, M->wd, M->d_secpix,
                                                        (int)M->h_secpix.size(), M->d_hyp, 1.0 / M->real_map,
                                                        M->real_map, dst);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && tmp)
        e = cudaMemcpyAsync(out, tmp, sizeof(float2) * per * nviews, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (tmp) cudaFree(tmp);
    if (e != cudaSuccess) return mfail(BSG_ERR_CUDA, "bsg_match_sections: %s", cudaGetErrorString(e));
    return BSG_OK;
}

extern "C" int bsg_match_set_images(bsg_match* h, const float* images, long nimg, const double* ctf,
                                    double file_avg, double file_std, int flags) {
    Match* M = reinterpret_cast<Match*>(h);
    if (!M || !images || !ctf || nimg < 1) return mfail(BSG_ERR_ARG, "bsg_match_set_images: bad argument");
    MCK(cudaSetDevice(M->device));
    const int n = M->n, D = M->D;
    const int npix = (int)M->h_pix.size();
    cudaStream_t s = M->stream;
    if (nimg > M->cap) {
        cudaFree(M->d_spec); cudaFree(M->d_ctf); cudaFree(M->d_dsum);
        cudaFree(M->d_scale); cudaFree(M->d_shift); cudaFree(M->d_ictf);
        M->d_spec = nullptr; M->d_ctf = nullptr; M->d_dsum = nullptr;
        M->d_scale = nullptr; M->d_shift = nullptr; M->d_ictf = nullptr;
        M->cap = 0;
        MCK(cudaMalloc(&M->d_spec, sizeof(float2) * (size_t)D * D * nimg));
        MCK(cudaMalloc(&M->d_ctf, sizeof(float) * (size_t)std::max(1, npix) * nimg));
        MCK(cudaMalloc(&M->d_dsum, sizeof(double) * (size_t)M->nshell * nimg));
        MCK(cudaMalloc(&M->d_scale, sizeof(double) * nimg));
        MCK(cudaMalloc(&M->d_shift, sizeof(double) * nimg));
        MCK(cudaMalloc(&M->d_ictf, sizeof(ImgCtf) * nimg));
        M->cap = nimg;
    }
    // CTF records: [volt, abw00, abw20, abw22, abw2m2, abw40, flags, 0];
    // img_recip_space_fom applies it only when the defocus is >= 1 angstrom
    std::vector<ImgCtf> ic(nimg);
    for (long i = 0; i < nimg; ++i) {
        const double* r = ctf + 8 * i;
        memset(&ic[i], 0, sizeof(ImgCtf));
        for (int j = 0; j < 5; ++j) ic[i].c[j] = r[1 + j];
        const int f = (int)r[6];
        const double t2 = -M_PI * electron_lambda(r[0]);
        const double def = t2 != 0 ? r[2] / t2 : 0;
        ic[i].apply = (f & BSG_MATCH_APPLY_CTF) && def >= 1 ? 1 : 0;
        ic[i].invert = (f & BSG_MATCH_INVERT) ? 1 : 0;
    }
    M->h_ictf = ic;
    M->h_volt.assign(nimg, 0.0);
    for (long i = 0; i < nimg; ++i) M->h_volt[i] = ctf[8 * i];
    MCK(cudaMemcpyAsync(M->d_ictf, ic.data(), sizeof(ImgCtf) * nimg, cudaMemcpyHostToDevice, s));
    if (file_std > 0) {
        std::vector<double> sc(nimg, 1.0 / file_std), sh(nimg, -file_avg / file_std);
        if (!(file_std > 1e-30)) { std::fill(sc.begin(), sc.end(), 1.0); std::fill(sh.begin(), sh.end(), -file_avg); }
        MCK(cudaMemcpyAsync(M->d_scale, sc.data(), sizeof(double) * nimg, cudaMemcpyHostToDevice, s));
        MCK(cudaMemcpyAsync(M->d_shift, sh.data(), sizeof(double) * nimg, cudaMemcpyHostToDevice, s));
        MCK(cudaStreamSynchronize(s));
    }
    // images in chunks through the work buffers
    const long n2 = (long)n * n;
    const long chunk = std::max<long>(1, std::min<long>(nimg, M->cfg.batch > 0 ? M->cfg.batch : 1024));
    int rc = ensure_work(*M, (size_t)n2 * chunk);
    if (rc) return rc;
    if (!(flags & BSG_DEVICE_PTR)) {
        rc = ensure_pinned(*M, sizeof(float) * n2 * chunk);
        if (rc) return rc;
    }
    for (long b0 = 0; b0 < nimg; b0 += chunk) {
        const long cnt = std::min(chunk, nimg - b0);
        const float* src = images + b0 * n2;
        if (!(flags & BSG_DEVICE_PTR)) {
            memcpy(M->h_pin, src, sizeof(float) * n2 * cnt);
            MCK(cudaMemcpyAsync(M->d_real, M->h_pin, sizeof(float) * n2 * cnt, cudaMemcpyHostToDevice, s));
            src = M->d_real;
        }
        if (!(file_std > 0)) {
            image_stats_kernel<<<(unsigned)cnt, 256, 0, s>>>(src, (int)n2, M->d_scale + b0, M->d_shift + b0);
            MCK(cudaGetLastError());
        }
        to_complex_kernel<<<148 * 8, 256, 0, s>>>(src, M->d_work, n2 * cnt, n2, M->d_scale + b0, M->d_shift + b0);
        MCK(cudaGetLastError());
        MCK(fft2_forward(M->d_work, n, cnt, M->d_tw_img, s));
        img_cut_kernel<<<148 * 8, 256, 0, s>>>(M->d_work, n, D, cnt, M->d_spec + (size_t)b0 * D * D);
        MCK(cudaGetLastError());
        img_shells_kernel<<<(unsigned)cnt, 256, 0, s>>>(M->d_spec + (size_t)b0 * D * D, D, M->d_pix, npix,
                                                         M->d_shell_start, M->nshell, M->d_ictf + b0,
                                                         1.0 / M->real_img, M->d_ctf + (size_t)b0 * npix,
                                                         M->d_dsum + (size_t)b0 * M->nshell);
        MCK(cudaGetLastError());
        if (!(flags & BSG_DEVICE_PTR)) MCK(cudaStreamSynchronize(s));   // staging reuse
    }
    MCK(cudaStreamSynchronize(s));
    M->nimg = nimg;
    return BSG_OK;
}

extern "C" int bsg_match_prepared(bsg_match* h, long first, long count, float* out, int flags) {
    Match* M = reinterpret_cast<Match*>(h);
    if (!M || !out || first < 0 || count < 1 || first + count > M->nimg)
        return mfail(BSG_ERR_ARG, "bsg_match_prepared: bad range");
    MCK(cudaSetDevice(M->device));
    const size_t per = (size_t)M->D * M->D;
    MCK(cudaMemcpyAsync(out, M->d_spec + per * first, sizeof(float2) * per * count,
                        (flags & BSG_DEVICE_PTR) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, M->stream));
    MCK(cudaStreamSynchronize(M->stream));
    return BSG_OK;
}

extern "C" int bsg_match_score(bsg_match* h, const double* hyps, long nhyp, double* fom, double* cv, int flags) {
    Match* M = reinterpret_cast<Match*>(h);
    if (!M || !hyps || !fom || nhyp < 1) return mfail(BSG_ERR_ARG, "bsg_match_score: bad argument");
    if (!M->have_ref || M->nimg < 1) return mfail(BSG_ERR_STATE, "bsg_match_score: set the reference and images first");
    MCK(cudaSetDevice(M->device));
    int rc = ensure_hyps(*M, nhyp);
    if (rc) return rc;
    std::vector<MHyp> hv(nhyp);
    for (long i = 0; i < nhyp; ++i) {
        const double* r = hyps + BSG_MATCH_HYP_DOUBLES * i;
        const long img = (long)r[0];
        if (img < 0 || img >= M->nimg) return mfail(BSG_ERR_ARG, "bsg_match_score: hypothesis %ld names image %ld", i, img);
        memset(&hv[i], 0, sizeof(MHyp));
        hv[i].img = (int)img;
        match_view_rows(*M, r + 1, hv[i].m);
        // origin in pixels of the uncut image, scaled with the cut
        // (Bimage_fft.cpp:433), then phase_shift_to_origin's 2 pi o / size
        const double ox = M->cut_scale * r[10], oy = M->cut_scale * r[11];
        hv[i].sx = ox / M->D * 2 * M_PI;
        hv[i].sy = oy / M->D * 2 * M_PI;
    }
    std::vector<MHypG> groups;
    std::vector<long> slot;
    group_hypotheses(hv, groups, slot);
    const long ng = (long)groups.size();
    int rc2 = ensure_groups(*M, ng);
    if (rc2) return rc2;
    cudaStream_t s = M->stream;
    MCK(cudaMemcpyAsync(M->d_grp, groups.data(), sizeof(MHypG) * ng, cudaMemcpyHostToDevice, s));
    MCK(launch_fom(*M, M->d_grp, ng, M->d_gout, M->d_gout + ng * MAXORG, s, (flags & BSG_MATCH_SCORE_FP64) != 0,
                   nullptr, nullptr, (flags & BSG_MATCH_SCORE_DPR) != 0));
    std::vector<double> go(2 * ng * MAXORG);
    MCK(cudaMemcpyAsync(go.data(), M->d_gout, sizeof(double) * go.size(), cudaMemcpyDeviceToHost, s));
    MCK(cudaStreamSynchronize(s));
    for (long i = 0; i < nhyp; ++i) {
        fom[i] = go[slot[i]];
        if (cv) cv[i] = go[ng * MAXORG + slot[i]];
    }
    return BSG_OK;
}


extern "C" int bsg_match_project(bsg_match* h, const double* mats, long nviews, double resolution,
                                 const double* origins, const double* ctf, float* out, int flags) {
    Match* M = reinterpret_cast<Match*>(h);
    if (!M || !mats || !out || nviews < 1) return mfail(BSG_ERR_ARG, "bsg_match_project: bad argument");
    if (!M->have_ref) return mfail(BSG_ERR_STATE, "bsg_match_project: no reference set");
    MCK(cudaSetDevice(M->device));
    const int N = M->N;
    const double u = M->cfg.map_sampling, real = N * u;
    if (!(resolution > 0)) resolution = u;                 // Bimage_project.cpp:291
    // section pixels of the uncut map within the limit, reference order
    std::vector<MPix> px;
    const double inv = 1.0 / real, maxs2 = 1.0 / (resolution * resolution);
    for (int yy = 0; yy < N; ++yy)
        for (int xx = 0; xx < N; ++xx) {
            const int hh = sfreq(xx, N), kk = sfreq(yy, N);
            const double ix = hh * inv, iy = kk * inv;
            if (ix * ix + iy * iy > maxs2) continue;
            MPix q{};
            q.h = (short)hh; q.k = (short)kk; q.idx = yy * N + xx; q.insec = 1;
            px.push_back(q);
        }
    const long per = (long)N * N;
    const long chunk = std::max(1L, std::min<long>(nviews, (512L << 20) / (long)(sizeof(double2) * per)));
    int rc = ensure_work(*M, (size_t)per * chunk);
    if (rc) return rc;
    cudaStream_t s = M->stream;
    MPix* d_px = nullptr;
    MHyp* d_v = nullptr;
    ImgCtf* d_c = nullptr;
    float* d_o = nullptr;
    cudaError_t e = cudaMalloc(&d_px, sizeof(MPix) * std::max<size_t>(1, px.size()));
    if (e == cudaSuccess) e = cudaMalloc(&d_v, sizeof(MHyp) * chunk);
    if (e == cudaSuccess && ctf) e = cudaMalloc(&d_c, sizeof(ImgCtf) * chunk);
    if (e == cudaSuccess && !(flags & BSG_DEVICE_PTR)) e = cudaMalloc(&d_o, sizeof(float) * per * chunk);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_px, px.data(), sizeof(MPix) * px.size(), cudaMemcpyHostToDevice, s);
    std::vector<MHyp> hv(chunk);
    std::vector<ImgCtf> hc(ctf ? chunk : 0);
    for (long v0 = 0; e == cudaSuccess && v0 < nviews; v0 += chunk) {
        const long cnt = std::min(chunk, nviews - v0);
        for (long i = 0; i < cnt; ++i) {
            memset(&hv[i], 0, sizeof(MHyp));
            memcpy(hv[i].m, mats + 9 * (v0 + i), sizeof(double) * 9);
            const double ox = origins ? origins[2 * (v0 + i)] : (double)(N / 2);
            const double oy = origins ? origins[2 * (v0 + i) + 1] : (double)(N / 2);
            hv[i].sx = -2 * M_PI * ox / N;
            hv[i].sy = -2 * M_PI * oy / N;
            if (ctf) {
                const double* r = ctf + BSG_MATCH_CTF_DOUBLES * (v0 + i);
                memset(&hc[i], 0, sizeof(ImgCtf));
                for (int j = 0; j < 5; ++j) hc[i].c[j] = r[1 + j];
                const int f = (int)r[6];
                const double t2 = -M_PI * electron_lambda(r[0]);
                hc[i].apply = (f & BSG_MATCH_APPLY_CTF) && t2 != 0 && r[2] / t2 >= 1 ? 1 : 0;
                hc[i].invert = (f & BSG_MATCH_INVERT) ? 1 : 0;
            }
        }
        e = cudaMemcpyAsync(d_v, hv.data(), sizeof(MHyp) * cnt, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && ctf) e = cudaMemcpyAsync(d_c, hc.data(), sizeof(ImgCtf) * cnt, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(M->d_work, 0, sizeof(double2) * per * cnt, s);
        if (e == cudaSuccess) {
            ProjArgs a{};
            a.vol = M->d_full; a.N = N; a.wd = M->wd; a.lut = M->d_lut; a.pix = d_px; a.npix = (int)px.size();
            a.views = d_v; a.ctf = ctf ? d_c : nullptr; a.inv = inv; a.real = real; a.fs = 1.0 / (N * M->cfg.pixel);
            a.out = M->d_work;
            project_kernel<<<(unsigned)cnt, 256, 0, s>>>(a);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = fft2_forward(M->d_work, N, cnt, M->d_tw_map, s);
        float* dst = (flags & BSG_DEVICE_PTR) ? out + per * v0 : d_o;
        if (e == cudaSuccess) {
            proj_real_kernel<<<148 * 8, 256, 0, s>>>(M->d_work, per * cnt, 1.0 / N, dst);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && !(flags & BSG_DEVICE_PTR))
            e = cudaMemcpyAsync(out + per * v0, d_o, sizeof(float) * per * cnt, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    cudaFree(d_px); cudaFree(d_v); cudaFree(d_c); cudaFree(d_o);
    if (e != cudaSuccess) return mfail(BSG_ERR_CUDA, "bsg_match_project: %s", cudaGetErrorString(e));
    return BSG_OK;
}

// img_recip_space_fom's shell weights (mg_refine.cpp:702-704): w[j] = 1,
// replaced by the caller's weight[j] where that is non-zero, for shells j
// < n; their sums over the FRC and cross-validation shells are formed in
// shell order as the reference's loops form them (:757-767).
extern "C" int bsg_match_set_shell_weights(bsg_match* h, const double* w, int n) {
    Match* M = reinterpret_cast<Match*>(h);
    if (!M || n < 0 || (n > 0 && !w)) return match_fail(BSG_ERR_ARG, "bsg_match_set_shell_weights: bad argument");
    std::vector<double> ws(M->nshell, 1.0);
    for (int j = 0; j < n && j < M->nshell; ++j) {
        if (!std::isfinite(w[j])) return match_fail(BSG_ERR_ARG, "bsg_match_set_shell_weights: weight %d not finite", j);
        if (w[j] != 0.0) ws[j] = w[j];
    }
    double wf = 0, wc = 0;
    for (int j = 0; j < M->nf; ++j) wf += ws[j];
    for (int j = M->cv0; j < M->cv1; ++j) wc += ws[j];
    cudaError_t e = cudaSetDevice(M->device);
    if (e == cudaSuccess) e = cudaStreamSynchronize(M->stream);
    if (e == cudaSuccess) e = cudaMemcpy(M->d_wshell, ws.data(), sizeof(double) * ws.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return match_fail(BSG_ERR_CUDA, "bsg_match_set_shell_weights: %s", cudaGetErrorString(e));
    M->h_wshell.swap(ws);
    M->wf = wf;
    M->wc = wc;
    return BSG_OK;
}
