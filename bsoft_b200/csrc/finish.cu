// finish.cu - from accumulated central sections to the real-space map.
// Reference steps (bsoft/src):
//   sum of partial maps + weigh   mg/mg_reconstruct.cpp:306-331,
//                                 img/Bimage_reconstruct.cpp:486-515
//   SNR (FOM) map                 img/Bimage_reconstruct.cpp:610-634
//   phase_shift_to_center         img/Bimage_complex.cpp:545-552 (= (-1)^(h+k+l))
//   fft_back (1/sqrt(N^3)), real  img/Bimage.h:903-908, Bimage_complex.cpp:170-186
//   filter_sinc (trilinear)       img/Bimage_filter.cpp:484-509
//
// weigh_kernel is one pass over the voxels; the 3-D inverse transform is
// three passes of warp FFTs (x lines contiguous; y and z lines staged 16 at
// a time through shared memory so global accesses stay coalesced).  The last
// pass writes only the real part, scaled and sinc-weighted.
#include "context.cuh"
#include "fft_dev.cuh"

#include <math.h>

namespace bsg {

#define SMALLFLOAT_F 1e-30f

struct WeighArgs {
    const double2* v0; const double* w0; const double* p0; const double* q0;
    const double2* v1; const double* w1; const double* p1; const double* q1;   // second half or null
    float2* out;      // weighed, centre-shifted complex volume
    float* fom;       // optional SNR map
    int N;
    int zsplit;       // > 0: half-space accumulators (insert.cu walk_edges)
    const double2* e0; const double* ew0;   // their unpaired pixels' sums below zsplit
    const double2* e1; const double* ew1;
};

// Index of the voxel at minus the frequency of voxel (x, y, z) (wrap-around).
__device__ __forceinline__ size_t mirror_index(size_t x, size_t y, size_t z, size_t N) {
    return ((((N - z) % N) * N + (N - y) % N) * N + (N - x) % N);
}

// The map's sums at voxel i.  Half-space accumulators (zsplit > 0) hold
// the paired pixels' sums P below zsplit, with the unpaired pixels' sums U
// there in (e, ew), and U alone at and above zsplit: the map is P(v) + U(v)
// below the split and conj(P(-v)) + U(v) above it.
__device__ __forceinline__ void read_sums(const double2* vol, const double* w, const double2* e, const double* ew,
                                          size_t i, size_t N, int zsplit, double2& v, double& wt) {
    v = vol[i];
    wt = w[i];
    if (zsplit <= 0) return;
    const size_t z = i / (N * N);
    if (z >= (size_t)zsplit) {
        const size_t m = mirror_index(i % N, (i / N) % N, z, N);
        const double2 u = vol[m];
        v.x += u.x;
        v.y -= u.y;
        wt += w[m];
    } else {
        const double2 u = e[i];
        v.x += u.x;
        v.y += u.y;
        wt += ew[i];
    }
}

__global__ void weigh_kernel(WeighArgs a) {
    const size_t N = a.N, N3 = N * N * N;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N3; i += (size_t)gridDim.x * blockDim.x) {
        double2 v;
        double w;
        read_sums(a.v0, a.w0, a.e0, a.ew0, i, N, a.zsplit, v, w);
        double p = a.p0 ? a.p0[i] : 0.0, q = a.q0 ? a.q0[i] : 0.0;
        if (a.v1) {
            double2 v1;
            double w1;
            read_sums(a.v1, a.w1, a.e1, a.ew1, i, N, a.zsplit, v1, w1);
            v.x += v1.x; v.y += v1.y;
            w += w1;
            if (a.p1) { p += a.p1[i]; q += a.q1[i]; }
        }
        float2 F = make_float2(0.f, 0.f);
        if (w > 1e-30) {
            q = w - q / w;
            F = make_float2((float)(v.x / w), (float)(v.y / w));
            if (q > 1.0) p /= q;
            else if (w > 1.0) p /= w;
            if (p < 0.0) p = 0.0;
        } else {
            p = 0.0;
            w = q = 1e-30;
        }
        if (a.fom) {
            // fspace_reconstruction_snr on the weighed channels
            const double signal = (double)F.x * F.x + (double)F.y * F.y;
            double noise = p - signal;
            if (noise < signal) noise = signal;
            float f = 0.f;
            if (w > 1.0 && signal > 1e-30 && noise > 1e-30) f = (float)((w * signal - p) / noise);
            a.fom[i] = (i == 0) ? 1.f : f;
        }
        // (-1)^(h+k+l): signed and unsigned indices share parity for even N
        const size_t x = i % N, y = (i / N) % N, z = i / (N * N);
        if ((x + y + z) & 1) { F.x = -F.x; F.y = -F.y; }
        a.out[i] = F;
    }
}

// Radix plan of a map edge: power of two -> in-place radix-2/4 DIT on
// bit-reversed input; otherwise mixed-radix Stockham (needs N scratch).
struct Radix {
    int mixed;
    int nstage;
    int r[16];
};

// x-lines: one warp per line, 8 lines per CTA
constexpr int XW = 8;
__global__ void __launch_bounds__(XW * 32) fft_x_kernel(float2* data, const float2* tw, int N, int logN, Radix rp) {
    extern __shared__ float2 sm[];
    float2* stw = sm;                              // N roots
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = rp.mixed ? 2 * N : N;
    float2* buf = sm + N + warp * per;
    for (int i = threadIdx.x; i < N; i += blockDim.x) stw[i] = tw[i];
    __syncthreads();
    const size_t line = (size_t)blockIdx.x * XW + warp;
    if (line >= (size_t)N * N) return;
    float2* p = data + line * N;
    if (rp.mixed) {
        for (int i = lane; i < N; i += 32) buf[i] = p[i];
        __syncwarp();
        warp_fft_mixed<true>(buf, buf + N, N, rp.r, rp.nstage, stw);
    } else {
        for (int i = lane; i < N; i += 32) buf[bitrev(i, logN)] = p[i];
        __syncwarp();
        warp_fft<true>(buf, N, logN, stw);
    }
    for (int i = lane; i < N; i += 32) p[i] = buf[i];
}

// strided lines (y: stride N, z: stride N*N): 16 adjacent x per CTA.
constexpr int SW = 16;
struct StridedArgs {
    float2* data;
    const float2* tw;
    int N, logN;
    int axis;          // 1 = y, 2 = z
    float* real_out;   // when set: write the real part * scale (* sinc) instead
    float scale;
    int sinc;
    Radix rp;
};

__global__ void __launch_bounds__(SW * 32) fft_strided_kernel(StridedArgs a) {
    extern __shared__ float2 sm[];
    const int N = a.N;
    const int per = a.rp.mixed ? 2 * N : N;
    float2* stw = sm;                 // N roots
    float2* tile = sm + N;            // SW lines of `per`
    for (int i = threadIdx.x; i < N; i += blockDim.x) stw[i] = a.tw[i];
    // blockIdx.x: x-chunk, blockIdx.y: the remaining coordinate (z for axis y, y for axis z)
    const int x0 = blockIdx.x * SW;
    const int other = blockIdx.y;
    const size_t stride = a.axis == 1 ? (size_t)N : (size_t)N * N;
    const size_t obase = a.axis == 1 ? (size_t)other * N * N : (size_t)other * N;
    for (int i = threadIdx.x; i < SW * N; i += blockDim.x) {
        const int c = i % SW, j = i / SW;
        const int x = x0 + c;
        float2 v = make_float2(0.f, 0.f);
        if (x < N) v = a.data[obase + (size_t)j * stride + x];
        tile[c * per + (a.rp.mixed ? j : (int)bitrev(j, a.logN))] = v;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    if (x0 + warp < N) {
        if (a.rp.mixed) warp_fft_mixed<true>(tile + warp * per, tile + warp * per + N, N, a.rp.r, a.rp.nstage, stw);
        else warp_fft<true>(tile + warp * N, N, a.logN, stw);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < SW * N; i += blockDim.x) {
        const int c = i % SW, j = i / SW;
        const int x = x0 + c;
        if (x >= N) continue;
        const size_t idx = obase + (size_t)j * stride + x;
        const float2 v = tile[c * per + j];
        if (a.real_out) {
            float r = v.x * a.scale;
            if (a.sinc) {
                // filter_sinc: r = pi |d|, d = (index - N/2) / N, weight (r / sin r)^2
                const int yy = a.axis == 1 ? j : other;
                const int zz = a.axis == 1 ? other : j;
                const double o = (double)(N / 2);
                const double dx = (x - o) / N, dy = (yy - o) / N, dz = (zz - o) / N;
                const double rr = 3.14159265358979323846 * sqrt(dx * dx + dy * dy + dz * dz);
                if (rr != 0.0) { const double w = rr / sin(rr); r = (float)(w * w * r); }
            }
            a.real_out[idx] = r;
        } else {
            a.data[idx] = v;
        }
    }
}

cudaError_t launch_weigh(const Context& c, int imap, cudaStream_t s) {
    WeighArgs a{};
    const int N = c.g.map;
    int h0 = 0;
    bool both = false;
    if (c.nhalves == 2) {
        if (imap == 0) both = true;
        else h0 = imap - 1;
    }
    a.v0 = c.d_vol[h0]; a.w0 = c.d_w[h0]; a.p0 = c.d_pow[h0]; a.q0 = c.d_w2[h0];
    if (both) { a.v1 = c.d_vol[1]; a.w1 = c.d_w[1]; a.p1 = c.d_pow[1]; a.q1 = c.d_w2[1]; }
    a.out = c.d_work;
    a.fom = c.g.fom ? c.d_fom : nullptr;
    a.N = N;
    a.zsplit = c.zsplit;
    a.e0 = c.d_evol[h0]; a.ew0 = c.d_ew[h0];
    if (both) { a.e1 = c.d_evol[1]; a.ew1 = c.d_ew[1]; }
    weigh_kernel<<<148 * 8, 256, 0, s>>>(a);
    return cudaGetLastError();
}

static Radix radix_plan(int N) {
    Radix rp{};
    rp.mixed = (N & (N - 1)) != 0;
    if (rp.mixed) rp.nstage = factor_radices(N, rp.r);
    return rp;
}

cudaError_t launch_ifft3(const Context& c, float2* vol, float* real_out, bool sinc, cudaStream_t s) {
    const int N = c.g.map, logN = ilog2i(N);
    const Radix rp = radix_plan(N);
    const size_t per = rp.mixed ? 2 * (size_t)N : (size_t)N;
    {
        const size_t lines = (size_t)N * N;
        const size_t smem = sizeof(float2) * ((size_t)N + XW * per);
        fft_x_kernel<<<(unsigned)((lines + XW - 1) / XW), XW * 32, smem, s>>>(vol, c.d_twmap, N, logN, rp);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    const size_t smem = sizeof(float2) * ((size_t)N + SW * per);
    dim3 grid((N + SW - 1) / SW, N);
    StridedArgs a{};
    a.data = vol; a.tw = c.d_twmap; a.N = N; a.logN = logN; a.rp = rp;
    a.axis = 1;
    fft_strided_kernel<<<grid, SW * 32, smem, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    a.axis = 2;
    a.real_out = real_out;
    a.scale = (float)(1.0 / sqrt((double)N * N * N));
    a.sinc = sinc ? 1 : 0;
    fft_strided_kernel<<<grid, SW * 32, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_finish(const Context& c, int imap, float* map_out, float* fom_out, bool sinc, cudaStream_t s) {
    (void)fom_out;
    cudaError_t e = launch_weigh(c, imap, s);
    if (e != cudaSuccess) return e;
    return launch_ifft3(c, c.d_work, map_out, sinc, s);
}

// Weighed (not centre-shifted) half map for the FSC: reuse weigh_kernel and
// undo nothing - the FSC only uses products F1 conj(F2) and |F|^2, which the
// (-1)^(h+k+l) factor leaves unchanged.
cudaError_t launch_weigh_into(const Context& c, int imap, float2* out, cudaStream_t s) {
    WeighArgs a{};
    const int h0 = imap - 1;
    a.v0 = c.d_vol[h0]; a.w0 = c.d_w[h0]; a.p0 = nullptr; a.q0 = nullptr;
    a.out = out; a.fom = nullptr; a.N = c.g.map;
    a.zsplit = c.zsplit;
    a.e0 = c.d_evol[h0]; a.ew0 = c.d_ew[h0];
    weigh_kernel<<<148 * 8, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// Half-space accumulators -> the map's sums (read_sums), into (dv, dw); in
// place (dv == vol) too: the voxels at and above zsplit are written first,
// from the paired sums below it, then (e, ew) is added below it.
__global__ void map_sums_upper_kernel(double2* dv, double* dw, const double2* vol, const double* w, int N,
                                      int zsplit) {
    const size_t n = N, n2 = n * n, first = (size_t)zsplit * n2, N3 = n2 * n;
    for (size_t i = first + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N3;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t m = mirror_index(i % n, (i / n) % n, i / n2, n);
        const double2 u = vol[m];
        double2 v = vol[i];
        v.x += u.x;
        v.y -= u.y;
        dv[i] = v;
        dw[i] = w[i] + w[m];
    }
}

__global__ void map_sums_lower_kernel(double2* dv, double* dw, const double2* vol, const double* w,
                                      const double2* e, const double* ew, size_t count) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        double2 v = vol[i];
        const double2 u = e[i];
        v.x += u.x;
        v.y += u.y;
        dv[i] = v;
        dw[i] = w[i] + ew[i];
    }
}

cudaError_t launch_map_sums(double2* dv, double* dw, const double2* vol, const double* w, const double2* e,
                            const double* ew, int N, int zsplit, cudaStream_t s) {
    if (zsplit <= 0) return cudaSuccess;
    map_sums_upper_kernel<<<148 * 8, 256, 0, s>>>(dv, dw, vol, w, N, zsplit);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    map_sums_lower_kernel<<<148 * 8, 256, 0, s>>>(dv, dw, vol, w, e, ew, (size_t)zsplit * N * N);
    return cudaGetLastError();
}

// FSC partial sums as Bimage::fsc(Bimage*) forms them
// (bsoft/src/img/Bimage_resolution.cpp:330-406 with fspace_radial_power,
// Bimage_fspace.cpp:848-958): radius = real * |index / real| (wrapped at
// (N-1)/2), a voxel adds (1 - f) to shell floor(radius) and f to the next,
// only voxels with floor(radius) < maxrad count.  One CTA per z-plane;
// thread r accumulates shell r of that plane in a fixed order (rows, then
// |h|, then sign), fsc_reduce sums the planes in order - deterministic,
// FP64 throughout.
__device__ __forceinline__ double fsc_radius(int h, int k, int l, double real) {
    const double fs = 1.0 / real;
    double rx = h * fs, ry = k * fs, rz = l * fs;
    rx *= rx; ry *= ry; rz *= rz;
    return real * sqrt(rx + ry + rz);
}

__global__ void fsc_plane_kernel(const float2* v1, const float2* v2, int N, int nshell, int maxrad, double real,
                                 double* part) {
    const int z = blockIdx.x;
    const int l = sfreq(z, N);
    for (int r = threadIdx.x; r < nshell; r += blockDim.x) {
        double num = 0, d1 = 0, d2 = 0;
        if (r < maxrad) {
            // voxels with floor(radius) in {r - 1, r}: radius in [r - 1, r + 1)
            const double rlo = r - 1.5, rhi = r + 1.5;      // index-space bounds with margin
            for (int y = 0; y < N; ++y) {
                const int k = sfreq(y, N);
                const double kl = (double)k * k + (double)l * l;
                if (kl >= rhi * rhi) continue;
                const int hlo = (rlo > 0 && rlo * rlo > kl) ? (int)floor(sqrt(rlo * rlo - kl)) : 0;
                const int hhi = min(N / 2, (int)ceil(sqrt(rhi * rhi - kl)));
                for (int hh = hlo; hh <= hhi; ++hh) {
                    for (int sgn = 0; sgn < 2; ++sgn) {
                        if (sgn && (hh == 0 || hh == N / 2)) continue;
                        const int x = sgn ? (N - hh) % N : hh;
                        const int h = sfreq(x, N);
                        const double rad = fsc_radius(h, k, l, real);
                        const int ir = (int)rad;
                        if (ir >= maxrad) continue;
                        double w;
                        if (ir == r) w = 1.0 - (rad - ir);
                        else if (ir + 1 == r) w = rad - ir;
                        else continue;
                        const size_t i = ((size_t)z * N + y) * N + x;
                        const float2 a = v1[i], b = v2[i];
                        num += w * ((double)a.x * b.x + (double)a.y * b.y);
                        d1 += w * ((double)a.x * a.x + (double)a.y * a.y);
                        d2 += w * ((double)b.x * b.x + (double)b.y * b.y);
                    }
                }
            }
        }
        double* o = part + ((size_t)z * nshell + r) * 3;
        o[0] = num; o[1] = d1; o[2] = d2;
    }
}

// FSC[0] = 1 (the reference sets it), FSC[r] = num / sqrt(d1 d2), 0 where
// not finite or beyond maxrad
__global__ void fsc_reduce_kernel(const double* part, int N, int nshell, int maxrad, double* fsc) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nshell) return;
    double num = 0, d1 = 0, d2 = 0;
    for (int z = 0; z < N; ++z) {
        const double* o = part + ((size_t)z * nshell + r) * 3;
        num += o[0]; d1 += o[1]; d2 += o[2];
    }
    double v = 0;
    if (r == 0) v = 1;
    else if (r < maxrad) {
        v = num / sqrt(d1 * d2);
        if (!isfinite(v)) v = 0;
    }
    fsc[r] = v;
}

cudaError_t launch_fsc(const Context& c, int nshell, double* out_dev, cudaStream_t s) {
    cudaError_t e = launch_weigh_into(c, 1, c.d_half_weighed[0], s);
    if (e != cudaSuccess) return e;
    e = launch_weigh_into(c, 2, c.d_half_weighed[1], s);
    if (e != cudaSuccess) return e;
    // fspace_maximum_radius (Bimage_fspace.cpp:26-38), sampling ratio 1
    const double real = c.g.map * c.cfg.map_sampling;
    const int maxrad = c.cfg.hi_res > 0.1 ? (int)(long)(real / c.cfg.hi_res) : c.g.map / 2;
    fsc_plane_kernel<<<c.g.map, 128, 0, s>>>(c.d_half_weighed[0], c.d_half_weighed[1], c.g.map, nshell, maxrad, real,
                                             c.d_fsc);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    fsc_reduce_kernel<<<(nshell + 127) / 128, 128, 0, s>>>(c.d_fsc, c.g.map, nshell, maxrad, out_dev);
    return cudaGetLastError();
}

cudaError_t prepare_finish_attributes() {
    cudaError_t e = cudaFuncSetAttribute(fft_x_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(sizeof(float2) * (512 + XW * 1024)));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(fft_strided_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(float2) * (512 + SW * 1024)));
}

}  // namespace bsg
