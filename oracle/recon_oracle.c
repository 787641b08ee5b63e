/*
 * recon_oracle.c - FP64 restatement of the reference's Fourier-space
 * reconstruction path (TEST INFRASTRUCTURE ONLY; see oracle.h).
 *
 * Per particle (bsoft/src/mg/mg_reconstruct.cpp:143-229):
 *   background      Bimage::calculate_background  Bimage_background.cpp:27-80
 *   pad             Bimage::pad -> resize          Bimage_resize.cpp:28-110, 347-357
 *   forward FFT     Bimage::fft(plan, 1)           Bimage_fft.cpp:176-234 (1/sqrt(ft^2))
 *   origin shift    Bimage::phase_shift_to_origin  Bimage_complex.cpp:490-534
 *   CTF             img_ctf_apply_complex          mg_ctf.cpp:661-676, 46-122; ctf.h:321-351
 *   insertion       Bimage::fspace_pack_2D         Bimage_reconstruct.cpp:112-174
 *                   Bimage::fspace_2D_interpolate  Bimage_reconstruct.cpp:25-88
 * Per map (mg_reconstruct.cpp:266-361, breconstruct.cpp:328-359):
 *   weigh           fspace_reconstruction_weigh    Bimage_reconstruct.cpp:486-515
 *   centre shift    phase_shift_to_center          Bimage_complex.cpp:545-552, 443-479
 *   inverse FFT     fft_back                       Bimage.h:903-908, Bimage_complex.cpp:170-186
 *   sinc            filter_sinc                    Bimage_filter.cpp:484-509
 */
#include "oracle.h"
#include "fft64.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SMALLFLOAT 1e-30

/* Bimage::calculate_background(nn, 0): mean of pixels outside the ellipse of
 * half-axes (x/2, y/2) (integer halves) around the image origin. */
static double background(const float* img, int n, const double* c)
{
    long h = n / 2;
    double sum = 0.0;
    long cnt = 0;
    for (int y = 0; y < n; ++y) {
        double y2 = (y - c[1]) / (double)h; y2 *= y2;
        for (int x = 0; x < n; ++x) {
            double x2 = (x - c[0]) / (double)h; x2 *= x2;
            if (x2 + y2 - 1 > 0) { sum += img[(long)y * n + x]; ++cnt; }
        }
    }
    return cnt ? sum / cnt : 0.0;
}

/* signed frequency index as Bimage wraps it: i > (size-1)/2 -> i - size */
static inline long sfreq(long i, long size) { return i > (size - 1) / 2 ? i - size : i; }

int orc_particle_transform(const orc_recon_cfg* cfg, const float* image,
                           const orc_particle* p, double* out)
{
    const int n = cfg->n, ft = cfg->ft;
    const long ft2 = (long)ft * ft;
    double bkg = background(image, n, p->bkg_center);
    /* pad into the ft x ft corner, fill = background (translate 0) */
    for (long i = 0; i < ft2; ++i) { out[2*i] = bkg; out[2*i+1] = 0.0; }
    if (ft < n) return -1;
    for (int y = 0; y < n; ++y)
        for (int x = 0; x < n; ++x)
            out[2*((long)y*ft + x)] = image[(long)y*n + x];
    long dims[2] = {ft, ft};
    if (fft64_nd(2, dims, out, -1)) return -2;
    double sc = sqrt(1.0 / (double)ft2);
    for (long i = 0; i < 2*ft2; ++i) out[i] *= sc;
    /* phase shift to origin: phi = h*2pi*ox/ft + k*2pi*oy/ft */
    double shx = p->origin[0] / ft * 2 * M_PI, shy = p->origin[1] / ft * 2 * M_PI;
    for (long yy = 0; yy < ft; ++yy) {
        long k = sfreq(yy, ft);
        for (long xx = 0; xx < ft; ++xx) {
            long h = sfreq(xx, ft);
            double phi = h * shx + k * shy;
            double c = cos(phi), s = sin(phi);
            double* v = out + 2*(yy*ft + xx);
            double re = v[0]*c - v[1]*s, im = v[0]*s + v[1]*c;
            v[0] = re; v[1] = im;
        }
    }
    if (cfg->ctf_action) {
        /* img_ctf_calculate(cp, flip, wiener, size, sam, 0, hires) */
        double hires = cfg->hi_res > 0 ? cfg->hi_res : p->pixel;
        double shi2 = 1.0 / (hires * hires);
        double fs = 1.0 / (ft * p->pixel);
        int flip = cfg->ctf_action == 1;
        double wiener = cfg->wiener;
        for (long yy = 0; yy < ft; ++yy) {
            double sy = sfreq(yy, ft) * fs;
            for (long xx = 0; xx < ft; ++xx) {
                double sx = sfreq(xx, ft) * fs;
                double s2 = sx*sx + sy*sy;
                double* v = out + 2*(yy*ft + xx);
                if (!(s2 >= 0 && s2 <= shi2)) { v[0] = v[1] = 0.0; continue; }
                double a = atan2(sy, sx);
                const double* c = p->ctf;
                double chi = c[0] + c[3]*s2*sin(2*a) + c[1]*s2 + c[2]*s2*cos(2*a) + c[4]*s2*s2;
                double w = sin(chi);
                if (flip) w = (w < 0) ? -1.0 : 1.0;
                else if (wiener) w = (wiener + 1) * w / (w*w + wiener);
                double s = sqrt(s2);
                double psi = c[6]*s*sin(a) + c[5]*s*cos(a);
                double cr = cos(psi) * w, ci = -sin(psi) * w;   /* conj(odd) * w */
                double re = v[0]*cr - v[1]*ci, im = v[0]*ci + v[1]*cr;
                v[0] = re; v[1] = im;
            }
        }
    }
    return 0;
}

static inline long wrap1(long j, long N) { if (j < 0) j += N; else if (j >= N) j -= N; return j; }

static void interpolate(long N, const double* cv, const double* m, double pw, int interp,
                        double* vol, double* weight, double* power, double* weight2)
{
    double pcv = cv[0]*cv[0] + cv[1]*cv[1];
    if (interp < 2) {
        long c[3];
        double w = pw;
        for (int i = 0; i < 3; ++i) c[i] = (long)floor(m[i] + 0.5);
        if (interp == 1) {
            double d0 = m[0]-c[0], d1 = m[1]-c[1], d2 = m[2]-c[2];
            w *= 1 - sqrt(d0*d0 + d1*d1 + d2*d2);
        }
        if (w > 0) {
            for (int i = 0; i < 3; ++i) { while (c[i] < 0) c[i] += N; while (c[i] >= N) c[i] -= N; }
            long j = (c[2]*N + c[1])*N + c[0];
            vol[2*j] += cv[0]*w; vol[2*j+1] += cv[1]*w;
            weight[j] += w;
            if (power) power[j] += w*pcv;
            if (weight2) weight2[j] += w*w;
        }
        return;
    }
    long c0 = (long)floor(m[0]), c1 = (long)floor(m[1]), c2 = (long)floor(m[2]);
    double f0 = m[0]-c0, f1 = m[1]-c1, f2 = m[2]-c2;
    for (int zz = 0; zz < 2; ++zz) {
        long jz = wrap1(c2 + zz, N);
        double dz = zz ? f2 : 1 - f2;
        for (int yy = 0; yy < 2; ++yy) {
            long jy = wrap1(c1 + yy, N);
            double dy = yy ? f1 : 1 - f1;
            for (int xx = 0; xx < 2; ++xx) {
                long jx = wrap1(c0 + xx, N);
                double dx = xx ? f0 : 1 - f0;
                double w = dx*dy*dz*pw;
                long j = (jz*N + jy)*N + jx;
                vol[2*j] += cv[0]*w; vol[2*j+1] += cv[1]*w;
                weight[j] += w;
                if (power) power[j] += w*pcv;
                if (weight2) weight2[j] += w*w;
            }
        }
    }
}

int orc_insert(const orc_recon_cfg* cfg, const float* images, const orc_particle* parts,
               long nparts, double* vol, double* weight, double* power, double* weight2)
{
    const int n = cfg->n, ft = cfg->ft;
    const long N = cfg->map;
    double* F = (double*)malloc(sizeof(double) * 2 * (long)ft * ft);
    if (!F) return -1;
    double hi_res = cfg->hi_res < 0.5 ? 0.5 : cfg->hi_res;
    double maxs2 = 1.0 / hi_res; maxs2 *= maxs2;
    double mins2 = 0.0;
    double mscale = N * cfg->map_sampling;
    for (long ip = 0; ip < nparts; ++ip) {
        const orc_particle* p = parts + ip;
        int rc = orc_particle_transform(cfg, images + ip * (long)n * n, p, F);
        if (rc) { free(F); return rc; }
        double pw = p->weight;
        double pad_ratio = ft * 1.0 / n;
        if (pad_ratio > 1) pw /= pad_ratio * pad_ratio * 0.6;
        double inv = p->scale / (ft * p->pixel);
        const double* R = p->mat;
        for (long yy = 0; yy < ft; ++yy) {
            double sy = sfreq(yy, ft) * inv;
            for (long xx = 0; xx < ft; ++xx) {
                double sx = sfreq(xx, ft) * inv;
                double s2 = sx*sx + sy*sy;
                if (s2 < mins2 || s2 > maxs2) continue;
                double w = pw;
                double d = (maxs2 - s2) * mscale;
                if (d < 1) w *= sqrt(d);
                double m[3];
                if (p->ewald) {
                    /* Ewald sphere (Bimage_reconstruct.cpp:157-168): s_z =
                     * +-(lambda/2) s2, m = (R s) mscale, inserted twice */
                    const double sz = p->ewald / 2 * s2;
                    for (int i = 0; i < 3; ++i) m[i] = (R[3*i]*sx + R[3*i+1]*sy + R[3*i+2]*sz) * mscale;
                    interpolate(N, F + 2*(yy*ft + xx), m, w, cfg->interp, vol, weight, power, weight2);
                    for (int i = 0; i < 3; ++i) m[i] = (R[3*i]*sx + R[3*i+1]*sy + R[3*i+2]*(-sz)) * mscale;
                    interpolate(N, F + 2*(yy*ft + xx), m, w, cfg->interp, vol, weight, power, weight2);
                    continue;
                }
                for (int i = 0; i < 3; ++i) m[i] = (R[3*i]*sx + R[3*i+1]*sy) * mscale;
                interpolate(N, F + 2*(yy*ft + xx), m, w, cfg->interp, vol, weight, power, weight2);
            }
        }
    }
    free(F);
    return 0;
}

long orc_finish(const orc_recon_cfg* cfg, double* vol, double* weight, double* power,
                double* weight2, double* map_out, int sinc)
{
    const long N = cfg->map, N3 = N * N * N;
    long cov = 0;
    for (long i = 0; i < N3; ++i) {
        if (weight[i] > SMALLFLOAT) {
            if (weight2) weight2[i] = weight[i] - weight2[i] / weight[i];
            vol[2*i] /= weight[i]; vol[2*i+1] /= weight[i];
            if (power && weight2) {
                if (weight2[i] > 1) power[i] /= weight2[i];
                else if (weight[i] > 1) power[i] /= weight[i];
                if (power[i] < 0) power[i] = 0;
            }
            ++cov;
        } else {
            vol[2*i] = vol[2*i+1] = 0.0;
            if (power) power[i] = 0;
            weight[i] = SMALLFLOAT;
            if (weight2) weight2[i] = SMALLFLOAT;
        }
    }
    if (power) power[0] = 1;
    /* phase shift to centre: phi = -2pi (h + k + l) * (N/2)/N */
    double t = -2 * M_PI * (double)(N / 2) / (double)N;
    for (long z = 0; z < N; ++z) {
        long l = sfreq(z, N);
        for (long y = 0; y < N; ++y) {
            long k = sfreq(y, N);
            for (long x = 0; x < N; ++x) {
                long h = sfreq(x, N);
                double phi = h*t + k*t + l*t;
                double c = cos(phi), s = sin(phi);
                double* v = vol + 2*((z*N + y)*N + x);
                double re = v[0]*c - v[1]*s, im = v[0]*s + v[1]*c;
                v[0] = re; v[1] = im;
            }
        }
    }
    double* tmp = (double*)malloc(sizeof(double) * 2 * N3);
    if (!tmp) return -1;
    memcpy(tmp, vol, sizeof(double) * 2 * N3);
    long dims[3] = {N, N, N};
    fft64_nd(3, dims, tmp, +1);
    double sc = sqrt(1.0 / (double)N3);
    for (long i = 0; i < N3; ++i) map_out[i] = tmp[2*i] * sc;
    free(tmp);
    if (sinc) {
        double o = (double)(N / 2);
        for (long z = 0, i = 0; z < N; ++z) {
            double d2 = (-o + z) / N;
            for (long y = 0; y < N; ++y) {
                double d1 = (-o + y) / N;
                for (long x = 0; x < N; ++x, ++i) {
                    double d0 = (-o + x) / N;
                    double r = M_PI * sqrt(d0*d0 + d1*d1 + d2*d2);
                    if (r) { double w = r / sin(r); map_out[i] *= w * w; }
                }
            }
        }
    }
    return cov;
}

int orc_fsc(int N, const double* v1, const double* v2, double real_size, double hi_res, int nshell, double* fsc)
{
    /* Bimage::fsc(Bimage*) (bsoft/src/img/Bimage_resolution.cpp:330-406)
     * with fspace_radial_power (bsoft/src/img/Bimage_fspace.cpp:848-958) on
     * two complex N^3 transforms (standard layout), sampling ratio 1:
     * radius = real_size * |s|, s = index / real_size (wrapped at (N-1)/2);
     * a voxel adds (1 - f) to shell floor(radius) and f to the next, f the
     * fraction, shells below maxrad = (long)(real_size / hi_res)
     * (fspace_maximum_radius, hi_res > 0.1); FSC[0] = 1, FSC[i] =
     * sum Re(F1 F2*) / sqrt(sum |F1|^2 sum |F2|^2) per shell (the shell
     * averages' common normalisation cancels), 0 where not finite.
     * Returns maxrad. */
    long maxrad = hi_res > 0.1 ? (long)(real_size / hi_res) : (long)(N / 2.0);
    double* num = (double*)calloc(maxrad + 1, sizeof(double));
    double* d1 = (double*)calloc(maxrad + 1, sizeof(double));
    double* d2 = (double*)calloc(maxrad + 1, sizeof(double));
    const double fs = 1.0 / real_size;
    const long half = (N - 1) / 2;
    for (long z = 0; z < N; ++z) {
        double rz = (double)(z > half ? z - N : z) * fs;
        rz *= rz;
        for (long y = 0; y < N; ++y) {
            double ry = (double)(y > half ? y - N : y) * fs;
            ry *= ry;
            for (long x = 0; x < N; ++x) {
                double rx = (double)(x > half ? x - N : x) * fs;
                rx *= rx;
                const double radius = real_size * sqrt(rx + ry + rz);
                const long ir = (long)radius;
                if (ir >= maxrad) continue;
                const double f = radius - ir, f1 = 1 - f;
                const long j = 2 * ((z * N + y) * N + x);
                const double p = v1[j] * v2[j] + v1[j + 1] * v2[j + 1];
                const double a = v1[j] * v1[j] + v1[j + 1] * v1[j + 1];
                const double b = v2[j] * v2[j] + v2[j + 1] * v2[j + 1];
                num[ir] += f1 * p; d1[ir] += f1 * a; d2[ir] += f1 * b;
                if (ir + 1 < maxrad) { num[ir + 1] += f * p; d1[ir + 1] += f * a; d2[ir + 1] += f * b; }
            }
        }
    }
    for (int r = 0; r < nshell; ++r) {
        double v = 0;
        if (r == 0) v = 1;
        else if (r < maxrad) {
            v = num[r] / sqrt(d1[r] * d2[r]);
            if (!isfinite(v)) v = 0;
        }
        fsc[r] = v;
    }
    free(num); free(d1); free(d2);
    return (int)maxrad;
}
