/*
 * match_oracle.c - FP64 restatement of the reference's central-section
 * projection matching (brefine's grid refinement and its scoring).
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h): the checker the CUDA matching
 * path is compared against, never the product.
 *
 * Reference functions restated here:
 *   FSI_Kernel::FSI_Kernel           bsoft/include/FSI_Kernel.h:28-68
 *   reference-map preparation        bsoft/src/mg/mg_refine.cpp:279-365
 *   Bimage::change_transform_size    bsoft/src/img/Bimage_fft.cpp:359-452
 *   Bimage::phase_shift_to_origin    bsoft/src/img/Bimage_complex.cpp:490-534
 *   Bimage::central_section          bsoft/src/img/Bimage_project.cpp:288-338
 *   Bimage::fspace_interpolate       bsoft/src/img/Bimage_fspace.cpp:85-147
 *   particle preparation             bsoft/src/mg/mg_refine.cpp:509-563
 *   Bimage::rescale_to_avg_std       bsoft/src/img/Bimage_rescale.cpp:163-182
 *   Bimage::statistics(long)         bsoft/src/img/Bimage_stats.cpp:101-150
 *   img_recip_space_fom              bsoft/src/mg/mg_refine.cpp:660-781
 *   CTFparam::calculate              bsoft/include/ctf.h:321-365
 */
#include "oracle.h"
#include "fft64.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define FSI_NDIV 512

int orc_fsi_kernel(int width, int power, double* table)
{
    /* FSI_Kernel.h:28-68.  Row r (fraction r/ndiv) holds the `wd` tap
     * weights; tap j sits at distance d = r/ndiv + (wd-1)/2 - j from the
     * sample, with weight sin(pi d) / (wd sin(pi d / wd)) * cos(pi d / wd)^power
     * (a periodic sinc under a cosine window).  Row 0 is the identity at tap
     * (wd-1)/2 and row ndiv the identity at tap (wd-1)/2 + 1.  A negative
     * power gives width 1 with all weights 1. */
    if (!table) return -1;
    const int wd = power < 0 ? 1 : width;
    if (wd < 1) return -1;
    const int wd_2 = (wd - 1) / 2;
    const long size = (long)(FSI_NDIV + 1) * wd;
    for (long i = 0; i < size; ++i) table[i] = power < 0 ? 1.0 : 0.0;
    if (power < 0) return wd;
    table[wd_2] = 1.0;
    for (int r = 1; r < FSI_NDIV; ++r) {
        const double frac = (double)r / FSI_NDIV;
        for (int j = 0; j < wd; ++j) {
            const double d = frac + wd_2 - j;
            const double a = M_PI * d / wd;
            table[(long)r * wd + j] = sin(M_PI * d) / (wd * sin(a)) * pow(cos(a), power);
        }
    }
    table[(long)FSI_NDIV * wd + wd_2 + 1] = 1.0;
    return wd;
}

int orc_match_diam(int N, double sampling, double hi_res)
{
    /* mg_refine.cpp:293-298: the transform is cut to an even edge of
     * 2.2 * real size / resolution (only ever reduced). */
    int diam = (int)(2.2 * N * sampling / hi_res + 0.5);
    if (diam % 2) diam += 1;
    return diam < N ? diam : N;
}

/* Bimage_fft.cpp:359-452 for a cut (nusize <= size): element xx of the new
 * edge comes from xx (xx <= (nu-1)/2) or from xx + size - nu. */
static long crop_src(long xx, long nu, long size)
{
    return xx > (nu - 1) / 2 ? xx + size - nu : xx;
}

static long wrap_freq(long i, long size)
{
    return i > (size - 1) / 2 ? i - size : i;
}

/* Bimage_complex.cpp:490-534: F(h,k,l) *= exp(i 2 pi (h ox + k oy + l oz) / size). */
static void phase_shift(int rank, long size, double* spec, const double* origin)
{
    double sh[3] = {0, 0, 0};
    for (int d = 0; d < rank; ++d) sh[d] = origin[d] / size * 2 * M_PI;
    const long nz = rank == 3 ? size : 1;
    long j = 0;
    for (long zz = 0; zz < nz; ++zz) {
        const double sl = wrap_freq(zz, size) * sh[2];
        for (long yy = 0; yy < size; ++yy) {
            const double skl = sl + wrap_freq(yy, size) * sh[1];
            for (long xx = 0; xx < size; ++xx, ++j) {
                const double phi = wrap_freq(xx, size) * sh[0] + skl;
                const double c = cos(phi), s = sin(phi);
                const double re = spec[2 * j], im = spec[2 * j + 1];
                spec[2 * j] = re * c - im * s;
                spec[2 * j + 1] = re * s + im * c;
            }
        }
    }
}

int orc_match_map(int N, const float* map, const double origin[3], double sampling, double hi_res,
                  double* spec, int* diam_out)
{
    /* mg_refine.cpp:279-365: fft() with 1/sqrt(N^3) scaling, cut to diam,
     * zero the zero-frequency term, phase shift to the (scaled) origin. */
    if (N < 2 || !map || !spec || !origin) return -1;
    const long n3 = (long)N * N * N;
    double* full = (double*)malloc(sizeof(double) * 2 * n3);
    if (!full) return -2;
    for (long i = 0; i < n3; ++i) { full[2 * i] = map[i]; full[2 * i + 1] = 0; }
    const long dims[3] = {N, N, N};
    if (fft64_nd(3, dims, full, -1)) { free(full); return -3; }
    const double sc = 1.0 / sqrt((double)n3);
    for (long i = 0; i < 2 * n3; ++i) full[i] *= sc;
    const int diam = orc_match_diam(N, sampling, hi_res);
    for (long z = 0; z < diam; ++z)
        for (long y = 0; y < diam; ++y)
            for (long x = 0; x < diam; ++x) {
                const long src = (crop_src(z, diam, N) * N + crop_src(y, diam, N)) * N + crop_src(x, diam, N);
                const long dst = (z * diam + y) * diam + x;
                spec[2 * dst] = full[2 * src];
                spec[2 * dst + 1] = full[2 * src + 1];
            }
    free(full);
    /* pref->set(0, 0); pref->set(1, 0): Bimage::set(long, double) writes the
     * j-th stored float, so the pair clears the real and imaginary parts of
     * the zero-frequency term */
    spec[0] = spec[1] = 0;
    const double scale = (double)diam / N;
    const double ori[3] = {origin[0] * scale, origin[1] * scale, origin[2] * scale};
    phase_shift(3, diam, spec, ori);
    if (diam_out) *diam_out = diam;
    return 0;
}

void orc_fspace_interpolate(int size, const double* spec, const double m[3], const double* kernel, int wd,
                            double out[2])
{
    /* Bimage_fspace.cpp:85-147: width^3 taps from floor(m) - (wd-1)/2 with a
     * single wrap per axis, weights kernel[kx] * kernel[ky] * kernel[kz]. */
    const long half = (wd - 1) / 2;
    long ib[3], ik[3];
    for (int d = 0; d < 3; ++d) {
        ib[d] = (long)floor(m[d]);
        ik[d] = ((long)((m[d] - ib[d]) * FSI_NDIV + 0.5)) * wd;
        ib[d] -= half;
    }
    double vr = 0, vi = 0;
    for (long zz = 0; zz < wd; ++zz) {
        long jz = ib[2] + zz;
        if (jz < 0) jz += size;
        if (jz >= size) jz -= size;
        for (long yy = 0; yy < wd; ++yy) {
            long jy = ib[1] + yy;
            if (jy < 0) jy += size;
            if (jy >= size) jy -= size;
            const double w = kernel[ik[1] + yy] * kernel[ik[2] + zz];
            const long row = (jz * size + jy) * size;
            for (long xx = 0; xx < wd; ++xx) {
                long jx = ib[0] + xx;
                if (jx < 0) jx += size;
                if (jx >= size) jx -= size;
                const double k = kernel[ik[0] + xx] * w;
                vr += spec[2 * (row + jx)] * k;
                vi += spec[2 * (row + jx) + 1] * k;
            }
        }
    }
    out[0] = vr;
    out[1] = vi;
}

int orc_central_section(int size, const double* spec, const double* mat, double real_size, double resolution,
                        const double* kernel, int wd, double* out)
{
    /* Bimage_project.cpp:288-338: every pixel (h, k) of the size^2 section
     * with s^2 = (h^2 + k^2) / real_size^2 <= 1/resolution^2 takes the map
     * value at m = mat (h, k, 0) (in voxels); the rest is zero. */
    if (size < 2 || !spec || !mat || !kernel || !out) return -1;
    const double inv = 1.0 / real_size;
    const double maxs2 = 1.0 / (resolution * resolution);
    memset(out, 0, sizeof(double) * 2 * size * size);
    long i = 0;
    for (long yy = 0; yy < size; ++yy) {
        const double iy = wrap_freq(yy, size) * inv;
        for (long xx = 0; xx < size; ++xx, ++i) {
            const double ix = wrap_freq(xx, size) * inv;
            const double s2 = ix * ix + iy * iy;
            if (s2 > maxs2) continue;
            double m[3];
            for (int r = 0; r < 3; ++r) m[r] = (mat[3 * r] * ix + mat[3 * r + 1] * iy) * real_size;
            orc_fspace_interpolate(size, spec, m, kernel, wd, out + 2 * i);
        }
    }
    return 0;
}

int orc_match_particle(int n, const float* image, int diam, double file_avg, double file_std, double* spec)
{
    /* mg_refine.cpp:509-563: rescale_to_avg_std(0, 1), unnormalised forward
     * FFT, zero the zero-frequency term, cut to the reference's transform
     * edge.  rescale_to_avg_std uses the image's stored average and standard
     * deviation; for a particle read from a stack those are the values of
     * the file header (MRC amean/arms, rwMRC.cpp:181-184), which the caller
     * passes as file_avg/file_std.  file_std <= 0 takes the population
     * statistics of this image (Bimage_stats.cpp:101-150) instead. */
    if (n < 2 || !image || !spec || diam < 2 || diam > n) return -1;
    const long n2 = (long)n * n;
    double avg = file_avg, std = file_std;
    if (!(file_std > 0)) {
        double sq = 0;
        avg = 0;
        for (long i = 0; i < n2; ++i) { avg += image[i]; sq += (double)image[i] * image[i]; }
        avg /= n2;
        std = sq / n2 - avg * avg;
        std = std > 0 ? sqrt(std) : 0;
    }
    const double scale = std > 1e-30 ? 1.0 / std : 1.0, shift = -avg * scale;
    double* full = (double*)malloc(sizeof(double) * 2 * n2);
    if (!full) return -2;
    for (long i = 0; i < n2; ++i) {
        full[2 * i] = (float)(image[i] * scale + shift);   /* stored as float */
        full[2 * i + 1] = 0;
    }
    const long dims[2] = {n, n};
    if (fft64_nd(2, dims, full, -1)) { free(full); return -3; }
    full[0] = full[1] = 0;   /* p->set(0, 0); p->set(1, 0): the zero-frequency term */
    for (long y = 0; y < diam; ++y)
        for (long x = 0; x < diam; ++x) {
            const long src = crop_src(y, diam, n) * n + crop_src(x, diam, n);
            spec[2 * (y * diam + x)] = full[2 * src];
            spec[2 * (y * diam + x) + 1] = full[2 * src + 1];
        }
    free(full);
    return 0;
}

void orc_phase_shift_2d(int size, double* spec, const double origin[2])
{
    phase_shift(2, size, spec, origin);
}

static double ctf_value(const double* c, double s2, double angle)
{
    /* CTFparam::calculate = sin(calculate_aberration_even) (ctf.h:321-365)
     * with the even aberration weights abw00, abw20, abw22, abw2-2, abw40. */
    const double chi = c[0] + s2 * (c[1] + c[2] * cos(2 * angle) + c[3] * sin(2 * angle)) + c[4] * s2 * s2;
    return sin(chi);
}

double orc_recip_space_fom(int size, const double* img, const double* ref, double img_real_size,
                           double ref_real_size, double ref_sampling, double hi_res, double lo_res,
                           int fom_type, const double* ctf, int invert, double* cv_out)
{
    /* mg_refine.cpp:660-781 with unit shell weights.  Shell j = floor(|(h,k)|)
     * in pixel units; FRC: sum_j<max_rad num_j / sqrt(dsum_j msum_j) averaged
     * over the shells below max_rad = real_size / hi_res, and the same over
     * [max_rad, 1.1 max_rad) as the cross-validation figure.  The reference
     * is multiplied by the CTF when one is given (the APPLY_CTF flag). */
    if (lo_res > 0 && hi_res > lo_res) { const double t = hi_res; hi_res = lo_res; lo_res = t; }
    /* pref->check_resolution on the 2-D section */
    if (hi_res > ref_real_size) hi_res = ref_real_size;
    else {
        const double rm = 2.0 / sqrt(2.0 / (ref_sampling * ref_sampling));
        if (hi_res < rm) hi_res = rm;
    }
    const double max_rad = ref_real_size / hi_res;
    double max_rad_cv = 1.1 * max_rad;
    if (max_rad_cv <= max_rad) max_rad_cv = max_rad + 1;
    const double max_rad_sq = max_rad_cv * max_rad_cv;
    double min_rad_sq = 0;
    if (lo_res > 0) { min_rad_sq = ref_real_size / lo_res; min_rad_sq *= min_rad_sq; }
    const double fs = 1.0 / img_real_size;
    double* fom = (double*)calloc(3 * (size_t)size, sizeof(double));
    if (!fom) return 0;
    double* dsum = fom + size;
    double* msum = dsum + size;
    long i = 0;
    for (long yy = 0; yy < size; ++yy) {
        const long k = wrap_freq(yy, size);
        const double sy2 = (fs * k) * (fs * k);
        for (long xx = 0; xx < size; ++xx, ++i) {
            const long h = wrap_freq(xx, size);
            const double sx2 = (fs * h) * (fs * h);
            const double d2 = (double)(h * h + k * k);
            if (d2 < min_rad_sq || d2 > max_rad_sq) continue;
            const long j = (long)sqrt(d2);
            if (j >= size) continue;
            double rr = ref[2 * i], ri = ref[2 * i + 1];
            if (ctf) {
                double c = ctf_value(ctf, sx2 + sy2, atan2((double)k, (double)h));
                if (invert) c = -c;
                rr *= c;
                ri *= c;
            }
            const double xr = img[2 * i], xi = img[2 * i + 1];
            if (fom_type < 1) {
                fom[j] += xr * rr + xi * ri;
                msum[j] += rr * rr + ri * ri;
                dsum[j] += xr * xr + xi * xi;
            } else {
                const double amp = sqrt(xr * xr + xi * xi) + sqrt(rr * rr + ri * ri);
                double dphi = atan2(xi, xr) - atan2(ri, rr);
                while (dphi < -M_PI) dphi += 2 * M_PI;
                while (dphi > M_PI) dphi -= 2 * M_PI;
                fom[j] += amp * dphi * dphi;
                msum[j] += amp;
            }
        }
    }
    double f = 0, wsum = 0, cv = 0;
    for (long j = 0; j < max_rad; ++j) {
        wsum += 1;
        if (fom_type < 1) {
            const double den = dsum[j] * msum[j];
            if (den > 0) f += fom[j] / sqrt(den);
        } else if (msum[j]) {
            f += cos(sqrt(fom[j] / msum[j]));
        }
    }
    f /= wsum;
    wsum = 0;
    for (long j = (long)max_rad; j < max_rad_cv; ++j) {
        wsum += 1;
        if (fom_type < 1) {
            const double den = dsum[j] * msum[j];
            if (den > 0) cv += fom[j] / sqrt(den);
        } else if (msum[j]) {
            cv += cos(sqrt(fom[j] / msum[j]));
        }
    }
    cv /= wsum;
    free(fom);
    if (cv_out) *cv_out = cv;
    return f;
}
