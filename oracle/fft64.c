/*
 * fft64.c - FP64 discrete Fourier transforms for the CPU oracle (test
 * infrastructure only; see fft64.h).  Written from the mathematics:
 * radix-2 decimation in time for powers of two, Bluestein's chirp-z
 * identity  jk = (j^2 + k^2 - (k-j)^2)/2  for all other lengths.
 */
#include "fft64.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct fft64_1d {
    long    n;
    int     sign;
    int     pow2;
    long    m;          /* convolution length (Bluestein) */
    long*   rev;        /* bit-reversal permutation (pow2 of length n or m) */
    double* tw;         /* twiddles exp(sign*2*pi*i*k/L), k < L/2 */
    double* chirp;      /* Bluestein: exp(sign*pi*i*k^2/n), k < n */
    double* bfft;       /* Bluestein: FFT_m of conj chirp sequence */
    struct fft64_1d* sub_f;   /* Bluestein forward length-m plan */
    struct fft64_1d* sub_b;   /* Bluestein backward length-m plan */
};

static int is_pow2(long n) { return n > 0 && (n & (n - 1)) == 0; }

static void radix2(const fft64_1d* p, double* x)
{
    long n = p->n;
    for (long i = 0; i < n; ++i) {
        long j = p->rev[i];
        if (j > i) {
            double tr = x[2*i], ti = x[2*i+1];
            x[2*i] = x[2*j]; x[2*i+1] = x[2*j+1];
            x[2*j] = tr; x[2*j+1] = ti;
        }
    }
    for (long len = 2; len <= n; len <<= 1) {
        long half = len >> 1, step = n / len;
        for (long s = 0; s < n; s += len) {
            for (long k = 0; k < half; ++k) {
                double wr = p->tw[2*(k*step)], wi = p->tw[2*(k*step)+1];
                double* a = x + 2*(s + k);
                double* b = x + 2*(s + k + half);
                double br = b[0]*wr - b[1]*wi;
                double bi = b[0]*wi + b[1]*wr;
                b[0] = a[0] - br; b[1] = a[1] - bi;
                a[0] += br;       a[1] += bi;
            }
        }
    }
}

fft64_1d* fft64_plan_1d(long n, int sign)
{
    if (n < 1) return NULL;
    fft64_1d* p = (fft64_1d*)calloc(1, sizeof(fft64_1d));
    if (!p) return NULL;
    p->n = n;
    p->sign = sign < 0 ? -1 : 1;
    p->pow2 = is_pow2(n);
    if (p->pow2) {
        p->rev = (long*)malloc(sizeof(long) * n);
        p->tw = (double*)malloc(sizeof(double) * (n > 1 ? n : 2));
        int bits = 0;
        while ((1L << bits) < n) ++bits;
        for (long i = 0; i < n; ++i) {
            long r = 0;
            for (int b = 0; b < bits; ++b) if (i & (1L << b)) r |= 1L << (bits - 1 - b);
            p->rev[i] = r;
        }
        for (long k = 0; k < n / 2 || k == 0; ++k) {
            double a = p->sign * 2.0 * M_PI * (double)k / (double)n;
            p->tw[2*k] = cos(a);
            p->tw[2*k+1] = sin(a);
            if (n < 2) break;
        }
        return p;
    }
    /* Bluestein */
    long m = 1;
    while (m < 2 * n - 1) m <<= 1;
    p->m = m;
    p->chirp = (double*)malloc(sizeof(double) * 2 * n);
    p->bfft = (double*)calloc(2 * m, sizeof(double));
    p->sub_f = fft64_plan_1d(m, -1);
    p->sub_b = fft64_plan_1d(m, +1);
    for (long k = 0; k < n; ++k) {
        /* k^2 mod 2n keeps the angle argument small and exact */
        long kk = (long)(((unsigned long long)k * (unsigned long long)k) % (unsigned long long)(2 * n));
        double a = p->sign * M_PI * (double)kk / (double)n;
        p->chirp[2*k] = cos(a);
        p->chirp[2*k+1] = sin(a);
    }
    /* b[k] = conj(chirp[k]) for |k| < n, circularly wrapped */
    for (long k = 0; k < n; ++k) {
        p->bfft[2*k] = p->chirp[2*k];
        p->bfft[2*k+1] = -p->chirp[2*k+1];
        if (k) {
            p->bfft[2*(m-k)] = p->chirp[2*k];
            p->bfft[2*(m-k)+1] = -p->chirp[2*k+1];
        }
    }
    radix2(p->sub_f, p->bfft);
    return p;
}

void fft64_free_1d(fft64_1d* p)
{
    if (!p) return;
    free(p->rev); free(p->tw); free(p->chirp); free(p->bfft);
    fft64_free_1d(p->sub_f); fft64_free_1d(p->sub_b);
    free(p);
}

long fft64_len(const fft64_1d* p) { return p ? p->n : 0; }

long fft64_work_size(const fft64_1d* p) { return p->pow2 ? 0 : 2 * p->m; }

void fft64_exec_1d(const fft64_1d* p, double* x, double* work)
{
    if (p->n == 1) return;
    if (p->pow2) { radix2(p, x); return; }
    long n = p->n, m = p->m;
    double* a = work;
    memset(a, 0, sizeof(double) * 2 * m);
    /* a[k] = x[k] * chirp[k] */
    for (long k = 0; k < n; ++k) {
        double cr = p->chirp[2*k], ci = p->chirp[2*k+1];
        a[2*k]   = x[2*k]*cr - x[2*k+1]*ci;
        a[2*k+1] = x[2*k]*ci + x[2*k+1]*cr;
    }
    radix2(p->sub_f, a);
    for (long k = 0; k < m; ++k) {
        double ar = a[2*k], ai = a[2*k+1];
        double br = p->bfft[2*k], bi = p->bfft[2*k+1];
        a[2*k]   = ar*br - ai*bi;
        a[2*k+1] = ar*bi + ai*br;
    }
    radix2(p->sub_b, a);
    double inv = 1.0 / (double)m;
    for (long k = 0; k < n; ++k) {
        double ar = a[2*k] * inv, ai = a[2*k+1] * inv;
        double cr = p->chirp[2*k], ci = p->chirp[2*k+1];
        x[2*k]   = ar*cr - ai*ci;
        x[2*k+1] = ar*ci + ai*cr;
    }
}

int fft64_nd(int rank, const long* dims, double* x, int sign)
{
    long total = 1;
    for (int d = 0; d < rank; ++d) total *= dims[d];
    for (int d = 0; d < rank; ++d) {
        long n = dims[d];
        if (n < 2) continue;
        long stride = 1;
        for (int e = d + 1; e < rank; ++e) stride *= dims[e];
        long outer = total / (n * stride);
        fft64_1d* p = fft64_plan_1d(n, sign);
        if (!p) return -1;
        double* line = (double*)malloc(sizeof(double) * 2 * n);
        double* work = (double*)malloc(sizeof(double) * (fft64_work_size(p) + 2));
        for (long o = 0; o < outer; ++o) {
            for (long s = 0; s < stride; ++s) {
                double* base = x + 2 * (o * n * stride + s);
                for (long k = 0; k < n; ++k) {
                    line[2*k] = base[2*k*stride];
                    line[2*k+1] = base[2*k*stride+1];
                }
                fft64_exec_1d(p, line, work);
                for (long k = 0; k < n; ++k) {
                    base[2*k*stride] = line[2*k];
                    base[2*k*stride+1] = line[2*k+1];
                }
            }
        }
        free(line); free(work);
        fft64_free_1d(p);
    }
    return 0;
}
