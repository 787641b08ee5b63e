/*
 * fftw3_standin.c - implementation of the FFTW3-API stand-in (test
 * infrastructure only; see fftw3.h).  Plans only record geometry and the
 * per-dimension FP64 sub-plans; every execute allocates its own scratch, so
 * one plan can be shared read-only across threads the way the reference
 * shares its plan between OpenMP workers (bsoft/src/breconstruct.cpp:280-291).
 */
#include "fftw3.h"
#include "../fft64.h"

#include <stdlib.h>
#include <string.h>

struct fftwf_plan_s {
    int rank;
    long n[3];
    int howmany;
    long istride, idist, ostride, odist;   /* advanced layout (rank 1 only) */
    int advanced;
    int sign;
    fftwf_complex* in;
    fftwf_complex* out;
    fft64_1d* sub[3];
};

static fftwf_plan make_plan(int rank, const int* n, int sign)
{
    if (rank < 1 || rank > 3) return NULL;
    fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
    if (!p) return NULL;
    p->rank = rank;
    p->sign = sign < 0 ? -1 : 1;
    p->howmany = 1;
    for (int d = 0; d < rank; ++d) {
        p->n[d] = n[d];
        p->sub[d] = fft64_plan_1d(n[d], p->sign);
        if (!p->sub[d]) { fftwf_destroy_plan(p); return NULL; }
    }
    return p;
}

fftwf_plan fftwf_plan_dft(int rank, const int* n, fftwf_complex* in,
                          fftwf_complex* out, int sign, unsigned flags)
{
    (void)flags;
    fftwf_plan p = make_plan(rank, n, sign);
    if (p) { p->in = in; p->out = out; }
    return p;
}

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags)
{
    int d[1] = {n};
    return fftwf_plan_dft(1, d, in, out, sign, flags);
}

fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags)
{
    int d[2] = {n0, n1};
    return fftwf_plan_dft(2, d, in, out, sign, flags);
}

fftwf_plan fftwf_plan_dft_3d(int n0, int n1, int n2, fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags)
{
    int d[3] = {n0, n1, n2};
    return fftwf_plan_dft(3, d, in, out, sign, flags);
}

fftwf_plan fftwf_plan_many_dft(int rank, const int* n, int howmany,
                               fftwf_complex* in, const int* inembed,
                               int istride, int idist,
                               fftwf_complex* out, const int* onembed,
                               int ostride, int odist,
                               int sign, unsigned flags)
{
    (void)inembed; (void)onembed; (void)flags;
    if (rank != 1) return NULL;   /* the reference only plans 1-D batches */
    fftwf_plan p = make_plan(rank, n, sign);
    if (!p) return NULL;
    p->advanced = 1;
    p->howmany = howmany;
    p->istride = istride; p->idist = idist;
    p->ostride = ostride; p->odist = odist;
    p->in = in; p->out = out;
    return p;
}

static void exec_advanced(const fftwf_plan p, fftwf_complex* in, fftwf_complex* out)
{
    long n = p->n[0];
    double* line = (double*)malloc(sizeof(double) * 2 * n);
    double* work = (double*)malloc(sizeof(double) * (fft64_work_size(p->sub[0]) + 2));
    for (long t = 0; t < p->howmany; ++t) {
        for (long k = 0; k < n; ++k) {
            const float* v = in[t * p->idist + k * p->istride];
            line[2*k] = v[0]; line[2*k+1] = v[1];
        }
        fft64_exec_1d(p->sub[0], line, work);
        for (long k = 0; k < n; ++k) {
            float* v = out[t * p->odist + k * p->ostride];
            v[0] = (float)line[2*k]; v[1] = (float)line[2*k+1];
        }
    }
    free(line); free(work);
}

void fftwf_execute_dft(const fftwf_plan p, fftwf_complex* in, fftwf_complex* out)
{
    if (!p || !in || !out) return;
    if (p->advanced) { exec_advanced(p, in, out); return; }
    long total = 1;
    for (int d = 0; d < p->rank; ++d) total *= p->n[d];
    double* x = (double*)malloc(sizeof(double) * 2 * total);
    if (!x) return;
    for (long i = 0; i < total; ++i) { x[2*i] = in[i][0]; x[2*i+1] = in[i][1]; }
    /* transform along each axis with the pre-planned 1-D sub-plans */
    for (int d = 0; d < p->rank; ++d) {
        long n = p->n[d];
        if (n < 2) continue;
        long stride = 1;
        for (int e = d + 1; e < p->rank; ++e) stride *= p->n[e];
        long outer = total / (n * stride);
        double* line = (double*)malloc(sizeof(double) * 2 * n);
        double* work = (double*)malloc(sizeof(double) * (fft64_work_size(p->sub[d]) + 2));
        for (long o = 0; o < outer; ++o)
            for (long s = 0; s < stride; ++s) {
                double* base = x + 2 * (o * n * stride + s);
                if (stride == 1) {
                    fft64_exec_1d(p->sub[d], base, work);
                    continue;
                }
                for (long k = 0; k < n; ++k) { line[2*k] = base[2*k*stride]; line[2*k+1] = base[2*k*stride+1]; }
                fft64_exec_1d(p->sub[d], line, work);
                for (long k = 0; k < n; ++k) { base[2*k*stride] = line[2*k]; base[2*k*stride+1] = line[2*k+1]; }
            }
        free(line); free(work);
    }
    for (long i = 0; i < total; ++i) { out[i][0] = (float)x[2*i]; out[i][1] = (float)x[2*i+1]; }
    free(x);
}

void fftwf_execute(const fftwf_plan p)
{
    if (p) fftwf_execute_dft(p, p->in, p->out);
}

void fftwf_destroy_plan(fftwf_plan p)
{
    if (!p) return;
    for (int d = 0; d < 3; ++d) fft64_free_1d(p->sub[d]);
    free(p);
}

int  fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int nthreads) { (void)nthreads; }
void fftwf_cleanup_threads(void) {}
