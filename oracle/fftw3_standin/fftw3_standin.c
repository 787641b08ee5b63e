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
    /* transform along each axis with the pre-planned 1-D sub-plans; strided
     * axes are gathered 16 lines at a time for cache locality, and large
     * transforms spread their lines over OpenMP threads (FFTW's threaded
     * planner does the equivalent; nested calls from the reference's own
     * parallel regions stay single-threaded) */
    for (int d = 0; d < p->rank; ++d) {
        long n = p->n[d];
        if (n < 2) continue;
        long stride = 1;
        for (int e = d + 1; e < p->rank; ++e) stride *= p->n[e];
        long outer = total / (n * stride);
        const long G = 16;
        long ngroups = outer * ((stride + G - 1) / G);
        const fft64_1d* sub = p->sub[d];
        #pragma omp parallel for schedule(dynamic, 4) if (total >= 65536)
        for (long gi = 0; gi < ngroups; ++gi) {
            long o = gi / ((stride + G - 1) / G);
            long s0 = (gi % ((stride + G - 1) / G)) * G;
            long cnt = stride - s0 < G ? stride - s0 : G;
            double* buf = (double*)malloc(sizeof(double) * 2 * n * G);
            double* work = (double*)malloc(sizeof(double) * (fft64_work_size(sub) + 2));
            double* base = x + 2 * (o * n * stride + s0);
            if (stride == 1) {
                fft64_exec_1d(sub, base, work);
            } else {
                for (long k = 0; k < n; ++k)
                    for (long c = 0; c < cnt; ++c) {
                        buf[2*(c*n + k)] = base[2*(k*stride + c)];
                        buf[2*(c*n + k)+1] = base[2*(k*stride + c)+1];
                    }
                for (long c = 0; c < cnt; ++c) fft64_exec_1d(sub, buf + 2*c*n, work);
                for (long k = 0; k < n; ++k)
                    for (long c = 0; c < cnt; ++c) {
                        base[2*(k*stride + c)] = buf[2*(c*n + k)];
                        base[2*(k*stride + c)+1] = buf[2*(c*n + k)+1];
                    }
            }
            free(buf); free(work);
        }
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
