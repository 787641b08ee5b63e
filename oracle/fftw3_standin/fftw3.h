/*
 * fftw3.h - project-written stand-in for the slice of the FFTW 3.3.x
 * single-precision API that the reference's sources call (FFTW itself is an
 * un-vendored dependency of the reference and is not installed here).
 *
 * Test infrastructure only: it lets the reference's own C++ sources be
 * compiled into the CPU oracle (oracle/_ref).  Arithmetic is FP64 internally
 * (fft64.c) with single-precision storage, FFTW's sign convention and no
 * normalisation.  Entry points follow FFTW's published interface:
 *   fftwf_plan_dft            <- bsoft/src/util/fft.cpp:66
 *   fftwf_plan_many_dft       <- bsoft/src/img/Bimage_fft.cpp:327
 *   fftwf_execute_dft         <- bsoft/src/util/fft.cpp:111
 *   fftwf_destroy_plan        <- bsoft/src/util/fft.cpp:89
 *   fftwf_{init,cleanup}_threads, fftwf_plan_with_nthreads
 *                             <- e.g. bsoft/src/brefine.cpp:182-183
 */
#ifndef BSOFT_FFTW3_STANDIN_H
#define BSOFT_FFTW3_STANDIN_H

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct fftwf_plan_s* fftwf_plan;

#define FFTW_FORWARD  (-1)
#define FFTW_BACKWARD (+1)

#define FFTW_MEASURE    (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED  (1U << 1)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT    (1U << 5)
#define FFTW_ESTIMATE   (1U << 6)

#define FFTW_VERSION "standin-fp64"

fftwf_plan fftwf_plan_dft(int rank, const int* n, fftwf_complex* in,
                          fftwf_complex* out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex* in, fftwf_complex* out,
                             int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex* in,
                             fftwf_complex* out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_3d(int n0, int n1, int n2, fftwf_complex* in,
                             fftwf_complex* out, int sign, unsigned flags);
fftwf_plan fftwf_plan_many_dft(int rank, const int* n, int howmany,
                               fftwf_complex* in, const int* inembed,
                               int istride, int idist,
                               fftwf_complex* out, const int* onembed,
                               int ostride, int odist,
                               int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex* in, fftwf_complex* out);
void fftwf_destroy_plan(fftwf_plan p);
int  fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int nthreads);
void fftwf_cleanup_threads(void);

#ifdef __cplusplus
}
#endif

#endif
