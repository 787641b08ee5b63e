/*
 * fft64.h - FP64 discrete Fourier transforms for the CPU oracle.
 *
 * Test infrastructure only: this is the checker's arithmetic, never the
 * product path.  Two users:
 *   - fftw3_standin/ : the FFTW3-API stand-in the reference's own sources are
 *     linked against (FFTW 3.3.x is an un-vendored dependency of the
 *     reference: bsoft/include/fft.h:12-20, bsoft/src/util/fft.cpp:31-114);
 *   - recon_oracle.c : the FP64 restatement of the reconstruction path.
 *
 * Convention (FFTW's): sign = -1 forward, +1 backward, unnormalised,
 * X[k] = sum_j x[j] exp(sign * 2 pi i j k / n).
 * Power-of-two lengths use an iterative radix-2 Cooley-Tukey transform with
 * twiddles evaluated in double; other lengths use Bluestein's chirp-z
 * algorithm over a power-of-two convolution.
 */
#ifndef BSOFT_ORACLE_FFT64_H
#define BSOFT_ORACLE_FFT64_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fft64_1d fft64_1d;

/* Plan a length-n transform of the given sign.  Returns NULL on failure. */
fft64_1d* fft64_plan_1d(long n, int sign);
void      fft64_free_1d(fft64_1d* p);
long      fft64_len(const fft64_1d* p);

/* Transform n complex doubles (interleaved re,im) in place.  `work` must hold
 * fft64_work_size(p) doubles; plans are read-only so one plan may be shared
 * by many threads as long as each passes its own work buffer. */
long      fft64_work_size(const fft64_1d* p);
void      fft64_exec_1d(const fft64_1d* p, double* x, double* work);

/* N-dimensional in-place transform of a row-major array (dims[0] slowest)
 * of complex doubles.  Allocates its own scratch.  Returns 0 on success. */
int       fft64_nd(int rank, const long* dims, double* x, int sign);

#ifdef __cplusplus
}
#endif

#endif
