/*
 * fftw3.h -- FFTW-subset shim used ONLY by the oracle (test infrastructure).
 *
 * FFTW3 is not installed in this environment, so the reference program
 * (main.c of slitvinov/dns) cannot be linked against it.  This header exposes
 * the handful of FFTW3 entry points that main.c calls (main.c:156-162,
 * 177-223, 249-251, 274, 345-347, 363-365, 378-380, 424-428) with the same
 * names, signatures and conventions, backed by a project-written double
 * precision FFT (shim_fft.c):
 *
 *   - r2c is the forward transform (exp(-i...)), c2r the backward one
 *     (exp(+i...)); neither is normalised;
 *   - multi-dimensional arrays are row-major, the last dimension is the real
 *     one and has n/2+1 complex outputs;
 *   - a multi-dimensional c2r first runs the complex backward transforms over
 *     the leading dimensions and then the 1D c2r along the last dimension,
 *     which ignores the imaginary parts of its DC and (even n) Nyquist inputs;
 *   - c2r may destroy its input; r2c never does (FFTW_PRESERVE_INPUT).
 *
 * Only the names and argument meanings are FFTW's; the algorithm (batched
 * Stockham radix-4/2, real transforms through a half-length complex FFT) and
 * all code are this project's own.  This file is never used by the product.
 */
#ifndef DNS_ORACLE_FFTW3_SHIM_H
#define DNS_ORACLE_FFTW3_SHIM_H

#include <complex.h>
#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double _Complex fftw_complex;
typedef struct shim_plan_s *fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_ESTIMATE (1U << 6)

int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_threads_set_callback(
    void (*parallel_loop)(void *(*work)(char *), char *jobdata, size_t elsize,
                          int njobs, void *data),
    void *data);
void fftw_cleanup_threads(void);
void fftw_cleanup(void);

double *fftw_alloc_real(size_t n);
fftw_complex *fftw_alloc_complex(size_t n);
void *fftw_malloc(size_t n);
void fftw_free(void *p);

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in,
                               fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in,
                               double *out, unsigned flags);
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out,
                               unsigned flags);
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

/* Project additions (not FFTW API): twiddle generator shared with tests. */
void shim_sincos2pi(long k, long n, double *c, double *s);

#ifdef __cplusplus
}
#endif
#endif
