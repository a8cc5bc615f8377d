/*
 * Minimal FFTW3-API stand-in, used ONLY to compile the reference NISE and
 * 2DFFT programs from their own unmodified sources as a test oracle
 * (oracle/_ref).  Test infrastructure: nothing in the product links this.
 *
 * Provides the subset the reference calls: complex-to-complex 1-D and 2-D
 * plans (any size, forward or backward, unnormalised, row-major like FFTW),
 * fftw_malloc/fftw_free and fftw_execute.  The transform is an FP64
 * mixed-radix FFT (fftw_shim.c) with the FFTW sign convention
 * out[k] = sum_j in[j] * exp(sign * 2*pi*i * j*k/n), sign = -1 forward.
 */
#ifndef ORACLE_FFTW3_SHIM_H
#define ORACLE_FFTW3_SHIM_H
#include <stddef.h>

typedef double fftw_complex[2];
typedef struct oracle_fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

/* Single-precision real<->complex subset (linked by techniques off the path). */
typedef float fftwf_complex[2];
typedef struct oracle_fftw_plan_s *fftwf_plan;
void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *in, float *out, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);

#endif
