/*
 * FP64 mixed-radix FFT behind the FFTW3 API subset declared in fftw3.h
 * (test infrastructure for the oracle build of the reference only).
 *
 * Algorithm: recursive decimation in time.  A length-n transform with
 * smallest prime factor p is split into p interleaved sub-transforms of
 * length n/p and recombined with twiddles; prime lengths fall back to a
 * direct DFT.  Twiddles are exp(sign*2*pi*i*k/n) evaluated in long double.
 */
#include "fftw3.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

struct oracle_fftw_plan_s {
    int n0, n1; /* n1 == 0 for 1-D */
    fftw_complex *in, *out;
    int sign;
    int kind; /* 0 complex (double), 1 r2c (float), 2 c2r (float) */
    void *fin, *fout;
};

void *fftw_malloc(size_t n) { return malloc(n ? n : 1); }
void fftw_free(void *p) { free(p); }

static int smallest_factor(int n) {
    for (int p = 2; p * p <= n; p++)
        if (n % p == 0) return p;
    return n;
}

static void twiddle(long n, long k, int sign, double *re, double *im) {
    const long double pi = 3.141592653589793238462643383279502884L;
    long double a = sign * 2.0L * pi * (long double)(k % n) / (long double)n;
    *re = (double)cosl(a);
    *im = (double)sinl(a);
}

/* x: input with stride s (complex units), y: contiguous output of length n. */
static void fft_rec(const double *x, long s, double *y, int n, int sign) {
    if (n == 1) { y[0] = x[0]; y[1] = x[1]; return; }
    int p = smallest_factor(n);
    if (p == n) { /* direct DFT for prime length */
        for (int k = 0; k < n; k++) {
            double sr = 0, si = 0;
            for (int j = 0; j < n; j++) {
                double wr, wi;
                twiddle(n, (long)j * k, sign, &wr, &wi);
                const double *xj = x + 2 * (long)j * s;
                sr += xj[0] * wr - xj[1] * wi;
                si += xj[0] * wi + xj[1] * wr;
            }
            y[2 * k] = sr; y[2 * k + 1] = si;
        }
        return;
    }
    int m = n / p;
    double *sub = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    for (int r = 0; r < p; r++) fft_rec(x + 2 * (long)r * s, s * p, sub + 2 * (long)r * m, m, sign);
    for (int k = 0; k < n; k++) {
        double sr = 0, si = 0;
        int km = k % m;
        for (int r = 0; r < p; r++) {
            double wr, wi;
            twiddle(n, (long)r * k, sign, &wr, &wi);
            const double *z = sub + 2 * ((long)r * m + km);
            sr += z[0] * wr - z[1] * wi;
            si += z[0] * wi + z[1] * wr;
        }
        y[2 * k] = sr; y[2 * k + 1] = si;
    }
    free(sub);
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
    (void)flags;
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->n0 = n; p->n1 = 0; p->in = in; p->out = out; p->sign = sign;
    return p;
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags) {
    (void)flags;
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->n0 = n0; p->n1 = n1; p->in = in; p->out = out; p->sign = sign;
    return p;
}

static void execute_real(const fftw_plan p) {
    int n = p->n0;
    double *x = (double *)calloc(2 * (size_t)n, sizeof(double));
    double *y = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    if (p->kind == 1) { /* real input, first n/2+1 outputs of the forward DFT */
        const float *in = (const float *)p->fin;
        for (int j = 0; j < n; j++) x[2 * j] = in[j];
        fft_rec(x, 1, y, n, FFTW_FORWARD);
        float *out = (float *)p->fout;
        for (int k = 0; k <= n / 2; k++) { out[2 * k] = (float)y[2 * k]; out[2 * k + 1] = (float)y[2 * k + 1]; }
    } else { /* Hermitian half-spectrum input, unnormalised backward DFT, real output */
        const float *in = (const float *)p->fin;
        for (int k = 0; k <= n / 2; k++) { x[2 * k] = in[2 * k]; x[2 * k + 1] = in[2 * k + 1]; }
        for (int k = n / 2 + 1; k < n; k++) { x[2 * k] = in[2 * (n - k)]; x[2 * k + 1] = -in[2 * (n - k) + 1]; }
        fft_rec(x, 1, y, n, FFTW_BACKWARD);
        float *out = (float *)p->fout;
        for (int j = 0; j < n; j++) out[j] = (float)y[2 * j];
    }
    free(x); free(y);
}

void *fftwf_malloc(size_t n) { return malloc(n ? n : 1); }
void fftwf_free(void *p) { free(p); }
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned flags) {
    (void)flags;
    fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
    p->n0 = n; p->kind = 1; p->fin = in; p->fout = out;
    return p;
}
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *in, float *out, unsigned flags) {
    (void)flags;
    fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
    p->n0 = n; p->kind = 2; p->fin = in; p->fout = out;
    return p;
}
void fftwf_execute(const fftwf_plan p) { execute_real(p); }
void fftwf_destroy_plan(fftwf_plan p) { free(p); }

void fftw_execute(const fftw_plan p) {
    if (p->n1 == 0) {
        int n = p->n0;
        double *tmp = (double *)malloc(sizeof(double) * 2 * (size_t)n);
        fft_rec((const double *)p->in, 1, tmp, n, p->sign);
        memcpy(p->out, tmp, sizeof(double) * 2 * (size_t)n);
        free(tmp);
        return;
    }
    int n0 = p->n0, n1 = p->n1;
    size_t tot = (size_t)n0 * n1;
    double *a = (double *)malloc(sizeof(double) * 2 * tot);
    double *col = (double *)malloc(sizeof(double) * 2 * (size_t)n0);
    double *colo = (double *)malloc(sizeof(double) * 2 * (size_t)n0);
    for (int r = 0; r < n0; r++) /* rows (contiguous, last index) */
        fft_rec((const double *)p->in + 2 * (size_t)r * n1, 1, a + 2 * (size_t)r * n1, n1, p->sign);
    for (int c = 0; c < n1; c++) {
        for (int r = 0; r < n0; r++) {
            col[2 * r] = a[2 * ((size_t)r * n1 + c)];
            col[2 * r + 1] = a[2 * ((size_t)r * n1 + c) + 1];
        }
        fft_rec(col, 1, colo, n0, p->sign);
        for (int r = 0; r < n0; r++) {
            a[2 * ((size_t)r * n1 + c)] = colo[2 * r];
            a[2 * ((size_t)r * n1 + c) + 1] = colo[2 * r + 1];
        }
    }
    memcpy(p->out, a, sizeof(double) * 2 * tot);
    free(a); free(col); free(colo);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
