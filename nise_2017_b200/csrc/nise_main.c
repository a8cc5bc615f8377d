/*
 * nise — NISE-compatible driver for the B200 engine.
 *
 * Usage: nise <inputfile>   (same keyword file as the reference's NISE program)
 *
 * Follows the reference driver (NISE.c:49-362) for the techniques on this
 * path: read the keywords, load the trajectory, run Absorption (writing
 * TD_Absorption.dat and Absorption.dat), the other linear techniques LD,
 * Raman, SFG, DOS and CD (their TD_*.dat and spectrum files), or the 2DIR
 * and 2DUVvis families (writing RparI.dat ... RcroII.dat), all through the C
 * ABI in nise_b200.h.  Engine controls come
 * from the environment: NISE_PRECISION=fp64, NISE_LAUNCH=plain, NISE_DEVICE=<n>.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "nise_b200.h"

static int fail(nise_ctx *c, const char *what, int rc) {
    fprintf(stderr, "%s failed (status %d): %s\n", what, rc, c ? nise_last_error(c) : nise_global_error());
    if (c) nise_destroy(c);
    return 1;
}

int main(int argc, char *argv[]) {
    if (argc < 2) {
        printf("Specify input file name on command line!\n");
        return 255;
    }
    nise_params p;
    nise_params_default(&p);
    int rc = nise_read_input(argv[1], &p);
    if (rc != NISE_OK) return fail(NULL, "reading input", rc);
    const char *prec = getenv("NISE_PRECISION");
    if (prec && !strcmp(prec, "fp64")) p.precision = NISE_FP64;
    const char *launch = getenv("NISE_LAUNCH");
    if (launch && !strcmp(launch, "plain")) p.launch_mode = NISE_PLAIN;
    const char *dev = getenv("NISE_DEVICE");
    if (dev) p.device = atoi(dev);

    FILE *log = fopen("NISE.log", "w");
    if (log) {
        fprintf(log, "Log\n");
        fclose(log);
    }
    nise_ctx *c = NULL;
    if ((rc = nise_create(&p, &c)) != NISE_OK) return fail(NULL, "creating context", rc);
    if ((rc = nise_load_files(c)) != NISE_OK) return fail(c, "loading trajectory", rc);

    if (p.technique == NISE_TECH_ABSORPTION) {
        double *re = calloc(p.tmax1, sizeof(double)), *im = calloc(p.tmax1, sizeof(double));
        int samples = 0;
        if ((rc = nise_absorption(c, re, im, &samples)) != NISE_OK) return fail(c, "absorption", rc);
        nise_write_td_absorption("TD_Absorption.dat", &p, re, im, samples);
        int fft = p.fft < p.tmax1 ? p.tmax1 : p.fft, rows = 0;
        double *w = calloc(fft, sizeof(double)), *sr = calloc(fft, sizeof(double)), *si = calloc(fft, sizeof(double));
        if ((rc = nise_absorption_fft(c, re, im, samples, w, sr, si, fft, &rows)) != NISE_OK)
            return fail(c, "absorption FFT", rc);
        nise_write_spectrum("Absorption.dat", w, sr, si, rows);
        free(re); free(im); free(w); free(sr); free(si);
        printf("----------------------------------------------\n");
        printf(" Absorption calculation succesfully completed\n");
        printf("----------------------------------------------\n\n");
    } else if (p.technique >= NISE_TECH_2DIR && p.technique <= NISE_TECH_NOEAUVVIS) {
        size_t plane = (size_t)p.tmax3 * p.tmax1;
        double *R = calloc(12 * plane, sizeof(double));
        int count = 0;
        if ((rc = nise_2dir(c, R, &count)) != NISE_OK) return fail(c, "2DIR", rc);
        static const char *names[6] = {"RparI.dat", "RparII.dat", "RperI.dat", "RperII.dat", "RcroI.dat", "RcroII.dat"};
        for (int k = 0; k < 6; k++) nise_write_2d(names[k], &p, R + 2 * k * plane, R + (2 * k + 1) * plane, count);
        free(R);
        printf("Samples %d\n", count);
        printf("----------------------------------------\n");
        printf(" %s calculation succesfully completed\n", p.technique >= NISE_TECH_2DUVVIS ? "2DES" : "2DIR");
        printf("----------------------------------------\n\n");
    } else if (p.technique >= NISE_TECH_LD && p.technique <= NISE_TECH_LUM) {
        double *re = calloc(4 * (size_t)p.tmax1, sizeof(double)), *im = calloc(4 * (size_t)p.tmax1, sizeof(double));
        int channels = 0, samples = 0;
        if ((rc = nise_linear(c, re, im, 4, &channels, &samples)) != NISE_OK) return fail(c, p.technique_name, rc);
        int fft = p.fft < p.tmax1 ? p.tmax1 : p.fft, rows = 0;
        double *w = calloc(fft, sizeof(double)), *sr = calloc(fft, sizeof(double)), *si = calloc(fft, sizeof(double));
        for (int k = 0; k < channels; k++) {
            const double *rk = re + (size_t)k * p.tmax1, *ik = im + (size_t)k * p.tmax1;
            /* TD_DOS.dat and TD_Lum.dat have no trailing blank (calc_DOS.c:209, luminescence.c:224), the
               others do; luminescence writes the total's time-domain file only */
            const char *td = nise_linear_file(p.technique, k, 1);
            if (td) nise_write_td(td, &p, rk, ik, samples, p.technique != NISE_TECH_DOS && p.technique != NISE_TECH_LUM);
            if ((rc = nise_absorption_fft(c, rk, ik, samples, w, sr, si, fft, &rows)) != NISE_OK)
                return fail(c, "1D FFT", rc);
            nise_write_spectrum(nise_linear_file(p.technique, k, 0), w, sr, si, rows);
        }
        free(re); free(im); free(w); free(sr); free(si);
        static const char *done[] = {"Linear Dichroism", "Raman", "SFG", "DOS", "CD", "Luminescence"};
        printf("----------------------------------------------\n");
        printf(" %s calculation succesfully completed\n", done[p.technique - NISE_TECH_LD]);
        printf("----------------------------------------------\n\n");
    } else {
        fprintf(stderr, "Technique '%s' is not on this engine's path (Absorption, LD, Raman, SFG, DOS, CD, Luminescence, "
                "2DIR, GBIR, SEIR, EAIR, noEAIR, "
                "2DUVvis, GBUVvis, SEUVvis, EAUVvis, noEAUVvis)\n",
                p.technique_name);
        nise_destroy(c);
        return 2;
    }
    double ms = 0, main_ms = 0;
    long launches = 0;
    nise_last_timing(c, &ms, &main_ms, &launches);
    printf(" Device time %.3f ms (propagation %.3f ms) in %ld kernel launches\n", ms, main_ms, launches);
    nise_destroy(c);
    return 0;
}
