/*
 * ORACLE / CPU-baseline harness — test and measurement infrastructure.
 *
 * Times the reference's own single-vector propagator (propagate_vector,
 * propagate.c:20-39, compiled from the reference sources by the Makefile in
 * this directory) on one frame of a trajectory: `threads` vectors are
 * propagated concurrently (one per OpenMP thread, as propagate_matrix does at
 * propagate.c:43-52), each for `steps` steps, and the wall time is printed as
 * one JSON line.  Site-steps = threads * steps * N.
 *
 * usage: ref_bench energy.bin coupling.bin|- N propagation couplingcut deltat
 *                  trotter threshold min1 max1 threads steps [in.bin out.bin]
 *   energy.bin holds diagonal-only records (HamiltonianType Coupling) when a
 *   coupling file is given, else Full records; frame 0 is used.
 *   With in.bin and out.bin the starting vectors are read from in.bin and the
 *   propagated ones written to out.bin (float32 [threads][re N, im N]): the
 *   reference's own propagated states, for the parity fixtures.
 */
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "types.h"
#include "propagate.h"

static float *read_floats(const char *path, long count, long offset_words) {
    FILE *f = fopen(path, "rb");
    if (!f) return NULL;
    float *b = (float *)malloc(sizeof(float) * count);
    fseek(f, 4 * offset_words, SEEK_SET);
    long got = (long)fread(b, sizeof(float), count, f);
    fclose(f);
    if (got != count) { free(b); return NULL; }
    return b;
}

int main(int argc, char **argv) {
    if (argc < 13) {
        fprintf(stderr, "usage: %s energy coupling|- N propagation cut deltat trotter thres min1 max1 threads steps\n",
                argv[0]);
        return 2;
    }
    int N = atoi(argv[3]);
    t_non *non = (t_non *)calloc(1, sizeof(t_non));
    non->singles = N;
    non->propagation = atoi(argv[4]);
    non->couplingcut = (float)atof(argv[5]);
    non->deltat = (float)atof(argv[6]);
    non->ts = atoi(argv[7]);
    non->thres = (float)atof(argv[8]);
    non->min1 = (float)atof(argv[9]);
    non->max1 = (float)atof(argv[10]);
    non->shifte = (non->max1 + non->min1) / 2;
    int threads = atoi(argv[11]), steps = atoi(argv[12]);
    long nn2 = (long)N * (N + 1) / 2;
    float *H;
    if (strcmp(argv[2], "-")) { /* coupling frame + diagonal frame 0 */
        H = read_floats(argv[2], nn2, 1);
        float *d = read_floats(argv[1], N, 1);
        if (!H || !d) return 3;
        for (int i = 0; i < N; i++) H[i * N + i - (i * (i + 1)) / 2] = d[i] - non->shifte;
        free(d);
    } else {
        H = read_floats(argv[1], nn2, 1);
        if (!H) return 3;
        for (int i = 0; i < N; i++) H[i * N + i - (i * (i + 1)) / 2] -= non->shifte;
    }
    for (int i = 0; i < N; i++) /* read cut, read_trajectory.c:305-311 */
        for (int j = i + 1; j < N; j++) {
            long idx = j + (long)i * ((N << 1) - i - 1) / 2;
            if (H[idx] < non->couplingcut && H[idx] > -non->couplingcut) H[idx] = 0;
        }
    float *vr = (float *)calloc((size_t)threads * N, sizeof(float));
    float *vi = (float *)calloc((size_t)threads * N, sizeof(float));
    for (long i = 0; i < (long)threads * N; i++) vr[i] = (float)((i * 7919 % 1000) / 1000.0 - 0.5);
    const char *in_path = argc >= 15 ? argv[13] : NULL, *out_path = argc >= 15 ? argv[14] : NULL;
    if (in_path) {
        FILE *f = fopen(in_path, "rb");
        if (!f) return 4;
        for (int v = 0; v < threads; v++)
            if (fread(vr + (size_t)v * N, sizeof(float), N, f) != (size_t)N ||
                fread(vi + (size_t)v * N, sizeof(float), N, f) != (size_t)N) {
                fclose(f);
                return 4;
            }
        fclose(f);
    }
    double t0 = omp_get_wtime();
#pragma omp parallel for num_threads(threads) schedule(static, 1)
    for (int v = 0; v < threads; v++)
        for (int s = 0; s < steps; s++) propagate_vector(non, H, vr + (size_t)v * N, vi + (size_t)v * N, 1, 1, 1);
    double t1 = omp_get_wtime();
    if (out_path) {
        FILE *f = fopen(out_path, "wb");
        if (!f) return 5;
        for (int v = 0; v < threads; v++) {
            fwrite(vr + (size_t)v * N, sizeof(float), N, f);
            fwrite(vi + (size_t)v * N, sizeof(float), N, f);
        }
        fclose(f);
    }
    double chk = 0;
    for (long i = 0; i < (long)threads * N; i++) chk += vr[i] * vr[i] + vi[i] * vi[i];
    printf("{\"seconds\": %.6f, \"threads\": %d, \"steps\": %d, \"sites\": %d, \"site_steps\": %ld, \"norm\": %.6e}\n",
           t1 - t0, threads, steps, N, (long)threads * steps * N, chk);
    return 0;
}
