/*
 * Seeded synthetic trajectory generator writing NISE's binary (GROBIN)
 * trajectory layout.
 *
 * Record layouts written (all little-endian, as the reference reads them with
 * fread, read_trajectory.c):
 *   Energy, HamiltonianType Full   : int32 tag + float32[N(N+1)/2]   (read_He, :157-178)
 *     packed upper triangle, row-major: index(a<=b) = b + a(2N-a-1)/2
 *     (Sindex, NISE_subs.h:54-65)
 *   Energy, HamiltonianType Coupling: int32 tag + float32[N] (read_Dia, :317-341)
 *   Couplingfile                    : one Full record (read_coupling, :47-70)
 *   Dipolefile                      : int32 tag + float32[3N] (x block, y block,
 *                                     z block; read_mue, :357-377)
 *   Anharmonicfile                  : int32 tag + float32[N] (read_A, :344-354)
 *   Overtonedipolefile              : int32 tag + float32[3N] (read_over, :402-414)
 *
 * Statistics: site energies eps0 + Ornstein-Uhlenbeck noise
 * x <- a x + sqrt(1-a^2) sigma xi, a = exp(-dt/tau), x0 ~ N(0, sigma^2)
 * (the form of the reference tutorial generator).  Couplings: chain
 * nearest-neighbour J = j_nn + N(0, j_sigma) redrawn every frame, or static
 * point-dipole couplings (the TDC formula of read_trajectory.c:199-215)
 * between unit dipoles on a cubic lattice or in a random cluster, zeroed when
 * |J| < jcut.  Dipoles: seeded random unit vectors plus an optional
 * per-frame Gaussian jitter per component.
 *
 * The random streams are xoshiro256** seeded through splitmix64 with Gaussian
 * deviates from the Box-Muller transform; every site has its own stream so
 * the output depends only on the seed.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "nise_synth.h"

typedef struct { uint64_t s[4]; int has_spare; double spare; } rng_t;

static uint64_t splitmix64(uint64_t *x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static void rng_seed(rng_t *r, uint64_t seed, uint64_t stream) {
    uint64_t x = seed * 0x100000001B3ULL + stream * 0x9E3779B97F4A7C15ULL + 12345;
    for (int i = 0; i < 4; i++) r->s[i] = splitmix64(&x);
    r->has_spare = 0;
}
static inline uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
static uint64_t rng_next(rng_t *r) {
    uint64_t *s = r->s;
    uint64_t res = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45);
    return res;
}
static double rng_uniform(rng_t *r) { return ((rng_next(r) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
static double rng_gauss(rng_t *r) {
    if (r->has_spare) { r->has_spare = 0; return r->spare; }
    double u = rng_uniform(r), v = rng_uniform(r);
    double rad = sqrt(-2.0 * log(u)), ang = 6.283185307179586 * v;
    r->spare = rad * sin(ang); r->has_spare = 1;
    return rad * cos(ang);
}

static inline long tri_index(int a, int b, int n) {
    if (a > b) { int t = a; a = b; b = t; }
    return (long)b + (long)a * (2L * n - a - 1) / 2;
}

static void unit_vector(rng_t *r, double v[3]) {
    double z = 2.0 * rng_uniform(r) - 1.0, ph = 6.283185307179586 * rng_uniform(r);
    double s = sqrt(1.0 - z * z);
    v[0] = s * cos(ph); v[1] = s * sin(ph); v[2] = z;
}

long nise_synth_energy_record_floats(const nise_synth_spec *sp) {
    return sp->ham_type == NISE_SYNTH_FULL ? (long)sp->n_sites * (sp->n_sites + 1) / 2 : sp->n_sites;
}

/* Geometry and static dipoles; positions in Angstrom. */
static int build_geometry(const nise_synth_spec *sp, double *pos, double *mu) {
    int n = sp->n_sites;
    rng_t g;
    rng_seed(&g, sp->seed, 0xD1B0LL);
    for (int i = 0; i < n; i++) unit_vector(&g, mu + 3 * i);
    if (sp->geometry == NISE_SYNTH_CHAIN) {
        for (int i = 0; i < n; i++) { pos[3 * i] = i * sp->spacing; pos[3 * i + 1] = 0; pos[3 * i + 2] = 0; }
    } else if (sp->geometry == NISE_SYNTH_LATTICE) {
        for (int i = 0; i < n; i++) {
            pos[3 * i] = (i % 8) * sp->spacing;
            pos[3 * i + 1] = ((i / 8) % 8) * sp->spacing;
            pos[3 * i + 2] = (i / 64) * sp->spacing;
        }
    } else {
        /* random sequential placement in a cube with a minimum separation */
        double side = sp->spacing * cbrt((double)n) * 1.25, dmin = 0.75 * sp->spacing;
        rng_t p;
        rng_seed(&p, sp->seed, 0xC1C1LL);
        for (int i = 0; i < n; i++) {
            int tries = 0;
            for (;;) {
                double x = side * rng_uniform(&p), y = side * rng_uniform(&p), z = side * rng_uniform(&p);
                int ok = 1;
                for (int j = 0; j < i && ok; j++) {
                    double dx = x - pos[3 * j], dy = y - pos[3 * j + 1], dz = z - pos[3 * j + 2];
                    if (dx * dx + dy * dy + dz * dz < dmin * dmin) ok = 0;
                }
                if (ok) { pos[3 * i] = x; pos[3 * i + 1] = y; pos[3 * i + 2] = z; break; }
                if (++tries > 100000) return -1;
            }
        }
    }
    return 0;
}

/* Static point-dipole couplings (cm^-1) into packed triangle Jp (diagonal untouched). */
static void point_dipole_couplings(const nise_synth_spec *sp, const double *pos, const double *mu, float *Jp) {
    int n = sp->n_sites;
    const double A = 5034.11861687; /* Debye^2/Angstrom^3 -> cm^-1 */
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            double R[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
            double r2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2], r = sqrt(r2);
            const double *m1 = mu + 3 * i, *m2 = mu + 3 * j;
            double f1 = m1[0] * m2[0] + m1[1] * m2[1] + m1[2] * m2[2];
            double f2 = -3.0 * (m1[0] * R[0] + m1[1] * R[1] + m1[2] * R[2]) *
                        (m2[0] * R[0] + m2[1] * R[1] + m2[2] * R[2]) / r2;
            double J = A * (f1 + f2) / (r2 * r);
            if (fabs(J) < sp->jcut) J = 0.0;
            Jp[tri_index(i, j, n)] = (float)J;
        }
}

int nise_synth_fill(const nise_synth_spec *sp, void *energy, void *dipole, void *coupling, void *anharm,
                    void *overtone) {
    int n = sp->n_sites;
    if (n <= 0 || sp->frames <= 0 || sp->dt_fs <= 0) return -1;
    long nn2 = (long)n * (n + 1) / 2;
    long erec = nise_synth_energy_record_floats(sp);
    double *pos = (double *)malloc(sizeof(double) * 3 * n), *mu = (double *)malloc(sizeof(double) * 3 * n);
    double *ou = (double *)malloc(sizeof(double) * n);
    float *Jstatic = (float *)calloc(nn2, sizeof(float));
    rng_t *site_rng = (rng_t *)malloc(sizeof(rng_t) * n);
    rng_t jrng, murng, arng;
    if (!pos || !mu || !ou || !Jstatic || !site_rng) return -2;
    if (build_geometry(sp, pos, mu) != 0) return -3;
    if (sp->geometry != NISE_SYNTH_CHAIN) point_dipole_couplings(sp, pos, mu, Jstatic);
    double a = exp(-sp->dt_fs / sp->tau_fs), b = sqrt(1.0 - a * a);
    for (int i = 0; i < n; i++) {
        rng_seed(&site_rng[i], sp->seed, 1000 + (uint64_t)i);
        ou[i] = sp->sigma * rng_gauss(&site_rng[i]);
    }
    rng_seed(&jrng, sp->seed, 0x7A7ALL);
    rng_seed(&murng, sp->seed, 0x3E3ELL);
    rng_seed(&arng, sp->seed, 0xA5A5LL);

    char *E = (char *)energy;
    size_t erec_bytes = 4 + 4 * (size_t)erec;
    for (long t = 0; t < sp->frames; t++) {
        int32_t tag = (int32_t)t;
        char *rec = E + (size_t)t * erec_bytes;
        memcpy(rec, &tag, 4);
        float *h = (float *)(rec + 4);
        if (sp->ham_type == NISE_SYNTH_FULL) {
            for (long k = 0; k < nn2; k++) h[k] = Jstatic[k];
            if (sp->geometry == NISE_SYNTH_CHAIN)
                for (int i = 0; i + 1 < n; i++)
                    h[tri_index(i, i + 1, n)] = (float)(sp->j_nn + sp->j_sigma * rng_gauss(&jrng));
            for (int i = 0; i < n; i++) h[tri_index(i, i, n)] = (float)(sp->eps0 + ou[i]);
        } else {
            for (int i = 0; i < n; i++) h[i] = (float)(sp->eps0 + ou[i]);
        }
        for (int i = 0; i < n; i++) ou[i] = a * ou[i] + b * sp->sigma * rng_gauss(&site_rng[i]);
    }

    if (coupling) {
        int32_t tag = 0;
        memcpy(coupling, &tag, 4);
        float *h = (float *)((char *)coupling + 4);
        for (long k = 0; k < nn2; k++) h[k] = Jstatic[k];
        if (sp->geometry == NISE_SYNTH_CHAIN)
            for (int i = 0; i + 1 < n; i++) h[tri_index(i, i + 1, n)] = (float)sp->j_nn;
        for (int i = 0; i < n; i++) h[tri_index(i, i, n)] = (float)sp->eps0;
    }

    int nd = sp->dipole_frames > 0 ? sp->dipole_frames : sp->frames;
    size_t drec_bytes = 4 + 4 * 3 * (size_t)n;
    for (long t = 0; dipole && t < nd; t++) {
        int32_t tag = (int32_t)t;
        char *rec = (char *)dipole + (size_t)t * drec_bytes;
        memcpy(rec, &tag, 4);
        float *m = (float *)(rec + 4);
        for (int x = 0; x < 3; x++)
            for (int i = 0; i < n; i++) {
                double v = mu[3 * i + x];
                if (sp->mu_jitter > 0) v += sp->mu_jitter * rng_gauss(&murng);
                m[x * n + i] = (float)v;
            }
    }
    for (long t = 0; anharm && t < sp->frames; t++) {
        int32_t tag = (int32_t)t;
        char *rec = (char *)anharm + (size_t)t * (4 + 4 * (size_t)n);
        memcpy(rec, &tag, 4);
        float *h = (float *)(rec + 4);
        for (int i = 0; i < n; i++) h[i] = (float)(sp->anharm_mean + sp->anharm_sigma * rng_gauss(&arng));
    }
    for (long t = 0; overtone && t < sp->frames; t++) {
        int32_t tag = (int32_t)t;
        char *rec = (char *)overtone + (size_t)t * drec_bytes;
        memcpy(rec, &tag, 4);
        float *m = (float *)(rec + 4);
        for (int x = 0; x < 3; x++)
            for (int i = 0; i < n; i++)
                m[x * n + i] = (float)(1.41421356237 * mu[3 * i + x] * (1.0 + 0.02 * rng_gauss(&arng)));
    }
    free(pos); free(mu); free(ou); free(Jstatic); free(site_rng);
    return 0;
}

static int write_file(const char *path, const void *buf, size_t bytes) {
    FILE *f = fopen(path, "wb");
    if (!f) return -10;
    size_t w = fwrite(buf, 1, bytes, f);
    fclose(f);
    return w == bytes ? 0 : -11;
}

int nise_synth_write(const nise_synth_spec *sp, const char *energy_path, const char *dipole_path,
                     const char *coupling_path, const char *anharm_path, const char *overtone_path) {
    int n = sp->n_sites;
    long nn2 = (long)n * (n + 1) / 2;
    size_t ebytes = (size_t)sp->frames * (4 + 4 * (size_t)nise_synth_energy_record_floats(sp));
    int nd = sp->dipole_frames > 0 ? sp->dipole_frames : sp->frames;
    size_t dbytes = (size_t)nd * (4 + 12 * (size_t)n);
    size_t abytes = (size_t)sp->frames * (4 + 4 * (size_t)n);
    size_t obytes = (size_t)sp->frames * (4 + 12 * (size_t)n);
    void *E = malloc(ebytes), *D = malloc(dbytes);
    void *C = coupling_path ? malloc(4 + 4 * nn2) : NULL;
    void *A = anharm_path ? malloc(abytes) : NULL;
    void *O = overtone_path ? malloc(obytes) : NULL;
    int rc = (!E || !D) ? -2 : nise_synth_fill(sp, E, D, C, A, O);
    if (rc == 0) rc = write_file(energy_path, E, ebytes);
    if (rc == 0) rc = write_file(dipole_path, D, dbytes);
    if (rc == 0 && C) rc = write_file(coupling_path, C, 4 + 4 * nn2);
    if (rc == 0 && A) rc = write_file(anharm_path, A, abytes);
    if (rc == 0 && O) rc = write_file(overtone_path, O, obytes);
    free(E); free(D); free(C); free(A); free(O);
    return rc;
}
