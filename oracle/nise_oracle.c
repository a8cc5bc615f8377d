/*
 * ORACLE — test infrastructure, not product code.
 *
 * CPU restatement of the reference NISE propagation path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, and only
 * as the checker.  Each function names the reference file:line it follows.
 *
 * Built twice (Makefile in this directory):
 *   -DORACLE_F32 : `real` and the response accumulators are float and every
 *                  expression keeps the reference's operand types and order,
 *                  so the FP32 build reproduces the reference's rounding
 *                  (pinned against the reference binary in tests/).
 *   default      : `real` and accumulators are double — the FP64 reference.
 * The float-rounded physical constants of the reference (src/types.h:5-12)
 * are used in both builds so the two differ only in arithmetic precision.
 *
 * Deviation (both builds): the reference diagonalises with LAPACK ssyev_
 * (propagate.c:1185-1221); this restatement uses a cyclic Jacobi eigensolver
 * in FP64.  Eigenvector sign/order freedom does not change U = V e^{-iEf} V^T.
 */
#include "nise_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef ORACLE_F32
typedef float real;
#ifdef ORACLE_ACC64
typedef double acc;
#else
typedef float acc;
#endif
#define RSIN sinf
#define RCOS cosf
#define RSQRT sqrtf
#else
typedef double real;
typedef double acc;
#define RSIN sin
#define RCOS cos
#define RSQRT sqrt
#endif

/* src/types.h:5-12 (declared float in the reference). */
static const float c_v = 2.99792458e-5;
static const float twoPi = 2 * 3.14159265359;
static const float icm2ifs = 2.99792458e-5;
static const float sqrt2 = 1.41421356237;
static const float ithirty = 1.0 / 30;

int oracle_real_size(void) { return (int)sizeof(real); }

/* NISE_subs.h:54-65 */
static inline int Sindex(int a, int b, int N) {
    if (a > b) return a + b * ((N << 1) - b - 1) / 2;
    return b + a * ((N << 1) - a - 1) / 2;
}

/* ------------------------------------------------------------------ */
/* Trajectory access: whole files in memory, frames addressed like     */
/* read_trajectory.c (record = int32 tag + floats).                    */
typedef struct {
    const oracle_params *p;
    float shifte;
    char *E; long nE;
    char *D; long nD;
    char *A; long nA;
    char *O; long nO;
    char *P; long nP;  /* Positionfile (TransitionDipole / ExtendedDipole) */
    char *B; long nB;  /* PBCfile */
    char *Al; long nAl; /* Alphafile */
    float *Hc;     /* coupling frame for HamiltonianType Coupling (read_coupling) */
    float *mu_xyz; /* static dipoles for HamiltonianType Coupling */
    int nshift; int *shift_site; float *shift_ab;
} traj_t;

static char *slurp(const char *path, long *bytes) {
    FILE *f = fopen(path, "rb");
    if (!f) return NULL;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *b = (char *)malloc(n > 0 ? n : 1);
    if (n > 0 && fread(b, 1, n, f) != (size_t)n) { free(b); fclose(f); return NULL; }
    fclose(f);
    *bytes = n;
    return b;
}

static void traj_free(traj_t *t) {
    free(t->E); free(t->D); free(t->A); free(t->O); free(t->P); free(t->B); free(t->Al); free(t->Hc); free(t->mu_xyz);
    free(t->shift_site); free(t->shift_ab);
    memset(t, 0, sizeof(*t));
}

static long full_frame_floats(const oracle_params *p) {
    return (long)p->singles * (p->singles + 1) / 2 + (long)p->doubles * (p->doubles + 1) / 2;
}

static int read_mue(const traj_t *t, const char *buf, long nbytes, float *mu, int pos, int x);

/* pbc1 (NISE_subs.c:641-648). */
static float pbc1(float r, int x, const float *box) {
    if (box[0] > 0.0) {
        if (r > box[x] / 2) r = r - box[x];
        if (r < -box[x] / 2) r = r + box[x];
    }
    return r;
}

/* Couplings computed on the fly (read_trajectory.c:180-303): transition
 * dipole coupling from one position per site, or extended dipoles from two
 * (records 2*pos and 2*pos+1 of the Positionfile), with the periodic box of
 * the PBCfile record pos when given.  Float arithmetic in the reference's
 * order; sqrt and 1.0/x in double as the reference's calls are. */
static int onfly_couplings(const traj_t *t, float *He, int pos) {
    const oracle_params *p = t->p;
    const int N = p->singles;
    const float A = 5034.11861687;
    float box[3] = {0, 0, 0};
    if (t->B) {
        long off = (long)pos * 16 + 4;
        if (off + 12 > t->nB) return 0;
        memcpy(box, t->B + off, 12);
    }
    float *R = (float *)calloc(3 * N, sizeof(float)), *R2 = (float *)calloc(3 * N, sizeof(float));
    float *mu = (float *)calloc(3 * N, sizeof(float));
    int ok = 1, rp = p->ham_onfly == 2 ? 2 * pos : pos;
    for (int x = 0; x < 3 && ok; x++) {
        ok = read_mue(t, t->P, t->nP, R + x * N, rp, x) && read_mue(t, t->D, t->nD, mu + x * N, pos, x);
        if (ok && p->ham_onfly == 2) ok = read_mue(t, t->P, t->nP, R2 + x * N, rp + 1, x);
    }
    if (ok && p->ham_onfly == 1) {
        for (int i = 0; i < N; i++) {
            float m1x = mu[i], m1y = mu[N + i], m1z = mu[2 * N + i];
            for (int j = i + 1; j < N; j++) {
                float Rx = pbc1(R[i] - R[j], 0, box);
                float Ry = pbc1(R[N + i] - R[N + j], 1, box);
                float Rz = pbc1(R[2 * N + i] - R[2 * N + j], 2, box);
                float m2x = mu[j], m2y = mu[N + j], m2z = mu[2 * N + j];
                float dist = sqrt(Rx * Rx + Ry * Ry + Rz * Rz);
                float idist = 1.0 / dist;
                float idist3 = idist * idist * idist;
                float f1 = m1x * m2x + m1y * m2y + m1z * m2z;
                float f2 = -3 * (m1x * Rx + m1y * Ry + m1z * Rz) * (m2x * Rx + m2y * Ry + m2z * Rz) * idist * idist;
                He[Sindex(i, j, N)] = A * (f1 + f2) * idist3;
            }
        }
    } else if (ok) {
        for (int i = 0; i < N; i++) {
            float Rx = pbc1(R2[i] - R[i], 0, box);
            float Ry = pbc1(R2[N + i] - R[N + i], 1, box);
            float Rz = pbc1(R2[2 * N + i] - R[2 * N + i], 2, box);
            float m1x = mu[i], m1y = mu[N + i], m1z = mu[2 * N + i];
            float dist = sqrt(Rx * Rx + Ry * Ry + Rz * Rz);
            float q1 = sqrt(m1x * m1x + m1y * m1y + m1z * m1z) / dist;
            for (int j = i + 1; j < N; j++) {
                Rx = pbc1(R2[j] - R[j], 0, box);
                Ry = pbc1(R2[N + j] - R[N + j], 1, box);
                Rz = pbc1(R2[2 * N + j] - R[2 * N + j], 2, box);
                dist = sqrt(Rx * Rx + Ry * Ry + Rz * Rz);
                /* the reference forms q2 from the first dipole (read_trajectory.c:246) */
                float q2 = sqrt(m1x * m1x + m1y * m1y + m1z * m1z) / dist;
                float J, idist;
                Rx = pbc1(R[i] - R[j], 0, box); Ry = pbc1(R[N + i] - R[N + j], 1, box);
                Rz = pbc1(R[2 * N + i] - R[2 * N + j], 2, box);
                dist = sqrt(Rx * Rx + Ry * Ry + Rz * Rz); idist = 1.0 / dist; J = idist;
                Rx = pbc1(R[i] - R2[j], 0, box); Ry = pbc1(R[N + i] - R2[N + j], 1, box);
                Rz = pbc1(R[2 * N + i] - R2[2 * N + j], 2, box);
                dist = sqrt(Rx * Rx + Ry * Ry + Rz * Rz); idist = 1.0 / dist; J = J - idist;
                Rx = pbc1(R2[i] - R[j], 0, box); Ry = pbc1(R2[N + i] - R[N + j], 1, box);
                Rz = pbc1(R2[2 * N + i] - R[2 * N + j], 2, box);
                dist = sqrt(Rx * Rx + Ry * Ry + Rz * Rz); idist = 1.0 / dist; J = J - idist;
                Rx = pbc1(R2[i] - R2[j], 0, box); Ry = pbc1(R2[N + i] - R2[N + j], 1, box);
                Rz = pbc1(R2[2 * N + i] - R2[2 * N + j], 2, box);
                dist = sqrt(Rx * Rx + Ry * Ry + Rz * Rz); idist = 1.0 / dist; J = J + idist;
                He[Sindex(i, j, N)] = A * q1 * q2 * J;
            }
        }
    }
    free(R); free(R2); free(mu);
    return ok;
}

/* read_He (read_trajectory.c:106-314): Full frame (:157-178) or diagonal-only
 * frame for HamiltonianType Coupling (:135-156); coupling cut (:305-311).
 * Returns 0 when the frame lies beyond the file (the reference exits). */
static int read_He_mem(const traj_t *t, const char *buf, long nbytes, float *He, int pos) {
    const oracle_params *p = t->p;
    int N = p->singles;
    if ((p->ham_coupling && pos >= 0) || p->ham_onfly) {
        long off = (long)pos * (4 + 4L * N);
        if (pos < 0 || off + 4 + 4L * N > nbytes) return 0;
        const float *h = (const float *)(buf + off + 4);
        for (int i = 0; i < N; i++) He[i * N + i - (i * (i + 1)) / 2] = h[i] - t->shifte;
        if (p->ham_onfly && !onfly_couplings(t, He, pos)) return 0;
    } else {
        if (pos == -1) pos = 0;
        long nn = (long)N * (N + 1) / 2;
        long off = (long)pos * (4 + 4L * full_frame_floats(p));
        if (off + 4 + 4L * nn > nbytes) return 0;
        memcpy(He, buf + off + 4, sizeof(float) * nn);
        for (int i = 0; i < N; i++) He[i * N + i - (i * (i + 1)) / 2] -= t->shifte;
    }
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++)
            if (fabs(He[Sindex(i, j, N)]) < p->couplingcut) He[Sindex(i, j, N)] = 0;
    return 1;
}

static int read_He(const traj_t *t, float *He, int pos) { return read_He_mem(t, t->E, t->nE, He, pos); }

/* read_mue (read_trajectory.c:357-377): component x of the dipole at frame pos. */
static int read_mue(const traj_t *t, const char *buf, long nbytes, float *mu, int pos, int x) {
    int N = t->p->singles;
    long rec = 4 + 4L * (3L * N + 3L * N * t->p->doubles);
    long off = (long)pos * rec + 4 + 4L * x * N;
    if (pos < 0 || off + 4L * N > nbytes) return 0;
    memcpy(mu, buf + off, sizeof(float) * N);
    return 1;
}

/* mureadE / read_dipole (read_trajectory.c:90-101, 428-441). */
static int mu_read(const traj_t *t, float *mu, int pos, int x) {
    int N = t->p->singles;
    if (t->p->ham_coupling) { memcpy(mu, t->mu_xyz + N * x, sizeof(float) * N); return 1; }
    return read_mue(t, t->D, t->nD, mu, pos, x);
}

/* read_A (:344-354) and read_over (:402-414). */
static int read_A(const traj_t *t, float *anh, int pos) {
    int N = t->p->singles;
    long off = (long)pos * (4 + 4L * N) + 4;
    if (pos < 0 || off + 4L * N > t->nA) return 0;
    memcpy(anh, t->A + off, sizeof(float) * N);
    return 1;
}
static int read_over(const traj_t *t, float *over, int pos, int x) {
    int N = t->p->singles;
    long off = (long)pos * (4 + 12L * N) + 4 + 4L * x * N;
    if (pos < 0 || off + 4L * N > t->nO) return 0;
    memcpy(over, t->O + off, sizeof(float) * N);
    return 1;
}

/* read_alpha (read_trajectory.c:380-399): component x of the polarisability at frame pos. */
static int read_alpha(const traj_t *t, float *alpha, int pos, int x) {
    int N = t->p->singles;
    long off = (long)pos * (4 + 24L * N) + 4 + 4L * x * N;
    if (pos < 0 || off + 4L * N > t->nAl) return 0;
    memcpy(alpha, t->Al + off, sizeof(float) * N);
    return 1;
}

/* apply_singleshift (hamshift.c:59-66), file format of read_shift (:13-47). */
static void apply_singleshift(const traj_t *t, float *H) {
    for (int i = 0; i < t->nshift; i++) {
        int idx = Sindex(t->shift_site[i], t->shift_site[i], t->p->singles);
        H[idx] = H[idx] * t->shift_ab[2 * i] + t->shift_ab[2 * i + 1];
    }
}

static int traj_open(traj_t *t, const oracle_params *p, float shifte, int need_anh) {
    memset(t, 0, sizeof(*t));
    t->p = p;
    t->shifte = shifte;
    int N = p->singles;
    t->E = slurp(p->energy, &t->nE);
    t->D = slurp(p->dipole, &t->nD);
    /* calc_DOS and raman.c open no dipole file */
    const int dipoles = !(p->technique == 12 || p->technique == 14);
    if (!t->E || (dipoles && !t->D)) return -1;
    if (p->technique == 12 || p->technique == 13) {
        t->Al = slurp(p->alpha, &t->nAl);
        if (!t->Al) return -1;
    }
    if (p->technique == 15) {
        t->P = slurp(p->position, &t->nP);
        if (!t->P) return -1;
    }
    if (p->ham_onfly) {
        t->P = slurp(p->position, &t->nP);
        if (!t->P) return -1;
        if (p->pbc[0] && !(t->B = slurp(p->pbc, &t->nB))) return -1;
    }
    if (need_anh) {
        t->A = slurp(p->anharm, &t->nA);
        t->O = slurp(p->overtone, &t->nO);
        if (!t->A || !t->O) return -1;
    }
    if (p->ham_coupling) {
        long nb;
        char *cb = slurp(p->coupling, &nb);
        if (!cb) return -1;
        t->Hc = (float *)calloc((size_t)N * (N + 1) / 2, sizeof(float));
        int ok = read_He_mem(t, cb, nb, t->Hc, -1);
        free(cb);
        if (!ok) return -1;
        t->mu_xyz = (float *)calloc(3 * (size_t)N, sizeof(float));
        for (int x = 0; x < 3 && dipoles; x++)
            if (!read_mue(t, t->D, t->nD, t->mu_xyz + N * x, 0, x)) return -1;
    }
    if (p->shift[0]) {
        FILE *f = fopen(p->shift, "r");
        if (f) {
            if (fscanf(f, "%d", &t->nshift) != 1) { fclose(f); return -1; }
            t->shift_site = (int *)calloc(t->nshift > 0 ? t->nshift : 1, sizeof(int));
            t->shift_ab = (float *)calloc(2 * (t->nshift > 0 ? t->nshift : 1), sizeof(float));
            for (int i = 0; i < t->nshift; i++)
                if (fscanf(f, "%d %f %f", &t->shift_site[i], &t->shift_ab[2 * i], &t->shift_ab[2 * i + 1]) != 3) {
                    fclose(f);
                    return -1;
                }
            fclose(f);
        }
    }
    return 0;
}

/* Hamiltonian buffer initialisation: HamiltonianType Coupling keeps the
 * coupling frame and only overwrites the diagonal on every read. */
static float *ham_alloc(const traj_t *t) {
    int N = t->p->singles;
    float *H = (float *)calloc((size_t)N * (N + 1) / 2, sizeof(float));
    if (t->Hc) memcpy(H, t->Hc, sizeof(float) * (size_t)N * (N + 1) / 2);
    return H;
}

/* ------------------------------------------------------------------ */
/* FP64 cyclic Jacobi eigensolver (replaces ssyev_).                   */
void oracle_eigh(int n, double *A, double *w, double *V) {
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) V[i * n + j] = (i == j);
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0, tot = 0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                tot += A[i * n + j] * A[i * n + j];
                if (i != j) off += A[i * n + j] * A[i * n + j];
            }
        if (off <= 1e-30 * (tot > 0 ? tot : 1)) break;
        for (int pq = 0; pq < n * n; pq++) {
            int P = pq / n, Q = pq % n;
            if (Q <= P) continue;
            double apq = A[P * n + Q];
            if (apq == 0.0) continue;
            double app = A[P * n + P], aqq = A[Q * n + Q];
            double theta = (aqq - app) / (2.0 * apq);
            double tt = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            double c = 1.0 / sqrt(tt * tt + 1.0), s = tt * c;
            for (int k = 0; k < n; k++) { /* columns P,Q */
                double akp = A[k * n + P], akq = A[k * n + Q];
                A[k * n + P] = c * akp - s * akq;
                A[k * n + Q] = s * akp + c * akq;
            }
            for (int k = 0; k < n; k++) { /* rows P,Q */
                double apk = A[P * n + k], aqk = A[Q * n + k];
                A[P * n + k] = c * apk - s * aqk;
                A[Q * n + k] = s * apk + c * aqk;
            }
            for (int k = 0; k < n; k++) {
                double vkp = V[k * n + P], vkq = V[k * n + Q];
                V[k * n + P] = c * vkp - s * vkq;
                V[k * n + Q] = s * vkp + c * vkq;
            }
        }
    }
    /* sort ascending like LAPACK */
    int *ord = (int *)malloc(sizeof(int) * n);
    for (int i = 0; i < n; i++) ord[i] = i;
    for (int i = 1; i < n; i++) {
        int k = ord[i], j = i - 1;
        while (j >= 0 && A[ord[j] * n + ord[j]] > A[k * n + k]) { ord[j + 1] = ord[j]; j--; }
        ord[j + 1] = k;
    }
    double *Vs = (double *)malloc(sizeof(double) * n * n);
    for (int j = 0; j < n; j++) {
        w[j] = A[ord[j] * n + ord[j]];
        for (int i = 0; i < n; i++) Vs[i * n + j] = V[i * n + ord[j]];
    }
    memcpy(V, Vs, sizeof(double) * n * n);
    free(Vs); free(ord);
}

/* Square Hamiltonian from packed (propagate.c:79-85) and its eigenvectors
 * in the layout diagonalizeLPD leaves in H: H[i*N+j] = component i of
 * eigenvector j (propagate.c:1211-1217). */
static void diag_packed(const float *Hp, int N, real *Hv, real *e) {
    double *A = (double *)malloc(sizeof(double) * N * N), *V = (double *)malloc(sizeof(double) * N * N);
    double *w = (double *)malloc(sizeof(double) * N);
    for (int a = 0; a < N; a++) {
        A[a + N * a] = Hp[a + N * a - (a * (a + 1)) / 2];
        for (int b = a + 1; b < N; b++) A[a + N * b] = A[b + N * a] = Hp[b + N * a - (a * (a + 1)) / 2];
    }
    oracle_eigh(N, A, w, V);
    for (int i = 0; i < N * N; i++) Hv[i] = (real)V[i];
    for (int i = 0; i < N; i++) e[i] = (real)w[i];
    free(A); free(V); free(w);
}

/* U = V e^{-i e f} V^T in the reference's storage (propagate.c:89-106).
 * crr/cri[a + c*N]. */
static void build_U(int N, const real *Hv, const real *e, real f, real *crr, real *cri) {
    real *re_U = (real *)calloc(N, sizeof(real)), *im_U = (real *)calloc(N, sizeof(real));
    real *cnr = (real *)calloc((size_t)N * N, sizeof(real)), *cni = (real *)calloc((size_t)N * N, sizeof(real));
    for (int a = 0; a < N; a++) {
        re_U[a] = cos(e[a] * f);
        im_U[a] = -sin(e[a] * f);
    }
    for (int a = 0; a < N; a++)
        for (int b = 0; b < N; b++) {
            cnr[b + a * N] += Hv[b + a * N] * re_U[b];
            cni[b + a * N] += Hv[b + a * N] * im_U[b];
        }
    memset(crr, 0, sizeof(real) * N * N);
    memset(cri, 0, sizeof(real) * N * N);
    for (int a = 0; a < N; a++)
        for (int b = 0; b < N; b++)
            for (int c = 0; c < N; c++) {
                crr[a + c * N] += Hv[b + a * N] * cnr[b + c * N];
                cri[a + c * N] += Hv[b + a * N] * cni[b + c * N];
            }
    free(re_U); free(im_U); free(cnr); free(cni);
}

/* ------------------------------------------------------------------ */
/* Singles propagators                                                 */

/* propagate_vec_DIA (propagate.c:60-125) and, with thres>0, the truncated
 * propagate_vec_DIA_S (:185-258).  Returns the number of kept elements. */
static int prop_DIA(const oracle_params *p, const float *Hp, real *cr, real *ci, int sign, int truncate) {
    int N = p->singles;
    real f = (real)p->deltat * (real)icm2ifs * (real)twoPi * sign;
    real *Hv = (real *)malloc(sizeof(real) * N * N), *e = (real *)malloc(sizeof(real) * N);
    real *crr = (real *)malloc(sizeof(real) * N * N), *cri = (real *)malloc(sizeof(real) * N * N);
    real *cnr = (real *)calloc(N, sizeof(real)), *cni = (real *)calloc(N, sizeof(real));
    diag_packed(Hp, N, Hv, e);
    build_U(N, Hv, e, f, crr, cri);
    int elements = 0;
    for (int a = 0; a < N; a++) {
        cnr[a] = 0, cni[a] = 0;
        for (int b = 0; b < N; b++) {
            if (truncate && !((crr[a + b * N] * crr[a + b * N] + cri[a + b * N] * cri[a + b * N]) > p->thres))
                continue;
            elements++;
            cnr[a] += crr[a + b * N] * cr[b] - cri[a + b * N] * ci[b];
            cni[a] += crr[a + b * N] * ci[b] + cri[a + b * N] * cr[b];
        }
    }
    for (int a = 0; a < N; a++) cr[a] = cnr[a], ci[a] = cni[a];
    free(Hv); free(e); free(crr); free(cri); free(cnr); free(cni);
    return elements;
}

/* propagate_vec_coupling_S (propagate.c:821-899): Trotter splitting with m
 * sub-steps of half diagonal phase, sequential 2x2 coupling rotations in
 * (a,b) lexicographic order, half diagonal phase. */
static void prop_coupling(const oracle_params *p, const float *Hp, real *cr, real *ci, int m, int sign) {
    int N = p->singles;
    real f = (real)p->deltat * (real)icm2ifs * (real)twoPi * sign / m;
    float *H0 = (float *)malloc(sizeof(float) * N), *H1 = (float *)malloc(sizeof(float) * (N * (N - 1) / 2 + 1));
    int *col = (int *)malloc(sizeof(int) * (N * (N - 1) / 2 + 1)), *row = (int *)malloc(sizeof(int) * (N * (N - 1) / 2 + 1));
    real *re_U = (real *)malloc(sizeof(real) * N), *im_U = (real *)malloc(sizeof(real) * N);
    real *ocr = (real *)malloc(sizeof(real) * N), *oci = (real *)malloc(sizeof(real) * N);
    int kmax = 0;
    for (int a = 0; a < N; a++) {
        H0[a] = Hp[Sindex(a, a, N)];
        for (int b = a + 1; b < N; b++) {
            int index = Sindex(a, b, N);
            if (fabs(Hp[index]) > p->couplingcut) { H1[kmax] = Hp[index]; col[kmax] = a; row[kmax] = b; kmax++; }
        }
    }
    for (int a = 0; a < N; a++) {
        re_U[a] = cos(0.5 * H0[a] * f);
        im_U[a] = -sin(0.5 * H0[a] * f);
    }
    for (int i = 0; i < m; i++) {
        for (int a = 0; a < N; a++) {
            ocr[a] = cr[a] * re_U[a] - ci[a] * im_U[a];
            oci[a] = ci[a] * re_U[a] + cr[a] * im_U[a];
        }
        for (int k = 0; k < kmax; k++) {
            int a = col[k], b = row[k];
            real J = H1[k];
            J = J * f;
            real si = -sin(J);
            real co = sqrt(1 - si * si);
            real cr1 = co * ocr[a] - si * oci[b];
            real ci1 = co * oci[a] + si * ocr[b];
            real cr2 = co * ocr[b] - si * oci[a];
            real ci2 = co * oci[b] + si * ocr[a];
            ocr[a] = cr1, oci[a] = ci1, ocr[b] = cr2, oci[b] = ci2;
        }
        for (int a = 0; a < N; a++) {
            cr[a] = ocr[a] * re_U[a] - oci[a] * im_U[a];
            ci[a] = oci[a] * re_U[a] + ocr[a] * im_U[a];
        }
    }
    free(H0); free(H1); free(col); free(row); free(re_U); free(im_U); free(ocr); free(oci);
}

/* find_norm / re_normalize (NISE_subs.c:125-148). */
static real find_norm(const real *r, const real *i, int N) {
    real norm = 0;
    for (int a = 0; a < N; a++) norm += r[a] * r[a] + i[a] * i[a];
    return norm;
}
static void re_normalize(real *r, real *i, int N, real norm) {
    real nn = find_norm(r, i, N);
    if (norm != nn) {
        real factor = sqrt(norm / nn);
        for (int a = 0; a < N; a++) { r[a] = r[a] * factor; i[a] = i[a] * factor; }
    }
}

/* propagate_vec_RK4 (propagate.c:261-373). */
static void prop_RK4(const oracle_params *p, const float *Hp, real *cr, real *ci, int m, int sign) {
    int N = p->singles, N2 = N * (N + 1) / 2;
    real f = (real)p->deltat * (real)icm2ifs * (real)twoPi * sign / m;
    real *H0 = (real *)malloc(sizeof(real) * N2);
    int *col = (int *)malloc(sizeof(int) * N2), *row = (int *)malloc(sizeof(int) * N2);
    real *k1r = (real *)calloc(N, sizeof(real)), *k1i = (real *)calloc(N, sizeof(real));
    real *k2r = (real *)calloc(N, sizeof(real)), *k2i = (real *)calloc(N, sizeof(real));
    real *k3r = (real *)calloc(N, sizeof(real)), *k3i = (real *)calloc(N, sizeof(real));
    real *k4r = (real *)calloc(N, sizeof(real)), *k4i = (real *)calloc(N, sizeof(real));
    int kmax = 0;
    for (int a = 0; a < N; a++)
        for (int b = a; b < N; b++) {
            int index = Sindex(a, b, N);
            if (fabs(Hp[index]) > p->couplingcut || a == b) {
                H0[kmax] = f * Hp[index];
                col[kmax] = a, row[kmax] = b;
                kmax++;
            }
        }
    for (int i = 0; i < m; i++) {
        if (i > 0) {
            memset(k1r, 0, sizeof(real) * N); memset(k1i, 0, sizeof(real) * N);
            memset(k2r, 0, sizeof(real) * N); memset(k2i, 0, sizeof(real) * N);
            memset(k3r, 0, sizeof(real) * N); memset(k3i, 0, sizeof(real) * N);
            memset(k4r, 0, sizeof(real) * N); memset(k4i, 0, sizeof(real) * N);
        }
        for (int k = 0; k < kmax; k++) {
            k1r[col[k]] += H0[k] * ci[row[k]];
            k1i[col[k]] -= H0[k] * cr[row[k]];
            if (row[k] != col[k]) {
                k1r[row[k]] += H0[k] * ci[col[k]];
                k1i[row[k]] -= H0[k] * cr[col[k]];
            }
        }
        for (int k = 0; k < kmax; k++) {
            k2r[col[k]] += H0[k] * (ci[row[k]] + k1i[row[k]] * 0.5);
            k2i[col[k]] -= H0[k] * (cr[row[k]] + k1r[row[k]] * 0.5);
            if (row[k] != col[k]) {
                k2r[row[k]] += H0[k] * (ci[col[k]] + k1i[col[k]] * 0.5);
                k2i[row[k]] -= H0[k] * (cr[col[k]] + k1r[col[k]] * 0.5);
            }
        }
        for (int k = 0; k < kmax; k++) {
            k3r[col[k]] += H0[k] * (ci[row[k]] + k2i[row[k]] * 0.5);
            k3i[col[k]] -= H0[k] * (cr[row[k]] + k2r[row[k]] * 0.5);
            if (row[k] != col[k]) {
                k3r[row[k]] += H0[k] * (ci[col[k]] + k2i[col[k]] * 0.5);
                k3i[row[k]] -= H0[k] * (cr[col[k]] + k2r[col[k]] * 0.5);
            }
        }
        for (int k = 0; k < kmax; k++) {
            k4r[col[k]] += H0[k] * (ci[row[k]] + k3i[row[k]]);
            k4i[col[k]] -= H0[k] * (cr[row[k]] + k3r[row[k]]);
            if (row[k] != col[k]) {
                k4r[row[k]] += H0[k] * (ci[col[k]] + k3i[col[k]]);
                k4i[row[k]] -= H0[k] * (cr[col[k]] + k3r[col[k]]);
            }
        }
        real norm = find_norm(cr, ci, N);
        for (int k = 0; k < N; k++) {
            cr[k] = cr[k] + (k1r[k] + 2 * k2r[k] + 2 * k3r[k] + k4r[k]) / 6.0;
            ci[k] = ci[k] + (k1i[k] + 2 * k2i[k] + 2 * k3i[k] + k4i[k]) / 6.0;
        }
        re_normalize(cr, ci, N, norm);
    }
    free(H0); free(col); free(row);
    free(k1r); free(k1i); free(k2r); free(k2i); free(k3r); free(k3i); free(k4r); free(k4i);
}

/* propagate_vector dispatch (propagate.c:20-39); propagation 2
 * ("Diagonal", rejected by the reference at readinput.c:243-248) is the
 * exact eigen propagator, i.e. the Sparse scheme at Threshold 0. */
static void propagate_vector(const oracle_params *p, const float *Hp, real *cr, real *ci, int sign) {
    if (p->propagation == 1) prop_coupling(p, Hp, cr, ci, p->ts, sign);
    else if (p->propagation == 3) prop_RK4(p, Hp, cr, ci, p->ts, sign);
    else if (p->propagation == 2) prop_DIA(p, Hp, cr, ci, sign, 0);
    else {
        if (p->thres == 0 || p->thres > 1) prop_DIA(p, Hp, cr, ci, sign, 0);
        else prop_DIA(p, Hp, cr, ci, sign, 1);
    }
}

void oracle_propagate_vector(const oracle_params *p, const float *H, void *cr, void *ci, int sign) {
    propagate_vector(p, H, (real *)cr, (real *)ci, sign);
}

/* propagate_t2_DIA (propagate.c:130-180) with matrix_on_vector,
 * vector_on_vector and trans_matrix_on_vector (NISE_subs.c:71-122):
 * one diagonalisation applied to nvec vectors (rows of cr/ci). */
static void prop_t2(const oracle_params *p, const float *Hp, real *cr, real *ci, int nvec) {
    int N = p->singles;
    real f = (real)p->deltat * (real)icm2ifs * (real)twoPi * 1;
    real *Hv = (real *)malloc(sizeof(real) * N * N), *e = (real *)malloc(sizeof(real) * N);
    real *re_U = (real *)malloc(sizeof(real) * N), *im_U = (real *)malloc(sizeof(real) * N);
    real *xr = (real *)malloc(sizeof(real) * N), *xi = (real *)malloc(sizeof(real) * N);
    diag_packed(Hp, N, Hv, e);
    for (int a = 0; a < N; a++) { re_U[a] = cos(e[a] * f); im_U[a] = -sin(e[a] * f); }
    for (int v = 0; v < nvec; v++) {
        real *vr = cr + (size_t)v * N, *vi = ci + (size_t)v * N;
        for (int a = 0; a < N; a++) {
            xr[a] = 0, xi[a] = 0;
            for (int b = 0; b < N; b++) { xr[a] += Hv[a + b * N] * vr[b]; xi[a] += Hv[a + b * N] * vi[b]; }
        }
        for (int a = 0; a < N; a++) {
            real re = re_U[a] * xr[a] - im_U[a] * xi[a];
            real im = im_U[a] * xr[a] + re_U[a] * xi[a];
            xr[a] = re, xi[a] = im;
        }
        for (int a = 0; a < N; a++) {
            vr[a] = 0, vi[a] = 0;
            for (int b = 0; b < N; b++) { vr[a] += Hv[b + a * N] * xr[b]; vi[a] += Hv[b + a * N] * xi[b]; }
        }
    }
    free(Hv); free(e); free(re_U); free(im_U); free(xr); free(xi);
}

void oracle_propagate_t2(const oracle_params *p, const float *H, void *cr, void *ci, int nvec) {
    prop_t2(p, H, (real *)cr, (real *)ci, nvec);
}

/* ------------------------------------------------------------------ */
/* Doubles (two-exciton) manifold                                      */

/* propagate_vec_coupling_S_doubles (propagate.c:902-1048); with es, the
 * two-level variant propagate_vec_coupling_S_doubles_ES (propagate.c:1051-1181):
 * no anharmonicity, no rotations of the c == a and c == b cases. */
static void prop_coupling_doubles(const oracle_params *p, const float *Hp, real *cr, real *ci, int m,
                                  const float *Anh, int es) {
    int N = p->singles, N2 = N * (N + 1) / 2;
    const real f = (real)p->deltat * (real)icm2ifs * (real)twoPi / m;
    real *H0 = (real *)malloc(sizeof(real) * N2);
    float *H1 = (float *)malloc(sizeof(float) * (N * N / 2 + 1));
    int *col = (int *)malloc(sizeof(int) * (N * N / 2 + 1)), *row = (int *)malloc(sizeof(int) * (N * N / 2 + 1));
    real *re_U = (real *)malloc(sizeof(real) * N2), *im_U = (real *)malloc(sizeof(real) * N2);
    real *ocr = (real *)malloc(sizeof(real) * N2), *oci = (real *)malloc(sizeof(real) * N2);
    for (int a = 0; a < N; a++) {
        int ia = Sindex(a, a, N);
        for (int b = a; b < N; b++) {
            int index = Sindex(a, b, N);
            H0[index] = (real)Hp[ia] + (real)Hp[Sindex(b, b, N)];
            if (a == b && !es) {
                if (p->anharmonicity == 0) H0[index] -= Anh[a];
                else H0[index] -= p->anharmonicity;
            }
        }
    }
    int kmax = 0;
    for (int a = 0; a < N; a++)
        for (int b = a + 1; b < N; b++) {
            int index = b + a * ((N << 1) - a - 1) / 2;
            if (fabsf(Hp[index]) > p->couplingcut) { H1[kmax] = Hp[index]; col[kmax] = a; row[kmax] = b; kmax++; }
        }
    for (int a = 0; a < N2; a++) {
        re_U[a] = RCOS((real)0.5f * H0[a] * f);
        im_U[a] = -RSIN((real)0.5f * H0[a] * f);
    }
    for (int i = 0; i < m; i++) {
        for (int a = 0; a < N2; a++) {
            ocr[a] = cr[a] * re_U[a] - ci[a] * im_U[a];
            oci[a] = cr[a] * im_U[a] + ci[a] * re_U[a];
        }
        for (int k = 0; k < kmax; k++) {
            int a = col[k], b = row[k], c = 0;
            real J = H1[k] * f;
            int aN = a * ((N << 1) - a - 1) / 2, bN = b * ((N << 1) - b - 1) / 2;
            real si = -RSIN(J), co = RSQRT(1 - si * si);
            real si2, co2;
#define ROT(i1, i2, CO, SI)                                                   \
    do {                                                                      \
        real cr1 = CO * ocr[i1] - SI * oci[i2];                               \
        real ci1 = CO * oci[i1] + SI * ocr[i2];                               \
        real cr2 = CO * ocr[i2] - SI * oci[i1];                               \
        real ci2 = CO * oci[i2] + SI * ocr[i1];                               \
        ocr[i1] = cr1, oci[i1] = ci1, ocr[i2] = cr2, oci[i2] = ci2;           \
    } while (0)
            for (; c < a; c++) ROT(a + c * ((N << 1) - c - 1) / 2, b + c * ((N << 1) - c - 1) / 2, co, si);
            si2 = -RSIN(J * sqrt2);
            co2 = RSQRT(1 - si2 * si2);
            for (; c == a; c++)
                if (!es) ROT(a + c * ((N << 1) - c - 1) / 2, b + c * ((N << 1) - c - 1) / 2, co2, si2);
            for (; c < b; c++) ROT(c + aN, b + c * ((N << 1) - c - 1) / 2, co, si);
            for (; c == b; c++)
                if (!es) ROT(c + aN, b + c * ((N << 1) - c - 1) / 2, co2, si2);
            for (; c < N; c++) ROT(c + aN, c + bN, co, si);
#undef ROT
        }
        for (int a = 0; a < N2; a++) {
            cr[a] = ocr[a] * re_U[a] - oci[a] * im_U[a];
            ci[a] = ocr[a] * im_U[a] + oci[a] * re_U[a];
        }
    }
    free(H0); free(H1); free(col); free(row); free(re_U); free(im_U); free(ocr); free(oci);
}

/* propagate_vec_RK4_doubles (propagate.c:376-590); with es the two-level
 * variant propagate_vec_RK4_doubles_ES (propagate.c:593-826): diagonal part
 * and update over |ab>, a < b, only; coupling terms with c == a or c == b
 * left out. */
static void prop_RK4_doubles(const oracle_params *p, const float *Hp, real *cr, real *ci, int m, const float *Anh,
                             int es) {
    int N = p->singles, N2 = N * (N + 1) / 2;
    real f = (real)p->deltat * (real)icm2ifs * (real)twoPi / m;
    real *H0 = (real *)malloc(sizeof(real) * N2), *HD = (real *)malloc(sizeof(real) * N2);
    int *col = (int *)malloc(sizeof(int) * N2), *row = (int *)malloc(sizeof(int) * N2);
    real *kr[4], *ki[4];
    for (int q = 0; q < 4; q++) { kr[q] = (real *)calloc(N2, sizeof(real)); ki[q] = (real *)calloc(N2, sizeof(real)); }
    char *isdiag = (char *)calloc(N2, 1);
    for (int a = 0; a < N; a++) isdiag[Sindex(a, a, N)] = 1;
    int kmax = 0;
    for (int a = 0; a < N; a++)
        for (int b = a + 1; b < N; b++) {
            int index = Sindex(a, b, N);
            if (fabs(Hp[index]) > p->couplingcut) { H0[kmax] = f * Hp[index]; col[kmax] = a, row[kmax] = b; kmax++; }
        }
    for (int a = 0; a < N; a++) {
        int ia = Sindex(a, a, N);
        for (int b = a; b < N; b++) {
            int index = Sindex(a, b, N);
            HD[index] = f * (Hp[ia] + Hp[Sindex(b, b, N)]);
            if (a == b && !es) {
                if (p->anharmonicity == 0) HD[index] -= Anh[a] * f;
                else HD[index] -= p->anharmonicity * f;
            }
        }
    }
    for (int i = 0; i < m; i++) {
        if (i > 0)
            for (int q = 0; q < 4; q++) { memset(kr[q], 0, sizeof(real) * N2); memset(ki[q], 0, sizeof(real) * N2); }
        for (int q = 0; q < 4; q++) {
            /* argument: c + s * k_{q-1}, s = 0, 0.5, 0.5, 1 */
            const real *pr = q ? kr[q - 1] : NULL, *pi = q ? ki[q - 1] : NULL;
            real *Kr = kr[q], *Ki = ki[q];
            for (int k = 0; k < N2; k++) {
                if (es && isdiag[k]) continue;
                if (q == 0) { Kr[k] += HD[k] * ci[k]; Ki[k] -= HD[k] * cr[k]; }
                else if (q < 3) { Kr[k] += HD[k] * (ci[k] + pi[k] * 0.5); Ki[k] -= HD[k] * (cr[k] + pr[k] * 0.5); }
                else { Kr[k] += HD[k] * (ci[k] + pi[k]); Ki[k] -= HD[k] * (cr[k] + pr[k]); }
            }
            for (int k = 0; k < kmax; k++) {
                int a = col[k], b = row[k];
                for (int c = 0; c < N; c++) {
                    if (es && (c == a || c == b)) continue;
                    int i1 = Sindex(a, c, N), i2 = Sindex(b, c, N);
                    float factor = 1.0;
                    if (c == a) factor = sqrt2;
                    if (b == c) factor = sqrt2;
                    if (q == 0) {
                        Kr[i1] += H0[k] * ci[i2] * factor; Ki[i1] -= H0[k] * cr[i2] * factor;
                        Kr[i2] += H0[k] * ci[i1] * factor; Ki[i2] -= H0[k] * cr[i1] * factor;
                    } else if (q < 3) {
                        Kr[i1] += H0[k] * (ci[i2] + pi[i2] * 0.5) * factor; Ki[i1] -= H0[k] * (cr[i2] + pr[i2] * 0.5) * factor;
                        Kr[i2] += H0[k] * (ci[i1] + pi[i1] * 0.5) * factor; Ki[i2] -= H0[k] * (cr[i1] + pr[i1] * 0.5) * factor;
                    } else {
                        Kr[i1] += H0[k] * (ci[i2] + pi[i2]) * factor; Ki[i1] -= H0[k] * (cr[i2] + pr[i2]) * factor;
                        Kr[i2] += H0[k] * (ci[i1] + pi[i1]) * factor; Ki[i2] -= H0[k] * (cr[i1] + pr[i1]) * factor;
                    }
                }
            }
        }
        real norm = find_norm(cr, ci, N2);
        for (int k = 0; k < N2; k++) {
            if (es && isdiag[k]) continue;
            cr[k] = cr[k] + (kr[0][k] + 2.0 * kr[1][k] + 2.0 * kr[2][k] + kr[3][k]) / 6.0;
            ci[k] = ci[k] + (ki[0][k] + 2.0 * ki[1][k] + 2.0 * ki[2][k] + ki[3][k]) / 6.0;
        }
        re_normalize(cr, ci, N2, norm);
    }
    free(H0); free(HD); free(col); free(row); free(isdiag);
    for (int q = 0; q < 4; q++) { free(kr[q]); free(ki[q]); }
}

/* time_evolution_mat (propagate.c:1241-1299): truncated one-sub-step U. */
static int time_evolution_mat(const oracle_params *p, const float *Hp, real *Ur, real *Ui, int *R, int *C, int m) {
    int N = p->singles;
    real f = (real)p->deltat * (real)icm2ifs * (real)twoPi / m;
    real *Hv = (real *)malloc(sizeof(real) * N * N), *e = (real *)malloc(sizeof(real) * N);
    real *cr = (real *)malloc(sizeof(real) * N * N), *ci = (real *)malloc(sizeof(real) * N * N);
    diag_packed(Hp, N, Hv, e);
    build_U(N, Hv, e, f, cr, ci);
    int elements = 0;
    for (int a = 0; a < N; a++)
        for (int b = 0; b < N; b++)
            if ((cr[a + b * N] * cr[a + b * N] + ci[a + b * N] * ci[a + b * N]) > p->thres) {
                Ur[elements] = cr[a + b * N], Ui[elements] = ci[a + b * N];
                R[elements] = a, C[elements] = b;
                elements++;
            }
    free(Hv); free(e); free(cr); free(ci);
    return elements;
}

/* propagate_double_sparce (propagate.c:1304-1394); with es the two-level
 * variant propagate_double_sparce_ES (propagate.c:1400-1473): plain copies
 * instead of the anharmonic phases, g = 0 where exactly one index differs. */
static void prop_double_sparse(const oracle_params *p, const real *Ur, const real *Ui, const int *R, const int *C,
                               real *fr, real *fi, int elements, int m, const float *Anh, int es) {
    int N = p->singles, Nf = N * (N + 1) / 2;
    real f = (real)p->deltat * (real)icm2ifs * (real)twoPi;
    real fm = f * 0.5 / m;
    real *vr = (real *)calloc(Nf, sizeof(real)), *vi = (real *)calloc(Nf, sizeof(real));
    real *co = (real *)calloc(N, sizeof(real)), *si = (real *)calloc(N, sizeof(real));
    for (int i = 0; i < N; i++) {
        if (es) { co[i] = 1, si[i] = 0; continue; }
        real an = p->anharmonicity != 0 ? (real)p->anharmonicity : (real)Anh[i];
        co[i] = cos(fm * an), si[i] = sin(fm * an);
    }
    for (int i = 0; i < m; i++) {
        memcpy(vr, fr, sizeof(real) * Nf);
        memcpy(vi, fi, sizeof(real) * Nf);
        for (int a = 0; a < N; a++) {
            int A = Sindex(a, a, N);
            if (es) { fr[A] = vr[A], fi[A] = vi[A]; continue; }
            fr[A] = co[a] * vr[A] - si[a] * vi[A];
            fi[A] = co[a] * vi[A] + si[a] * vr[A];
        }
        memset(vr, 0, sizeof(real) * Nf);
        memset(vi, 0, sizeof(real) * Nf);
        for (int a = 0; a < elements; a++) {
            int s = R[a], t = C[a];
            real Uar = Ur[a], Uai = Ui[a];
            for (int b = 0; b <= a; b++) {
                int u = R[b], v = C[b];
                real Ubr = Ur[b], Ubi = Ui[b];
                real g = 1;
                int iA = Sindex(s, u, N), iB = Sindex(t, v, N);
                if (s != u) g = es ? 0 : sqrt2;
                if (v != t) g = es ? 0 : sqrt2;
                if (s != u && v != t) g = 1;
                vr[iA] += (Uar * Ubr - Uai * Ubi) * fr[iB] * g;
                vr[iA] -= (Uai * Ubr + Uar * Ubi) * fi[iB] * g;
                vi[iA] += (Uar * Ubr - Uai * Ubi) * fi[iB] * g;
                vi[iA] += (Uai * Ubr + Uar * Ubi) * fr[iB] * g;
            }
        }
        memcpy(fr, vr, sizeof(real) * Nf);
        memcpy(fi, vi, sizeof(real) * Nf);
        for (int a = 0; a < N; a++) {
            int A = Sindex(a, a, N);
            if (es) { fr[A] = vr[A], fi[A] = vi[A]; continue; }
            fr[A] = co[a] * vr[A] - si[a] * vi[A];
            fi[A] = co[a] * vi[A] + si[a] * vr[A];
        }
    }
    free(vr); free(vi); free(co); free(si);
}

/* propagate_double_2DIR_control / propagate_double_2DES_control
 * (propagate.c:1476-1591, 1594-1710) for one vector: the UVvis techniques
 * (technique >= 6) take the two-level propagators. */
void oracle_propagate_doubles(const oracle_params *p, const float *H, void *cr, void *ci, const float *anh) {
    int N = p->singles, es = p->technique >= 6;
    if (p->propagation == 1) prop_coupling_doubles(p, H, (real *)cr, (real *)ci, p->ts, anh, es);
    else if (p->propagation == 3) prop_RK4_doubles(p, H, (real *)cr, (real *)ci, p->ts, anh, es);
    else {
        real *Ur = (real *)calloc((size_t)N * N, sizeof(real)), *Ui = (real *)calloc((size_t)N * N, sizeof(real));
        int *Rs = (int *)calloc((size_t)N * N, sizeof(int)), *Cs = (int *)calloc((size_t)N * N, sizeof(int));
        /* the reference passes (Cs, Rs) in swapped order (propagate.c:1495-1496) */
        int el = time_evolution_mat(p, H, Ur, Ui, Cs, Rs, p->ts);
        prop_double_sparse(p, Ur, Ui, Rs, Cs, (real *)cr, (real *)ci, el, p->ts, anh, es);
        free(Ur); free(Ui); free(Rs); free(Cs);
    }
}

/* dipole_double (NISE_subs.c:485-509). */
static void dipole_double(const oracle_params *p, const float *dipole, const real *cr, const real *ci, real *fr,
                          real *fi, float *over) {
    int n = p->singles, N = n * (n + 1) / 2;
    for (int i = 0; i < N; i++) fr[i] = 0, fi[i] = 0;
    if (p->anharmonicity != 0)
        for (int i = 0; i < n; i++) over[i] = sqrt2 * dipole[i];
    for (int i = 0; i < n; i++) {
        int index = Sindex(i, i, n);
        fr[index] += over[i] * cr[i];
        fi[index] += over[i] * ci[i];
        for (int j = i + 1; j < n; j++) {
            index = Sindex(i, j, n);
            fr[index] += dipole[i] * cr[j];
            fi[index] += dipole[i] * ci[j];
            fr[index] += dipole[j] * cr[i];
            fi[index] += dipole[j] * ci[i];
        }
    }
}

/* dipole_double_last (NISE_subs.c:552-575). */
static void dipole_double_last(const oracle_params *p, const float *dipole, const real *cr, const real *ci,
                               real *fr, real *fi, float *over) {
    int n = p->singles;
    for (int i = 0; i < n; i++) fr[i] = 0, fi[i] = 0;
    if (p->anharmonicity != 0)
        for (int i = 0; i < n; i++) over[i] = sqrt2 * dipole[i];
    for (int i = 0; i < n; i++) {
        int index = Sindex(i, i, n);
        fr[i] += over[i] * cr[index];
        fi[i] += over[i] * ci[index];
        for (int j = i + 1; j < n; j++) {
            index = Sindex(i, j, n);
            fr[j] += dipole[i] * cr[index];
            fi[j] += dipole[i] * ci[index];
            fr[i] += dipole[j] * cr[index];
            fi[i] += dipole[j] * ci[index];
        }
    }
}

/* dipole_double_ES (NISE_subs.c:533-548): no |aa> term. */
static void dipole_double_ES(const oracle_params *p, const float *dipole, const real *cr, const real *ci, real *fr,
                             real *fi) {
    int n = p->singles, N = n * (n + 1) / 2;
    for (int i = 0; i < N; i++) fr[i] = 0, fi[i] = 0;
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            int index = Sindex(i, j, n);
            fr[index] += dipole[i] * cr[j];
            fi[index] += dipole[i] * ci[j];
            fr[index] += dipole[j] * cr[i];
            fi[index] += dipole[j] * ci[i];
        }
}

/* dipole_double_last_ES (NISE_subs.c:578-592). */
static void dipole_double_last_ES(const oracle_params *p, const float *dipole, const real *cr, const real *ci,
                                  real *fr, real *fi) {
    int n = p->singles;
    for (int i = 0; i < n; i++) fr[i] = 0, fi[i] = 0;
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            int index = Sindex(i, j, n);
            fr[j] += dipole[i] * cr[index];
            fi[j] += dipole[i] * ci[index];
            fr[i] += dipole[j] * cr[index];
            fi[i] += dipole[j] * ci[index];
        }
}

void oracle_dipole_double(const oracle_params *p, const float *dipole, const void *cr, const void *ci, void *fr,
                          void *fi, float *over) {
    dipole_double(p, dipole, (const real *)cr, (const real *)ci, (real *)fr, (real *)fi, over);
}
void oracle_dipole_double_last(const oracle_params *p, const float *dipole, const void *cr, const void *ci,
                               void *fr, void *fi, float *over) {
    dipole_double_last(p, dipole, (const real *)cr, (const real *)ci, (real *)fr, (real *)fi, over);
}

/* ------------------------------------------------------------------ */
/* Linear absorption (absorption.c:18-202, calc_S1 :205-212).          */
int oracle_absorption(const oracle_params *p, double *re_out, double *im_out, int *samples_out) {
    int N = p->singles;
    float shift1 = (p->max1 + p->min1) / 2;
    traj_t t;
    if (traj_open(&t, p, shift1, 0) != 0) { traj_free(&t); return -1; }
    int N_samples = (p->length - p->tmax1 - 1) / p->sample + 1; /* determine_samples, NISE_subs.c:197-221 */
    if (N_samples <= 0) { traj_free(&t); return -2; }
    int end = p->end == 0 ? N_samples : p->end;
    if (end > N_samples) { traj_free(&t); return -3; }
    int tmax = p->tmax1;
    acc *re_S = (acc *)calloc(tmax, sizeof(acc)), *im_S = (acc *)calloc(tmax, sizeof(acc));
    float *H = ham_alloc(&t), *mu = (float *)malloc(sizeof(float) * N);
    real *vr = (real *)malloc(sizeof(real) * N), *vi = (real *)malloc(sizeof(real) * N);
    float *mu0 = (float *)malloc(sizeof(float) * N);
    int rc = 0, samples;
    for (samples = p->begin; samples < end && rc == 0; samples++) {
        int ti = samples * p->sample;
        for (int x = 0; x < 3 && rc == 0; x++) {
            if (!mu_read(&t, mu0, ti, x)) { rc = -4; break; }
            for (int i = 0; i < N; i++) vr[i] = mu0[i], vi[i] = 0;
            for (int t1 = 0; t1 < tmax; t1++) {
                int tj = ti + t1;
                if (!read_He(&t, H, tj)) { rc = -5; break; }
                apply_singleshift(&t, H);
                if (!mu_read(&t, mu, tj, x)) { rc = -4; break; }
                for (int i = 0; i < N; i++) {
                    re_S[t1] += mu[i] * vr[i];
                    im_S[t1] += mu[i] * vi[i];
                }
                propagate_vector(p, H, vr, vi, 1);
            }
        }
    }
    for (int i = 0; i < tmax; i++) re_out[i] = re_S[i], im_out[i] = im_S[i];
    *samples_out = samples;
    free(re_S); free(im_S); free(H); free(mu); free(vr); free(vi); free(mu0);
    traj_free(&t);
    return rc;
}

/* Linear techniques besides absorption: the sample loops of LD
 * (calc_LD.c:149-220, calc_LD :286-296), Raman (raman.c:139-226, :293-310),
 * SFG (sfg.c:143-205, :281-298), DOS (calc_DOS.c:120-172, :225-234) and CD
 * (calc_CD.c:172-327, :381-392), each with its own read-outs and channels.
 * LD, Raman, DOS and CD read frames with read_He (no SingleShift); SFG with
 * read_Hamiltonian.  SFG's x and y start vectors have no read-out and are not
 * propagated here. */
/* Boltzmann weighting of a luminescence initial vector by the equilibrium
 * density matrix of the packed Hamiltonian H (luminescence.c:246-314,
 * bltz_weight): v <- rho v, rho = V exp(-E/kT) V^T / Q, the products in the
 * reference's loop order.  Q is summed from zero (the reference leaves it
 * uninitialised, luminescence.c:262,277).  FP64 eigendecomposition in place
 * of ssyev_. */
static void lum_weight_exact(const oracle_params *p, const float *H, real *v) {
    const int N = p->singles;
    real *Hv = (real *)malloc(sizeof(real) * N * N), *e = (real *)malloc(sizeof(real) * N);
    real *c2 = (real *)malloc(sizeof(real) * N), *c1 = (real *)calloc(N, sizeof(real));
    real *cnr = (real *)calloc((size_t)N * N, sizeof(real)), *crr = (real *)calloc((size_t)N * N, sizeof(real));
    diag_packed(H, N, Hv, e);
    const float kBT = p->temperature * 0.695;  /* Kelvin to cm^-1 */
    real Q = 0;
    for (int a = 0; a < N; a++) {
        c2[a] = (real)exp(-e[a] / kBT);
        Q = Q + c2[a];
    }
    const real iQ = (real)(1.0 / Q);
    for (int a = 0; a < N; a++)
        for (int b = 0; b < N; b++) cnr[b + a * N] += Hv[b + a * N] * c2[b] * iQ;
    for (int a = 0; a < N; a++)
        for (int b = 0; b < N; b++)
            for (int c = 0; c < N; c++) crr[a + c * N] += Hv[b + a * N] * cnr[b + c * N];
    for (int a = 0; a < N; a++)
        for (int b = 0; b < N; b++) c1[a] += crr[a + b * N] * v[b];
    for (int a = 0; a < N; a++) v[a] = c1[a];
    free(Hv); free(e); free(c2); free(c1); free(cnr); free(crr);
}

/* The same weighting by m imaginary-time Trotter steps (luminescence.c:318-
 * 409, bltz_weight_itime): per step the diagonal half-factors
 * exp(-H_aa f/2), the couplings |J| > Couplingcut in lexicographic order as
 * (cosh, -sinh) pairs of J f, the half-factors again; f = 1/(m kT); then
 * the vector is scaled back to its initial norm. */
static void lum_weight_itime(const oracle_params *p, const float *H, real *cr) {
    const int N = p->singles, m = p->imag_steps;
    const float kBT = p->temperature * 0.695;
    const real f = (real)(1.0 / (m * kBT));  /* float in the reference, real here */
    real *reU = (real *)malloc(sizeof(real) * N), *ocr = (real *)malloc(sizeof(real) * N);
    real norm = 0, Q = 0;
    for (int a = 0; a < N; a++) norm += cr[a] * cr[a];
    for (int a = 0; a < N; a++) reU[a] = (real)exp(-0.5 * H[Sindex(a, a, N)] * f);
    for (int i = 0; i < m; i++) {
        for (int a = 0; a < N; a++) ocr[a] = cr[a] * reU[a];
        for (int a = 0; a < N; a++)
            for (int b = a + 1; b < N; b++) {
                real J = H[Sindex(a, b, N)];
                if (!(fabs(J) > p->couplingcut)) continue;
                J = -J * f;
                const real eJ = (real)(exp(J) * 0.5), emJ = (real)(exp(-J) * 0.5);
                const real sih = eJ - emJ, coh = eJ + emJ;
                const real r1 = coh * ocr[a] + sih * ocr[b], r2 = coh * ocr[b] + sih * ocr[a];
                ocr[a] = r1, ocr[b] = r2;
            }
        for (int a = 0; a < N; a++) cr[a] = ocr[a] * reU[a];
    }
    for (int a = 0; a < N; a++) Q += cr[a] * cr[a];
    const real iQ = (real)sqrt(norm / Q);
    for (int a = 0; a < N; a++) cr[a] = cr[a] * iQ;
    free(reU); free(ocr);
}

int oracle_linear(const oracle_params *p, double *re_out, double *im_out, int *nch_out, int *samples_out) {
    const int N = p->singles, tech = p->technique, tmax = p->tmax1;
    if (tech < 11 || tech > 16) return -6;
    float shift1 = (p->max1 + p->min1) / 2;
    traj_t t;
    if (traj_open(&t, p, shift1, 0) != 0) { traj_free(&t); return -1; }
    int N_samples = (p->length - p->tmax1 - 1) / p->sample + 1;
    if (N_samples <= 0) { traj_free(&t); return -2; }
    int end = p->end == 0 ? N_samples : p->end;
    if (end > N_samples) { traj_free(&t); return -3; }
    const int nch = (tech == 12 || tech == 13) ? 2 : (tech == 16 ? 4 : 1);  /* Luminescence: total, x, y, z */
    const int nvec = tech == 14 ? N : (tech == 15 ? N : 1);  /* vectors propagated together */
    acc *S = (acc *)calloc(2 * (size_t)nch * tmax, sizeof(acc));   /* [ch][re/im][t1] */
    acc *Sj = (acc *)calloc(2 * (size_t)N * tmax, sizeof(acc));    /* CD: per initial site */
    float *H = ham_alloc(&t), *mu = (float *)malloc(sizeof(float) * N), *op = (float *)malloc(sizeof(float) * N);
    float *pos = (float *)malloc(sizeof(float) * N), *pos0 = (float *)malloc(sizeof(float) * 3 * N);
    real *vr = (real *)calloc((size_t)nvec * N, sizeof(real)), *vi = (real *)calloc((size_t)nvec * N, sizeof(real));
    int rc = 0, samples;
#define SRE(ch, t1) S[(2 * (size_t)(ch)) * tmax + (t1)]
#define SIM(ch, t1) S[(2 * (size_t)(ch) + 1) * tmax + (t1)]
    if (tech == 15 && p->ham_coupling)  /* static positions of frame 0 (calc_CD.c:164-170) */
        for (int x = 0; x < 3; x++)
            if (!read_mue(&t, t.P, t.nP, pos0 + N * x, 0, x)) rc = -4;
    const int nx = tech == 12 ? 6 : (tech == 13 || tech == 14 ? 1 : 3);
    for (samples = p->begin; samples < end && rc == 0; samples++) {
        const int ti = samples * p->sample;
        for (int x = 0; x < nx && rc == 0; x++) {
            /* initial vectors */
            memset(vr, 0, sizeof(real) * nvec * N);
            memset(vi, 0, sizeof(real) * nvec * N);
            if (tech == 11 || tech == 13) {        /* mu_x(ti); SFG: mu_z */
                if (!mu_read(&t, mu, ti, tech == 13 ? 2 : x)) { rc = -4; break; }
                for (int i = 0; i < N; i++) vr[i] = mu[i];
            } else if (tech == 12) {               /* alpha_x(ti) */
                if (!read_alpha(&t, op, ti, x)) { rc = -4; break; }
                for (int i = 0; i < N; i++) vr[i] = op[i];
            } else if (tech == 16) {               /* mu_x(ti) weighted by the Hamiltonian read last */
                if (!mu_read(&t, mu, ti, x)) { rc = -4; break; }
                for (int i = 0; i < N; i++) vr[i] = mu[i];
                if (p->imag_steps == 0) lum_weight_exact(p, H, vr);
                else lum_weight_itime(p, H, vr);
            } else if (tech == 14) {               /* unitmat */
                for (int j = 0; j < N; j++) vr[(size_t)j * N + j] = 1;
            } else {                               /* CD: mu_x(ti)_j on site j */
                if (!mu_read(&t, mu, ti, x)) { rc = -4; break; }
                for (int j = 0; j < N; j++) vr[(size_t)j * N + j] = mu[j];
            }
            for (int t1 = 0; t1 < tmax; t1++) {
                const int tj = ti + t1;
                if (!read_He(&t, H, tj)) { rc = -5; break; }
                if (tech == 13 || tech == 16) apply_singleshift(&t, H);  /* read_Hamiltonian */
                if (tech == 11) {
                    if (!mu_read(&t, mu, tj, x)) { rc = -4; break; }
                    float factor = x == 2 ? 1 : -0.5;
                    for (int i = 0; i < N; i++) {
                        SRE(0, t1) += mu[i] * vr[i] * factor;
                        SIM(0, t1) += mu[i] * vi[i] * factor;
                    }
                } else if (tech == 12) {
                    if (!read_alpha(&t, op, tj, x)) { rc = -4; break; }
                    if (x == 0 || x == 3 || x == 5)
                        for (int i = 0; i < N; i++) { SRE(0, t1) += op[i] * vr[i]; SIM(0, t1) += op[i] * vi[i]; }
                    else
                        for (int i = 0; i < N; i++) { SRE(1, t1) += 2 * op[i] * vr[i]; SIM(1, t1) += 2 * op[i] * vi[i]; }
                } else if (tech == 13) {
                    for (int xa = 0; xa < 6; xa++) {
                        if (!read_alpha(&t, op, tj, xa)) { rc = -4; break; }
                        if (xa == 5)
                            for (int i = 0; i < N; i++) { SRE(0, t1) += op[i] * vr[i]; SIM(0, t1) += op[i] * vi[i]; }
                        if (xa == 0 || xa == 3)
                            for (int i = 0; i < N; i++) {
                                SRE(1, t1) += op[i] * vr[i] / 2;
                                SIM(1, t1) += op[i] * vi[i] / 2;
                            }
                    }
                    if (rc) break;
                } else if (tech == 16) {  /* calc_LUM: the total and component x's channel */
                    if (!mu_read(&t, mu, tj, x)) { rc = -4; break; }
                    for (int i = 0; i < N; i++) {
                        SRE(0, t1) += mu[i] * vr[i];
                        SIM(0, t1) += mu[i] * vi[i];
                    }
                    for (int i = 0; i < N; i++) {
                        SRE(1 + x, t1) += mu[i] * vr[i];
                        SIM(1 + x, t1) += mu[i] * vi[i];
                    }
                } else if (tech == 14) {
                    for (int i = 0; i < N; i++) {
                        SRE(0, t1) += vr[(size_t)i * N + i];
                        SIM(0, t1) += vi[(size_t)i * N + i];
                    }
                } else {
                    for (int y = 0; y < 3; y++) {
                        if (y == x) continue;
                        int z = 3 - x - y, sign = 0;
                        if (z == 0 && y == 1 && x == 2) sign = 1;
                        if (z == 0 && y == 2 && x == 1) sign = -1;
                        if (z == 1 && y == 0 && x == 2) sign = -1;
                        if (z == 2 && y == 0 && x == 1) sign = 1;
                        if (z == 2 && y == 1 && x == 0) sign = -1;
                        if (z == 1 && y == 2 && x == 0) sign = 1;
                        /* static dipoles: the reference copies component x (calc_CD.c:250) */
                        if (!mu_read(&t, mu, tj, p->ham_coupling ? x : y)) { rc = -4; break; }
                        if (p->ham_coupling) memcpy(pos, pos0 + N * z, sizeof(float) * N);
                        else if (!read_mue(&t, t.P, t.nP, pos, tj, z)) { rc = -4; break; }
                        for (int j = 0; j < N; j++)
                            for (int i = 0; i < N; i++) {
                                Sj[(size_t)j * tmax + t1] += sign * (pos[i] - pos[j]) * mu[i] * vr[(size_t)j * N + i];
                                Sj[((size_t)N + j) * tmax + t1] += sign * (pos[i] - pos[j]) * mu[i] * vi[(size_t)j * N + i];
                            }
                    }
                    if (rc) break;
                }
                for (int v = 0; v < nvec; v++) propagate_vector(p, H, vr + (size_t)v * N, vi + (size_t)v * N, 1);
            }
        }
    }
    if (tech == 15)  /* sum over the initial sites (calc_CD.c:334-342) */
        for (int t1 = 0; t1 < tmax; t1++)
            for (int j = 0; j < N; j++) {
                SRE(0, t1) += Sj[(size_t)j * tmax + t1];
                SIM(0, t1) += Sj[((size_t)N + j) * tmax + t1];
            }
    for (int ch = 0; ch < nch; ch++)
        for (int t1 = 0; t1 < tmax; t1++) {
            re_out[(size_t)ch * tmax + t1] = SRE(ch, t1);
            im_out[(size_t)ch * tmax + t1] = SIM(ch, t1);
        }
#undef SRE
#undef SIM
    *nch_out = nch;
    *samples_out = samples;
    free(S); free(Sj); free(H); free(mu); free(op); free(pos); free(pos0); free(vr); free(vi);
    traj_free(&t);
    return rc;
}

/* 1D FFT and output axis (1DFFT.c:144-228), DFT in FP64. */
int oracle_1dfft(const oracle_params *p, const double *re_S, const double *im_S, int samples, double *freq,
                 double *spec_re, double *spec_im, int max_rows) {
    float shift1 = (p->max1 + p->min1) / 2;
    int fft = p->fft < p->tmax1 ? p->tmax1 : p->fft;
    int tmax = p->tmax1;
    double *in = (double *)calloc(2 * (size_t)fft, sizeof(double));
    double *out = (double *)calloc(2 * (size_t)fft, sizeof(double));
    real *spr = (real *)calloc(fft, sizeof(real)), *spi = (real *)calloc(fft, sizeof(real));
    for (int i = 0; i < tmax; i++) {
        in[2 * i] = (acc)im_S[i] / samples;
        in[2 * i + 1] = (acc)re_S[i] / samples;
        if (p->lifetime > 0.0) {
            double d = exp((real)(-i) * (real)p->deltat / (2 * (real)p->lifetime));
            in[2 * i] *= d; in[2 * i + 1] *= d;
        }
        if (p->homogen > 0.0) {
            double d = exp((real)(-i) * (real)p->deltat / (2 * (real)p->homogen));
            in[2 * i] *= d; in[2 * i + 1] *= d;
        }
        if (p->inhomogen > 0.0) {
            double d = exp((real)(-i) * (real)p->deltat * i * (real)p->deltat /
                           (2 * (real)p->inhomogen * (real)p->inhomogen));
            in[2 * i] *= d; in[2 * i + 1] *= d;
        }
        if (p->window == 1) {
            double w = cos(i * (real)twoPi / (4 * tmax - 4)) * cos(i * (real)twoPi / (4 * tmax - 4));
            in[2 * i] *= w; in[2 * i + 1] *= w;
        }
    }
    in[0] *= 0.5;
    in[1] *= 0.5;
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < fft; k++) {
        long double sr = 0, si = 0;
        for (int j = 0; j < fft; j++) {
            long double a = -2.0L * pi * (long double)(((long)j * k) % fft) / fft;
            long double c = cosl(a), s = sinl(a);
            sr += in[2 * j] * c - in[2 * j + 1] * s;
            si += in[2 * j] * s + in[2 * j + 1] * c;
        }
        out[2 * k] = (double)sr, out[2 * k + 1] = (double)si;
    }
    for (int i = 0; i < fft; i++) {
        spr[i] = out[2 * i + 1] * 2 * (real)p->deltat * (real)c_v;
        spi[i] = out[2 * i] * 2 * (real)p->deltat * (real)c_v;
    }
    int rows = 0;
    for (int i = fft / 2; i <= fft - 1; i++) {
        real w = -((fft - i) / (real)p->deltat / (real)c_v / fft - (real)shift1);
        if (w > p->min1 && w < p->max1 && rows < max_rows) {
            freq[rows] = w; spec_re[rows] = spr[i]; spec_im[rows] = spi[i]; rows++;
        }
    }
    for (int i = 0; i <= fft / 2 - 1; i++) {
        real w = -((-i) / (real)p->deltat / (real)c_v / fft - (real)shift1);
        if (w > p->min1 && w < p->max1 && rows < max_rows) {
            freq[rows] = w; spec_re[rows] = spr[i]; spec_im[rows] = spi[i]; rows++;
        }
    }
    free(in); free(out); free(spr); free(spi);
    return rows;
}

/* ------------------------------------------------------------------ */
/* 2DIR (calc_2DIR.c:22-629), polar.c:12-105, print2D MPI_subs.c:20-34  */

static float polarweight(int pol, int x) {
    float weight = 0;
    if (pol == 0) {
        if (x <= 2) weight = 6 * ithirty;
        if (x >= 3) weight = 2 * ithirty;
    }
    if (pol == 1) {
        if (x <= 2) weight = 2 * ithirty;
        if (x >= 3 && x <= 8) weight = 4 * ithirty;
        if (x >= 9) weight = -1 * ithirty;
    }
    if (pol == 2) {
        if (x <= 2) weight = 0.0;
        if (x >= 3 && x <= 8) weight = 0.0;
        if (x >= 9 && x <= 14) weight = 2.5 * ithirty;
        if (x >= 15) weight = -2.5 * ithirty;
    }
    return weight;
}

static void polar(int xp[4], int x) {
    static const int tab[21][4] = {
        {0, 0, 0, 0}, {1, 1, 1, 1}, {2, 2, 2, 2}, {0, 0, 1, 1}, {0, 0, 2, 2}, {1, 1, 0, 0}, {1, 1, 2, 2},
        {2, 2, 0, 0}, {2, 2, 1, 1}, {0, 1, 0, 1}, {0, 2, 0, 2}, {1, 0, 1, 0}, {1, 2, 1, 2}, {2, 0, 2, 0},
        {2, 1, 2, 1}, {0, 1, 1, 0}, {0, 2, 2, 0}, {1, 0, 0, 1}, {1, 2, 2, 1}, {2, 0, 0, 2}, {2, 1, 1, 2}};
    for (int i = 0; i < 4; i++) xp[i] = tab[x][i];
}

void oracle_print2d_normalize(const oracle_params *p, double *re, double *im, int sample_count) {
    for (int t1 = 0; t1 < p->tmax1; t1++)
        for (int t3 = 0; t3 < p->tmax3; t3++) {
            acc r = (acc)re[t3 * p->tmax1 + t1], i = (acc)im[t3 * p->tmax1 + t1];
            r /= sample_count;
            i /= sample_count;
            if (t3 == 0) r /= 2, i /= 2;
            re[t3 * p->tmax1 + t1] = r, im[t3 * p->tmax1 + t1] = i;
        }
}

/* calc_2DIR (calc_2DIR.c:22-629); for the UVvis techniques 6-10 calc_2DES
 * (calc_2DES.c:22-586), which differs only in the doubles operators and
 * propagators (dipole_double_ES, dipole_double_last_ES, the _ES propagators)
 * and in reading no anharmonicity or overtone files. */
int oracle_2dir(const oracle_params *p, double *Rout, int *sample_count) {
    int N = p->singles, nn2 = N * (N + 1) / 2, T1 = p->tmax1, T3 = p->tmax3;
    int tech = p->technique, es = tech >= 6;
    if (es) tech -= 5; /* 2DUVvis GBUVvis SEUVvis EAUVvis noEAUVvis -> 2DIR ... noEAIR */
    int do_gb = (tech == 1 || tech == 2 || tech == 5), do_se = (tech == 1 || tech == 3 || tech == 5);
    int do_ea = (tech == 1 || tech == 4);
    float shift1 = (p->max1 + p->min1) / 2;
    traj_t t;
    int need_anh = (p->anharmonicity == 0 && !es && (tech >= 1 && tech <= 5));
    if (traj_open(&t, p, shift1, need_anh) != 0) { traj_free(&t); return -1; }
    /* calculateWorkset (MPI_subs.c:36-110) */
    int total = (p->length - p->tmax1 - p->tmax2 - p->tmax3 - 1) / p->sample + 1;
    if (total <= 0) { traj_free(&t); return -2; }
    int end = p->end == 0 ? total : p->end;
    int sc = end - p->begin;
    if (sc == 0) sc = 1;
    *sample_count = sc;

    acc *R = (acc *)calloc(12 * (size_t)T3 * T1, sizeof(acc));
#define RA(k, t3, t1) R[((size_t)(k) * T3 + (t3)) * T1 + (t1)]
    float *lt = (float *)malloc(sizeof(float) * T3 * T1);
    for (int t1 = 0; t1 < T1; t1++)
        for (int t3 = 0; t3 < T3; t3++)
            lt[t3 * T1 + t1] = p->lifetime > 0
                                   ? (float)exp(-(double)(t1 + t3) * p->deltat / (2 * p->lifetime))
                                   : 1.0f;
    float *H = ham_alloc(&t);
    float *Anh = (float *)calloc(N, sizeof(float)), *over = (float *)calloc(N, sizeof(float));
    real *leftrr = (real *)calloc(N, sizeof(real)), *leftri = (real *)calloc(N, sizeof(real));
    real *leftnr = (real *)calloc((size_t)T1 * N, sizeof(real)), *leftni = (real *)calloc((size_t)T1 * N, sizeof(real));
    real *rightrr = (real *)calloc((size_t)T1 * N, sizeof(real)), *rightri = (real *)calloc((size_t)T1 * N, sizeof(real));
    real *rightnr = (real *)calloc(N, sizeof(real)), *rightni = (real *)calloc(N, sizeof(real));
    float *mut2 = (float *)calloc(N, sizeof(float)), *mut4 = (float *)calloc(N, sizeof(float));
    float *mtmp = (float *)calloc(N, sizeof(float));
    real *mut3r = (real *)calloc(N, sizeof(real)), *mut3i = (real *)calloc(N, sizeof(real));
    real *fr = (real *)calloc(nn2, sizeof(real)), *fi = (real *)calloc(nn2, sizeof(real));
    real *ft1r = (real *)calloc((size_t)T1 * nn2, sizeof(real)), *ft1i = (real *)calloc((size_t)T1 * nn2, sizeof(real));
    acc *t1nr = (acc *)calloc(T1, sizeof(acc)), *t1ni = (acc *)calloc(T1, sizeof(acc));
    acc *t1rr = (acc *)calloc(T1, sizeof(acc)), *t1ri = (acc *)calloc(T1, sizeof(acc));
    int rc = 0;
#define CHK(x) do { if (!(x)) { rc = -5; goto done; } } while (0)
    for (int s = p->begin; s < end; s++) {
        for (int molPol = 0; molPol < 21; molPol++) {
            int tj = s * p->sample + p->tmax1, tk = tj + p->tmax2, px[4];
            polar(px, molPol);
            float w0 = polarweight(0, molPol), w1 = polarweight(1, molPol), w2 = polarweight(2, molPol);
            CHK(mu_read(&t, mut2, tj, px[1]));
            /* GB: t1 vectors (calc_2DIR.c:214-239) */
            for (int t1 = 0; t1 < T1; t1++) {
                CHK(mu_read(&t, mtmp, tj - t1, px[0]));
                for (int i = 0; i < N; i++) leftnr[t1 * N + i] = mtmp[i], leftni[t1 * N + i] = 0;
                for (int tm = 0; tm < t1; tm++) {
                    CHK(read_He(&t, H, tj - t1 + tm));
                    propagate_vector(p, H, leftnr + t1 * N, leftni + t1 * N, 1);
                }
            }
            for (int t1 = 0; t1 < T1; t1++) {
                t1nr[t1] = 0, t1ni[t1] = 0;
                for (int i = 0; i < N; i++) {
                    t1nr[t1] += mut2[i] * leftnr[t1 * N + i];
                    t1ni[t1] += mut2[i] * leftni[t1 * N + i];
                }
            }
            /* GB: t3 (calc_2DIR.c:255-299) */
            CHK(mu_read(&t, mtmp, tk, px[2]));
            for (int i = 0; i < N; i++) mut3r[i] = mtmp[i], mut3i[i] = 0;
            for (int t3 = 0; t3 < T3; t3++) {
                int tl = tk + t3;
                CHK(mu_read(&t, mut4, tl, px[3]));
                if (do_gb) {
                    acc t3nr = 0, t3ni = 0;
                    for (int i = 0; i < N; i++) { t3nr += mut4[i] * mut3r[i]; t3ni += mut4[i] * mut3i[i]; }
                    for (int t1 = 0; t1 < T1; t1++) {
                        float lw = lt[t3 * T1 + t1];
                        float pw[3] = {w0 * lw, w1 * lw, w2 * lw};
                        for (int q = 0; q < 3; q++) {
                            RA(4 * q + 0, t3, t1) -= (t3ni * t1nr[t1] - t3nr * t1ni[t1]) * pw[q];
                            RA(4 * q + 1, t3, t1) -= (t3nr * t1nr[t1] + t3ni * t1ni[t1]) * pw[q];
                            RA(4 * q + 2, t3, t1) -= (t3ni * t1nr[t1] + t3nr * t1ni[t1]) * pw[q];
                            RA(4 * q + 3, t3, t1) -= (t3nr * t1nr[t1] - t3ni * t1ni[t1]) * pw[q];
                        }
                    }
                }
                CHK(read_He(&t, H, tl));
                propagate_vector(p, H, mut3r, mut3i, 1);
            }
            /* SE: t2 (calc_2DIR.c:303-326) */
            CHK(mu_read(&t, mtmp, tj, px[1]));
            for (int i = 0; i < N; i++) leftrr[i] = mtmp[i], leftri[i] = 0;
            for (int t2 = 0; t2 < p->tmax2; t2++) {
                CHK(read_He(&t, H, tj + t2));
                prop_t2(p, H, leftrr, leftri, 1);
                prop_t2(p, H, leftnr, leftni, T1);
            }
            CHK(mu_read(&t, mtmp, tk, px[2]));
            for (int i = 0; i < N; i++) mut3r[i] = mtmp[i];
            if (do_ea) { /* calc_2DIR.c:331-348 */
                if (es) {
                    dipole_double_ES(p, mtmp, leftrr, leftri, fr, fi);
                    for (int t1 = 0; t1 < T1; t1++)
                        dipole_double_ES(p, mtmp, leftnr + t1 * N, leftni + t1 * N, ft1r + (size_t)t1 * nn2,
                                         ft1i + (size_t)t1 * nn2);
                } else {
                    if (p->anharmonicity == 0) CHK(read_over(&t, over, tk, px[2]));
                    dipole_double(p, mtmp, leftrr, leftri, fr, fi, over);
                    for (int t1 = 0; t1 < T1; t1++)
                        dipole_double(p, mtmp, leftnr + t1 * N, leftni + t1 * N, ft1r + (size_t)t1 * nn2,
                                      ft1i + (size_t)t1 * nn2, over);
                }
                for (int i = 0; i < T1 * N; i++) rightrr[i] = leftnr[i], rightri[i] = -leftni[i];
                for (int i = 0; i < N; i++) rightnr[i] = leftrr[i], rightni[i] = -leftri[i];
            }
            for (int i = 0; i < N; i++) mut3i[i] = 0;
            acc t3nr = 0, t3ni = 0;
            for (int i = 0; i < N; i++) { t3nr += leftrr[i] * mut3r[i]; t3ni -= leftri[i] * mut3r[i]; }
            for (int t1 = 0; t1 < T1; t1++) {
                t1rr[t1] = 0, t1ri[t1] = 0;
                for (int i = 0; i < N; i++) {
                    t1rr[t1] += leftnr[t1 * N + i] * mut3r[i];
                    t1ri[t1] -= leftni[t1 * N + i] * mut3r[i];
                }
            }
            /* SE: t3 (calc_2DIR.c:372-443) */
            for (int t3 = 0; t3 < T3; t3++) {
                int tl = tk + t3;
                CHK(mu_read(&t, mut4, tl, px[3]));
                acc t3rr = 0, t3ri = 0;
                for (int i = 0; i < N; i++) { t3rr += mut4[i] * leftrr[i]; t3ri += mut4[i] * leftri[i]; }
                for (int t1 = 0; t1 < T1; t1++) {
                    t1nr[t1] = 0, t1ni[t1] = 0;
                    for (int i = 0; i < N; i++) {
                        t1nr[t1] += leftnr[t1 * N + i] * mut4[i];
                        t1ni[t1] += leftni[t1 * N + i] * mut4[i];
                    }
                }
                if (do_se)
                    for (int t1 = 0; t1 < T1; t1++) {
                        float lw = lt[t3 * T1 + t1];
                        float pw[3] = {w0 * lw, w1 * lw, w2 * lw};
                        for (int q = 0; q < 3; q++) {
                            RA(4 * q + 0, t3, t1) -= (t3rr * t1ri[t1] + t3ri * t1rr[t1]) * pw[q];
                            RA(4 * q + 1, t3, t1) -= (t3rr * t1rr[t1] - t3ri * t1ri[t1]) * pw[q];
                            RA(4 * q + 2, t3, t1) -= (t3ni * t1nr[t1] + t3nr * t1ni[t1]) * pw[q];
                            RA(4 * q + 3, t3, t1) -= (t3nr * t1nr[t1] - t3ni * t1ni[t1]) * pw[q];
                        }
                    }
                CHK(read_He(&t, H, tl));
                propagate_vector(p, H, leftrr, leftri, 1);
                for (int t1 = 0; t1 < T1; t1++) propagate_vector(p, H, leftnr + t1 * N, leftni + t1 * N, 1);
            }
            /* EA (calc_2DIR.c:445-506) */
            if (do_ea)
                for (int t3 = 0; t3 < T3; t3++) {
                    int tl = tk + t3;
                    CHK(mu_read(&t, mut4, tl, px[3]));
                    if (es) {
                        dipole_double_last_ES(p, mut4, fr, fi, leftrr, leftri);
                        for (int t1 = 0; t1 < T1; t1++)
                            dipole_double_last_ES(p, mut4, ft1r + (size_t)t1 * nn2, ft1i + (size_t)t1 * nn2,
                                                  leftnr + t1 * N, leftni + t1 * N);
                    } else {
                        if (p->anharmonicity == 0) CHK(read_over(&t, over, tl, px[3]));
                        dipole_double_last(p, mut4, fr, fi, leftrr, leftri, over);
                        for (int t1 = 0; t1 < T1; t1++)
                            dipole_double_last(p, mut4, ft1r + (size_t)t1 * nn2, ft1i + (size_t)t1 * nn2,
                                               leftnr + t1 * N, leftni + t1 * N, over);
                    }
                    for (int t1 = 0; t1 < T1; t1++) {
                        acc rrI = 0, riI = 0, rrII = 0, riII = 0;
                        const real *Rr = rightrr + t1 * N, *Ri = rightri + t1 * N;
                        const real *Lr = leftnr + t1 * N, *Li = leftni + t1 * N;
                        for (int i = 0; i < N; i++) {
                            rrI += leftri[i] * Rr[i] + leftrr[i] * Ri[i];
                            riI += leftrr[i] * Rr[i] - Ri[i] * leftri[i];
                            rrII += rightnr[i] * Li[i] + rightni[i] * Lr[i];
                            riII += rightnr[i] * Lr[i] - rightni[i] * Li[i];
                        }
                        float lw = lt[t3 * T1 + t1];
                        float pw[3] = {w0 * lw, w1 * lw, w2 * lw};
                        for (int q = 0; q < 3; q++) {
                            RA(4 * q + 0, t3, t1) += rrI * pw[q];
                            RA(4 * q + 1, t3, t1) += riI * pw[q];
                            RA(4 * q + 2, t3, t1) += rrII * pw[q];
                            RA(4 * q + 3, t3, t1) += riII * pw[q];
                        }
                    }
                    CHK(read_He(&t, H, tl));
                    if (p->anharmonicity == 0 && !es) CHK(read_A(&t, Anh, tl));
                    /* propagate_double_2DIR_control (propagate.c:1476-1591) */
                    oracle_propagate_doubles(p, H, fr, fi, Anh);
                    for (int t1 = 0; t1 < T1; t1++)
                        oracle_propagate_doubles(p, H, ft1r + (size_t)t1 * nn2, ft1i + (size_t)t1 * nn2, Anh);
                    if (p->propagation == 0 || p->propagation == 2) {
                        prop_DIA(p, H, rightnr, rightni, -1, 1);
                        for (int t1 = 0; t1 < T1; t1++) prop_DIA(p, H, rightrr + t1 * N, rightri + t1 * N, -1, 1);
                    } else if (p->propagation == 1) {
                        prop_coupling(p, H, rightnr, rightni, p->ts, -1);
                        for (int t1 = 0; t1 < T1; t1++) prop_coupling(p, H, rightrr + t1 * N, rightri + t1 * N, p->ts, -1);
                    } else {
                        prop_RK4(p, H, rightnr, rightni, p->ts, -1);
                        for (int t1 = 0; t1 < T1; t1++) prop_RK4(p, H, rightrr + t1 * N, rightri + t1 * N, p->ts, -1);
                    }
                }
        }
    }
done:
    for (size_t i = 0; i < 12 * (size_t)T3 * T1; i++) Rout[i] = R[i];
#undef RA
#undef CHK
    free(R); free(lt); free(H); free(Anh); free(over); free(leftrr); free(leftri); free(leftnr); free(leftni);
    free(rightrr); free(rightri); free(rightnr); free(rightni); free(mut2); free(mut4); free(mtmp);
    free(mut3r); free(mut3i); free(fr); free(fi); free(ft1r); free(ft1i); free(t1nr); free(t1ni); free(t1rr); free(t1ri);
    traj_free(&t);
    return rc;
}
