/*
 * ORACLE — test infrastructure, not product code.
 *
 * CPU restatement of the reference NISE wavefunction-propagation path
 * (GHlacour/NISE_2017) used only by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py as the checker.  Compiled twice from
 * nise_oracle.c: ORACLE_REAL=float (the reference's own single-precision
 * arithmetic, pinned against the reference binary built in _ref/) and
 * ORACLE_REAL=double (the FP64 reference every result's error is stated
 * against).
 */
#ifndef NISE_ORACLE_H
#define NISE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Path subset of the reference's t_non (src/types.h:37-90). */
typedef struct {
    int singles, doubles;
    int length, sample, begin, end;
    int tmax1, tmax2, tmax3;
    float deltat;
    int ts;
    float lifetime, homogen, inhomogen;
    int window, fft;
    float thres;         /* already rescaled by (dt*icm2ifs*2pi/ts)^2 (readinput.c:264-267) */
    float couplingcut;
    float anharmonicity;
    float min1, max1, min2, max2, min3, max3;
    int ham_coupling;    /* 1: HamiltonianType Coupling, 0: Full */
    int propagation;     /* 0 Sparse, 1 Coupling, 2 Diagonal, 3 RK4 */
    int technique;       /* 0 Absorption, 1 2DIR, 2 GBIR, 3 SEIR, 4 EAIR, 5 noEAIR, 6-10 the UVvis names,
                            11 LD, 12 Raman, 13 SFG, 14 DOS, 15 CD, 16 Luminescence */
    char energy[256], dipole[256], coupling[256], anharm[256], overtone[256], shift[256];
    int ham_onfly;       /* 1: TransitionDipole, 2: ExtendedDipole (couplings from positions) */
    char position[256], pbc[256];
    char alpha[256];     /* Alphafile (Raman, SFG) */
    float temperature;   /* Temperature (K), Luminescence */
    int imag_steps;      /* ImaginaryTimesteps: 0 exact Boltzmann weights, else imaginary-time steps */
} oracle_params;

int oracle_real_size(void);
/* Raw response sums (before normalisation); *samples = end (absorption.c:185). */
int oracle_absorption(const oracle_params *p, double *re_S, double *im_S, int *samples);
/* Raw 2D response sums, 12 arrays of tmax3*tmax1 ([t3][t1]) in the order
 * rrIpar riIpar rrIIpar riIIpar rrIper riIper rrIIper riIIper rrIcro riIcro rrIIcro riIIcro. */
int oracle_2dir(const oracle_params *p, double *R, int *sample_count);
/* LD, Raman, SFG, DOS, CD, Luminescence (calc_LD.c, raman.c, sfg.c, calc_DOS.c, calc_CD.c, luminescence.c):
 * raw response sums of each output channel, re/im[channel][tmax1]; *samples = end. */
int oracle_linear(const oracle_params *p, double *re_S, double *im_S, int *channels, int *samples);
/* print2D normalisation (MPI_subs.c:20-34) applied in place to one array pair. */
void oracle_print2d_normalize(const oracle_params *p, double *re, double *im, int sample_count);
/* do_1DFFT (1DFFT.c:144-274): returns the number of rows written to freq/spec. */
int oracle_1dfft(const oracle_params *p, const double *re_S, const double *im_S, int samples, double *freq,
                 double *spec_re, double *spec_im, int max_rows);

/* Single-vector propagators on a packed, already shifted Hamiltonian. */
void oracle_propagate_vector(const oracle_params *p, const float *H, void *cr, void *ci, int sign);
void oracle_propagate_doubles(const oracle_params *p, const float *H, void *cr, void *ci, const float *anh);
void oracle_propagate_t2(const oracle_params *p, const float *H, void *cr, void *ci, int nvec);
void oracle_dipole_double(const oracle_params *p, const float *dipole, const void *cr, const void *ci, void *fr,
                          void *fi, float *over);
void oracle_dipole_double_last(const oracle_params *p, const float *dipole, const void *cr, const void *ci,
                               void *fr, void *fi, float *over);
/* Symmetric eigensolver (cyclic Jacobi, FP64): A row-major n*n (destroyed),
 * eigenvalues ascending in w, eigenvectors as columns of V (row-major). */
void oracle_eigh(int n, double *A, double *w, double *V);

#ifdef __cplusplus
}
#endif
#endif
