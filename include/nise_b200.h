/*
 * nise_b200 — C ABI of the B200 engine for the NISE wavefunction-propagation
 * path (linear absorption and 2DIR).  Plain C types only; the caller owns
 * every output buffer; every entry returns an int status (NISE_OK == 0) and
 * never exits the process.  One context per host thread; all device work of a
 * context runs on a stream the context owns.
 *
 * Reference interfaces replaced (GHlacour/NISE_2017, src/):
 *   nise_params            <- t_non (types.h:37-90), the fields on this path
 *   nise_params_default    <- defaults in readInput (readinput.c:24-44)
 *   nise_read_input        <- readInput (readinput.c:13-289)
 *   nise_load_files        <- open_files/read_coupling/read_shift and the
 *                             fseek+fread frame readers (read_trajectory.c:15-457,
 *                             hamshift.c:13-47), as one bulk load into HBM
 *   nise_set_trajectory    <- the same, from record images already in host memory
 *   nise_absorption        <- absorption() (absorption.c:18-202), the response part
 *   nise_absorption_fft    <- do_1DFFT() (1DFFT.c:144-228)
 *   nise_2dir              <- calc_2DIR() (calc_2DIR.c:22-629) and calc_2DES()
 *                             (calc_2DES.c:22-586), one GPU instead of MPI ranks
 *   nise_linear            <- LD(), raman(), sfg(), calc_DOS(), calc_CD(), luminescence()
 *                             (calc_LD.c, raman.c, sfg.c, calc_DOS.c, calc_CD.c, luminescence.c)
 *   nise_translate         <- translate's main() (translate.c:25-65)
 *   nise_propagate         <- propagate_vector() (propagate.c:20-39), batched
 *   nise_propagate_doubles <- propagate_vec_coupling_S_doubles / _RK4_doubles /
 *                             propagate_double_sparce (propagate.c:376-1394)
 *   nise_write_*           <- the output writers (absorption.c:181-189,
 *                             1DFFT.c:208-228, print2D in MPI_subs.c:20-34)
 */
#ifndef NISE_B200_H
#define NISE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NISE_B200_ABI_VERSION 1

/* Status codes. */
#define NISE_OK 0
#define NISE_ERR_ARG (-1)         /* invalid argument or keyword value */
#define NISE_ERR_IO (-2)          /* file missing or trajectory too short */
#define NISE_ERR_SHAPE (-3)       /* sizes inconsistent with the parameters */
#define NISE_ERR_DEVICE (-4)      /* CUDA error (message in nise_last_error) */
#define NISE_ERR_TIMEOUT (-5)     /* a bounded device wait gave up */
#define NISE_ERR_UNSUPPORTED (-6) /* combination not implemented */
#define NISE_ERR_NOMEM (-7)       /* host or device allocation failed */
#define NISE_ERR_STATE (-8)       /* call order (e.g. no trajectory loaded) */

/* Propagation keyword (readinput.c:236-254).  Any string other than
 * Coupling/Diagonal/RK4 selects SPARSE, as in the reference. */
enum { NISE_PROP_SPARSE = 0, NISE_PROP_COUPLING = 1, NISE_PROP_DIAGONAL = 2, NISE_PROP_RK4 = 3 };
/* HamiltonianType keyword. */
/* HamiltonianType: Full records, Coupling (diagonal frames + one static
 * coupling record), TransitionDipole / ExtendedDipole (diagonal frames,
 * couplings computed for every frame from the Positionfile and the dipoles,
 * read_trajectory.c:180-303). */
enum { NISE_HAM_FULL = 0, NISE_HAM_COUPLING = 1, NISE_HAM_TDC = 2, NISE_HAM_EDC = 3 };
/* Technique keyword (techniques on this path).  The UVvis family
 * (calc_2DES.c) is the 2DIR family with two-level sites: no overtone, no
 * anharmonicity, doubles |ab> with a != b only. */
enum {
    NISE_TECH_ABSORPTION = 0,
    NISE_TECH_2DIR = 1,
    NISE_TECH_GBIR = 2,
    NISE_TECH_SEIR = 3,
    NISE_TECH_EAIR = 4,
    NISE_TECH_NOEAIR = 5,
    NISE_TECH_2DUVVIS = 6,
    NISE_TECH_GBUVVIS = 7,
    NISE_TECH_SEUVVIS = 8,
    NISE_TECH_EAUVVIS = 9,
    NISE_TECH_NOEAUVVIS = 10,
    NISE_TECH_LD = 11,
    NISE_TECH_RAMAN = 12,
    NISE_TECH_SFG = 13,
    NISE_TECH_DOS = 14,
    NISE_TECH_CD = 15,
    NISE_TECH_LUM = 16,            /* Luminescence, PL, Fluorescence (luminescence.c) */
    NISE_TECH_OTHER = 99
};
/* Arithmetic of the propagation.  FP32 reproduces the reference's single
 * precision operations (same formulas and order, no fused multiply-add) and
 * accumulates responses in FP64; FP64 propagates in double precision. */
enum { NISE_FP32 = 0, NISE_FP64 = 1 };
/* Launch mode: BATCHED runs every start point and polarisation of the job in
 * one launch; PLAIN launches one start point (three polarisations) at a time,
 * the structure of the reference's sample loop. */
enum { NISE_BATCHED = 0, NISE_PLAIN = 1 };

typedef struct {
    /* t_non fields on the path (types.h:37-90), keyword names in comments */
    int singles, doubles;          /* Singles, Doubles */
    int length, sample;            /* Length, Samplerate */
    int begin, end;                /* BeginPoint, EndPoint (0 = all samples) */
    int tmax1, tmax2, tmax3;       /* RunTimes */
    float deltat;                  /* Timestep (fs) */
    int ts;                        /* Trotter */
    float lifetime, homogen, inhomogen; /* Lifetime, Homogeneous, Inhomogeneous (fs) */
    int window;                    /* Window: 0 none, 1 Hann */
    int fft;                       /* FFT */
    float thres;                   /* Threshold as written (scaled internally, readinput.c:264-267) */
    float couplingcut;             /* Couplingcut (cm^-1) */
    float anharmonicity;           /* Anharmonicity (0: read Anharmonicfile/Overtonedipolefile) */
    float min1, max1, min2, max2, min3, max3; /* MinFrequencies, MaxFrequencies */
    int hamiltonian;               /* HamiltonianType: NISE_HAM_* */
    int propagation;               /* Propagation: NISE_PROP_* */
    int technique;                 /* Technique: NISE_TECH_* */
    char technique_name[64];       /* Technique string as written */
    char energyFName[256];         /* Hamiltonianfile */
    char dipoleFName[256];         /* Dipolefile */
    char couplingFName[256];       /* Couplingfile */
    char anharFName[256];          /* Anharmonicfile */
    char overdipFName[256];        /* Overtonedipolefile */
    char singleShiftFName[256];    /* SingleShiftfile */
    /* engine controls (no reference counterpart) */
    int precision;                 /* NISE_FP32 or NISE_FP64 */
    int launch_mode;               /* NISE_BATCHED or NISE_PLAIN */
    int device;                    /* CUDA device ordinal */
    int kernel_config;             /* absorption kernel: 0 automatic (autotuned or default);
                                      Trotter: 1 thread per vector, 64/128/256 level-scheduled
                                      rotations with that many threads per start point, 32/33 a
                                      warp per vector with the rotation table in shared/global
                                      memory, 34 a warp per two vectors (static couplings) (all
                                      bitwise identical);
                                      Sparse/Diagonal (static couplings): 3 or 9 k_abs_taylor2 with
                                      4 or 8 vectors per CTA, 8 the Taylor series (row-owner
                                      layout where it fits, else sliced ELL), 13 the sliced-ELL
                                      Taylor kernel, 14 the row-owner Taylor kernel with 32 warps
                                      per CTA, 10 the sliced-ELL Chebyshev kernel (FP32), 15 the
                                      row-owner Chebyshev kernel (FP32), 12 the sliced-ELL Taylor
                                      kernel with 4 vectors per CTA (FP32);
                                      2 the eigen route (explicit per-frame propagators, up to
                                      2048 sites batched in FP32, else 1024), 16 / 17 its
                                      propagators applied per start point / on the tensor cores;
                                      2D techniques, Trotter doubles: 1 one warp per doubles
                                      vector (else two warps per vector for 32 < N <= 64,
                                      bitwise the same result) */
    char positionFName[256];       /* Positionfile (TransitionDipole / ExtendedDipole; CD) */
    char pbcFName[256];            /* PBCfile: periodic box per frame (optional) */
    char alphaFName[256];          /* Alphafile: polarisabilities (Raman, SFG) */
    float temperature;             /* Temperature (K; default 300), Luminescence */
    int imag_steps;                /* ImaginaryTimesteps: 0 (default) exact Boltzmann weights from an
                                      eigendecomposition, m > 0 m imaginary-time Trotter steps */
} nise_params;

typedef struct nise_ctx nise_ctx;

/* Defaults of readInput (readinput.c:24-44) plus engine controls. */
int nise_params_default(nise_params *p);
/* Parse a NISE keyword file with readInput's matching rules (first token
 * compared by strncmp over its own length; last occurrence wins; unknown
 * lines ignored).  Applies the post-parse rules on this path: tmax3 = tmax1
 * for 2D techniques, length checks.  Diagonal is accepted (the reference
 * exits on it).  Returns NISE_ERR_IO if the file is missing. */
int nise_read_input(const char *path, nise_params *p);

int nise_create(const nise_params *p, nise_ctx **out);
void nise_destroy(nise_ctx *ctx);
/* Message of the last failed call on this context ("" if none). */
const char *nise_last_error(const nise_ctx *ctx);
/* Message of the last failed call that had no context (nise_create etc.). */
const char *nise_global_error(void);

/* Read the files named in the parameters (binary layouts of
 * read_trajectory.c) and copy every record to device memory once. */
int nise_load_files(nise_ctx *ctx);
/* Same from caller memory: byte images of the files (records with their
 * int32 tags).  coupling is required for HamiltonianType Coupling;
 * anharm/overtone when Anharmonicity is 0 on a 2D technique; others NULL. */
int nise_set_trajectory(nise_ctx *ctx, const void *energy, size_t energy_bytes, const void *dipole,
                        size_t dipole_bytes, const void *coupling, size_t coupling_bytes, const void *anharm,
                        size_t anharm_bytes, const void *overtone, size_t overtone_bytes);
/* SingleShiftfile contents: H_ii <- H_ii * a + b (hamshift.c:59-66); n = 0 clears. */
int nise_set_singleshift(nise_ctx *ctx, int n, const int *sites, const float *a, const float *b);

/* Linear absorption response (absorption.c:92-154): raw sums over samples
 * and polarisations, re_S/im_S of length tmax1, and the normaliser (end). */
int nise_absorption(nise_ctx *ctx, double *re_S, double *im_S, int *samples);
/* 1D spectrum of a response (1DFFT.c:144-228), FFT on the device.  Writes
 * up to max_rows rows (frequency cm^-1, Re, Im) in the reference's order. */
int nise_absorption_fft(nise_ctx *ctx, const double *re_S, const double *im_S, int samples, double *freq,
                        double *spec_re, double *spec_im, int max_rows, int *rows);

/* 2DIR family (calc_2DIR.c:22-629) and, for the UVvis techniques, calc_2DES
 * (calc_2DES.c:22-586): raw sums of the 12 response arrays,
 * R[12][tmax3][tmax1] in the order rrIpar riIpar rrIIpar riIIpar rrIper
 * riIper rrIIper riIIper rrIcro riIcro rrIIcro riIIcro, and the sample
 * count print2D divides by. */
int nise_2dir(nise_ctx *ctx, double *R, int *sample_count);

/* Batched propagate_vector: nvec vectors (rows of re/im, float for FP32 or
 * double for FP64 contexts), vector v propagated one step with the packed,
 * already shifted Hamiltonian H + v*N(N+1)/2, sign +1 or -1. */
int nise_propagate(nise_ctx *ctx, const float *H, void *re, void *im, int nvec, int sign);
/* Batched doubles propagation (propagate_double_2DIR_control's per-vector
 * step) for vectors of length N(N+1)/2; anh is per-site (or NULL). */
int nise_propagate_doubles(nise_ctx *ctx, const float *H, void *re, void *im, int nvec, const float *anh);

/* Output files in the reference's text formats.  nise_write_td writes a
 * time-domain response "t Re Im" per line divided by samples; the files of
 * absorption.c:181-189 and most techniques end each line with a blank
 * (trailing_blank 1), TD_DOS.dat does not (calc_DOS.c:207-210). */
int nise_write_td(const char *path, const nise_params *p, const double *re_S, const double *im_S, int samples,
                  int trailing_blank);
int nise_write_td_absorption(const char *path, const nise_params *p, const double *re_S, const double *im_S,
                             int samples);
int nise_write_spectrum(const char *path, const double *freq, const double *spec_re, const double *spec_im,
                        int rows);
/* print2D: divides by sample_count, halves the t3 = 0 row, writes t1 t2 t3 Re Im. */
int nise_write_2d(const char *path, const nise_params *p, const double *re, const double *im, int sample_count);

/* Launch autotuner: times the candidate kernel configurations of this
 * context's absorption job (Trotter: thread per vector or level-scheduled
 * rotations with 64/128/256 threads per start point; Sparse: the Taylor
 * kernel variants) and keeps the fastest for every later job of the same
 * scheme, precision and size in this process.  Results do not depend on the
 * choice (Trotter variants are bitwise identical). */
int nise_absorption_tune(nise_ctx *ctx);

/* HamiltonianType TransitionDipole / ExtendedDipole (read_He with the TDC/EDC
 * couplings of read_trajectory.c:180-303): energy holds the diagonal records
 * (int32 tag + N floats per frame), position the Positionfile records (the
 * dipole-file layout; two records per frame for extended dipoles), pbc the
 * PBCfile records (int32 tag + box, or NULL).  Every frame's couplings are
 * computed once on the device and kept as Full records; nise_load_files calls
 * this for those types. */
int nise_set_trajectory_onfly(nise_ctx *ctx, const void *energy, size_t energy_bytes, const void *dipole,
                              size_t dipole_bytes, const void *position, size_t position_bytes, const void *pbc,
                              size_t pbc_bytes, const void *anharm, size_t anharm_bytes, const void *overtone,
                              size_t overtone_bytes);

/* Trajectory format translation (the reference's translate program,
 * translate.c:25-940): reads its keyword file (InputFormat/OutputFormat among
 * GROBIN, GROASC, MITASC, MITTXT, SPECTRON, SKIBIN; the InputX and OutputX file
 * names; Singles, Doubles, Length, Anharmonicity, Skip Doubles and the
 * Modify Select/Label/Shift block) and writes the translated files.  Host
 * only.  Returns NISE_ERR_IO for a missing file, NISE_ERR_ARG for a bad
 * keyword file (message in nise_global_error). */
int nise_translate(const char *keyword_file);

/* Operator records of the linear techniques: alpha the Alphafile (read_alpha,
 * read_trajectory.c:380-399: int32 tag + 6N floats per frame, components
 * xx xy xz yy yz zz) for Raman and SFG; position the CD Positionfile (the
 * dipole-file layout, int32 tag + 3N floats per frame).  Either may be NULL;
 * nise_load_files calls this for Raman, SFG and CD. */
int nise_set_operators(nise_ctx *ctx, const void *alpha, size_t alpha_bytes, const void *position,
                       size_t position_bytes);

/* Linear techniques besides absorption: LD (calc_LD.c:15-290), Raman
 * (raman.c:15-307), SFG (sfg.c:15-297), DOS (calc_DOS.c:15-234), CD
 * (calc_CD.c:15-392) and Luminescence (luminescence.c:17-409), chosen by the
 * context's technique.  Writes the raw response sums of each output channel,
 * re_S/im_S[channel][tmax1] (LD, DOS, CD: one channel; Raman: VV, VH; SFG:
 * PPP, SSP; Luminescence: total, x, y, z), the channel count and the sample
 * count the reference divides by.  Each channel's spectrum is
 * nise_absorption_fft of its response.  Luminescence sums the partition
 * function from zero (the reference starts it uninitialised). */
int nise_linear(nise_ctx *ctx, double *re_S, double *im_S, int max_channels, int *channels, int *samples);
/* Output file of channel k of a linear technique: the time-domain file
 * (td != 0, e.g. TD_Raman_VV.dat) or the spectrum (Raman_VV.dat); NULL past
 * the last channel. */
const char *nise_linear_file(int technique, int channel, int td);

/* Batched linear absorption of many contexts (trajectories of any size and
 * scheme, one device): nise_batch_create plans every job (optionally
 * autotuning), then captures all of them, each on its own stream, with their
 * 1D transforms into one CUDA graph; nise_batch_run launches the graph once
 * and waits.  Results per job: the response (as nise_absorption) and the
 * Absorption.dat rows (as nise_absorption_fft).  Destroy the batch before its
 * contexts.  No reference counterpart (the reference runs one trajectory per
 * process). */
typedef struct nise_batch nise_batch;
int nise_batch_create(nise_ctx *const *ctxs, int n, int autotune, nise_batch **out);
int nise_batch_run(nise_batch *batch);
int nise_batch_result(nise_batch *batch, int job, double *re_S, double *im_S, int *samples);
int nise_batch_spectrum(nise_batch *batch, int job, double *freq, double *spec_re, double *spec_im, int max_rows,
                        int *rows);
/* Device time of the last nise_batch_run (ms) and the kernels in the graph. */
int nise_batch_timing(const nise_batch *batch, double *ms, long *kernel_launches);
const char *nise_batch_error(const nise_batch *batch);
void nise_batch_destroy(nise_batch *batch);

/* The reference's 2DFFT program (2DFFT.c:20-830): reads the keyword file at
 * `input_path` (FFT, Timestep, RunTimes, Min/MaxFrequencies, Homogeneous,
 * Inhomogeneous, Window, Format, Technique) and the 2D response files
 * R{par,per,cro}{I,II}.dat of the current directory (per waiting time when a
 * Waitingtime.dat lists them, the .IRraman files for 2DIRraman), and writes
 * Rw*.dat, 2D.*.dat and PP.*.dat there.  The fft x fft transforms run on
 * `device`. */
int nise_2dfft_files(const char *input_path, int device);

/* Run this context's device work on the caller's CUDA stream (a
 * cudaStream_t passed as a pointer; NULL restores the context's own stream). */
int nise_set_stream(nise_ctx *ctx, void *stream);
/* Device time of the last compute call (ms, CUDA events on the context's
 * stream): the whole call and its main propagation kernel(s), and how many of
 * this library's kernels it launched. */
int nise_last_timing(const nise_ctx *ctx, double *total_ms, double *main_kernel_ms, long *launches);
/* Algorithmic work of the last compute call's main kernel(s): floating-point
 * operations and HBM bytes (every trajectory frame and dipole record read
 * once, state kept on chip). */
int nise_last_work(const nise_ctx *ctx, double *flops, double *hbm_bytes);
/* Measured FP32 FMA throughput of a device (TFLOP/s), the roofline
 * denominator of the CUDA-core kernels. */
int nise_probe_fp32_peak(int device, double *tflops);

/* No counterpart in the reference (it has no derivatives).  A differentiable
 * FP64 model of linear absorption with Propagation Coupling, RK4, Diagonal or
 * Sparse with Threshold 0: the Trotter scheme of propagate_vec_coupling_S
 * (propagate.c:821-899), the RK4 scheme of propagate_vec_RK4
 * (propagate.c:261-373) or the exact propagator exp(-i H f) of
 * propagate_vec_DIA (propagate.c:60-125; a degree-18 Taylor polynomial of
 * exp(-i H f/m), m sub-steps per frame with ||H|| f/m <= 1, remainder below
 * 2e-17), every nonzero coupling of the pattern kept, on the loaded
 * trajectory with site_shift[a] (cm^-1, N values) added to every shifted
 * diagonal energy (a SingleShift with a = 1), every coupling multiplied by
 * coupling_scale after the read cut, and the transform of do_1DFFT
 * (1DFFT.c:144-228) with the given lifetime (fs; 0 = none).  A SingleShift
 * loaded in the context is not applied.  Writes the Absorption.dat rows. */
int nise_absorption_model(nise_ctx *ctx, const double *site_shift, double coupling_scale, double lifetime,
                          double *freq, double *spec_re, double *spec_im, int max_rows, int *rows);
/* Gradient of a loss L of that spectrum: given dL/dspec_re and dL/dspec_im at
 * its `rows` rows, returns dL/dsite_shift (N values), dL/dcoupling_scale and
 * dL/dlifetime, by reverse-time propagation from checkpoints stored every 32
 * steps of a forward recomputation (RK4 and the exact propagator: the states
 * of each checkpoint block recomputed forward, then the sub-steps'
 * polynomials differentiated in reverse).  The truncated propagator (Sparse
 * with a Threshold in (0, 1], propagate_vec_DIA_S) returns
 * NISE_ERR_UNSUPPORTED. */
int nise_backward_absorption(nise_ctx *ctx, const double *site_shift, double coupling_scale, double lifetime,
                             const double *dL_dspec_re, const double *dL_dspec_im, int rows, double *g_shift,
                             double *g_scale, double *g_lifetime);

/* Host-only: the order in which the engine applies the Trotter rotations of
 * a coupling list (propagate.c:876-888 applies them in the list's
 * lexicographic order, one after another).  ab holds k pairs (a, b), a < b,
 * in that order.  Rotation q gets level 1 + the highest level of the earlier
 * rotations sharing one of its sites; perm (k values) lists the rotations by
 * level, lvptr (nlev + 1 values, at most k + 1) bounds the levels in perm,
 * and chkptr (nchk + 1 values, at most k + 1) splits every level into chunks
 * of at most 32 rotations, one warp step each.  Within a chunk the rotations
 * are ordered, and flip[q] = 1 (k values; may be NULL) applies rotation
 * perm[q] as (b, a), to spread the lanes' shared-memory loads over the banks;
 * the rotations of a chunk are disjoint and the rotation is symmetric in its
 * sites, so neither changes the float operations.  Touches no GPU. */
int nise_rotation_schedule(const int *ab, int k, int n, int *perm, int *lvptr, int *nlev, int *chkptr, int *nchk,
                           int *flip);

/* No counterpart in the reference.  Linear absorption with the Trotter
 * "Coupling" scheme (HamiltonianType Full) for callers whose device memory is
 * owned by their own allocator and who therefore cannot let the library call
 * cudaMalloc/cudaFree: inputs (record images of the Hamiltonian and dipole
 * files) and outputs (re_S/im_S, tmax1 doubles each) are caller-allocated
 * DEVICE buffers, every intermediate table lives in one static device array
 * of 32 MiB that each GPU loading the library keeps until exit, and larger
 * jobs return NISE_ERR_SHAPE.  Work is enqueued on `stream` (a cudaStream_t,
 * NULL = default stream) on the current device; the call reads a count back
 * to the host and synchronises `stream` before it returns.  All calls share
 * the array: calls whose device work overlaps (other streams, other host
 * threads) race, so the caller serialises them.
 * The first call on a device looks up the array's device address; make it
 * before any stream capture.  Results equal nise_absorption's. */
int nise_absorption_noalloc(const nise_params *p, const void *d_energy, size_t energy_bytes, const void *d_dipole,
                            size_t dipole_bytes, double *d_re_S, double *d_im_S, int *samples, void *stream);

#ifdef __cplusplus
}
#endif
#endif
