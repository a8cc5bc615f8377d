// Host-side launch interface of the engine's kernels (implemented in the
// .cu files, called by api.cpp).  Every launcher returns a cudaError_t value
// cast to int (0 = success) and only enqueues work on the given stream.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "devtypes.h"

// Per-frame coefficients of the Trotter "Coupling" scheme
// (propagate_vec_coupling_S, propagate.c:821-899) for frames [f0, f0+nf):
//   U[t][a]   = (cos(h_a f/2), -sin(h_a f/2))     half-step diagonal phase
//   rot[t][k] = (co, si), si = -sin(J_k f), co = sqrt(1 - si^2)
// for the coupling pattern pairs[k] = (a, b), a < b, in lexicographic order.
// With a static coupling frame, rot has one row shared by all frames.
struct TrotterPlan {
    int n, k;
    const int2 *pairs;  // device [k]
    long f0, nf;
    void *U;            // R2 [nf][n]
    void *rot;          // R2 [nf][k] or [k]
    int rot_static;
    int singleshift;    // apply SingleShift to the diagonal (absorption path)
};

// Per-frame sparse lists of the RK4 scheme (propagate_vec_RK4,
// propagate.c:261-373): entries[k] = (a, b), a <= b, diagonal always kept,
// val[t][k] = f * H_ab (0 where |H_ab| <= cut in that frame).
struct Rk4Plan {
    int n, k;
    const int2 *entries;
    long f0, nf;
    void *val;          // R [nf][k]
    int singleshift;
};

// Complex numbers per site row of the sliced-ELL Taylor kernel's state (the
// 8 vectors of a CTA, unpadded): FP32 rows are 64 bytes, so even and odd rows
// fall on the two halves of the shared-memory banks.
#define NISE_T3_ROW 8

// Sparse exact propagator exp(-i H f) by a Taylor series on a static CSR
// coupling matrix plus the per-frame diagonal.
struct TaylorPlan {
    int n, nnz;
    const int *row_ptr, *col;
    const void *val;       // R [nnz], static couplings (HamiltonianType Coupling)
    const int *pidx;       // packed index of every CSR entry (per-frame couplings)
    int static_j;
    long f0, nf;
    const int *order;      // [nf] Taylor order per frame
    int singleshift;
    // sliced-ELL copy of the couplings for the shared-memory kernel: slices of
    // 4 rows, entries (state offset = column * NISE_T3_ROW, weight) [slot][row]
    const void *ell;
    const int *ell_sptr;   // [nslices + 1] entry offset of each slice
    const int *ell_rows;   // [nslices][4] site of each slice row (n for padding)
    int ell_nslices, ell_nent;
    int only_v2;           // 1: use k_abs_taylor2 even where the sliced-ELL kernel fits
    // Chebyshev tables (set by launch_prep_cheb; then launch_abs_taylor runs
    // the FP32 Chebyshev kernel): 1/R per frame and [nf][NISE_CHEB_KMAX+1]
    // complex coefficients a_k
    const float *cheb_inv_r;
    const float *cheb_center;  // c_t: the centre subtracted from the diagonal
    const float2 *cheb_coef;
    // 4-vector variant (k_abs_taylor4, FP32): 8-row slices, entries (column * 4,
    // weight bits) as int2 [slot][row], rows [nslices][8]
    int use_v4;
    const void *ell4;
    const int *ell4_sptr, *ell4_rows;
    int ell4_nslices, ell4_nent;
    // row-owner layout (k_abs_taylor_rv, FP32): 8-row slices of alternating
    // parity, couplings in slot triples [group][row]: float4 of the three
    // weights and the bits of the three neighbours' row indices (10 bits
    // each); tptr [nslices + 1] first group of each slice, rows [nslices][8];
    // wsl[s] the slices of each warp of launch shape s (24 or 32 warps,
    // [warp][8], -1 = none), it[s] the most slices of a warp; no_rv keeps the
    // 8-vector waves on k_abs_taylor3
    const float4 *ell8_tri;
    const int *ell8_tptr, *ell8_rows;
    const int *ell8_wsl[2];
    int ell8_it[2];
    int ell8_nslices, ell8_ntg;
    int rv_shape;
    int no_rv;
    int rv_cheb;           // with the Chebyshev tables: the row-owner kernel's Chebyshev form
    const int *order_taylor;  // the Taylor orders next to the Chebyshev ones (10, 15)
    int *err;              // device flag: 1 = a bounded wait for a staged frame gave up
};
#define NISE_CHEB_KMAX 40

// A batch of linear-absorption start points: vectors v = 3*(s-begin)+x for
// samples s in [begin, begin+nsamp), polarisations x = 0..2.
struct AbsJob {
    int begin, nsamp, sample, tmax, ts;
    double f;              // full-step phase factor deltat*icm2ifs*2pi (no /ts)
    float f32_sub;         // same / ts in the reference's float arithmetic
    double f64_sub;        // same / ts in double
    float f32_full;        // deltat*icm2ifs*2pi in float arithmetic
};

int launch_prep_trotter(int prec, const DevTraj &T, const TrotterPlan &P, double fsub, float fsub32,
                        cudaStream_t s);
int launch_abs_trotter(int prec, const DevTraj &T, const TrotterPlan &P, const AbsJob &J, double2 *resp,
                       cudaStream_t s);
// Trotter absorption with level-scheduled rotations (CTA per start point):
// P.pairs holds the couplings in level order, lvptr[l]..lvptr[l+1] the
// rotations of level l.  Bitwise identical to launch_abs_trotter.
int launch_abs_trotter_lv(int prec, const DevTraj &T, const TrotterPlan &P, const AbsJob &J, double2 *resp,
                          const int *lvptr, int nlev, int threads, cudaStream_t s);
// Streaming multiprocessors of the current device.
int sm_count();
// The same with a warp per vector (the lanes share a level's rotations),
// bitwise identical to both.  chk[c]..chk[c+1] are the rotations of
// chunk c (a level, or at most 32 of its rotations).  tables = 1: the
// rotation table in shared memory where it fits; 0: read from global memory.
int launch_abs_trotter_wv(int prec, const DevTraj &T, const TrotterPlan &P, const AbsJob &J, double2 *resp,
                          const int *chk, int nchk, int tables, cudaStream_t s);
// Two vectors per warp sharing the schedule (static coefficients only),
// bitwise identical to launch_abs_trotter_wv.
int launch_abs_trotter_wv2(int prec, const DevTraj &T, const TrotterPlan &P, const AbsJob &J, double2 *resp,
                           const int *chk, int nchk, cudaStream_t s);
int launch_prep_rk4(int prec, const DevTraj &T, const Rk4Plan &P, double fsub, float fsub32, cudaStream_t s);
int launch_abs_rk4(int prec, const DevTraj &T, const Rk4Plan &P, const AbsJob &J, double2 *resp, cudaStream_t s);
int launch_prep_taylor(int prec, const DevTraj &T, TaylorPlan &P, double rowabs_max, double f, int *order,
                       cudaStream_t s);
// kernels (optional): the number of kernels launched (the sliced-ELL Taylor
// kernel runs whole waves of 8-vector CTAs plus 1-vector CTAs for the rest).
// The row-owner Taylor kernel (FP32, static couplings, 8 vectors per CTA)
// for vectors v0 .. v0+nvec-1; cudaErrorNotSupported when the job does not
// fit its layout (shared memory, dipoles not static).
int launch_abs_taylor_rv(const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp, int v0, int nvec,
                         cudaStream_t s);
bool taylor_rv_fits(const DevTraj &T, const TaylorPlan &P);
// Vectors [v0, v0 + nvec) of an FP32 static-coupling job: on the row-owner
// kernel (whole CTAs of 8), or on 1-vector CTAs of the sliced-ELL Taylor
// kernel (one).
int launch_abs_taylor_part(const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp, int v0, int nvec,
                           bool one, cudaStream_t s);
int launch_abs_taylor(int prec, const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp,
                      int vec_per_cta, cudaStream_t s, int *kernels = nullptr);
// Chebyshev coefficients of the exact step per frame (FP32 kernel); sets
// P.order, P.cheb_inv_r and P.cheb_coef.
int launch_prep_cheb(const DevTraj &T, TaylorPlan &P, double rowabs_max, double f, int *order, float *inv_r,
                     float *center, float2 *coef, cudaStream_t s);
// flag[idx] = 1 for packed off-diagonals with |J| > cut in any frame of [f0, f0+nf).
int launch_pattern_scan(const DevTraj &T, long f0, long nf, int *flag, cudaStream_t s);
// Sum resp[v][t] over v in order (deterministic) into out[t].
int launch_reduce_resp(const double2 *resp, int nvec, int tmax, double2 *out, cudaStream_t s);
// 1D spectrum (1DFFT.c:144-228) of the response on the device.
struct FftJob {
    int tmax, fft, samples, window, fp32;
    double deltat, lifetime, homogen, inhomogen;
};
int launch_fft1d(const FftJob &J, const double2 *resp, double2 *spec, cudaStream_t s);
// Same with a caller work buffer in[fft] (no allocation: usable in stream capture).
int launch_fft1d_buf(const FftJob &J, const double2 *resp, double2 *spec, double2 *in, cudaStream_t s);

// Batched single steps on caller Hamiltonians (nise_propagate): vector v
// uses packed H + v*n(n+1)/2.
int launch_step_coupling(int prec, int n, float cut, const float *H, void *re, void *im, int nvec, int ts,
                         double fsub, float fsub32, cudaStream_t s);
int launch_step_rk4(int prec, int n, float cut, const float *H, void *re, void *im, int nvec, int ts,
                    double fsub, float fsub32, cudaStream_t s);
int launch_step_taylor(int prec, int n, const float *H, void *re, void *im, int nvec, double f, cudaStream_t s);

// Eigen route (diag.cu).  U[t][a][c] = sum_k V[t][a][k] V[t][c][k] exp(-i w[t][k] f)
// for nfr frames, rounded to the working precision (prec 0 FP32, 1 FP64) and,
// when `truncate`, zeroed where |U_ac|^2 <= thres (propagate_vec_DIA_S).
int launch_build_u(int prec, const double *V, const double *w, long nfr, int n, double f, float thres, int truncate,
                   void *U, cudaStream_t s);
// The eigen-route absorption with the propagators applied on the tensor cores
// (FP32, time-major; dia_tc.cu): X is 4 * tc_dia_columns(J) * n floats of
// workspace, err a device flag set when a bounded wait gives up.  The
// _frames form runs frames ta..tb (clipped to the job's first and last
// frames) with the propagator of frame t at U + (t - ufirst) n^2, so the
// propagators can be built and applied chunk by chunk.
int tc_dia_columns(const AbsJob &J);
bool tc_dia_fits(const AbsJob &J, int n);
long tc_dia_first_frame(const AbsJob &J);
long tc_dia_last_frame(const AbsJob &J);
int launch_abs_dia_tc(const DevTraj &T, const void *U, long f0, int n, const AbsJob &J, double2 *resp, float *X,
                      int *err, cudaStream_t s);
int launch_abs_dia_tc_frames(const DevTraj &T, const void *U, long ufirst, int n, const AbsJob &J, double2 *resp,
                             float *X, int *err, long ta, long tb, cudaStream_t s);
// Linear absorption of the start points of J with the per-frame propagators
// U (frames from f0): one CTA per start point, n <= 1024.
int launch_abs_dia(int prec, const DevTraj &T, const void *U, long f0, int n, const AbsJob &J, double2 *resp,
                   cudaStream_t s);

// Differentiable FP64 Trotter absorption (adjoint.cu).  Tables for frames
// [f0, f0+nf): U[t][a] half-step phases with the site shifts, rot[t][k]
// (co, si) of the scaled couplings, jf[t][k] = J f; checkpoints every K
// steps plus the last state (nck slots per vector).
struct AdjPlan {
    int n, k, ts, K, nck;
    const int2 *pairs;
    long f0, nf;
    const double *shift;   // [n] device
    double scale, f;       // coupling scale, deltat*icm2ifs*2pi/ts
    double2 *U, *rot;
    double *jf;
};
int launch_adj_prep(const DevTraj &T, const AdjPlan &P, cudaStream_t s);
int launch_adj_fwd(const DevTraj &T, const AdjPlan &P, const AbsJob &J, double2 *resp, double2 *ckpt,
                   cudaStream_t s);
int launch_adj_bwd(const DevTraj &T, const AdjPlan &P, const AbsJob &J, const double2 *G, const double2 *ckpt,
                   double *gshift_part, double *gscale_part, double *gshift, double *gscale, cudaStream_t s);

// Full record images for couplings computed on the fly (onfly.cu): diag are
// the Hamiltonian file's diagonal records (int32 tag + n floats), pos the
// Positionfile records (one per frame, two for extended dipoles), dip the
// dipole records (dip_words words each), pbc the PBCfile records (int32 tag +
// box, or NULL).  out receives frames records of full_words words.
struct OnflyJob {
    const float *diag, *pos, *dip, *pbc;
    long frames, full_words, dip_words;
    int n, edc;
};
int launch_onfly(const OnflyJob &J, float *out, cudaStream_t s);

