// Batched FP64 eigendecomposition of per-frame Hamiltonians (eigen.cu).
#pragma once
#include <cuda_runtime.h>

#include "devtypes.h"

#define NISE_EIG_MAX_N 120

struct EigJob {
    DevTraj T;
    int n;
    int singleshift;
};

// Shared memory needed per frame.
size_t eig_smem_bytes(int n);
// Diagonalise the (shifted, cut) Hamiltonian of every frame in frames_dev:
// V[f][i][j] = component i of eigenvector j, w[f][j] ascending.
// n <= NISE_EIG_MAX_N (two FP64 n x n matrices in one CTA's shared memory).
int launch_eig(const EigJob &J, const long *frames_dev, long nframes, double *V, double *w, cudaStream_t s);

// Any n (eigen_large.cu): the Jacobi above up to NISE_EIG_MAX_N, else
// Householder tridiagonalisation + implicit QR (frames in parallel, one CTA
// each) with eig_any_ws_doubles(n, nframes) doubles of workspace A_ws and a
// status word set to 1 when a frame does not converge.  V's layout is
// private to the pair: pass it to launch_build_u_any.
size_t eig_any_ws_doubles(int n, long frames);
int launch_eig_any(const EigJob &J, const long *frames_dev, long nframes, double *V, double *w, double *A_ws,
                   int *status, cudaStream_t s);
// U[t] = V exp(-i w f) V^T (complex, working precision; |U|^2 <= thres
// dropped when truncate), for the layout of launch_eig_any.
int launch_build_u_any(int prec, const double *V, const double *w, long nfr, int n, double f, float thres,
                       int truncate, void *U, cudaStream_t s);
