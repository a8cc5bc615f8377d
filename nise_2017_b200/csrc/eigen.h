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
