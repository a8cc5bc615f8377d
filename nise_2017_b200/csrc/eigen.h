// Batched FP64 eigendecomposition of per-frame Hamiltonians (eigen.cu).
#pragma once
#include <cuda_runtime.h>

#include "devtypes.h"

struct EigJob {
    DevTraj T;
    int n;
    int singleshift;
};

// Shared memory needed per frame.
size_t eig_smem_bytes(int n);
// Diagonalise the (shifted, cut) Hamiltonian of every frame in frames_dev:
// V[f][i][j] = component i of eigenvector j, w[f][j] ascending.  n <= 128.
int launch_eig(const EigJob &J, const long *frames_dev, long nframes, double *V, double *w, cudaStream_t s);
