// Batched FP64 symmetric eigensolver for per-frame Hamiltonians.
//
// Replaces the reference's LAPACK ssyev_ calls (diagonalizeLPD,
// propagate.c:1185-1221) used by propagate_t2_DIA and the exact propagators.
// One CTA diagonalises one frame with the parallel (Brent-Luk round-robin)
// cyclic Jacobi method in shared memory: every round applies N/2 disjoint
// rotations, rows then columns, and accumulates the eigenvectors.  Odd N is
// padded with one decoupled index that is dropped afterwards.  Eigenvalues
// come out ascending with V[i][j] = component i of eigenvector j, the layout
// diagonalizeLPD leaves behind.
#include "common.cuh"
#include "eigen.h"

namespace {

// Round-robin pairing: position 0 fixed, the others rotate.
__device__ __forceinline__ void rr_pair(int r, int k, int M, int *p, int *q) {
    auto pos = [&](int i) { return i == 0 ? 0 : 1 + (i - 1 + r) % (M - 1); };
    int a = pos(k), b = pos(M - 1 - k);
    *p = min(a, b);
    *q = max(a, b);
}

__global__ void k_eig_jacobi(EigJob J, const long *frames, double *V_out, double *w_out) {
    extern __shared__ double sh[];
    const int n = J.n, M = n + (n & 1), tid = threadIdx.x, NT = blockDim.x;
    double *A = sh, *V = A + (size_t)M * M, *cs = V + (size_t)M * M;  // cs: [M/2][2]
    double *red = cs + M;
    long t = frames[blockIdx.x];
    const DevTraj &T = J.T;
    for (int e = tid; e < M * M; e += NT) {
        int i = e / M, j = e % M;
        double v = 0;
        if (i < n && j < n) {
            if (i == j) v = (double)traj_diag(T, t, i, J.singleshift != 0);
            else v = (double)traj_coupling(T, t, min(i, j), max(i, j));
        } else if (i == j) {
            v = 0;  // padding index: decoupled
        }
        A[e] = v;
        V[e] = (i == j) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int sweep = 0; sweep < 60; sweep++) {
        // convergence test: off-diagonal Frobenius norm vs total
        double off = 0, tot = 0;
        for (int e = tid; e < M * M; e += NT) {
            double a = A[e];
            tot += a * a;
            if (e / M != e % M) off += a * a;
        }
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            tot += __shfl_xor_sync(0xffffffffu, tot, o);
        }
        if ((tid & 31) == 0) { red[2 * (tid >> 5)] = off; red[2 * (tid >> 5) + 1] = tot; }
        __syncthreads();
        if (tid == 0) {
            double so = 0, st = 0;
            for (int w = 0; w < NT / 32; w++) { so += red[2 * w]; st += red[2 * w + 1]; }
            red[2 * 32] = (so <= 1e-30 * (st > 0 ? st : 1.0)) ? 1.0 : 0.0;
        }
        __syncthreads();
        if (red[2 * 32] != 0.0) break;
        __syncthreads();
        for (int r = 0; r < M - 1; r++) {
            for (int k = tid; k < M / 2; k += NT) {
                int p, q;
                rr_pair(r, k, M, &p, &q);
                double apq = A[p * M + q], c = 1, s = 0;
                if (apq != 0.0) {
                    double theta = (A[q * M + q] - A[p * M + p]) / (2.0 * apq);
                    double tt = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    c = 1.0 / sqrt(tt * tt + 1.0);
                    s = tt * c;
                }
                cs[2 * k] = c;
                cs[2 * k + 1] = s;
            }
            __syncthreads();
            // columns p,q of A and V: A <- A J, V <- V J
            for (int e = tid; e < (M / 2) * M; e += NT) {
                int k = e / M, row = e % M, p, q;
                rr_pair(r, k, M, &p, &q);
                double c = cs[2 * k], s = cs[2 * k + 1];
                double ap = A[row * M + p], aq = A[row * M + q];
                A[row * M + p] = c * ap - s * aq;
                A[row * M + q] = s * ap + c * aq;
                double vp = V[row * M + p], vq = V[row * M + q];
                V[row * M + p] = c * vp - s * vq;
                V[row * M + q] = s * vp + c * vq;
            }
            __syncthreads();
            // rows p,q of A: A <- J^T A
            for (int e = tid; e < (M / 2) * M; e += NT) {
                int k = e / M, col = e % M, p, q;
                rr_pair(r, k, M, &p, &q);
                double c = cs[2 * k], s = cs[2 * k + 1];
                double ap = A[p * M + col], aq = A[q * M + col];
                A[p * M + col] = c * ap - s * aq;
                A[q * M + col] = s * ap + c * aq;
            }
            __syncthreads();
        }
    }
    // ascending order of the n physical eigenvalues (drop the padding index,
    // identified as the eigenvector with no weight on the physical sites)
    __shared__ int order[256];
    if (tid == 0) {
        int cnt = 0;
        int pad = -1;
        if (M != n) {
            double best = -1;
            for (int j = 0; j < M; j++) {
                double wgt = fabs(V[(M - 1) * M + j]);
                if (wgt > best) { best = wgt; pad = j; }
            }
        }
        for (int j = 0; j < M; j++)
            if (j != pad) order[cnt++] = j;
        for (int i = 1; i < cnt; i++) {
            int k = order[i], j = i - 1;
            while (j >= 0 && A[order[j] * M + order[j]] > A[k * M + k]) { order[j + 1] = order[j]; j--; }
            order[j + 1] = k;
        }
    }
    __syncthreads();
    double *Vo = V_out + (size_t)blockIdx.x * n * n, *wo = w_out + (size_t)blockIdx.x * n;
    for (int e = tid; e < n * n; e += NT) {
        int i = e / n, j = e % n;
        Vo[e] = V[i * M + order[j]];
    }
    for (int j = tid; j < n; j += NT) wo[j] = A[order[j] * M + order[j]];
}

}  // namespace

size_t eig_smem_bytes(int n) {
    int M = n + (n & 1);
    return sizeof(double) * (2 * (size_t)M * M + M + 2 * 33);
}

int launch_eig(const EigJob &J, const long *frames_dev, long nframes, double *V, double *w, cudaStream_t s) {
    if (J.n > NISE_EIG_MAX_N) return (int)cudaErrorNotSupported;
    size_t smem = eig_smem_bytes(J.n);
    cudaError_t e = cudaFuncSetAttribute(k_eig_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e) return (int)e;
    if (nframes <= 0) return 0;
    k_eig_jacobi<<<(unsigned)nframes, 256, smem, s>>>(J, frames_dev, V, w);
    return (int)cudaGetLastError();
}
