// Batched FP64 symmetric eigensolver for per-frame Hamiltonians.
//
// Replaces the reference's LAPACK ssyev_ calls (diagonalizeLPD,
// propagate.c:1185-1221) used by propagate_t2_DIA and the exact propagators.
// One CTA diagonalises one frame with the parallel (Brent-Luk round-robin)
// cyclic Jacobi method in shared memory: every round applies N/2 disjoint
// rotations to both sides of A at once, block by block, and accumulates the
// eigenvectors.  Odd N is
// padded with one decoupled index that is dropped afterwards.  Eigenvalues
// come out ascending with V[i][j] = component i of eigenvector j, the layout
// diagonalizeLPD leaves behind.
#include "common.cuh"
#include "eigen.h"

namespace {

__device__ __forceinline__ int rr_pos(int i, int r, int M) {
    if (i == 0) return 0;
    int v = i - 1 + r;
    if (v >= M - 1) v -= M - 1;
    return 1 + v;
}

// CTA of 32 x 16 threads per frame.  Per round: the M/2 rotation angles,
// then every 2x2 block of A is rotated on both sides at once (rows by the
// pair of its row block, columns by the pair of its column block; the
// rotated pair's own off-diagonal element is set to its exact value 0) and
// the eigenvector columns are rotated, all independent, so a round costs two
// barriers.
__global__ void __launch_bounds__(512) k_eig_jacobi(EigJob J, const long *frames, double *V_out, double *w_out) {
    extern __shared__ double sh[];
    const int n = J.n, M = n + (n & 1), H = M / 2;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx, NT = 512;
    double *A = sh, *V = A + (size_t)M * M;
    double2 *cs = (double2 *)(V + (size_t)M * M);  // [H] (c, s)
    int2 *pq = (int2 *)(cs + H);                   // [H] (p, q), p < q
    double *red = (double *)(pq + H + (H & 1));    // [2 * 16 + 1]
    long t = frames[blockIdx.x];
    const DevTraj &T = J.T;
    for (int e = tid; e < M * M; e += NT) {
        int i = e / M, j = e % M;
        double v = 0;
        if (i < n && j < n) {
            if (i == j) v = (double)traj_diag(T, t, i, J.singleshift != 0);
            else v = (double)traj_coupling(T, t, min(i, j), max(i, j));
        }
        A[e] = v;  // a padding index (odd n) is decoupled with a zero diagonal
        V[e] = (i == j) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int sweep = 0; sweep < 60; sweep++) {
        // convergence test: off-diagonal Frobenius norm against the total
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
        if (tx == 0) { red[2 * ty] = off; red[2 * ty + 1] = tot; }
        __syncthreads();
        if (tid == 0) {
            double so = 0, st = 0;
            for (int w = 0; w < 16; w++) { so += red[2 * w]; st += red[2 * w + 1]; }
            red[32] = (so <= 1e-30 * (st > 0 ? st : 1.0)) ? 1.0 : 0.0;
        }
        __syncthreads();
        if (red[32] != 0.0) break;
        for (int r = 0; r < M - 1; r++) {
            for (int k = tid; k < H; k += NT) {
                int a = rr_pos(k, r, M), b = rr_pos(M - 1 - k, r, M);
                int p = min(a, b), q = max(a, b);
                double apq = A[p * M + q], c = 1, sn = 0;
                if (apq != 0.0) {
                    double theta = (A[q * M + q] - A[p * M + p]) / (2.0 * apq);
                    double tt = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    c = 1.0 / sqrt(tt * tt + 1.0);
                    sn = tt * c;
                }
                cs[k] = make_double2(c, sn);
                pq[k] = make_int2(p, q);
            }
            __syncthreads();
            // A <- J^T A J by 2x2 blocks: rows (p_k, q_k), columns (p_l, q_l)
            for (int k = ty; k < H; k += 16) {
                const int2 rk = pq[k];
                const double2 ck = cs[k];
                double *Ap = A + (size_t)rk.x * M, *Aq = A + (size_t)rk.y * M;
                for (int l = tx; l < H; l += 32) {
                    const int2 cl = pq[l];
                    const double2 dl = cs[l];
                    double a00 = Ap[cl.x], a01 = Ap[cl.y], a10 = Aq[cl.x], a11 = Aq[cl.y];
                    double b00 = dl.x * a00 - dl.y * a01, b01 = dl.y * a00 + dl.x * a01;
                    double b10 = dl.x * a10 - dl.y * a11, b11 = dl.y * a10 + dl.x * a11;
                    Ap[cl.x] = ck.x * b00 - ck.y * b10;
                    Ap[cl.y] = ck.x * b01 - ck.y * b11;
                    Aq[cl.x] = ck.y * b00 + ck.x * b10;
                    Aq[cl.y] = ck.y * b01 + ck.x * b11;
                    if (l == k) Ap[cl.y] = Aq[cl.x] = 0.0;  // the rotation annihilates A_pq
                }
            }
            // V <- V J: columns (p_k, q_k) of every row
            for (int row = ty; row < M; row += 16) {
                double *Vr = V + (size_t)row * M;
                for (int k = tx; k < H; k += 32) {
                    const int2 rk = pq[k];
                    const double2 ck = cs[k];
                    double vp = Vr[rk.x], vq = Vr[rk.y];
                    Vr[rk.x] = ck.x * vp - ck.y * vq;
                    Vr[rk.y] = ck.y * vp + ck.x * vq;
                }
            }
            __syncthreads();
        }
    }
    // ascending order of the n physical eigenvalues (drop the padding index,
    // identified as the eigenvector with no weight on the physical sites);
    // the order reuses the rotation table's shared memory
    int *order = (int *)cs;
    __syncthreads();
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
    int M = n + (n & 1), H = M / 2;
    return sizeof(double) * 2 * (size_t)M * M + sizeof(double2) * H + sizeof(int2) * (H + (H & 1)) +
           sizeof(double) * 33;
}

int launch_eig(const EigJob &J, const long *frames_dev, long nframes, double *V, double *w, cudaStream_t s) {
    if (J.n > NISE_EIG_MAX_N) return (int)cudaErrorNotSupported;
    size_t smem = eig_smem_bytes(J.n);
    cudaError_t e = cudaFuncSetAttribute(k_eig_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e) return (int)e;
    if (nframes <= 0) return 0;
    k_eig_jacobi<<<(unsigned)nframes, dim3(32, 16), smem, s>>>(J, frames_dev, V, w);
    return (int)cudaGetLastError();
}
