// Batched FP64 symmetric eigensolver for frames above the shared-memory
// Jacobi's size limit (eigen.cu), and the eigen-propagator builder for them.
//
// Replaces the reference's LAPACK ssyev_ (diagonalizeLPD,
// propagate.c:1185-1221) and its naive N^3 transform to the site basis
// (propagate_vec_DIA, propagate.c:89-106) for the exact propagators of
// Propagation Sparse / Diagonal and the t2 step.  One CTA per frame, the
// matrix in global memory:
//
//  1. Householder tridiagonalisation, A = Q T Q^T (Golub & Van Loan,
//     Matrix Computations, Alg. 8.3.1 with the reflector of Alg. 5.1.1): for
//     column k a reflector H_k = I - beta v v^T maps A[k+1:, k] onto a
//     multiple of e_1; the trailing matrix gets A <- A - v w^T - w v^T with
//     p = beta A v, w = p - (beta p^T v / 2) v.  v_k is kept in row k of A
//     (right of the diagonal, free after step k), beta_k in shared memory;
//  2. implicit symmetric QR steps with the Wilkinson shift on T (Alg. 8.3.2
//     and 8.3.3): each step chases the bulge from the top of the unreduced
//     block to its bottom with Givens rotations, computed by one thread, and
//     every thread then applies the step's rotations to its own components
//     of all eigenvectors (Z <- Z G^T, the eigenvectors stored one per row,
//     so a warp's loads are contiguous);
//  3. back-transformation Z <- Q Z with the reflectors in reverse order.
//
// Output: w[f][j] (not sorted) and Z[f][j][i] = component i of eigenvector
// j.  A frame that does not converge in 30 n QR steps sets its status word.
#include <cstdint>

#include "common.cuh"
#include "eigen.h"
#include "engine.h"

namespace {

constexpr int kEgNT = 512;
constexpr int kEgNW = kEgNT / 32;

__device__ __forceinline__ double block_sum(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();  // red may still be read by a previous sum
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0;
    for (int w = 0; w < kEgNW; w++) s += red[w];
    return s;
}

// Smallest-magnitude-safe sqrt(a^2 + b^2).
__device__ __forceinline__ double hyp(double a, double b) { return hypot(a, b); }

__global__ void __launch_bounds__(kEgNT) k_eig_large(EigJob J, const long *frames, double *A_ws, double *Z_out,
                                                     double *w_out, int *status) {
    extern __shared__ double sh[];
    const int n = J.n, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double *d = sh, *e = d + n, *beta = e + n, *v = beta + n, *p = v + n, *cs = p + n;  // cs: [2n]
    double *red = cs + 2 * n;                                                          // [kEgNW + 8]
    int *ctl = (int *)(red + kEgNW + 8);
    const long t = frames[blockIdx.x];
    double *A = A_ws + (size_t)blockIdx.x * n * n;
    double *Z = Z_out + (size_t)blockIdx.x * n * n;
    const DevTraj &T = J.T;

    // the frame's shifted, cut Hamiltonian (read_He / read_Hamiltonian)
    for (int i = warp; i < n; i += kEgNW)
        for (int j = lane; j < n; j += 32) {
            double h;
            if (i == j) h = (double)traj_diag(T, t, i, J.singleshift != 0);
            else h = (double)traj_coupling(T, t, min(i, j), max(i, j));
            A[(size_t)i * n + j] = h;
            Z[(size_t)i * n + j] = i == j ? 1.0 : 0.0;
        }
    __syncthreads();

    // 1. tridiagonalisation
    for (int k = 0; k + 2 < n; k++) {
        const int m = n - k - 1;  // length of x = A[k+1:, k] = A[k, k+1:]
        const double *row = A + (size_t)k * n + k + 1;
        double s = 0;
        for (int i = tid; i < m; i += kEgNT) {
            const double x = row[i];
            v[i] = x;
            if (i > 0) s += x * x;
        }
        const double sigma = block_sum(s, red);
        const double alpha = v[0];
        if (tid == 0) d[k] = A[(size_t)k * n + k];
        if (sigma == 0.0) {  // already reduced: H_k = I
            if (tid == 0) {
                e[k] = alpha;
                beta[k] = 0.0;
            }
            __syncthreads();
            continue;
        }
        const double mu = sqrt(alpha * alpha + sigma);
        const double v0 = alpha <= 0.0 ? alpha - mu : -sigma / (alpha + mu);
        const double b = 2.0 * v0 * v0 / (sigma + v0 * v0);
        const double inv0 = 1.0 / v0;
        __syncthreads();
        for (int i = tid; i < m; i += kEgNT) v[i] = i == 0 ? 1.0 : v[i] * inv0;
        __syncthreads();
        // p = b * A[k+1:, k+1:] v: a warp per row, lanes over columns
        for (int i = warp; i < m; i += kEgNW) {
            const double *ar = A + (size_t)(k + 1 + i) * n + k + 1;
            double acc = 0;
            for (int j = lane; j < m; j += 32) acc += ar[j] * v[j];
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) p[i] = b * acc;
        }
        __syncthreads();
        double pv = 0;
        for (int i = tid; i < m; i += kEgNT) pv += p[i] * v[i];
        const double K = 0.5 * b * block_sum(pv, red);
        for (int i = tid; i < m; i += kEgNT) p[i] -= K * v[i];  // w
        __syncthreads();
        // A[k+1:, k+1:] -= v w^T + w v^T
        for (int i = warp; i < m; i += kEgNW) {
            double *ar = A + (size_t)(k + 1 + i) * n + k + 1;
            const double vi = v[i], pi = p[i];
            for (int j = lane; j < m; j += 32) ar[j] -= vi * p[j] + pi * v[j];
        }
        // keep v_k in row k right of the diagonal (its first entry, 1, implied)
        for (int i = tid; i < m; i += kEgNT) A[(size_t)k * n + k + 1 + i] = v[i];
        if (tid == 0) {
            e[k] = mu;
            beta[k] = b;
        }
        __syncthreads();
    }
    if (tid == 0) {
        if (n >= 2) {
            d[n - 2] = A[(size_t)(n - 2) * n + n - 2];
            e[n - 2] = A[(size_t)(n - 1) * n + n - 2];
            beta[n - 2] = 0.0;
        }
        d[n - 1] = A[(size_t)(n - 1) * n + n - 1];
        e[n - 1] = 0.0;
        beta[n - 1] = 0.0;
        ctl[0] = n - 1;  // m: bottom of the active block
        ctl[3] = 0;      // failure
    }
    __syncthreads();

    // 2. implicit QR steps with the Wilkinson shift
    const double eps = 2.220446049250313e-16;
    int steps = 0;
    while (true) {
        if (tid == 0) {
            int m = ctl[0], l = -1;
            while (m > 0) {
                // deflate at the bottom; find the top l of the unreduced block [l, m]
                if (fabs(e[m - 1]) <= eps * (fabs(d[m - 1]) + fabs(d[m]))) {
                    e[m - 1] = 0.0;
                    m--;
                    continue;
                }
                l = m - 1;
                while (l > 0 && fabs(e[l - 1]) > eps * (fabs(d[l - 1]) + fabs(d[l]))) l--;
                if (l > 0) e[l - 1] = 0.0;
                break;
            }
            ctl[0] = m;
            ctl[1] = l;
            if (m > 0) {
                // Wilkinson shift from the trailing 2x2 of the block
                const double dd = 0.5 * (d[m - 1] - d[m]), bm = e[m - 1];
                const double mu = d[m] - bm * bm / (dd + copysign(hyp(dd, bm), dd == 0.0 ? 1.0 : dd));
                // the active 2x2 (a, bb; bb, cc) and the bulge travel in
                // registers; d[k+2] and e[k+1] are read one rotation ahead
                double x = d[l] - mu, z = e[l];
                double a = d[l], bb = e[l], cc = d[l + 1];
                for (int k = l; k < m; k++) {
                    const double bn = k + 1 < m ? e[k + 1] : 0.0, dn = k + 1 < m ? d[k + 2] : 0.0;
                    // G = [c s; -s c] with c = x / r, s = z / r, r = sqrt(x^2 + z^2)
                    const double rr = x * x + z * z;
                    double c = 1.0, s = 0.0, r = 0.0;
                    if (rr > 0.0) {
                        const double ri = rsqrt(rr);
                        c = x * ri;
                        s = z * ri;
                        r = rr * ri;
                    }
                    if (k > l) e[k - 1] = r;
                    // T <- G T G^T on rows/columns k, k+1
                    const double c2 = c * c, s2 = s * s, c2s = 2.0 * c * s;
                    const double dk = c2 * a + c2s * bb + s2 * cc;
                    const double dk1 = s2 * a - c2s * bb + c2 * cc;
                    const double ek = c * s * (cc - a) + (c2 - s2) * bb;
                    d[k] = dk;
                    cs[2 * k] = c;
                    cs[2 * k + 1] = s;
                    if (k + 1 < m) {
                        x = ek;
                        z = s * bn;  // the bulge at (k, k+2)
                        a = dk1;
                        bb = c * bn;
                        cc = dn;
                    } else {
                        d[k + 1] = dk1;
                        e[k] = ek;
                    }
                }
            }
        }
        __syncthreads();
        const int m = ctl[0], l = ctl[1];
        if (m <= 0) break;
        if (++steps > 30 * n) {
            if (tid == 0) ctl[3] = 1;
            break;
        }
        // Z <- Z G^T for the step's rotations: component i of eigenvectors k, k+1
        // two components per thread at a time (independent chains), eight
        // rows ahead of the rotations
        for (int i0 = tid; i0 < n; i0 += 2 * kEgNT) {
            const int i1 = i0 + kEgNT;
            const bool two = i1 < n;
            const int j1 = two ? i1 : i0;  // a second chain on the same column when there is none
            double *z0p = Z + i0, *z1p = Z + j1;
            double zk0 = z0p[(size_t)l * n], zk1 = z1p[(size_t)l * n];
            int k = l;
            for (; k + 8 <= m; k += 8) {
                double a0[8], a1[8];
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    a0[q] = z0p[(size_t)(k + 1 + q) * n];
                    a1[q] = z1p[(size_t)(k + 1 + q) * n];
                }
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const double c = cs[2 * (k + q)], s = cs[2 * (k + q) + 1];
                    const double o0 = c * zk0 + s * a0[q], o1 = c * zk1 + s * a1[q];
                    zk0 = -s * zk0 + c * a0[q];
                    zk1 = -s * zk1 + c * a1[q];
                    z0p[(size_t)(k + q) * n] = o0;
                    if (two) z1p[(size_t)(k + q) * n] = o1;
                }
            }
            for (; k < m; k++) {
                const double c = cs[2 * k], s = cs[2 * k + 1];
                const double a0 = z0p[(size_t)(k + 1) * n], a1 = z1p[(size_t)(k + 1) * n];
                const double o0 = c * zk0 + s * a0, o1 = c * zk1 + s * a1;
                zk0 = -s * zk0 + c * a0;
                zk1 = -s * zk1 + c * a1;
                z0p[(size_t)k * n] = o0;
                if (two) z1p[(size_t)k * n] = o1;
            }
            z0p[(size_t)m * n] = zk0;
            if (two) z1p[(size_t)m * n] = zk1;
        }
        __syncthreads();
    }

    // 3. Z <- H_0 H_1 ... H_(n-3) Z (rows of Z are the eigenvectors)
    for (int k = n - 3; k >= 0; k--) {
        const double b = beta[k];
        if (b == 0.0) continue;
        const int m = n - k - 1;
        __syncthreads();
        for (int i = tid; i < m; i += kEgNT) v[i] = i == 0 ? 1.0 : A[(size_t)k * n + k + 1 + i];
        __syncthreads();
        for (int j = warp; j < n; j += kEgNW) {
            double *zr = Z + (size_t)j * n + k + 1;
            double acc = 0;
            for (int i = lane; i < m; i += 32) acc += v[i] * zr[i];
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            acc *= b;
            for (int i = lane; i < m; i += 32) zr[i] -= acc * v[i];
        }
    }
    for (int j = tid; j < n; j += kEgNT) w_out[(size_t)blockIdx.x * n + j] = d[j];
    if (tid == 0 && ctl[3]) atomicExch(status, 1);
}

// U[t][a][c] = sum_k Z[k][a] exp(-i w_k f) Z[k][c] (the eigen-propagator of
// propagate_vec_DIA in FP64, rounded to the working precision; elements with
// |U_ac|^2 <= thres in the working precision dropped when truncating,
// propagate_vec_DIA_S).  64 x 64 tiles of U, 256 threads with 4 x 4
// elements each, k in chunks of 16 staged in shared memory; only tiles on or
// above the diagonal are computed and mirrored (U is symmetric).
template <typename R>
__global__ void __launch_bounds__(256) k_build_u_large(const double *Zall, const double *wall, int n, double f,
                                                       float thres, int truncate, typename Vec2<R>::T *Uall) {
    typedef typename Vec2<R>::T R2;
    __shared__ double zc[16][64], zs[16][64], zb[16][64];
    const int nb = (n + 63) / 64;
    int ta = 0, tc = blockIdx.x;  // upper-triangular tile index -> (ta, tc), ta <= tc
    while (tc >= nb - ta) {
        tc -= nb - ta;
        ta++;
    }
    tc += ta;
    const int fr = blockIdx.y;
    const double *Z = Zall + (size_t)fr * n * n, *w = wall + (size_t)fr * n;
    R2 *U = Uall + (size_t)fr * n * n;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int a0 = ta * 64, c0 = tc * 64;
    double ur[4][4] = {}, ui[4][4] = {};
    for (int k0 = 0; k0 < n; k0 += 16) {
        for (int q = threadIdx.x; q < 16 * 64; q += 256) {
            const int kk = q / 64, x = q % 64, k = k0 + kk;
            double za = 0, zcv = 0, co = 0, si = 0;
            if (k < n) {
                if (a0 + x < n) za = Z[(size_t)k * n + a0 + x];
                if (c0 + x < n) zcv = Z[(size_t)k * n + c0 + x];
                sincos(w[k] * f, &si, &co);
            }
            zc[kk][x] = za * co;
            zs[kk][x] = -za * si;
            zb[kk][x] = zcv;
        }
        __syncthreads();
#pragma unroll 4
        for (int kk = 0; kk < 16; kk++) {
            double bc[4];
#pragma unroll
            for (int j = 0; j < 4; j++) bc[j] = zb[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const double pc = zc[kk][ty + 16 * i], ps = zs[kk][ty + 16 * i];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    ur[i][j] = fma(pc, bc[j], ur[i][j]);
                    ui[i][j] = fma(ps, bc[j], ui[i][j]);
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int a = a0 + ty + 16 * i, c = c0 + tx + 16 * j;
            if (a >= n || c >= n || (ta == tc && c < a)) continue;
            R2 z;
            z.x = (R)ur[i][j];
            z.y = (R)ui[i][j];
            if (truncate) {
                bool keep;
                if (sizeof(R) == 4)
                    keep = __fadd_rn(__fmul_rn((float)z.x, (float)z.x), __fmul_rn((float)z.y, (float)z.y)) > thres;
                else
                    keep = (double)z.x * z.x + (double)z.y * z.y > (double)thres;
                if (!keep) z.x = z.y = (R)0;
            }
            U[(size_t)a * n + c] = z;
            U[(size_t)c * n + a] = z;
        }
}

}  // namespace

size_t eig_large_smem(int n) { return sizeof(double) * ((size_t)7 * n + kEgNW + 8) + 16; }

int launch_eig_large(const EigJob &J, const long *frames_dev, long nframes, double *A_ws, double *Z, double *w,
                     int *status, cudaStream_t s) {
    if (nframes <= 0) return 0;
    const size_t sm = eig_large_smem(J.n);
    cudaError_t e = cudaFuncSetAttribute(k_eig_large, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return (int)e;
    k_eig_large<<<(unsigned)nframes, kEgNT, sm, s>>>(J, frames_dev, A_ws, Z, w, status);
    return (int)cudaGetLastError();
}

int launch_build_u_large(int prec, const double *Z, const double *w, long nfr, int n, double f, float thres,
                         int truncate, void *U, cudaStream_t s) {
    if (nfr <= 0) return 0;
    const int nb = (n + 63) / 64;
    const dim3 grid(nb * (nb + 1) / 2, (unsigned)nfr);
    if (prec == 0) k_build_u_large<float><<<grid, 256, 0, s>>>(Z, w, n, f, thres, truncate, (float2 *)U);
    else k_build_u_large<double><<<grid, 256, 0, s>>>(Z, w, n, f, thres, truncate, (double2 *)U);
    return (int)cudaGetLastError();
}

// Either solver by size: eigen.cu's shared-memory Jacobi (V[a][k]) up to
// NISE_EIG_MAX_N sites, the tridiagonal QR above (Z[k][a]); the matching
// propagator builder reads its own layout.
size_t eig_any_ws_doubles(int n, long frames) { return n > NISE_EIG_MAX_N ? (size_t)frames * n * n : 0; }

int launch_eig_any(const EigJob &J, const long *frames_dev, long nframes, double *V, double *w, double *A_ws,
                   int *status, cudaStream_t s) {
    if (J.n <= NISE_EIG_MAX_N) return launch_eig(J, frames_dev, nframes, V, w, s);
    if (!A_ws || !status) return (int)cudaErrorInvalidValue;
    return launch_eig_large(J, frames_dev, nframes, A_ws, V, w, status, s);
}

int launch_build_u_any(int prec, const double *V, const double *w, long nfr, int n, double f, float thres,
                       int truncate, void *U, cudaStream_t s) {
    if (n <= NISE_EIG_MAX_N) return launch_build_u(prec, V, w, nfr, n, f, thres, truncate, U, s);
    return launch_build_u_large(prec, V, w, nfr, n, f, thres, truncate, U, s);
}
