// Eigen-route exact propagator for linear absorption: Propagation Diagonal,
// and Propagation Sparse where the static-coupling Taylor route does not
// apply (HamiltonianType Full, or a Threshold that truncates U).
//
// The reference computes, per vector and per step, the full one-step
// propagator U = V diag(exp(-i e f)) V^T from an FP32 LAPACK ssyev of the
// frame and applies it (propagate_vec_DIA, propagate.c:60-125), or applies
// only the elements with |U_ab|^2 > Threshold (propagate_vec_DIA_S,
// :185-258; Threshold pre-scaled by (f/ts)^2 at input, readinput.c:264-267).
// Here every frame is diagonalised once (FP64 Jacobi, eigen.cu), U is built
// once per frame in FP64 and rounded to the working precision, truncated by
// the same test in the working precision, and shared by every start point
// and polarisation that crosses the frame.  U is complex symmetric (V is
// real orthogonal), so it is stored once and read along rows.
#include "common.cuh"
#include "engine.h"

namespace {

// U[t][a][c] for the frames of one eigen chunk: CTA per frame, V^T and the
// phases in shared memory, one packed (a <= c) element per thread-iteration,
// mirrored so that U is exactly symmetric.
template <typename R>
__global__ void k_build_u(const double *V, const double *w, int n, double f, float thres, int truncate,
                          typename Vec2<R>::T *U) {
    typedef typename Vec2<R>::T R2;
    extern __shared__ double sh[];
    double *Vt = sh, *ph = Vt + (size_t)n * n;  // Vt[k][a] = V[a][k]; ph[2k], ph[2k+1]
    const double *Vf = V + (size_t)blockIdx.x * n * n;
    const double *wf = w + (size_t)blockIdx.x * n;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        int a = e / n, k = e % n;
        Vt[(size_t)k * n + a] = Vf[e];
    }
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double s, c;
        sincos(wf[k] * f, &s, &c);
        ph[2 * k] = c;
        ph[2 * k + 1] = -s;
    }
    __syncthreads();
    R2 *Uf = U + (size_t)blockIdx.x * n * n;
    const int np = n * (n + 1) / 2;
    for (int e = threadIdx.x; e < np; e += blockDim.x) {
        // packed upper-triangle e -> (a, c), a <= c
        int a = 0, rem = e;
        while (rem >= n - a) { rem -= n - a; a++; }
        int c = a + rem;
        double ur = 0, ui = 0;
        for (int k = 0; k < n; k++) {
            double p = Vt[(size_t)k * n + a] * Vt[(size_t)k * n + c];
            ur = fma(p, ph[2 * k], ur);
            ui = fma(p, ph[2 * k + 1], ui);
        }
        R2 z;
        z.x = (R)ur;
        z.y = (R)ui;
        if (truncate) {
            bool keep;
            if (sizeof(R) == 4)
                keep = __fadd_rn(__fmul_rn((float)z.x, (float)z.x), __fmul_rn((float)z.y, (float)z.y)) > thres;
            else
                keep = (double)z.x * z.x + (double)z.y * z.y > (double)thres;
            if (!keep) z.x = z.y = (R)0;
        }
        Uf[(size_t)a * n + c] = z;
        Uf[(size_t)c * n + a] = z;
    }
}

// Linear absorption with per-frame propagators: CTA per start point, its
// three polarisation vectors in shared memory, thread a owns site a.  The
// response is taken before each step (absorption.c:119-145): float products,
// double sums over sites (warp shuffles, then warps in order).  The step is
// c_a <- sum_b U_ab c_b in site order b, the reference's float accumulation
// (propagate.c:109-119) in FP32 mode.
template <typename R>
__global__ void k_abs_dia(DevTraj T, const typename Vec2<R>::T *__restrict__ U, long f0, int n, AbsJob J,
                          double2 *resp) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int a = threadIdx.x, lane = a & 31, warp = a >> 5, NW = blockDim.x >> 5;
    double2 *red = (double2 *)smem_raw;          // [3][warps]
    R2 *C = (R2 *)(red + 3 * NW);                // [3][n]
    const int sl = blockIdx.x;
    const long ti = (long)(J.begin + sl) * J.sample;
    for (int x = 0; x < 3; x++)
        if (a < n) {
            R2 z;
            z.x = (R)traj_mu(T, ti, x, a);
            z.y = 0;
            C[x * n + a] = z;
        }
    __syncthreads();
    for (int t1 = 0; t1 < J.tmax; t1++) {
        const long t = ti + t1;
        for (int x = 0; x < 3; x++) {
            double re = 0, im = 0;
            if (a < n) {
                R m = (R)traj_mu(T, t, x, a);
                R2 z = C[x * n + a];
                re = (double)A::mul(m, z.x);
                im = (double)A::mul(m, z.y);
            }
            for (int o = 16; o > 0; o >>= 1) {
                re += __shfl_xor_sync(0xffffffffu, re, o);
                im += __shfl_xor_sync(0xffffffffu, im, o);
            }
            if (lane == 0) red[x * NW + warp] = make_double2(re, im);
        }
        __syncthreads();
        if (a < 3) {
            double sr = 0, si = 0;
            for (int w = 0; w < NW; w++) {
                sr += red[a * NW + w].x;
                si += red[a * NW + w].y;
            }
            resp[(size_t)(3 * sl + a) * J.tmax + t1] = make_double2(sr, si);
        }
        if (t1 == J.tmax - 1) break;
        R2 acc[3];
        for (int x = 0; x < 3; x++) acc[x].x = acc[x].y = 0;
        if (a < n) {
            const R2 *Ut = U + (size_t)(t - f0) * n * n;
            for (int b = 0; b < n; b++) {
                R2 u = Ut[(size_t)b * n + a];  // = U[a][b]
#pragma unroll
                for (int x = 0; x < 3; x++) {
                    R2 z = C[x * n + b];
                    acc[x].x = A::add(acc[x].x, A::sub(A::mul(u.x, z.x), A::mul(u.y, z.y)));
                    acc[x].y = A::add(acc[x].y, A::add(A::mul(u.x, z.y), A::mul(u.y, z.x)));
                }
            }
        }
        __syncthreads();
        if (a < n)
            for (int x = 0; x < 3; x++) C[x * n + a] = acc[x];
        __syncthreads();
    }
}

}  // namespace

size_t dia_build_smem(int n) { return sizeof(double) * ((size_t)n * n + 2 * n); }

int launch_build_u(int prec, const double *V, const double *w, long nfr, int n, double f, float thres, int truncate,
                   void *U, cudaStream_t s) {
    if (nfr <= 0) return 0;
    size_t sm = dia_build_smem(n);
    cudaError_t e;
    if (prec == 0) {
        if ((e = cudaFuncSetAttribute(k_build_u<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)))
            return (int)e;
        k_build_u<float><<<(unsigned)nfr, 256, sm, s>>>(V, w, n, f, thres, truncate, (float2 *)U);
    } else {
        if ((e = cudaFuncSetAttribute(k_build_u<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)))
            return (int)e;
        k_build_u<double><<<(unsigned)nfr, 256, sm, s>>>(V, w, n, f, thres, truncate, (double2 *)U);
    }
    return (int)cudaGetLastError();
}

int launch_abs_dia(int prec, const DevTraj &T, const void *U, long f0, int n, const AbsJob &J, double2 *resp,
                   cudaStream_t s) {
    if (J.nsamp <= 0) return 0;
    const int threads = ((n + 31) / 32) * 32;
    const int nw = threads / 32;
    if (threads > 1024) return (int)cudaErrorNotSupported;
    if (prec == 0) {
        size_t sm = sizeof(float2) * 3 * n + sizeof(double2) * 3 * nw;
        cudaError_t e = cudaFuncSetAttribute(k_abs_dia<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return (int)e;
        k_abs_dia<float><<<J.nsamp, threads, sm, s>>>(T, (const float2 *)U, f0, n, J, resp);
    } else {
        size_t sm = sizeof(double2) * 3 * n + sizeof(double2) * 3 * nw;
        cudaError_t e = cudaFuncSetAttribute(k_abs_dia<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return (int)e;
        k_abs_dia<double><<<J.nsamp, threads, sm, s>>>(T, (const double2 *)U, f0, n, J, resp);
    }
    return (int)cudaGetLastError();
}
