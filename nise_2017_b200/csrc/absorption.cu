// Linear-absorption kernels: per-frame coefficient preparation, the three
// singles propagation schemes applied to every start point and polarisation
// of a job, and the deterministic response reduction.
//
// Work decomposition.  A job is the set of vectors v = 3*(s-begin)+x: start
// point s (frame ti = s*Samplerate) and dipole component x.  Each vector runs
// the sample loop of absorption.c:119-145: S[t1] += mu(ti+t1).psi, then psi
// <- U(ti+t1) psi, for t1 < tmax (the step after the last response is not
// taken; it cannot change any output).  The Trotter and RK4 schemes are
// sequential inside a vector (each rotation/update reads the previous one),
// so a thread owns a vector and keeps it in shared memory, interleaved by
// lane ([site][lane]) so a warp's accesses to one site are conflict-free.
// Per-frame coefficients (phases, rotation cos/sin, RK4 values) are computed
// once per frame by a preparation kernel and read by every vector that
// crosses the frame.  The sparse Taylor scheme is a sparse-matrix product per
// Taylor order: a CTA owns G vectors and spreads the sites over its threads.
#include <algorithm>
#include <cstdio>

#include "common.cuh"
#include "engine.h"
#include "schemes.cuh"

namespace {

// ------------------------------------------------------------ Trotter
template <typename R>
__global__ void k_prep_trotter(DevTraj T, TrotterPlan P, R fsub) {
    typedef typename Vec2<R>::T R2;
    long per = P.n + (P.rot_static ? 0 : P.k);
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (tid >= P.nf * per) return;
    long fi = tid / per;
    int e = (int)(tid % per);
    long t = P.f0 + fi;
    if (e < P.n) {
        float h = traj_diag(T, t, e, P.singleshift != 0);
        double arg = 0.5 * (double)h * (double)fsub;  // cos(0.5 * H0[a] * f), propagate.c:864
        R2 u;
        u.x = (R)cos(arg);
        u.y = (R)(-sin(arg));
        ((R2 *)P.U)[fi * P.n + e] = u;
    } else {
        int k = e - P.n;
        int2 ab = P.pairs[k];
        ((R2 *)P.rot)[fi * P.k + k] = Cst<R>::rot(traj_coupling(T, t, ab.x, ab.y), fsub, T.cut);
    }
}

template <typename R>
__global__ void k_prep_trotter_static(DevTraj T, TrotterPlan P, R fsub) {
    typedef typename Vec2<R>::T R2;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= P.k) return;
    int2 ab = P.pairs[k];
    ((R2 *)P.rot)[k] = Cst<R>::rot(traj_coupling(T, 0, ab.x, ab.y), fsub, T.cut);
}

template <typename R>
__global__ void k_abs_trotter(DevTraj T, TrotterPlan P, AbsJob J, double2 *resp, int nvec) {
    typedef typename Vec2<R>::T R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *S = (R2 *)smem_raw;
    const int B = blockDim.x, lane = threadIdx.x, n = P.n;
    int v = blockIdx.x * B + lane;
    if (v >= nvec) return;
    int s = J.begin + v / 3, x = v % 3;
    long ti = (long)s * J.sample;
    for (int i = 0; i < n; i++) {
        R2 z;
        z.x = (R)traj_mu(T, ti, x, i);
        z.y = 0;
        S[i * B + lane] = z;
    }
    const R2 *U = (const R2 *)P.U, *rot = (const R2 *)P.rot;
    for (int t1 = 0; t1 < J.tmax; t1++) {
        long tj = ti + t1;
        resp[(size_t)v * J.tmax + t1] = dot_mu<R>(T, tj, x, S, B, lane, n);
        if (t1 == J.tmax - 1) break;
        const R2 *Uf = U + (tj - P.f0) * n;
        const R2 *Rf = P.rot_static ? rot : rot + (tj - P.f0) * P.k;
        trotter_apply<R>(S, B, lane, n, P.k, P.pairs, Uf, Rf, J.ts);
    }
}

// Trotter absorption with the rotations of a sub-step grouped into levels:
// rotation k gets level 1 + the highest level of the earlier rotations that
// share one of its sites, so the rotations of one level touch disjoint sites
// and applying a level in parallel reproduces the sequential lexicographic
// order of propagate.c:876-888 operation for operation.  The coupling pairs
// are stored in level order: level l is pairs[lvptr[l] .. lvptr[l+1]).  CTA per start
// point, its three polarisation vectors in shared memory; the response is
// summed by one thread per polarisation in the order of dot_mu, so every
// Trotter kernel gives bitwise identical results.
template <typename R>
__global__ void k_abs_trotter_lv(DevTraj T, TrotterPlan P, AbsJob J, double2 *resp, const int *__restrict__ lvptr,
                                 int nlev) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = P.n, tid = threadIdx.x, NT = blockDim.x;
    R2 *C = (R2 *)smem_raw;             // [3][n]
    float *mu = (float *)(C + 3 * n);   // [3][n]
    const int sl = blockIdx.x;
    const long ti = (long)(J.begin + sl) * J.sample;
    for (int e = tid; e < 3 * n; e += NT) {
        R2 z;
        z.x = (R)traj_mu(T, ti, e / n, e % n);
        z.y = 0;
        C[e] = z;
    }
    const R2 *U = (const R2 *)P.U, *rot = (const R2 *)P.rot;
    for (int t1 = 0; t1 < J.tmax; t1++) {
        const long t = ti + t1;
        for (int e = tid; e < 3 * n; e += NT) mu[e] = traj_mu(T, t, e / n, e % n);
        __syncthreads();
        if (tid < 3) {  // the residue order of dot_mu
            double re = 0, im = 0;
            for (int r = 0; r < 32 && r < n; r++) {
                double pr = 0, pi = 0;
                for (int a = r; a < n; a += 32) {
                    R m = (R)mu[tid * n + a];
                    R2 z = C[tid * n + a];
                    pr += (double)A::mul(m, z.x);
                    pi += (double)A::mul(m, z.y);
                }
                re += pr;
                im += pi;
            }
            resp[(size_t)(3 * sl + tid) * J.tmax + t1] = make_double2(re, im);
        }
        __syncthreads();
        if (t1 == J.tmax - 1) break;
        const R2 *Uf = U + (t - P.f0) * n;
        const R2 *Rf = P.rot_static ? rot : rot + (t - P.f0) * P.k;
        for (int sub = 0; sub < J.ts; sub++) {
            for (int half = 0; half < 2; half++) {
                for (int e = tid; e < 3 * n; e += NT) {  // propagate.c:870-873 / 891-894
                    R2 z = C[e], u = Uf[e % n], o;
                    o.x = A::sub(A::mul(z.x, u.x), A::mul(z.y, u.y));
                    o.y = A::add(A::mul(z.y, u.x), A::mul(z.x, u.y));
                    C[e] = o;
                }
                __syncthreads();
                if (half == 1) break;
                for (int l = 0; l < nlev; l++) {
                    const int r0 = lvptr[l], cnt = lvptr[l + 1] - r0;
                    for (int e = tid; e < 3 * cnt; e += NT) {
                        const int k = r0 + e / 3, x = e % 3;
                        const int2 ab = P.pairs[k];
                        const R2 cs = Rf[k];
                        R2 *ca = C + x * n + ab.x, *cb = C + x * n + ab.y;
                        R2 xa = *ca, xb = *cb, ya, yb;
                        ya.x = A::sub(A::mul(cs.x, xa.x), A::mul(cs.y, xb.y));
                        ya.y = A::add(A::mul(cs.x, xa.y), A::mul(cs.y, xb.x));
                        yb.x = A::sub(A::mul(cs.x, xb.x), A::mul(cs.y, xa.y));
                        yb.y = A::add(A::mul(cs.x, xb.y), A::mul(cs.y, xa.x));
                        *ca = ya;
                        *cb = yb;
                    }
                    __syncthreads();
                }
            }
        }
    }
}

// Trotter absorption, warp per vector.  The rotations of one level touch
// disjoint sites (on lattices a level holds ~20 of them and there are ~N/3.6
// levels, because rotations that share a site keep their lexicographic
// order); the host splits every level into chunks of at most 32 rotations
// (chunk c = pairs[chk[c] .. chk[c+1])), the lanes apply one chunk and a
// __syncwarp separates chunks.  A two-deep register pipeline loads the bounds
// of chunk c+2 and the pairs and coefficients of chunk c+1 while chunk c is
// applied, so only the state loads sit on the critical path.  A lane with no
// rotation in a chunk rotates a spare site of its own (n .. n+31) by the
// identity (cos 1, sin 0; the spare sites stay zero), so the warp never
// diverges; in shared memory these identity rotations are table entries
// K .. K+31, and an idle lane reads the one congruent mod 32 to the entry it
// stands in for.  Every vector sees the reference's float operations
// (propagate.c:868-895); the response is summed in the order of dot_mu (lane
// r sums the sites r, r+32, ...), so all Trotter kernels give bitwise
// identical results.  W warps = W vectors per CTA; vector v is polarisation
// v % 3 of start point v / 3.
//
// SM: the rotation table lives in shared memory (pairs packed a | b << 16,
// coefficients as R2).  Static coefficients are loaded once; per-frame
// coefficients are reloaded every frame, and then the CTA is the three
// polarisations of one start point (W = 3, every warp active), which cross
// the same frames.  ustage: each warp copies the frame's half-step phases
// into shared memory with the response loads, once per frame instead of
// reading them twice per sub-step.
template <typename R, bool SM>
__global__ void k_abs_trotter_wv(DevTraj T, TrotterPlan P, AbsJob J, double2 *resp, int nvec,
                                 const int *__restrict__ chk_g, int nchk, int ustage) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = P.n, K = P.k, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, W = blockDim.x >> 5;
    unsigned char *sp = smem_raw;
    int *chk = (int *)sp;  // [nchk + 4]: chunk bounds, then K (empty chunks)
    sp += ((size_t)(nchk + 4) * sizeof(int) + 15) & ~(size_t)15;
    R2 *tcs = (R2 *)sp;  // SM: [K + 32] coefficients
    unsigned *tab = (unsigned *)(sp + (SM ? (((size_t)(K + 32) * sizeof(R2) + 15) & ~(size_t)15) : 0));  // SM: pairs
    if (SM) sp = (unsigned char *)tab + (((size_t)(K + 32) * sizeof(unsigned) + 15) & ~(size_t)15);
    const int nc = n + 32;  // sites and the 32 spare sites
    R2 *C = (R2 *)sp + (size_t)warp * nc * (ustage ? 2 : 1);
    R2 *Us = C + nc;  // ustage: [n] phases of the frame
    for (int e = threadIdx.x; e < nchk + 4; e += blockDim.x) chk[e] = e <= nchk ? chk_g[e] : K;
    if (SM) {
        for (int e = threadIdx.x; e < K + 32; e += blockDim.x) {
            const int2 ab = e < K ? P.pairs[e] : make_int2(n + e - K, n + e - K);
            tab[e] = (unsigned)ab.x | ((unsigned)ab.y << 16);
        }
        for (int e = threadIdx.x; e < K + 32; e += blockDim.x) {
            R2 u;
            u.x = 1;
            u.y = 0;
            if (e >= K) tcs[e] = u;
            else if (P.rot_static) tcs[e] = ((const R2 *)P.rot)[e];
        }
    }
    __syncthreads();
    const int v = blockIdx.x * W + warp;
    if (v >= nvec) return;  // never with per-frame coefficients in shared memory (W = 3)
    const int x = v % 3;
    const long ti = (long)(J.begin + v / 3) * J.sample;
    for (int a = lane; a < nc; a += 32) {
        R2 z;
        z.x = a < n ? (R)traj_mu(T, ti, x, a) : (R)0;
        z.y = 0;
        C[a] = z;
    }
    const R2 *U = (const R2 *)P.U, *rot = (const R2 *)P.rot;
    const int2 spare = make_int2(n + lane, n + lane);  // global-table kernel
    R2 unit;
    unit.x = 1;
    unit.y = 0;
    auto pair = [&](int k) -> int2 {
        if (SM) {
            const unsigned w = tab[k];
            return make_int2((int)(w & 0xffffu), (int)(w >> 16));
        }
        return P.pairs[k];
    };
    for (int t1 = 0; t1 < J.tmax; t1++) {
        const long t = ti + t1;
        const bool step = t1 + 1 < J.tmax;  // the frame's phases exist only for propagated frames
        const R2 *Uf = U + (t - P.f0) * n;
        double re = 0, im = 0;
#pragma unroll 4
        for (int a = lane; a < n; a += 32) {
            R m = (R)traj_mu(T, t, x, a);
            if (ustage && step) Us[a] = Uf[a];
            R2 z = C[a];
            re += (double)A::mul(m, z.x);
            im += (double)A::mul(m, z.y);
        }
        const double2 rs = resp_sum_warp(re, im, n);
        if (lane == 0) resp[(size_t)v * J.tmax + t1] = rs;
        if (!step) break;
        const R2 *Rf;
        if (SM) {
            if (!P.rot_static) {
                __syncthreads();  // every warp is done with the previous frame's coefficients
                const R2 *src = rot + (t - P.f0) * K;
                for (int e = threadIdx.x; e < K; e += blockDim.x) tcs[e] = src[e];
                __syncthreads();
            }
            Rf = tcs;
        } else {
            Rf = P.rot_static ? rot : rot + (t - P.f0) * K;
        }
        // half-step phases (propagate.c:870-873 / 891-894), from the staged copy (a lane
        // reads back only the phases it copied) or from global memory: two instances,
        // so that each reads one address space
        auto phase = [&](const R2 *uu) {
#pragma unroll 4
            for (int a = lane; a < n; a += 32) {
                R2 z = C[a], u = uu[a], o;
                o.x = A::sub(A::mul(z.x, u.x), A::mul(z.y, u.y));
                o.y = A::add(A::mul(z.y, u.x), A::mul(z.x, u.y));
                C[a] = o;
            }
        };
        for (int sub = 0; sub < J.ts; sub++) {
            if (ustage) phase(Us);
            else phase(Uf);
            __syncwarp();
            // chunk c = pairs[chk[c] .. e0): this lane's rotation (ab0, cs0);
            // e1 = end of chunk c+1
            int e0 = chk[1], e1 = chk[2];
            int2 ab0;
            R2 cs0;
            auto fetch = [&](int k, int end, int2 &ab, R2 &cs) {
                if (SM) {  // identity entry congruent to k mod 32: no bank conflict with the chunk
                    k = k < end ? k : K + ((k - K) & 31);
                    ab = pair(k);
                    cs = Rf[k];
                } else {
                    ab = k < end ? pair(k) : spare;
                    cs = k < end ? Rf[k] : unit;
                }
            };
            fetch(chk[0] + lane, e0, ab0, cs0);
#pragma unroll 2
            for (int c = 0; c < nchk; c++) {
                int2 ab1;
                R2 cs1;
                fetch(e0 + lane, e1, ab1, cs1);
                const int e2 = chk[c + 3];
                {  // propagate.c:876-888
                    R2 xa = C[ab0.x], xb = C[ab0.y], ya, yb;
                    ya.x = A::sub(A::mul(cs0.x, xa.x), A::mul(cs0.y, xb.y));
                    ya.y = A::add(A::mul(cs0.x, xa.y), A::mul(cs0.y, xb.x));
                    yb.x = A::sub(A::mul(cs0.x, xb.x), A::mul(cs0.y, xa.y));
                    yb.y = A::add(A::mul(cs0.x, xb.y), A::mul(cs0.y, xa.x));
                    C[ab0.x] = ya;
                    C[ab0.y] = yb;
                }
                __syncwarp();
                e0 = e1;
                e1 = e2;
                ab0 = ab1;
                cs0 = cs1;
            }
            if (ustage) phase(Us);
            else phase(Uf);
            __syncwarp();
        }
    }
}

// Two vectors per warp (static coefficients): both follow the same rotation
// schedule with the same coefficients, so a lane fetches its chunk's pair and
// coefficients once and rotates the pair in both vectors; a site's amplitudes
// of the two vectors sit next to each other (one 16-byte shared load in FP32).
// Each vector keeps its own start frame, half-step phases and response, and
// sees the float operations of k_abs_trotter_wv, so the results are bitwise
// those of that kernel.
template <typename R> struct TPair {
    typename Vec2<R>::T a, b;
};

template <typename R, bool SM>
__global__ void k_abs_trotter_wv2(DevTraj T, TrotterPlan P, AbsJob J, double2 *resp, int nvec,
                                  const int *__restrict__ chk_g, int nchk) {
    typedef typename Vec2<R>::T R2;
    typedef TPair<R> P2;
    typedef Ar<R> A;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = P.n, K = P.k, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, W = blockDim.x >> 5;
    unsigned char *sp = smem_raw;
    int *chk = (int *)sp;  // [nchk + 4]: chunk bounds, then K (empty chunks)
    sp += ((size_t)(nchk + 4) * sizeof(int) + 15) & ~(size_t)15;
    R2 *tcs = (R2 *)sp;  // SM: [K + 32] coefficients
    unsigned *tab = (unsigned *)(sp + (SM ? (((size_t)(K + 32) * sizeof(R2) + 15) & ~(size_t)15) : 0));  // SM: pairs
    if (SM) sp = (unsigned char *)tab + (((size_t)(K + 32) * sizeof(unsigned) + 15) & ~(size_t)15);
    const int nc = n + 32;  // sites and the 32 spare sites
    P2 *C = (P2 *)sp + (size_t)warp * nc;
    for (int e = threadIdx.x; e < nchk + 4; e += blockDim.x) chk[e] = e <= nchk ? chk_g[e] : K;
    R2 unit;
    unit.x = 1;
    unit.y = 0;
    if (SM) {
        for (int e = threadIdx.x; e < K + 32; e += blockDim.x) {
            const int2 ab = e < K ? P.pairs[e] : make_int2(n + e - K, n + e - K);
            tab[e] = (unsigned)ab.x | ((unsigned)ab.y << 16);
            tcs[e] = e < K ? ((const R2 *)P.rot)[e] : unit;
        }
    }
    __syncthreads();
    const int v0 = (blockIdx.x * W + warp) * 2, v1 = v0 + 1;
    if (v0 >= nvec) return;
    const bool has1 = v1 < nvec;
    const int x0 = v0 % 3, x1 = v1 % 3;
    const long ti0 = (long)(J.begin + v0 / 3) * J.sample, ti1 = (long)(J.begin + (has1 ? v1 : v0) / 3) * J.sample;
    for (int a = lane; a < nc; a += 32) {
        P2 z;
        z.a.x = a < n ? (R)traj_mu(T, ti0, x0, a) : (R)0;
        z.b.x = a < n && has1 ? (R)traj_mu(T, ti1, x1, a) : (R)0;
        z.a.y = z.b.y = 0;
        C[a] = z;
    }
    const R2 *U = (const R2 *)P.U;
    const R2 *Rf = SM ? tcs : (const R2 *)P.rot;
    const int2 spare = make_int2(n + lane, n + lane);
    auto rot1 = [&](R2 &xa, R2 &xb, const R2 cs) {  // propagate.c:876-888
        R2 ya, yb;
        ya.x = A::sub(A::mul(cs.x, xa.x), A::mul(cs.y, xb.y));
        ya.y = A::add(A::mul(cs.x, xa.y), A::mul(cs.y, xb.x));
        yb.x = A::sub(A::mul(cs.x, xb.x), A::mul(cs.y, xa.y));
        yb.y = A::add(A::mul(cs.x, xb.y), A::mul(cs.y, xa.x));
        xa = ya;
        xb = yb;
    };
    auto mulu = [&](R2 z, R2 u) {
        R2 o;
        o.x = A::sub(A::mul(z.x, u.x), A::mul(z.y, u.y));
        o.y = A::add(A::mul(z.y, u.x), A::mul(z.x, u.y));
        return o;
    };
    for (int t1 = 0; t1 < J.tmax; t1++) {
        const long ta = ti0 + t1, tb = ti1 + t1;
        const bool step = t1 + 1 < J.tmax;
        const R2 *Ua = U + (ta - P.f0) * n, *Ub = U + (tb - P.f0) * n;
        double re0 = 0, im0 = 0, re1 = 0, im1 = 0;
#pragma unroll 4
        for (int a = lane; a < n; a += 32) {
            const P2 z = C[a];
            const R m0 = (R)traj_mu(T, ta, x0, a), m1 = (R)traj_mu(T, tb, x1, a);
            re0 += (double)A::mul(m0, z.a.x);
            im0 += (double)A::mul(m0, z.a.y);
            re1 += (double)A::mul(m1, z.b.x);
            im1 += (double)A::mul(m1, z.b.y);
        }
        const double2 rs0 = resp_sum_warp(re0, im0, n), rs1 = resp_sum_warp(re1, im1, n);
        if (lane == 0) {
            resp[(size_t)v0 * J.tmax + t1] = rs0;
            if (has1) resp[(size_t)v1 * J.tmax + t1] = rs1;
        }
        if (!step) break;
        auto phase = [&]() {  // propagate.c:870-873 / 891-894, each vector with its frame's phases
#pragma unroll 4
            for (int a = lane; a < n; a += 32) {
                P2 z = C[a];
                z.a = mulu(z.a, Ua[a]);
                z.b = mulu(z.b, Ub[a]);
                C[a] = z;
            }
        };
        for (int sub = 0; sub < J.ts; sub++) {
            phase();
            __syncwarp();
            int e0 = chk[1], e1 = chk[2];
            int2 ab0;
            R2 cs0;
            auto fetch = [&](int k, int end, int2 &ab, R2 &cs) {
                if (SM) {  // identity entry congruent to k mod 32: no bank conflict with the chunk
                    k = k < end ? k : K + ((k - K) & 31);
                    const unsigned w = tab[k];
                    ab = make_int2((int)(w & 0xffffu), (int)(w >> 16));
                    cs = Rf[k];
                } else {
                    ab = k < end ? P.pairs[k] : spare;
                    cs = k < end ? Rf[k] : unit;
                }
            };
            fetch(chk[0] + lane, e0, ab0, cs0);
#pragma unroll 2
            for (int c = 0; c < nchk; c++) {
                int2 ab1;
                R2 cs1;
                fetch(e0 + lane, e1, ab1, cs1);
                const int e2 = chk[c + 3];
                P2 pa = C[ab0.x], pb = C[ab0.y];
                rot1(pa.a, pb.a, cs0);
                rot1(pa.b, pb.b, cs0);
                C[ab0.x] = pa;
                C[ab0.y] = pb;
                __syncwarp();
                e0 = e1;
                e1 = e2;
                ab0 = ab1;
                cs0 = cs1;
            }
            phase();
            __syncwarp();
        }
    }
}

// ------------------------------------------------------------ RK4
template <typename R>
__global__ void k_prep_rk4(DevTraj T, Rk4Plan P, R fsub) {
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (tid >= P.nf * P.k) return;
    long fi = tid / P.k;
    int k = (int)(tid % P.k);
    long t = P.f0 + fi;
    int2 ab = P.entries[k];
    float h;
    bool keep;
    if (ab.x == ab.y) {
        h = traj_diag(T, t, ab.x, P.singleshift != 0);
        keep = true;
    } else {
        h = traj_coupling(T, t, ab.x, ab.y);
        keep = fabsf(h) > T.cut;  // propagate.c:298
    }
    R v = keep ? Ar<R>::mul((R)fsub, (R)h) : (R)0;
    ((R *)P.val)[fi * P.k + k] = v;
}

template <typename R>
__global__ void k_abs_rk4(DevTraj T, Rk4Plan P, AbsJob J, double2 *resp, int nvec) {
    typedef typename Vec2<R>::T R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *S = (R2 *)smem_raw;
    const int B = blockDim.x, lane = threadIdx.x, n = P.n;
    int v = blockIdx.x * B + lane;
    if (v >= nvec) return;
    int s = J.begin + v / 3, x = v % 3;
    long ti = (long)s * J.sample;
    for (int i = 0; i < n; i++) {
        R2 z;
        z.x = (R)traj_mu(T, ti, x, i);
        z.y = 0;
        S[i * B + lane] = z;
    }
    for (int t1 = 0; t1 < J.tmax; t1++) {
        long tj = ti + t1;
        resp[(size_t)v * J.tmax + t1] = dot_mu<R>(T, tj, x, S, B, lane, n);
        if (t1 == J.tmax - 1) break;
        rk4_apply<R>(S, B, lane, n, P.k, P.entries, (const R *)P.val + (tj - P.f0) * P.k, J.ts);
    }
}

// ------------------------------------------------------------ sparse Taylor
// Truncation tolerance of the exact propagator's series per step, relative
// to the vector's norm: below the unit roundoff of the arithmetic (FP32
// 6.0e-8, FP64 1.1e-16), so truncation adds less than one rounding of the
// step it ends.
constexpr double kSeriesTolF32 = 1e-8, kSeriesTolF64 = 1e-16;

// Order of the Taylor series of exp(-i H f) per frame: the smallest K with
// b^(K+1)/(K+1)! <= tol, b = |f| * (max|h_ii| + max row sum |J|) >= ||H f||_2.
// H is Hermitian, so the remainder's 2-norm is the largest remainder of the
// scalar series of exp(-i x) over the eigenvalues, and |x|^(K+1)/(K+1)!
// bounds that for real x (Lagrange form).
template <typename R>
__global__ void k_prep_taylor(DevTraj T, TaylorPlan P, double rowabs, double f, double tol, int *order) {
    long fi = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (fi >= P.nf) return;
    long t = P.f0 + fi;
    double dmax = 0;
    for (int i = 0; i < P.n; i++) dmax = fmax(dmax, fabs((double)traj_diag(T, t, i, P.singleshift != 0)));
    double b = fabs(f) * (dmax + rowabs), term = 1.0;
    int K = 0;
    for (K = 0; K < 60; K++) {
        term *= b / (K + 1);
        if (term <= tol) break;
    }
    order[fi] = K < 1 ? 1 : K;
}

template <typename R, int G, int RPT>
__global__ void __launch_bounds__(512) k_abs_taylor(DevTraj T, TaylorPlan P, AbsJob J, double2 *resp, int nvec) {
    typedef typename Vec2<R>::T R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = P.n, tid = threadIdx.x, NT = blockDim.x;
    R2 *cur = (R2 *)smem_raw, *nxt = cur + (size_t)n * G;
    double *red = (double *)(nxt + (size_t)n * G);  // [NT/32][2G]
    const int v0 = blockIdx.x * G;
    int xg[G];
    long tig[G];
    bool valid[G];
#pragma unroll
    for (int g = 0; g < G; g++) {
        int v = v0 + g;
        valid[g] = v < nvec;
        int vv = valid[g] ? v : v0;
        xg[g] = vv % 3;
        tig[g] = (long)(J.begin + vv / 3) * J.sample;
    }
    R2 psi[RPT][G];
    float dg[RPT][G];
#pragma unroll
    for (int r = 0; r < RPT; r++) {
        int i = tid + r * NT;
#pragma unroll
        for (int g = 0; g < G; g++) {
            psi[r][g].x = (i < n) ? (R)traj_mu(T, tig[g], xg[g], i) : (R)0;
            psi[r][g].y = 0;
        }
    }
    const R *jval = (const R *)P.val;
    for (int t1 = 0; t1 < J.tmax; t1++) {
        // response (absorption.c:128-130): block reduction of mu.psi per vector
        double part[2 * G];
#pragma unroll
        for (int g = 0; g < G; g++) {
            double re = 0, im = 0;
#pragma unroll
            for (int r = 0; r < RPT; r++) {
                int i = tid + r * NT;
                if (i < n) {
                    R m = (R)traj_mu(T, tig[g] + t1, xg[g], i);
                    re += (double)(m * psi[r][g].x);
                    im += (double)(m * psi[r][g].y);
                }
            }
            part[2 * g] = re;
            part[2 * g + 1] = im;
        }
#pragma unroll
        for (int q = 0; q < 2 * G; q++)
            for (int o = 16; o > 0; o >>= 1) part[q] += __shfl_xor_sync(0xffffffffu, part[q], o);
        if ((tid & 31) == 0)
#pragma unroll
            for (int q = 0; q < 2 * G; q++) red[(tid >> 5) * 2 * G + q] = part[q];
        __syncthreads();
        if (tid < G && valid[tid]) {
            double re = 0, im = 0;
            for (int w = 0; w < NT / 32; w++) { re += red[w * 2 * G + 2 * tid]; im += red[w * 2 * G + 2 * tid + 1]; }
            resp[(size_t)(v0 + tid) * J.tmax + t1] = make_double2(re, im);
        }
        if (t1 == J.tmax - 1) break;
        // per-frame diagonal and series order
        int K = 1;
#pragma unroll
        for (int g = 0; g < G; g++) {
            long tj = tig[g] + t1;
            K = max(K, P.order[tj - P.f0]);
#pragma unroll
            for (int r = 0; r < RPT; r++) {
                int i = tid + r * NT;
                dg[r][g] = (i < n) ? traj_diag(T, tj, i, P.singleshift != 0) : 0.0f;
            }
        }
        // psi <- sum_k (-i f H)^k / k! psi ; cur holds the current term
#pragma unroll
        for (int r = 0; r < RPT; r++) {
            int i = tid + r * NT;
            if (i < n)
#pragma unroll
                for (int g = 0; g < G; g++) cur[(size_t)i * G + g] = psi[r][g];
        }
        for (int k = 1; k <= K; k++) {
            __syncthreads();
            R c = (R)(J.f / k);
#pragma unroll
            for (int r = 0; r < RPT; r++) {
                int i = tid + r * NT;
                if (i >= n) continue;
                R2 y[G];
#pragma unroll
                for (int g = 0; g < G; g++) {
                    R2 z = cur[(size_t)i * G + g];
                    y[g].x = (R)dg[r][g] * z.x;
                    y[g].y = (R)dg[r][g] * z.y;
                }
                for (int e = P.row_ptr[i]; e < P.row_ptr[i + 1]; e++) {
                    int j = P.col[e];
                    R w = jval[e];
                    const R2 *cj = cur + (size_t)j * G;
#pragma unroll
                    for (int g = 0; g < G; g++) {
                        R2 z = cj[g];
                        y[g].x += w * z.x;
                        y[g].y += w * z.y;
                    }
                }
#pragma unroll
                for (int g = 0; g < G; g++) {
                    R2 nz;
                    nz.x = c * y[g].y;   // (-i)(c)(y) = c*y.im - i c*y.re
                    nz.y = -c * y[g].x;
                    nxt[(size_t)i * G + g] = nz;
                    psi[r][g].x += nz.x;
                    psi[r][g].y += nz.y;
                }
            }
            __syncthreads();
            R2 *tmp = cur;
            cur = nxt;
            nxt = tmp;
        }
        __syncthreads();
    }
}

// Coupling pattern of HamiltonianType Full trajectories: flag[idx] = 1 for
// packed off-diagonal idx when |J| > cut in any frame of [f0, f0+nf).
__global__ void k_pattern_scan(DevTraj T, long f0, long nf, int *flag) {
    long nn2 = (long)T.n * (T.n + 1) / 2;
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (tid >= nn2) return;
    int a = 0;
    long rem = tid;
    while (rem >= T.n - a) { rem -= T.n - a; a++; }
    int b = a + (int)rem;
    if (a == b) return;
    int any = 0;
    for (long t = f0; t < f0 + nf && !any; t++) any = fabsf(traj_coupling(T, t, a, b)) > T.cut;
    flag[tid] = any;
}


// Sparse Taylor propagation, vectors across lanes.  A CTA owns G vectors
// (G in {4, 8}); lane = g + G*q handles vector g for row slot q, so one warp
// instruction covers 32/G consecutive rows of G vectors and reads, for each
// neighbour j, the G contiguous vector entries of row j (rows padded to G+2
// complex numbers to spread the rows over the shared-memory banks).  Rows
// are interleaved over warps (row = q + QR*(warp + NW*it)); the current
// Taylor term lives in shared memory (double buffered) and the partial sum
// psi and the frame diagonals in registers.
template <typename R, int G, int IT>
__global__ void __launch_bounds__(512) k_abs_taylor2(DevTraj T, TaylorPlan P, AbsJob J, double2 *resp, int nvec) {
    typedef typename Vec2<R>::T R2;
    constexpr int QR = 32 / G, RS = G + 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = P.n, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, NW = blockDim.x >> 5;
    const int g = lane % G, q = lane / G;
    R2 *cur = (R2 *)smem_raw, *nxt = cur + (size_t)n * RS;
    double *red = (double *)(nxt + (size_t)n * RS);  // [NW][G][2]
    const int v = blockIdx.x * G + g;
    const bool valid = v < nvec;
    const int vv = valid ? v : blockIdx.x * G;
    const int x = vv % 3;
    const long ti = (long)(J.begin + vv / 3) * J.sample;
    int rows[IT];
    R2 psi[IT];
    float dg[IT];
#pragma unroll
    for (int it = 0; it < IT; it++) {
        int i = q + QR * (warp + NW * it);
        rows[it] = i < n ? i : -1;
        psi[it].x = i < n ? (R)traj_mu(T, ti, x, i) : (R)0;
        psi[it].y = 0;
    }
    const R *jval = (const R *)P.val;
    for (int t1 = 0; t1 < J.tmax; t1++) {
        const long tj = ti + t1;
        double re = 0, im = 0;
#pragma unroll
        for (int it = 0; it < IT; it++)
            if (rows[it] >= 0) {
                R m = (R)traj_mu(T, tj, x, rows[it]);
                re += (double)(m * psi[it].x);
                im += (double)(m * psi[it].y);
            }
        for (int o = G; o < 32; o <<= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, o);
            im += __shfl_xor_sync(0xffffffffu, im, o);
        }
        if (q == 0) { red[(warp * G + g) * 2] = re; red[(warp * G + g) * 2 + 1] = im; }
        __syncthreads();
        if (tid < G && blockIdx.x * G + tid < nvec) {
            double sr = 0, si = 0;
            for (int w = 0; w < NW; w++) { sr += red[(w * G + tid) * 2]; si += red[(w * G + tid) * 2 + 1]; }
            resp[(size_t)(blockIdx.x * G + tid) * J.tmax + t1] = make_double2(sr, si);
        }
        if (t1 == J.tmax - 1) break;
        // series order: the largest over the CTA's vectors (their frames differ)
        int K = P.order[tj - P.f0];
        for (int o = 1; o < G; o <<= 1) K = max(K, __shfl_xor_sync(0xffffffffu, K, o));
#pragma unroll
        for (int it = 0; it < IT; it++) {
            dg[it] = rows[it] >= 0 ? traj_diag(T, tj, rows[it], P.singleshift != 0) : 0.0f;
            if (rows[it] >= 0) cur[(size_t)rows[it] * RS + g] = psi[it];
        }
        R2 *a = cur, *b = nxt;
        for (int k = 1; k <= K; k++) {
            __syncthreads();
            const R c = (R)(J.f / k);
#pragma unroll
            for (int it = 0; it < IT; it++) {
                const int i = rows[it];
                if (i < 0) continue;
                R2 z = a[(size_t)i * RS + g];
                R yr = (R)dg[it] * z.x, yi = (R)dg[it] * z.y;
                const int e1 = P.row_ptr[i + 1];
                for (int e = P.row_ptr[i]; e < e1; e++) {
                    const int j = P.col[e];
                    const R w = jval[e];
                    R2 zz = a[(size_t)j * RS + g];
                    yr += w * zz.x;
                    yi += w * zz.y;
                }
                R2 nz;
                nz.x = c * yi;  // (-i)(c)(y)
                nz.y = -c * yr;
                b[(size_t)i * RS + g] = nz;
                psi[it].x += nz.x;
                psi[it].y += nz.y;
            }
            R2 *tmp = a;
            a = b;
            b = tmp;
        }
        __syncthreads();
    }
}

// Sparse Taylor propagation with the coupling matrix in shared memory as a
// sliced ELL: slice s = rows 4s..4s+3, Ls entries per row (the slice's
// longest row, shorter rows padded with zero weights), entry = (offset of the
// neighbour row in a state of NISE_T3_ROW vectors per row, weight), stored
// [slot][row in slice] so 4 lanes read 4 consecutive entries.  The state is
// single-buffered: the next Taylor term of a thread's rows is kept in
// registers until every warp has read the current term, then written back.
//
// G vectors per CTA: lane = (vector g, row q of a slice, slice so of the
// 8 / G slices a warp instruction covers).  G = 8 is the throughput layout
// (one slice per warp instruction, rows of 8 vectors); G = 1 covers 8 slices
// per warp instruction, so a CTA finishes its vector several times sooner:
// the launcher gives it the vectors of a last, partial wave, or every vector
// when there are fewer than the SMs.  Vectors v0 .. v0+nvec-1.
//
// NT threads per CTA.  NT = 512 keeps each row's diagonal element in
// registers; above 512 (fewer registers per thread, more warps to hide the
// shared-memory latency) the diagonal of every (row, vector) is kept in
// shared memory instead.
template <typename R> struct EllEnt;
template <> struct EllEnt<float> { int off; float v; };
template <> struct EllEnt<double> { int off; int pad; double v; };

// CHEB: the Chebyshev form of the same exact step (FP32; P.order holds the
// Chebyshev orders, P.cheb_inv_r and P.cheb_coef the frame's 1/R and
// coefficients, as k_prep_cheb writes them): per own row T_(k-2) stays in a
// register next to the accumulated result.
template <typename R, int IT, int G, int NT, bool CHEB = false>
__global__ void __launch_bounds__(NT, 1) k_abs_taylor3(DevTraj T, TaylorPlan P, AbsJob J, double2 *resp, int v0, int nvec,
                                                    const EllEnt<R> *__restrict__ ell_g, const int *__restrict__ sptr_g,
                                                    int nslices, int nent, const int *__restrict__ rows_g) {
    typedef typename Vec2<R>::T R2;
    constexpr int QR = 4, SPW = 8 / G, RS = G == 8 ? NISE_T3_ROW : G, KC = NISE_CHEB_KMAX + 1;
    static_assert(G == 8 || G == 1, "G = 8 or 1 vectors per CTA");
    static_assert(!CHEB || sizeof(R) == 4, "the Chebyshev tables are FP32");
    constexpr bool kDgShared = NT > 512;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = P.n, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, NW = blockDim.x >> 5;
    const int g = lane % G, q = (lane / G) % QR, so = lane / (G * QR);
    R2 *cur = (R2 *)smem_raw;
    float *dgs = (float *)(cur + (size_t)n * RS);  // [n][G] diagonal of each vector's frame (kDgShared)
    EllEnt<R> *ell = (EllEnt<R> *)(dgs + (kDgShared ? (size_t)n * G : 0));
    int *sptr = (int *)(ell + nent);
    int *rows = sptr + nslices + 1;  // [nslices][4] site of each slice row (n: padding)
    double *red = (double *)(((uintptr_t)(rows + 4 * nslices) + 15) & ~(uintptr_t)15);
    for (int e = tid; e < nent; e += blockDim.x) ell[e] = ell_g[e];
    for (int e = tid; e <= nslices; e += blockDim.x) sptr[e] = sptr_g[e];
    for (int e = tid; e < 4 * nslices; e += blockDim.x) rows[e] = rows_g[e];
    __syncthreads();
    auto rowof = [&](int sl) { return sl < nslices ? rows[q + QR * sl] : n; };
    auto slice = [&](int it) { return (warp + NW * it) * SPW + so; };
    // a neighbour's state: entry offsets are byte offsets of rows of NISE_T3_ROW vectors
    const R2 *curg = cur + g;
    auto nbr = [&](int offb) -> R2 {
        if (RS == NISE_T3_ROW) return *(const R2 *)((const char *)curg + offb);
        return curg[(offb / (int)(NISE_T3_ROW * sizeof(R2))) * RS];
    };
    const int v = blockIdx.x * G + g;
    const bool valid = v < nvec;
    const int vv = v0 + (valid ? v : blockIdx.x * G);
    const int x = vv % 3;
    const long ti = (long)(J.begin + vv / 3) * J.sample;
    R2 psi[IT], nx[IT], prev[CHEB ? IT : 1];
    float dg[kDgShared ? 1 : IT];
#pragma unroll
    for (int it = 0; it < IT; it++) {
        int i = rowof(slice(it));
        psi[it].x = i < n ? (R)traj_mu(T, ti, x, i) : (R)0;
        psi[it].y = 0;
    }
    __syncthreads();
    for (int t1 = 0; t1 < J.tmax; t1++) {
        const long tj = ti + t1;
        double re = 0, im = 0;
#pragma unroll
        for (int it = 0; it < IT; it++) {
            int i = rowof(slice(it));
            if (i < n) {
                R m = (R)traj_mu(T, tj, x, i);
                re += (double)(m * psi[it].x);
                im += (double)(m * psi[it].y);
            }
        }
        for (int o = G; o < 32; o <<= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, o);
            im += __shfl_xor_sync(0xffffffffu, im, o);
        }
        if (lane < G) { red[(warp * G + g) * 2] = re; red[(warp * G + g) * 2 + 1] = im; }
        __syncthreads();
        if (tid < G && blockIdx.x * G + tid < nvec) {
            double sr = 0, si = 0;
            for (int w = 0; w < NW; w++) { sr += red[(w * G + tid) * 2]; si += red[(w * G + tid) * 2 + 1]; }
            resp[(size_t)(v0 + blockIdx.x * G + tid) * J.tmax + t1] = make_double2(sr, si);
        }
        if (t1 == J.tmax - 1) break;
        const long fl = tj - P.f0;
        int K = P.order[fl];
        for (int o = 1; o < G; o <<= 1) K = max(K, __shfl_xor_sync(0xffffffffu, K, o));
        R ir = 0, ir2 = 0;
        const float2 *cf = nullptr;
        float cen = 0.f;  // Chebyshev: the diagonal relative to the frame's centre
        if constexpr (CHEB) {
            ir = (R)P.cheb_inv_r[fl];
            ir2 = 2 * ir;
            cf = P.cheb_coef + fl * KC;
            cen = P.cheb_center[fl];
        }
#pragma unroll
        for (int it = 0; it < IT; it++) {
            int i = rowof(slice(it));
            float d = i < n ? traj_diag(T, tj, i, P.singleshift != 0) : 0.0f;
            if constexpr (CHEB) d = i < n ? __fsub_rn(d, cen) : 0.0f;
            if (kDgShared) {
                if (i < n) dgs[(size_t)i * G + g] = d;
            } else {
                dg[it] = d;
            }
            if (i < n) cur[(size_t)i * RS + g] = psi[it];
            if constexpr (CHEB) {  // psi becomes a_0 T_0 (a_0 complex: the centre's phase); T_0 is kept
                const float2 a0 = cf[0];
                const R2 z = psi[it];
                prev[it] = z;
                psi[it].x = (R)a0.x * z.x - (R)a0.y * z.y;
                psi[it].y = (R)a0.x * z.y + (R)a0.y * z.x;
            }
        }
        for (int k = 1; k <= K; k++) {
            __syncthreads();
            const R c = (R)(J.f / k);
#pragma unroll
            for (int it = 0; it < IT; it++) {
                const int sl = slice(it), i = rowof(sl);
                if (sl >= nslices) continue;
                const int ic = i < n ? i : 0;
                R2 z = cur[(size_t)ic * RS + g];
                const R d = kDgShared ? (R)dgs[(size_t)ic * G + g] : (R)dg[kDgShared ? 0 : it];
                R yr = d * z.x, yi = d * z.y;
                const int b0 = sptr[sl], b1 = sptr[sl + 1];
                // the next entry is loaded one iteration ahead (past the slice it
                // is not used; the read stays inside this CTA's shared memory)
                EllEnt<R> en = ell[b0 + q];
                for (int e = b0 + q; e < b1; e += QR) {
                    const EllEnt<R> nen = ell[e + QR];
                    R2 zz = nbr(en.off);
                    yr += en.v * zz.x;
                    yi += en.v * zz.y;
                    en = nen;
                }
                if constexpr (CHEB) {  // T_1 = (H/R) T_0, T_k = 2 (H/R) T_(k-1) - T_(k-2)
                    if (k == 1) {
                        nx[it].x = ir * yr;
                        nx[it].y = ir * yi;
                    } else {
                        nx[it].x = ir2 * yr - prev[it].x;
                        nx[it].y = ir2 * yi - prev[it].y;
                    }
                    prev[it] = z;
                } else {
                    nx[it].x = c * yi;  // (-i)(c)(y)
                    nx[it].y = -c * yr;
                }
            }
            __syncthreads();
            R2 a;
            if constexpr (CHEB) {
                const float2 ak = cf[k];
                a.x = (R)ak.x;
                a.y = (R)ak.y;
            }
#pragma unroll
            for (int it = 0; it < IT; it++) {
                const int sl = slice(it), i = rowof(sl);
                if (sl >= nslices || i >= n) continue;
                cur[(size_t)i * RS + g] = nx[it];
                if constexpr (CHEB) {
                    psi[it].x += a.x * nx[it].x - a.y * nx[it].y;
                    psi[it].y += a.x * nx[it].y + a.y * nx[it].x;
                } else {
                    psi[it].x += nx[it].x;
                    psi[it].y += nx[it].y;
                }
            }
        }
        __syncthreads();
    }
}

// The sliced-ELL Taylor kernel with 4 vectors per CTA (FP32): half the
// register state of k_abs_taylor3 per CTA, so two CTAs (32 warps) share an
// SM and hide the shared-memory latency better; the ELL (8-row slices whose
// rows cover the four residues of the site index mod 4 twice, rows of 4
// complex numbers = 32 bytes, so each residue class owns a quarter of the
// banks) stays in global memory and is read through the L1 cache.
template <int IT>
__global__ void __launch_bounds__(512, 2) k_abs_taylor4(DevTraj T, TaylorPlan P, AbsJob J, double2 *resp, int nvec) {
    constexpr int G = 4, QR = 8, RS = 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = P.n, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, NW = blockDim.x >> 5;
    const int g = lane % G, q = lane / G;
    float2 *cur = (float2 *)smem_raw;
    double *red = (double *)(cur + (size_t)n * RS);
    const int2 *__restrict__ ell = (const int2 *)P.ell4;  // (state offset, weight bits)
    const int *__restrict__ sptr = P.ell4_sptr;
    const int *__restrict__ rows = P.ell4_rows;
    const int nslices = P.ell4_nslices;
    auto rowof = [&](int sl) { return sl < nslices ? __ldg(rows + q + QR * sl) : n; };
    const int v = blockIdx.x * G + g;
    const bool valid = v < nvec;
    const int vv = valid ? v : blockIdx.x * G;
    const int x = vv % 3;
    const long ti = (long)(J.begin + vv / 3) * J.sample;
    float2 psi[IT], nx[IT];
    float dg[IT];
#pragma unroll
    for (int it = 0; it < IT; it++) {
        int i = rowof(warp + NW * it);
        psi[it].x = i < n ? traj_mu(T, ti, x, i) : 0.f;
        psi[it].y = 0;
    }
    for (int t1 = 0; t1 < J.tmax; t1++) {
        const long tj = ti + t1;
        double re = 0, im = 0;
#pragma unroll
        for (int it = 0; it < IT; it++) {
            int i = rowof(warp + NW * it);
            if (i < n) {
                float m = traj_mu(T, tj, x, i);
                re += (double)(m * psi[it].x);
                im += (double)(m * psi[it].y);
            }
        }
        for (int o = G; o < 32; o <<= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, o);
            im += __shfl_xor_sync(0xffffffffu, im, o);
        }
        if (q == 0) { red[(warp * G + g) * 2] = re; red[(warp * G + g) * 2 + 1] = im; }
        __syncthreads();
        if (tid < G && blockIdx.x * G + tid < nvec) {
            double sr = 0, si = 0;
            for (int w = 0; w < NW; w++) { sr += red[(w * G + tid) * 2]; si += red[(w * G + tid) * 2 + 1]; }
            resp[(size_t)(blockIdx.x * G + tid) * J.tmax + t1] = make_double2(sr, si);
        }
        if (t1 == J.tmax - 1) break;
        int K = P.order[tj - P.f0];
        for (int o = 1; o < G; o <<= 1) K = max(K, __shfl_xor_sync(0xffffffffu, K, o));
#pragma unroll
        for (int it = 0; it < IT; it++) {
            int i = rowof(warp + NW * it);
            dg[it] = i < n ? traj_diag(T, tj, i, P.singleshift != 0) : 0.0f;
            if (i < n) cur[(size_t)i * RS + g] = psi[it];
        }
        for (int k = 1; k <= K; k++) {
            __syncthreads();
            const float c = (float)(J.f / k);
#pragma unroll
            for (int it = 0; it < IT; it++) {
                const int sl = warp + NW * it, i = rowof(sl);
                if (sl >= nslices) continue;
                float2 z = cur[(size_t)(i < n ? i : 0) * RS + g];
                float yr = dg[it] * z.x, yi = dg[it] * z.y;
                const int b0 = __ldg(sptr + sl), b1 = __ldg(sptr + sl + 1);
                for (int e = b0 + q; e < b1; e += QR) {
                    const int2 en = __ldg(ell + e);
                    const float w = __int_as_float(en.y);
                    float2 zz = cur[en.x + g];
                    yr += w * zz.x;
                    yi += w * zz.y;
                }
                nx[it].x = c * yi;  // (-i)(c)(y)
                nx[it].y = -c * yr;
            }
            __syncthreads();
#pragma unroll
            for (int it = 0; it < IT; it++) {
                const int sl = warp + NW * it, i = rowof(sl);
                if (sl >= nslices || i >= n) continue;
                cur[(size_t)i * RS + g] = nx[it];
                psi[it].x += nx[it].x;
                psi[it].y += nx[it].y;
            }
        }
        __syncthreads();
    }
}

// Chebyshev expansion of the exact step (FP32, sliced ELL in shared memory).
//
// With c_t the centre of frame t's diagonal range, R_t the Gershgorin radius
// of H - c_t (half the diagonal range + max row sum of |J|) and x = f R_t,
// exp(-i f H) = exp(-i f c_t) sum_k a_k T_k((H - c_t) / R_t) with
// a_0 = J_0(x), a_k = 2 (-i)^k J_k(x) (the Jacobi-Anger expansion; the phase
// exp(-i f c_t) is folded into the stored coefficients); the
// T_k((H - c)/R) psi follow the three-term recurrence
// T_k = 2 ((H - c)/R) T_(k-1) - T_(k-2).  Centring shrinks R_t, so the order
// drops for frames whose diagonal range is off centre.  For the small
// x of a time step the Bessel coefficients fall off like (x/2)^k / k!,
// against x^k / k! for the Taylor terms, so fewer sparse products reach the
// same tolerance.  Per frame the prep kernel stores 1/R_t, c_t, the
// coefficients and the order K_t (2 * sum_(k>K) |J_k(x)| <= tol).
__global__ void k_prep_cheb(DevTraj T, TaylorPlan P, double rowabs, double f, double tol, int *order,
                            float *inv_r, float *center, float2 *coef) {
    long fi = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (fi >= P.nf) return;
    long t = P.f0 + fi;
    double lo = 0, hi = 0;
    for (int i = 0; i < P.n; i++) {
        const double d = (double)traj_diag(T, t, i, P.singleshift != 0);
        lo = i ? fmin(lo, d) : d;
        hi = i ? fmax(hi, d) : d;
    }
    const float cen = (float)(0.5 * (lo + hi));
    double R = fmax(hi - (double)cen, (double)cen - lo) + rowabs;
    if (!(R > 0)) R = 1;
    const double x = fabs(f) * R;
    // J_k(x), k = 0..KMAX+8, by Miller's downward recurrence normalised with
    // J_0 + 2 sum J_2k = 1 (valid for every x > 0; x is below 20 here).
    constexpr int KM = NISE_CHEB_KMAX + 8;
    double jv[KM + 1];
    for (int k = 0; k <= KM; k++) jv[k] = 0;
    if (x < 1e-300) {
        jv[0] = 1;
    } else {
        int M = (int)x + KM + 16;  // start well above the orders kept
        if (M & 1) M++;
        double jp = 0, j = 1e-280, sum = 0;
        for (int k = M; k >= 1; k--) {
            double jm = 2.0 * k / x * j - jp;  // J_(k-1)
            jp = j;
            j = jm;
            if (fabs(j) > 1e250) {  // rescale to stay in range
                j *= 1e-250;
                jp *= 1e-250;
                sum *= 1e-250;
                for (int q = 0; q <= KM; q++) jv[q] *= 1e-250;
            }
            if (k - 1 <= KM) jv[k - 1] = j;
            if (((k - 1) & 1) == 0 && k - 1 > 0) sum += 2 * j;
        }
        sum += jv[0];
        for (int k = 0; k <= KM; k++) jv[k] /= sum;
    }
    int K = NISE_CHEB_KMAX;
    for (int k = 1; k <= NISE_CHEB_KMAX; k++) {
        double tail = 0;
        for (int q = k + 1; q <= KM; q++) tail += fabs(jv[q]);
        if (2 * tail <= tol) {
            K = k;
            break;
        }
    }
    order[fi] = K;
    inv_r[fi] = (float)(1.0 / R);
    center[fi] = cen;
    // a_k times the phase exp(-i f c) = (pc, -ps)
    double ps, pc;
    sincos(f * (double)cen, &ps, &pc);
    float2 *c = coef + fi * (NISE_CHEB_KMAX + 1);
    for (int k = 0; k <= NISE_CHEB_KMAX; k++) {
        const double a = k ? 2 * jv[k] : jv[0];
        double ar = 0, ai = 0;
        switch (k & 3) {  // (-i)^k
        case 0: ar = a; break;
        case 1: ai = -a; break;
        case 2: ar = -a; break;
        default: ai = a; break;
        }
        c[k] = make_float2((float)(ar * pc + ai * ps), (float)(ai * pc - ar * ps));
    }
}

// k_abs_taylor3's layout (8 vectors per CTA, sliced ELL, rows of NISE_T3_ROW)
// with the Chebyshev recurrence: per own row the accumulated result, T_(k-2)
// and the new T_k stay in registers, the diagonal of the current frame in
// shared memory.
template <int IT>
__global__ void __launch_bounds__(512) k_abs_cheb3(DevTraj T, TaylorPlan P, AbsJob J, double2 *resp, int nvec,
                                                  const EllEnt<float> *__restrict__ ell_g,
                                                  const int *__restrict__ sptr_g, int nslices, int nent,
                                                  const float *__restrict__ inv_r, const float2 *__restrict__ coef,
                                                  const int *__restrict__ rows_g) {
    constexpr int G = 8, QR = 4, RS = NISE_T3_ROW, KC = NISE_CHEB_KMAX + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = P.n, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, NW = blockDim.x >> 5;
    const int g = lane % G, q = lane / G;
    float2 *cur = (float2 *)smem_raw;
    const float2 *curg = cur + g;  // ELL entry offsets are byte offsets of state rows
    float *dgs = (float *)(cur + (size_t)n * RS);  // [row][g]
    EllEnt<float> *ell = (EllEnt<float> *)(dgs + (size_t)n * G);
    int *sptr = (int *)(ell + nent);
    int *rows = sptr + nslices + 1;  // [nslices][4] site of each slice row (n: padding)
    double *red = (double *)(((uintptr_t)(rows + 4 * nslices) + 15) & ~(uintptr_t)15);
    for (int e = tid; e < nent; e += blockDim.x) ell[e] = ell_g[e];
    for (int e = tid; e <= nslices; e += blockDim.x) sptr[e] = sptr_g[e];
    for (int e = tid; e < 4 * nslices; e += blockDim.x) rows[e] = rows_g[e];
    __syncthreads();
    auto rowof = [&](int sl) { return sl < nslices ? rows[q + QR * sl] : n; };
    const int v = blockIdx.x * G + g;
    const bool valid = v < nvec;
    const int vv = valid ? v : blockIdx.x * G;
    const int x = vv % 3;
    const long ti = (long)(J.begin + vv / 3) * J.sample;
    float2 psi[IT], prev[IT], nx[IT];
#pragma unroll
    for (int it = 0; it < IT; it++) {
        int i = rowof(warp + NW * it);
        psi[it].x = i < n ? traj_mu(T, ti, x, i) : 0.f;
        psi[it].y = 0;
    }
    __syncthreads();
    for (int t1 = 0; t1 < J.tmax; t1++) {
        const long tj = ti + t1;
        double re = 0, im = 0;
#pragma unroll
        for (int it = 0; it < IT; it++) {
            int i = rowof(warp + NW * it);
            if (i < n) {
                float m = traj_mu(T, tj, x, i);
                re += (double)(m * psi[it].x);
                im += (double)(m * psi[it].y);
            }
        }
        for (int o = G; o < 32; o <<= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, o);
            im += __shfl_xor_sync(0xffffffffu, im, o);
        }
        if (q == 0) { red[(warp * G + g) * 2] = re; red[(warp * G + g) * 2 + 1] = im; }
        __syncthreads();
        if (tid < G && blockIdx.x * G + tid < nvec) {
            double sr = 0, si = 0;
            for (int w = 0; w < NW; w++) { sr += red[(w * G + tid) * 2]; si += red[(w * G + tid) * 2 + 1]; }
            resp[(size_t)(blockIdx.x * G + tid) * J.tmax + t1] = make_double2(sr, si);
        }
        if (t1 == J.tmax - 1) break;
        const long fl = tj - P.f0;
        int K = P.order[fl];
        for (int o = 1; o < G; o <<= 1) K = max(K, __shfl_xor_sync(0xffffffffu, K, o));
        const float ir = inv_r[fl], ir2 = 2.f * ir;
        const float2 *cf = coef + fl * KC;
        const float2 a0 = cf[0];  // J_0 times the centre's phase
        const float cen = P.cheb_center[fl];
#pragma unroll
        for (int it = 0; it < IT; it++) {
            int i = rowof(warp + NW * it);
            if (i < n) {
                dgs[(size_t)i * G + g] = __fsub_rn(traj_diag(T, tj, i, P.singleshift != 0), cen);
                cur[(size_t)i * RS + g] = psi[it];
            }
            prev[it] = psi[it];
            const float2 z = psi[it];
            psi[it].x = a0.x * z.x - a0.y * z.y;
            psi[it].y = a0.x * z.y + a0.y * z.x;
        }
        for (int k = 1; k <= K; k++) {
            __syncthreads();
            const float2 a = cf[k];
#pragma unroll
            for (int it = 0; it < IT; it++) {
                const int sl = warp + NW * it, i = rowof(sl);
                if (sl >= nslices) continue;
                const int ic = i < n ? i : 0;
                float2 z = cur[(size_t)ic * RS + g];
                const float d = dgs[(size_t)ic * G + g];
                float yr = d * z.x, yi = d * z.y;
                const int b0 = sptr[sl], b1 = sptr[sl + 1];
                int e = b0 + q;
                float yr2 = 0.f, yi2 = 0.f;
                for (; e + QR < b1; e += 2 * QR) {
                    EllEnt<float> e0 = ell[e], e1 = ell[e + QR];
                    float2 z0 = *(const float2 *)((const char *)curg + e0.off);
                    float2 z1 = *(const float2 *)((const char *)curg + e1.off);
                    yr += e0.v * z0.x;
                    yi += e0.v * z0.y;
                    yr2 += e1.v * z1.x;
                    yi2 += e1.v * z1.y;
                }
                if (e < b1) {
                    EllEnt<float> e0 = ell[e];
                    float2 z0 = *(const float2 *)((const char *)curg + e0.off);
                    yr += e0.v * z0.x;
                    yi += e0.v * z0.y;
                }
                yr += yr2;
                yi += yi2;
                float2 tk;
                if (k == 1) {
                    tk.x = ir * yr;
                    tk.y = ir * yi;
                } else {
                    tk.x = ir2 * yr - prev[it].x;
                    tk.y = ir2 * yi - prev[it].y;
                }
                prev[it] = z;
                nx[it] = tk;
            }
            __syncthreads();
#pragma unroll
            for (int it = 0; it < IT; it++) {
                const int sl = warp + NW * it, i = rowof(sl);
                if (sl >= nslices || i >= n) continue;
                cur[(size_t)i * RS + g] = nx[it];
                psi[it].x += a.x * nx[it].x - a.y * nx[it].y;
                psi[it].y += a.x * nx[it].y + a.y * nx[it].x;
            }
        }
        __syncthreads();
    }
}

// Sum of the per-vector responses resp[v][t] over v, in one fixed order: a
// CTA owns 32 consecutive t (lane = t, coalesced rows); warp w sums the
// vectors v = w, w + 32, ... in increasing v, then the 32 warp partials are
// added in warp order.
__global__ void __launch_bounds__(1024) k_reduce_resp(const double2 *resp, int nvec, int tmax, double2 *out) {
    __shared__ double2 part[32][33];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, t = blockIdx.x * 32 + lane;
    double re = 0, im = 0;
    if (t < tmax)
#pragma unroll 8
        for (int v = w; v < nvec; v += 32) {
            const double2 z = resp[(size_t)v * tmax + t];
            re += z.x;
            im += z.y;
        }
    part[w][lane] = make_double2(re, im);
    __syncthreads();
    if (w == 0 && t < tmax) {
        double sr = 0, si = 0;
        for (int q = 0; q < 32; q++) {
            sr += part[q][lane].x;
            si += part[q][lane].y;
        }
        out[t] = make_double2(sr, si);
    }
}

// ------------------------------------------------------------ single steps
// nise_propagate: each thread propagates one vector with its own packed H.
template <typename R>
__global__ void k_step_coupling(int n, float cut, const float *H, R *re, R *im, int nvec, int ts, R fsub) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *S = (R2 *)smem_raw;
    const int B = blockDim.x, lane = threadIdx.x;
    int v = blockIdx.x * B + lane;
    if (v >= nvec) return;
    const float *h = H + (size_t)v * n * (n + 1) / 2;
    for (int a = 0; a < n; a++) {
        R2 z;
        z.x = re[(size_t)v * n + a];
        z.y = im[(size_t)v * n + a];
        S[a * B + lane] = z;
    }
    for (int sub = 0; sub < ts; sub++) {
        for (int pass = 0; pass < 2; pass++) {
            if (pass == 1) {
                for (int a = 0; a < n; a++)
                    for (int b = a + 1; b < n; b++) {
                        float j = h[sindex(a, b, n)];
                        if (!(fabsf(j) > cut)) continue;
                        R2 cs = Cst<R>::rot(j, fsub, cut);
                        R2 xa = S[a * B + lane], xb = S[b * B + lane], ya, yb;
                        ya.x = A::sub(A::mul(cs.x, xa.x), A::mul(cs.y, xb.y));
                        ya.y = A::add(A::mul(cs.x, xa.y), A::mul(cs.y, xb.x));
                        yb.x = A::sub(A::mul(cs.x, xb.x), A::mul(cs.y, xa.y));
                        yb.y = A::add(A::mul(cs.x, xb.y), A::mul(cs.y, xa.x));
                        S[a * B + lane] = ya;
                        S[b * B + lane] = yb;
                    }
            }
            for (int a = 0; a < n; a++) {
                double arg = 0.5 * (double)h[sindex(a, a, n)] * (double)fsub;
                R ur = (R)cos(arg), ui = (R)(-sin(arg));
                R2 z = S[a * B + lane], o;
                o.x = A::sub(A::mul(z.x, ur), A::mul(z.y, ui));
                o.y = A::add(A::mul(z.y, ur), A::mul(z.x, ui));
                S[a * B + lane] = o;
            }
        }
    }
    for (int a = 0; a < n; a++) {
        R2 z = S[a * B + lane];
        re[(size_t)v * n + a] = z.x;
        im[(size_t)v * n + a] = z.y;
    }
}

template <typename R>
__global__ void k_step_rk4(int n, float cut, const float *H, R *re, R *im, int nvec, int ts, R fsub, int2 *ent_ws,
                           R *val_ws, int kmax_all) {
    typedef typename Vec2<R>::T R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *S = (R2 *)smem_raw;
    const int B = blockDim.x, lane = threadIdx.x;
    int v = blockIdx.x * B + lane;
    if (v >= nvec) return;
    const float *h = H + (size_t)v * n * (n + 1) / 2;
    int2 *ent = ent_ws + (size_t)v * kmax_all;
    R *val = val_ws + (size_t)v * kmax_all;
    int K = 0;
    for (int a = 0; a < n; a++)
        for (int b = a; b < n; b++) {
            float x = h[sindex(a, b, n)];
            if (fabsf(x) > cut || a == b) {
                ent[K] = make_int2(a, b);
                val[K] = Ar<R>::mul((R)fsub, (R)x);
                K++;
            }
        }
    for (int a = 0; a < n; a++) {
        R2 z;
        z.x = re[(size_t)v * n + a];
        z.y = im[(size_t)v * n + a];
        S[a * B + lane] = z;
    }
    rk4_apply<R>(S, B, lane, n, K, ent, val, ts);
    for (int a = 0; a < n; a++) {
        R2 z = S[a * B + lane];
        re[(size_t)v * n + a] = z.x;
        im[(size_t)v * n + a] = z.y;
    }
}

// Exact step exp(-i H f) psi by a Taylor series on the dense packed H
// (one thread per vector, for small n).
template <typename R>
__global__ void k_step_taylor(int n, const float *H, R *re, R *im, int nvec, double f) {
    typedef typename Vec2<R>::T R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int B = blockDim.x, lane = threadIdx.x;
    R2 *cur = (R2 *)smem_raw, *nxt = cur + (size_t)n * B, *acc = nxt + (size_t)n * B;
    int v = blockIdx.x * B + lane;
    if (v >= nvec) return;
    const float *h = H + (size_t)v * n * (n + 1) / 2;
    double bound = 0;
    for (int a = 0; a < n; a++) {
        double rs = 0;
        for (int b = 0; b < n; b++) rs += fabs((double)h[sindex(a, b, n)]);
        bound = fmax(bound, rs);
    }
    double bnd = fabs(f) * bound, term = exp(bnd), tol = sizeof(R) == 4 ? 1e-12 : 1e-18;
    int K;
    for (K = 0; K < 80; K++) {
        term *= bnd / (K + 1);
        if (term <= tol) break;
    }
    for (int a = 0; a < n; a++) {
        R2 z;
        z.x = re[(size_t)v * n + a];
        z.y = im[(size_t)v * n + a];
        cur[a * B + lane] = z;
        acc[a * B + lane] = z;
    }
    for (int k = 1; k <= K; k++) {
        R c = (R)(f / k);
        for (int a = 0; a < n; a++) {
            R yr = 0, yi = 0;
            for (int b = 0; b < n; b++) {
                R w = (R)h[sindex(a, b, n)];
                R2 z = cur[b * B + lane];
                yr += w * z.x;
                yi += w * z.y;
            }
            R2 nz;
            nz.x = c * yi;
            nz.y = -c * yr;
            nxt[a * B + lane] = nz;
            R2 s = acc[a * B + lane];
            s.x += nz.x;
            s.y += nz.y;
            acc[a * B + lane] = s;
        }
        R2 *tmp = cur;
        cur = nxt;
        nxt = tmp;
    }
    for (int a = 0; a < n; a++) {
        R2 z = acc[a * B + lane];
        re[(size_t)v * n + a] = z.x;
        im[(size_t)v * n + a] = z.y;
    }
}

int lanes_for(size_t bytes_per_lane, int want) {
    const size_t budget = 200 * 1024;
    int b = want;
    while (b > 1 && (size_t)b * bytes_per_lane > budget) b >>= 1;
    return b;
}

const size_t kMaxSmem = 227 * 1024;  // dynamic shared memory per CTA on sm_100

template <typename K>
int set_smem(K kernel, size_t bytes) {
    if (bytes > 48 * 1024)
        return (int)cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return 0;
}

}  // namespace

// ------------------------------------------------------------ launchers
int launch_prep_trotter(int prec, const DevTraj &T, const TrotterPlan &P, double fsub, float fsub32,
                        cudaStream_t s) {
    long per = P.n + (P.rot_static ? 0 : P.k);
    long tot = P.nf * per;
    int bs = 256;
    long grid = (tot + bs - 1) / bs;
    if (prec == 0) {
        if (tot) k_prep_trotter<float><<<grid, bs, 0, s>>>(T, P, fsub32);
        if (P.rot_static && P.k) k_prep_trotter_static<float><<<(P.k + 255) / 256, 256, 0, s>>>(T, P, fsub32);
    } else {
        if (tot) k_prep_trotter<double><<<grid, bs, 0, s>>>(T, P, fsub);
        if (P.rot_static && P.k) k_prep_trotter_static<double><<<(P.k + 255) / 256, 256, 0, s>>>(T, P, fsub);
    }
    return (int)cudaGetLastError();
}

int launch_abs_trotter(int prec, const DevTraj &T, const TrotterPlan &P, const AbsJob &J, double2 *resp,
                       cudaStream_t s) {
    int nvec = 3 * J.nsamp;
    size_t per_lane = (size_t)P.n * (prec == 0 ? sizeof(float2) : sizeof(double2));
    int B = lanes_for(per_lane, 64);
    size_t smem = per_lane * B;
    int grid = (nvec + B - 1) / B;
    int e;
    if (prec == 0) {
        if ((e = set_smem(k_abs_trotter<float>, smem))) return e;
        k_abs_trotter<float><<<grid, B, smem, s>>>(T, P, J, resp, nvec);
    } else {
        if ((e = set_smem(k_abs_trotter<double>, smem))) return e;
        k_abs_trotter<double><<<grid, B, smem, s>>>(T, P, J, resp, nvec);
    }
    return (int)cudaGetLastError();
}

int launch_abs_trotter_lv(int prec, const DevTraj &T, const TrotterPlan &P, const AbsJob &J, double2 *resp,
                          const int *lvptr, int nlev, int threads, cudaStream_t s) {
    if (J.nsamp <= 0) return 0;
    const size_t smem = (size_t)3 * P.n * ((prec == 0 ? sizeof(float2) : sizeof(double2)) + sizeof(float));
    int e;
    if (prec == 0) {
        if ((e = set_smem(k_abs_trotter_lv<float>, smem))) return e;
        k_abs_trotter_lv<float><<<J.nsamp, threads, smem, s>>>(T, P, J, resp, lvptr, nlev);
    } else {
        if ((e = set_smem(k_abs_trotter_lv<double>, smem))) return e;
        k_abs_trotter_lv<double><<<J.nsamp, threads, smem, s>>>(T, P, J, resp, lvptr, nlev);
    }
    return (int)cudaGetLastError();
}

// Warps per CTA for `units` warps of work when shared memory allows W: one CTA
// runs per SM, so the job takes rounds = ceil(units / (W * nsm)) CTA times;
// the fewest warps per CTA with that many rounds spread the work evenly (a
// CTA's time grows with its warps).  On the 1024-site lattice with 5985
// vectors (2993 warps of two): 9 warps give 333 CTAs, 2.25 rounds run as 3,
// 7 warps give 428 CTAs in the same 3 rounds.
static int even_width(int units, int W, int nsm) {
    const long rounds = ((long)units + (long)W * nsm - 1) / ((long)W * nsm);
    return (int)std::max(1L, ((long)units + rounds * nsm - 1) / (rounds * nsm));
}

// Shared memory of k_abs_trotter_wv: chunk table, rotation table (sm), W
// vectors (and their phases with ustage).
static size_t trotter_wv_smem(int prec, const TrotterPlan &P, int nchk, bool sm, bool ustage, int W) {
    const size_t r2 = prec == 0 ? sizeof(float2) : sizeof(double2);
    size_t b = ((size_t)(nchk + 4) * sizeof(int) + 15) & ~(size_t)15;
    if (sm) b += (((size_t)(P.k + 32) * r2 + 15) & ~(size_t)15) + (((size_t)(P.k + 32) * sizeof(unsigned) + 15) & ~(size_t)15);
    return b + (size_t)W * (P.n + 32) * r2 * (ustage ? 2 : 1);
}

// tables = 1: the rotation table in shared memory where it fits (else in
// global memory), 0: in global memory.  With static coefficients W vectors
// share a CTA, W = the vectors per SM (at most 16, as shared memory allows),
// so that small jobs spread over every SM; the phases are staged where
// shared memory has room for them at that W.
int launch_abs_trotter_wv(int prec, const DevTraj &T, const TrotterPlan &P, const AbsJob &J, double2 *resp,
                          const int *chk, int nchk, int tables, cudaStream_t s) {
    if (J.nsamp <= 0) return 0;
    const int nvec = 3 * J.nsamp, nsm = sm_count();
    bool sm = tables != 0 && P.n + 32 <= 65536, ustage = false;
    int W = 3;
    auto fits = [&](bool m, bool u, int w) { return trotter_wv_smem(prec, P, nchk, m, u, w) <= kMaxSmem; };
    auto widest = [&](bool m) {
        int w = std::min(16, std::max(1, (nvec + nsm - 1) / nsm));
        while (w > 1 && !fits(m, false, w)) w--;
        return w;
    };
    if (sm && !P.rot_static) {
        if (!fits(true, false, 3)) sm = false;
    } else if (sm && !fits(true, false, widest(true))) {
        sm = false;
    }
    if (sm && P.rot_static) W = widest(true);
    if (!sm) W = widest(false);
    if (!fits(sm, false, W)) return (int)cudaErrorNotSupported;
    if (sm ? P.rot_static : true) W = even_width(nvec, W, nsm);
    ustage = fits(sm, true, W);
    const size_t smem = trotter_wv_smem(prec, P, nchk, sm, ustage, W);
    const int grid = (nvec + W - 1) / W, us = ustage ? 1 : 0;
    int e;
#define NISE_WV(RT, SMT)                                                                         \
    do {                                                                                       \
        if ((e = set_smem(k_abs_trotter_wv<RT, SMT>, smem))) return e;                         \
        k_abs_trotter_wv<RT, SMT><<<grid, 32 * W, smem, s>>>(T, P, J, resp, nvec, chk, nchk, us); \
    } while (0)
    if (prec == 0) {
        if (sm) NISE_WV(float, true);
        else NISE_WV(float, false);
    } else {
        if (sm) NISE_WV(double, true);
        else NISE_WV(double, false);
    }
#undef NISE_WV
    return (int)cudaGetLastError();
}

// Two vectors per warp (static coefficients only): W warps of 2 vectors per
// CTA, W = half the vectors per SM (at most 16, as shared memory allows), the
// rotation table in shared memory where it fits.
int launch_abs_trotter_wv2(int prec, const DevTraj &T, const TrotterPlan &P, const AbsJob &J, double2 *resp,
                           const int *chk, int nchk, cudaStream_t s) {
    if (J.nsamp <= 0) return 0;
    if (!P.rot_static) return (int)cudaErrorNotSupported;
    const int nvec = 3 * J.nsamp, nsm = sm_count(), npair = (nvec + 1) / 2;
    const size_t r2 = prec == 0 ? sizeof(float2) : sizeof(double2);
    auto bytes = [&](bool m, int w) {
        size_t b = ((size_t)(nchk + 4) * sizeof(int) + 15) & ~(size_t)15;
        if (m) b += (((size_t)(P.k + 32) * r2 + 15) & ~(size_t)15) + (((size_t)(P.k + 32) * sizeof(unsigned) + 15) & ~(size_t)15);
        return b + (size_t)w * (P.n + 32) * 2 * r2;
    };
    bool sm = P.n + 32 <= 65536;
    int W = std::min(16, std::max(1, (npair + nsm - 1) / nsm));
    while (W > 1 && bytes(sm, W) > kMaxSmem) W--;
    if (sm && bytes(sm, W) > kMaxSmem) sm = false;
    if (!sm) {
        W = std::min(16, std::max(1, (npair + nsm - 1) / nsm));
        while (W > 1 && bytes(false, W) > kMaxSmem) W--;
    }
    if (bytes(sm, W) > kMaxSmem) return (int)cudaErrorNotSupported;
    W = even_width(npair, W, nsm);
    const size_t smem = bytes(sm, W);
    const int grid = (npair + W - 1) / W;
    int e;
#define NISE_WV2(RT, SMT)                                                                    \
    do {                                                                                   \
        if ((e = set_smem(k_abs_trotter_wv2<RT, SMT>, smem))) return e;                    \
        k_abs_trotter_wv2<RT, SMT><<<grid, 32 * W, smem, s>>>(T, P, J, resp, nvec, chk, nchk); \
    } while (0)
    if (prec == 0) {
        if (sm) NISE_WV2(float, true);
        else NISE_WV2(float, false);
    } else {
        if (sm) NISE_WV2(double, true);
        else NISE_WV2(double, false);
    }
#undef NISE_WV2
    return (int)cudaGetLastError();
}

int launch_prep_rk4(int prec, const DevTraj &T, const Rk4Plan &P, double fsub, float fsub32, cudaStream_t s) {
    long tot = P.nf * P.k;
    if (!tot) return 0;
    if (prec == 0) k_prep_rk4<float><<<(tot + 255) / 256, 256, 0, s>>>(T, P, fsub32);
    else k_prep_rk4<double><<<(tot + 255) / 256, 256, 0, s>>>(T, P, fsub);
    return (int)cudaGetLastError();
}

int launch_abs_rk4(int prec, const DevTraj &T, const Rk4Plan &P, const AbsJob &J, double2 *resp, cudaStream_t s) {
    int nvec = 3 * J.nsamp;
    size_t per_lane = 5 * (size_t)P.n * (prec == 0 ? sizeof(float2) : sizeof(double2));
    int B = lanes_for(per_lane, 64);
    size_t smem = per_lane * B;
    int grid = (nvec + B - 1) / B;
    int e;
    if (prec == 0) {
        if ((e = set_smem(k_abs_rk4<float>, smem))) return e;
        k_abs_rk4<float><<<grid, B, smem, s>>>(T, P, J, resp, nvec);
    } else {
        if ((e = set_smem(k_abs_rk4<double>, smem))) return e;
        k_abs_rk4<double><<<grid, B, smem, s>>>(T, P, J, resp, nvec);
    }
    return (int)cudaGetLastError();
}

int launch_prep_taylor(int prec, const DevTraj &T, TaylorPlan &P, double rowabs_max, double f, int *order,
                       cudaStream_t s) {
    double tol = prec == 0 ? kSeriesTolF32 : kSeriesTolF64;
    if (P.nf) k_prep_taylor<float><<<(P.nf + 127) / 128, 128, 0, s>>>(T, P, rowabs_max, f, tol, order);
    P.order = order;
    return (int)cudaGetLastError();
}

template <typename R, int G, int RPT>
static int run_taylor(const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp, int nvec,
                      cudaStream_t s) {
    int NT = 512;
    size_t smem = 2 * (size_t)P.n * G * sizeof(typename Vec2<R>::T) + (NT / 32) * 2 * G * sizeof(double);
    int e;
    if ((e = set_smem(k_abs_taylor<R, G, RPT>, smem))) return e;
    int grid = (nvec + G - 1) / G;
    k_abs_taylor<R, G, RPT><<<grid, NT, smem, s>>>(T, P, J, resp, nvec);
    return (int)cudaGetLastError();
}

template <typename R, int G, int IT>
static int run_taylor2(const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp, int nvec,
                       cudaStream_t s) {
    const int NT = 512;
    size_t smem = 2 * (size_t)P.n * (G + 2) * sizeof(typename Vec2<R>::T) + (NT / 32) * G * 2 * sizeof(double);
    int e;
    if ((e = set_smem(k_abs_taylor2<R, G, IT>, smem))) return e;
    k_abs_taylor2<R, G, IT><<<(nvec + G - 1) / G, NT, smem, s>>>(T, P, J, resp, nvec);
    return (int)cudaGetLastError();
}

size_t taylor3_smem(const TaylorPlan &P, size_t rsz, int G = 8, int NT = 512) {
    size_t ent = rsz == 4 ? 8 : 16;
    return (size_t)P.n * (G == 8 ? NISE_T3_ROW : G) * 2 * rsz + (NT > 512 ? (size_t)P.n * G * sizeof(float) : 0) +
           (size_t)P.ell_nent * ent + sizeof(int) * (5 * P.ell_nslices + 1) + 16 + (NT / 32) * 8 * 2 * sizeof(double);
}

template <int IT>
static int run_taylor4(const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp, int nvec, cudaStream_t s) {
    size_t smem = (size_t)P.n * 4 * sizeof(float2) + 16 * 4 * 2 * sizeof(double);
    int e;
    if ((e = set_smem(k_abs_taylor4<IT>, smem))) return e;
    k_abs_taylor4<IT><<<(nvec + 3) / 4, 512, smem, s>>>(T, P, J, resp, nvec);
    return (int)cudaGetLastError();
}

size_t cheb3_smem(const TaylorPlan &P) {
    return (size_t)P.n * NISE_T3_ROW * sizeof(float2) + (size_t)P.n * 8 * sizeof(float) + (size_t)P.ell_nent * 8 +
           sizeof(int) * (5 * P.ell_nslices + 1) + 16 + 16 * 8 * 2 * sizeof(double);
}

template <int IT>
static int run_cheb3(const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp, int nvec, cudaStream_t s) {
    size_t smem = cheb3_smem(P);
    int e;
    if ((e = set_smem(k_abs_cheb3<IT>, smem))) return e;
    k_abs_cheb3<IT><<<(nvec + 7) / 8, 512, smem, s>>>(T, P, J, resp, nvec, (const EllEnt<float> *)P.ell, P.ell_sptr,
                                                      P.ell_nslices, P.ell_nent, P.cheb_inv_r, P.cheb_coef,
                                                      P.ell_rows);
    return (int)cudaGetLastError();
}

template <typename R, int IT, int G, int NT = 512, bool CHEB = false>
static int run_taylor3_g(const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp, int v0, int nvec,
                         cudaStream_t s) {
    if (nvec <= 0) return 0;
    size_t smem = taylor3_smem(P, sizeof(R), G, NT);
    int e;
    if ((e = set_smem(k_abs_taylor3<R, IT, G, NT, CHEB>, smem))) return e;
    k_abs_taylor3<R, IT, G, NT, CHEB><<<(nvec + G - 1) / G, NT, smem, s>>>(
        T, P, J, resp, v0, nvec, (const EllEnt<R> *)P.ell, P.ell_sptr, P.ell_nslices, P.ell_nent, P.ell_rows);
    return (int)cudaGetLastError();
}

// Vectors of a job's last partial wave on 1-vector CTAs (k_abs_taylor3 with
// G = 1), 512 threads with IT1 rows per lane (1024 threads with one row per
// lane measured slower on the 1024-site lattice: 52.3 against 51.0 ms per
// job; the per-term barriers, not the lanes' gather chains, set its pace).
// With the Chebyshev tables of the row-owner waves (P.rv_cheb) the tail runs
// the same Chebyshev series.
template <typename R, int IT1>
static int run_taylor3_tail(const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp, int v0, int nvec,
                            cudaStream_t s) {
    if constexpr (sizeof(R) == 4)
        if (P.rv_cheb && P.cheb_coef) return run_taylor3_g<R, IT1, 1, 512, true>(T, P, J, resp, v0, nvec, s);
    return run_taylor3_g<R, IT1, 1>(T, P, J, resp, v0, nvec, s);
}

// Streaming multiprocessors of the current device (wave sizes).
int sm_count() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
}

// One CTA per SM at G = 8: whole waves of 8-vector CTAs, and the vectors of a
// last wave that would be less than half full on 1-vector CTAs (which finish
// several times sooner); fewer vectors than SMs all on 1-vector CTAs.  FP32
// lattices of 513..1056 sites (16 rows per thread at 512 threads) run their
// 8-vector CTAs with 768 threads, 11 rows each (measured on N = 1024: 75.3 ms
// instead of 81.7 ms per step; 640 threads 76.3 ms, 896 threads spill).
template <typename R, int IT>
static int run_taylor3(const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp, int nvec,
                       cudaStream_t s, int *kernels) {
    constexpr int IT1 = IT <= 8 ? 1 : IT / 8;  // rows per thread at G = 1: 8 slices per warp instruction
    const int nsm = sm_count(), ctas = (nvec + 7) / 8;
    int main = nvec;
    if (nvec <= nsm) main = 0;
    else if (ctas % nsm != 0 && ctas % nsm < nsm / 2 && ctas >= nsm) main = (ctas / nsm) * nsm * 8;
    if (kernels) *kernels = (main > 0) + (nvec > main);
    int e = -1;
    if constexpr (sizeof(R) == 4)  // the row-owner kernel for the 8-vector waves
        if (!P.no_rv && main > 0 && taylor_rv_fits(T, P)) {
            // the 1-vector CTAs take the first vectors, the waves the rest: the
            // order in which a trajectory copied in frame chunks arrives (the
            // chunked path runs the same split), at the same job length
            if ((e = run_taylor3_tail<R, IT1>(T, P, J, resp, 0, nvec - main, s))) return e;
            return launch_abs_taylor_rv(T, P, J, resp, nvec - main, main, s);
        }
    if (P.rv_cheb) {  // the Chebyshev series on 1-vector CTAs only (no whole wave)
        if (main > 0) return (int)cudaErrorNotSupported;
        return run_taylor3_tail<R, IT1>(T, P, J, resp, 0, nvec, s);
    }
    if constexpr (sizeof(R) == 4 && IT == 16)
        if (e < 0 && P.ell_nslices <= 24 * 11 && taylor3_smem(P, 4, 8, 768) <= 220 * 1024)
            e = run_taylor3_g<R, 11, 8, 768>(T, P, J, resp, 0, main, s);
    if (e < 0) e = run_taylor3_g<R, IT, 8>(T, P, J, resp, 0, main, s);
    if (e) return e;
    return run_taylor3_tail<R, IT1>(T, P, J, resp, main, nvec - main, s);
}

int launch_abs_taylor_part(const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp, int v0, int nvec,
                           bool one, cudaStream_t s) {
    if (nvec <= 0) return 0;
    if (!one) return launch_abs_taylor_rv(T, P, J, resp, v0, nvec, s);
    const TaylorPlan &Pt = P;  // 1-vector CTAs: the same series as the waves
    const int it = (P.ell_nslices + 15) / 16;
    if (!P.ell || it > 32) return (int)cudaErrorNotSupported;
    const int IT = it <= 1 ? 1 : it <= 2 ? 2 : it <= 4 ? 4 : it <= 8 ? 8 : it <= 16 ? 16 : 32;
    switch (IT <= 8 ? 1 : IT / 8) {
    case 1: return run_taylor3_tail<float, 1>(T, Pt, J, resp, v0, nvec, s);
    case 2: return run_taylor3_tail<float, 2>(T, Pt, J, resp, v0, nvec, s);
    default: return run_taylor3_tail<float, 4>(T, Pt, J, resp, v0, nvec, s);
    }
}

int launch_abs_taylor(int prec, const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp,
                      int vec_per_cta, cudaStream_t s, int *kernels) {
    if (kernels) *kernels = 1;
    if (P.use_v4) {  // the 4-vector sliced-ELL kernel (FP32, ELL through L1)
        if (prec != 0 || !P.ell4) return (int)cudaErrorNotSupported;
        int nvec = 3 * J.nsamp;
        int it = (P.ell4_nslices + 15) / 16;
        if (it > 32 || (size_t)P.n * 4 * sizeof(float2) + 1024 > kMaxSmem) return (int)cudaErrorNotSupported;
        int IT = it <= 1 ? 1 : it <= 2 ? 2 : it <= 4 ? 4 : it <= 8 ? 8 : it <= 16 ? 16 : 32;
        switch (IT) {
        case 1: return run_taylor4<1>(T, P, J, resp, nvec, s);
        case 2: return run_taylor4<2>(T, P, J, resp, nvec, s);
        case 4: return run_taylor4<4>(T, P, J, resp, nvec, s);
        case 8: return run_taylor4<8>(T, P, J, resp, nvec, s);
        case 16: return run_taylor4<16>(T, P, J, resp, nvec, s);
        default: return run_taylor4<32>(T, P, J, resp, nvec, s);
        }
    }
    if (P.cheb_coef && P.rv_cheb) {  // the row-owner kernel with the Chebyshev expansion (FP32)
        if (prec != 0 || !P.ell || !taylor_rv_fits(T, P)) return (int)cudaErrorNotSupported;
        const int it = (P.ell_nslices + 15) / 16;
        if (it > 32 || taylor3_smem(P, 4) > 220 * 1024) return (int)cudaErrorNotSupported;
        const int nvec = 3 * J.nsamp;
        switch (it <= 1 ? 1 : it <= 2 ? 2 : it <= 4 ? 4 : it <= 8 ? 8 : it <= 16 ? 16 : 32) {
        case 1: return run_taylor3<float, 1>(T, P, J, resp, nvec, s, kernels);
        case 2: return run_taylor3<float, 2>(T, P, J, resp, nvec, s, kernels);
        case 4: return run_taylor3<float, 4>(T, P, J, resp, nvec, s, kernels);
        case 8: return run_taylor3<float, 8>(T, P, J, resp, nvec, s, kernels);
        case 16: return run_taylor3<float, 16>(T, P, J, resp, nvec, s, kernels);
        default: return run_taylor3<float, 32>(T, P, J, resp, nvec, s, kernels);
        }
    }
    if (P.cheb_coef) {  // Chebyshev tables present: the FP32 sliced-ELL Chebyshev kernel
        if (prec != 0 || !P.ell || cheb3_smem(P) > kMaxSmem) return (int)cudaErrorNotSupported;
        int nvec = 3 * J.nsamp;
        int it = (P.ell_nslices + 15) / 16;
        if (it > 32) return (int)cudaErrorNotSupported;
        int IT = it <= 1 ? 1 : it <= 2 ? 2 : it <= 4 ? 4 : it <= 8 ? 8 : it <= 16 ? 16 : 32;
        switch (IT) {
        case 1: return run_cheb3<1>(T, P, J, resp, nvec, s);
        case 2: return run_cheb3<2>(T, P, J, resp, nvec, s);
        case 4: return run_cheb3<4>(T, P, J, resp, nvec, s);
        case 8: return run_cheb3<8>(T, P, J, resp, nvec, s);
        case 16: return run_cheb3<16>(T, P, J, resp, nvec, s);
        default: return run_cheb3<32>(T, P, J, resp, nvec, s);
        }
    }
    if (!P.only_v2 && P.static_j && P.ell && vec_per_cta > 4 && taylor3_smem(P, prec == 0 ? 4 : 8) <= 220 * 1024) {
        int nvec = 3 * J.nsamp;
        int it = (P.ell_nslices + 15) / 16;  // 16 warps, one slice (4 rows) per warp instruction
        int IT = it <= 1 ? 1 : it <= 2 ? 2 : it <= 4 ? 4 : it <= 8 ? 8 : it <= 16 ? 16 : 32;
        if (it <= 32) {
#define T3(R)                                                                    \
    switch (IT) {                                                                \
    case 1: return run_taylor3<R, 1>(T, P, J, resp, nvec, s, kernels);  \
    case 2: return run_taylor3<R, 2>(T, P, J, resp, nvec, s, kernels);  \
    case 4: return run_taylor3<R, 4>(T, P, J, resp, nvec, s, kernels);  \
    case 8: return run_taylor3<R, 8>(T, P, J, resp, nvec, s, kernels);  \
    case 16: return run_taylor3<R, 16>(T, P, J, resp, nvec, s, kernels); \
    default: return run_taylor3<R, 32>(T, P, J, resp, nvec, s, kernels); \
    }
            if (prec == 0) { T3(float) }
            T3(double)
#undef T3
        }
    }
    {
        // vectors across lanes (k_abs_taylor2): 16 warps cover 512 rows per
        // iteration at G = 8 (4 rows per warp) and 128 at G = 4... rows per
        // thread IT = ceil(n / (16 * 32 / G)).
        int nvec = 3 * J.nsamp;
        if (P.static_j) {
            const size_t r2 = prec == 0 ? sizeof(float2) : sizeof(double2);
            auto t2_smem = [&](int g) { return 2 * (size_t)P.n * (g + 2) * r2 + 16 * (size_t)g * 2 * sizeof(double); };
            int G = vec_per_cta <= 4 ? 4 : 8;
            if (prec != 0) G = 4;
            if (G == 8 && t2_smem(8) > kMaxSmem) G = 4;
            int per_iter = 16 * (32 / G);
            int it = (P.n + per_iter - 1) / per_iter;
            int IT = it <= 1 ? 1 : it <= 2 ? 2 : it <= 4 ? 4 : it <= 8 ? 8 : it <= 16 ? 16 : 32;
            if (it <= 32 && t2_smem(G) <= kMaxSmem) {
#define T2(R, GG)                                                                              \
    switch (IT) {                                                                              \
    case 1: return run_taylor2<R, GG, 1>(T, P, J, resp, nvec, s);                              \
    case 2: return run_taylor2<R, GG, 2>(T, P, J, resp, nvec, s);                              \
    case 4: return run_taylor2<R, GG, 4>(T, P, J, resp, nvec, s);                              \
    case 8: return run_taylor2<R, GG, 8>(T, P, J, resp, nvec, s);                              \
    case 16: return run_taylor2<R, GG, 16>(T, P, J, resp, nvec, s);                            \
    default: return run_taylor2<R, GG, 32>(T, P, J, resp, nvec, s);                            \
    }
                if (prec == 0) {
                    if (G == 4) { T2(float, 4) }
                    T2(float, 8)
                }
                T2(double, 4)
#undef T2
            }
        }
    }
    int nvec = 3 * J.nsamp;
    int rpt = (P.n + 511) / 512;
    if (rpt > 4 || !P.static_j) return (int)cudaErrorNotSupported;
    rpt = rpt <= 1 ? 1 : (rpt <= 2 ? 2 : 4);
    {  // k_abs_taylor keeps two full copies of G vectors: fall back to G = 3 where 8 (4) does not fit
        const size_t r2 = prec == 0 ? sizeof(float2) : sizeof(double2);
        const int gbig = prec == 0 ? 8 : 4;
        if (2 * (size_t)P.n * gbig * r2 + 16 * 2 * (size_t)gbig * sizeof(double) > kMaxSmem) vec_per_cta = 3;
        if (2 * (size_t)P.n * 3 * r2 + 16 * 2 * 3 * sizeof(double) > kMaxSmem) return (int)cudaErrorNotSupported;
    }
#define TAY(R, G)                                                                                  \
    do {                                                                                           \
        if (rpt == 1) return run_taylor<R, G, 1>(T, P, J, resp, nvec, s);                          \
        if (rpt == 2) return run_taylor<R, G, 2>(T, P, J, resp, nvec, s);                          \
        return run_taylor<R, G, 4>(T, P, J, resp, nvec, s);                                        \
    } while (0)
    if (prec == 0) {
        if (vec_per_cta <= 3) TAY(float, 3);
        TAY(float, 8);
    } else {
        if (vec_per_cta <= 3) TAY(double, 3);
        TAY(double, 4);
    }
#undef TAY
}

int launch_prep_cheb(const DevTraj &T, TaylorPlan &P, double rowabs_max, double f, int *order, float *inv_r,
                     float *center, float2 *coef, cudaStream_t s) {
    if (P.nf)
        k_prep_cheb<<<(P.nf + 127) / 128, 128, 0, s>>>(T, P, rowabs_max, f, kSeriesTolF32, order, inv_r, center, coef);
    P.order = order;
    P.cheb_inv_r = inv_r;
    P.cheb_center = center;
    P.cheb_coef = coef;
    return (int)cudaGetLastError();
}

int launch_pattern_scan(const DevTraj &T, long f0, long nf, int *flag, cudaStream_t s) {
    long nn2 = (long)T.n * (T.n + 1) / 2;
    k_pattern_scan<<<(nn2 + 255) / 256, 256, 0, s>>>(T, f0, nf, flag);
    return (int)cudaGetLastError();
}

int launch_reduce_resp(const double2 *resp, int nvec, int tmax, double2 *out, cudaStream_t s) {
    k_reduce_resp<<<(tmax + 31) / 32, 1024, 0, s>>>(resp, nvec, tmax, out);
    return (int)cudaGetLastError();
}

int launch_step_coupling(int prec, int n, float cut, const float *H, void *re, void *im, int nvec, int ts,
                         double fsub, float fsub32, cudaStream_t s) {
    size_t per_lane = (size_t)n * (prec == 0 ? sizeof(float2) : sizeof(double2));
    int B = lanes_for(per_lane, 64);
    size_t smem = per_lane * B;
    int e;
    if (prec == 0) {
        if ((e = set_smem(k_step_coupling<float>, smem))) return e;
        k_step_coupling<float><<<(nvec + B - 1) / B, B, smem, s>>>(n, cut, H, (float *)re, (float *)im, nvec, ts,
                                                                   fsub32);
    } else {
        if ((e = set_smem(k_step_coupling<double>, smem))) return e;
        k_step_coupling<double><<<(nvec + B - 1) / B, B, smem, s>>>(n, cut, H, (double *)re, (double *)im, nvec,
                                                                    ts, fsub);
    }
    return (int)cudaGetLastError();
}

int launch_step_rk4(int prec, int n, float cut, const float *H, void *re, void *im, int nvec, int ts, double fsub,
                    float fsub32, cudaStream_t s) {
    size_t rsz = prec == 0 ? sizeof(float) : sizeof(double);
    size_t per_lane = 5 * (size_t)n * 2 * rsz;
    int B = lanes_for(per_lane, 64);
    size_t smem = per_lane * B;
    int kmax = n * (n + 1) / 2;
    int2 *ent = nullptr;
    void *val = nullptr;
    int e;
    if ((e = (int)cudaMallocAsync((void **)&ent, sizeof(int2) * (size_t)kmax * nvec, s))) return e;
    if ((e = (int)cudaMallocAsync(&val, rsz * (size_t)kmax * nvec, s))) return e;
    if (prec == 0) {
        if ((e = set_smem(k_step_rk4<float>, smem))) return e;
        k_step_rk4<float><<<(nvec + B - 1) / B, B, smem, s>>>(n, cut, H, (float *)re, (float *)im, nvec, ts, fsub32,
                                                              ent, (float *)val, kmax);
    } else {
        if ((e = set_smem(k_step_rk4<double>, smem))) return e;
        k_step_rk4<double><<<(nvec + B - 1) / B, B, smem, s>>>(n, cut, H, (double *)re, (double *)im, nvec, ts,
                                                               fsub, ent, (double *)val, kmax);
    }
    e = (int)cudaGetLastError();
    cudaFreeAsync(ent, s);
    cudaFreeAsync(val, s);
    return e;
}

int launch_step_taylor(int prec, int n, const float *H, void *re, void *im, int nvec, double f, cudaStream_t s) {
    size_t per_lane = 3 * (size_t)n * (prec == 0 ? sizeof(float2) : sizeof(double2));
    int B = lanes_for(per_lane, 64);
    size_t smem = per_lane * B;
    int e;
    if (prec == 0) {
        if ((e = set_smem(k_step_taylor<float>, smem))) return e;
        k_step_taylor<float><<<(nvec + B - 1) / B, B, smem, s>>>(n, H, (float *)re, (float *)im, nvec, f);
    } else {
        if ((e = set_smem(k_step_taylor<double>, smem))) return e;
        k_step_taylor<double><<<(nvec + B - 1) / B, B, smem, s>>>(n, H, (double *)re, (double *)im, nvec, f);
    }
    return (int)cudaGetLastError();
}
