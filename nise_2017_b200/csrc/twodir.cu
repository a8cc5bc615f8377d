// 2DIR family (calc_2DIR.c:22-629) on one GPU, and the UVvis family
// (calc_2DES.c:22-586), which is the same calculation for two-level sites:
// the doubles basis keeps |ab> with a != b only (dipole_double_ES,
// dipole_double_last_ES, NISE_subs.c:533-592) and the doubles propagators
// have neither anharmonicity nor the sqrt(2) couplings to |aa>
// (propagate_vec_coupling_S_doubles_ES, propagate_vec_RK4_doubles_ES,
// propagate_double_sparce_ES; propagate.c:593-826, 1051-1181, 1400-1473).
// The |aa> slots stay in the packed layout and stay exactly zero.
//
// The reference loops over (start point, molecular polarisation) work items
// and, inside each, propagates dozens of vectors frame by frame.  Here the
// work of a chunk of start points is reorganised by linearity and shared:
//
//  * singles vectors depend on one dipole component only, so the t1 vectors
//    (leftn), the GB t3 vector (mut3), leftr and their t2/t3 propagations are
//    computed once per component x in {x,y,z} instead of once per molecular
//    polarisation (21);
//  * the excited-state-absorption (EA) "right" vectors are propagated
//    backwards in the reference (sign -1, propagate.c:1552-1560); they equal
//    the complex conjugates of the SE vectors propagated forwards, operation
//    by operation, for every scheme here (Trotter rotations, RK4, eigen
//    propagator), so the conjugated SE snapshots are used bit for bit;
//  * the doubles vectors depend on a pair of components: fr on (px1,px2) and
//    ft1[t1] on (px0,px2), 9 + 9*tmax1 vectors instead of 21*(1+tmax1).
//
// Kernels (one chunk of start points at a time):
//   k2d_gb1      leftn_x[t1]: mu_x(tj-t1) propagated t1 steps; GB t1 dots
//   k2d_gb3      mut3_x: mu_x(tk) propagated through t3; GB t3 dots
//   k2d_t2       t2 eigen steps (propagate_t2_DIA) of leftr_x and leftn_x[t1]
//   k2d_se       SE t3 propagation of leftr_x and leftn_x[t1], snapshots per t3
//   k2d_doubles  doubles (two-exciton) Trotter propagation of fr / ft1[t1],
//                dipole_double_last projections and EA dot products per t3
//   k2d_response GB + SE + EA contributions per (start point, t3, t1) with the
//                21 molecular-frame weights and the lifetime factors
// followed by a deterministic sum over start points.
//
// FP32 contexts keep the reference's single-precision operations (states,
// rotations, dipole operators) and accumulate every dot product and response
// sum in FP64, like the FP32/FP64-sum oracle.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "eigen.h"
#include "engine.h"
#include "nise_internal.h"
#include "schemes.cuh"

namespace {

// polar() (polar.c:36-105); the weights of polarweight() (polar.c:12-33)
// are uploaded to c_w as the float values the reference computes.
__constant__ int c_px[21][4] = {{0, 0, 0, 0}, {1, 1, 1, 1}, {2, 2, 2, 2}, {0, 0, 1, 1}, {0, 0, 2, 2}, {1, 1, 0, 0},
                                 {1, 1, 2, 2}, {2, 2, 0, 0}, {2, 2, 1, 1}, {0, 1, 0, 1}, {0, 2, 0, 2}, {1, 0, 1, 0},
                                 {1, 2, 1, 2}, {2, 0, 2, 0}, {2, 1, 2, 1}, {0, 1, 1, 0}, {0, 2, 2, 0}, {1, 0, 0, 1},
                                 {1, 2, 2, 1}, {2, 0, 0, 2}, {2, 1, 1, 2}};
__constant__ float c_w[3][21];

// The singles tables (SinglesTab: n, ts, prop, f0, the Trotter/RK4/eigen
// tables) are the base; the fields below are the 2D job's.
struct TwoD : SinglesTab {
    DevTraj T;
    int T1, T2, T3, sample, s0, S;  // S start points in this chunk, the first is s0
    int gb, se, ea;
    int es;                   // UVvis family: two-level doubles (no |aa>)
    float anh;                // Anharmonicity keyword (0: per-frame files)
    const void *Us;           // Sparse/Diagonal doubles: substep propagators U[t][n][n] (f/ts, truncated)
    long e0;                  // eigen data for frames [e0, e0 + ne)
    const double *eV, *ew;    // V [ne][n][n], w [ne][n]
    float f32_full;           // deltat*icm2ifs*2pi in float
    double f64_full;
    float f32_dsub;           // deltat*icm2ifs*2pi/ts in float (propagate.c:905)
    double f64_dsub;
    void *L;                  // [S][3][T1][n] R2  leftn_x[t1]
    void *Lr;                 // [S][3][n] R2      leftr_x
    void *SE;                 // [S][T3][NV][n] R2 snapshots, NV = 3 + 3*T1 (leftr_x, then leftn_x[t1])
    double2 *gbt1;            // [S][3 p0][3 p1][T1]
    double2 *gbt3;            // [S][3 p2][3 p3][T3]
    double2 *eaI, *eaII;      // [S][T3][21][T1]
    double *Rs;               // [S][12][T3][T1]
    const float *lt;          // [T3][T1]
};

__device__ __forceinline__ long tj_of(const TwoD &D, int s) { return (long)(D.s0 + s) * D.sample + D.T1; }
__device__ __forceinline__ long tk_of(const TwoD &D, int s) { return tj_of(D, s) + D.T2; }
__device__ __forceinline__ int nvec_se(const TwoD &D) { return 3 + 3 * D.T1; }

// sum_i mu_i * psi_i with float products (FP32) and an FP64 sum.
template <typename R>
__device__ __forceinline__ double2 dot_col(const DevTraj &T, long t, int x, const typename Vec2<R>::T *S, int B,
                                           int lane, int n) {
    return dot_mu<R>(T, t, x, S, B, lane, n);
}

// ---------------------------------------------------------------- GB t1
// Thread per (start point, x, pair p): t1 = p and t1 = T1-1-p, so every
// thread does T1-1 steps (the triangle of calc_2DIR.c:215-239 balanced).
template <typename R>
__global__ void k2d_gb1(TwoD D) {
    typedef typename Vec2<R>::T R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *S = (R2 *)smem_raw;
    const int B = blockDim.x, lane = threadIdx.x, n = D.n;
    const int P = (D.T1 + 1) / 2;
    int g = blockIdx.x * B + lane;
    if (g >= D.S * 3 * P) return;
    int s = g / (3 * P), rem = g % (3 * P), x = rem / P, p = rem % P;
    long tj = tj_of(D, s);
    for (int pass = 0; pass < 2; pass++) {
        int t1 = pass == 0 ? p : D.T1 - 1 - p;
        if (pass == 1 && t1 == p) break;
        for (int i = 0; i < n; i++) {
            R2 z;
            z.x = (R)traj_mu(D.T, tj - t1, x, i);
            z.y = 0;
            S[i * B + lane] = z;
        }
        for (int tm = 0; tm < t1; tm++) singles_step<R>(D, S, B, lane, tj - t1 + tm);
        R2 *out = (R2 *)D.L + (((size_t)s * 3 + x) * D.T1 + t1) * n;
        for (int i = 0; i < n; i++) out[i] = S[i * B + lane];
        if (D.gb)  // t1nr/t1ni (calc_2DIR.c:244-250) for every p1
            for (int p1 = 0; p1 < 3; p1++)
                D.gbt1[(((size_t)s * 3 + x) * 3 + p1) * D.T1 + t1] = dot_col<R>(D.T, tj, p1, S, B, lane, n);
    }
}

// ---------------------------------------------------------------- GB t3
template <typename R>
__global__ void k2d_gb3(TwoD D) {
    typedef typename Vec2<R>::T R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *S = (R2 *)smem_raw;
    const int B = blockDim.x, lane = threadIdx.x, n = D.n;
    int g = blockIdx.x * B + lane;
    if (g >= D.S * 3) return;
    int s = g / 3, x = g % 3;
    long tk = tk_of(D, s);
    for (int i = 0; i < n; i++) {
        R2 z;
        z.x = (R)traj_mu(D.T, tk, x, i);
        z.y = 0;
        S[i * B + lane] = z;
    }
    for (int t3 = 0; t3 < D.T3; t3++) {  // calc_2DIR.c:257-299
        long tl = tk + t3;
        for (int p3 = 0; p3 < 3; p3++)
            D.gbt3[(((size_t)s * 3 + x) * 3 + p3) * D.T3 + t3] = dot_col<R>(D.T, tl, p3, S, B, lane, n);
        if (t3 < D.T3 - 1) singles_step<R>(D, S, B, lane, tl);
    }
}

// ---------------------------------------------------------------- t2
// propagate_t2_DIA (propagate.c:130-180): V^T, phase, V per frame, with the
// eigenvectors in the reference's storage and FP32 operands in FP32 mode.
template <typename R>
__global__ void k2d_t2(TwoD D) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int B = blockDim.x, lane = threadIdx.x, n = D.n;
    R2 *S = (R2 *)smem_raw, *X = S + (size_t)n * B;
    const int NV = nvec_se(D);
    int g = blockIdx.x * B + lane;
    if (g >= D.S * NV) return;
    int s = g / NV, v = g % NV;
    R2 *vec = v < 3 ? (R2 *)D.Lr + ((size_t)s * 3 + v) * n
                    : (R2 *)D.L + (((size_t)s * 3 + (v - 3) / D.T1) * D.T1 + (v - 3) % D.T1) * n;
    for (int i = 0; i < n; i++) S[i * B + lane] = vec[i];
    long tj = tj_of(D, s);
    for (int t2 = 0; t2 < D.T2; t2++) {
        long fi = tj + t2 - D.e0;
        const double *V = D.eV + fi * n * n, *w = D.ew + fi * n;
        for (int a = 0; a < n; a++) {  // matrix_on_vector: x = V^T v
            R xr = 0, xi = 0;
            for (int b = 0; b < n; b++) {
                R c = (R)V[b * n + a];
                R2 z = S[b * B + lane];
                xr = A::add(xr, A::mul(c, z.x));
                xi = A::add(xi, A::mul(c, z.y));
            }
            R ev = (R)w[a], arg = A::mul(ev, sizeof(R) == 4 ? (R)D.f32_full : (R)D.f64_full);
            R ur = (R)cos((double)arg), ui = (R)(-sin((double)arg));
            R2 o;  // vector_on_vector (NISE_subs.c:71-80)
            o.x = A::sub(A::mul(ur, xr), A::mul(ui, xi));
            o.y = A::add(A::mul(ui, xr), A::mul(ur, xi));
            X[a * B + lane] = o;
        }
        for (int a = 0; a < n; a++) {  // trans_matrix_on_vector: v = V x
            R yr = 0, yi = 0;
            for (int b = 0; b < n; b++) {
                R c = (R)V[a * n + b];
                R2 z = X[b * B + lane];
                yr = A::add(yr, A::mul(c, z.x));
                yi = A::add(yi, A::mul(c, z.y));
            }
            R2 o;
            o.x = yr;
            o.y = yi;
            S[a * B + lane] = o;
        }
    }
    for (int i = 0; i < n; i++) vec[i] = S[i * B + lane];
}

// ---------------------------------------------------------------- SE t3
template <typename R>
__global__ void k2d_se(TwoD D) {
    typedef typename Vec2<R>::T R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *S = (R2 *)smem_raw;
    const int B = blockDim.x, lane = threadIdx.x, n = D.n;
    const int NV = nvec_se(D);
    int g = blockIdx.x * B + lane;
    if (g >= D.S * NV) return;
    int s = g / NV, v = g % NV;
    const R2 *vec = v < 3 ? (const R2 *)D.Lr + ((size_t)s * 3 + v) * n
                          : (const R2 *)D.L + (((size_t)s * 3 + (v - 3) / D.T1) * D.T1 + (v - 3) % D.T1) * n;
    for (int i = 0; i < n; i++) S[i * B + lane] = vec[i];
    long tk = tk_of(D, s);
    for (int t3 = 0; t3 < D.T3; t3++) {  // calc_2DIR.c:372-443
        R2 *snap = (R2 *)D.SE + (((size_t)s * D.T3 + t3) * NV + v) * n;
        for (int i = 0; i < n; i++) snap[i] = S[i * B + lane];
        if (t3 < D.T3 - 1) singles_step<R>(D, S, B, lane, tk + t3);
    }
}

// ---------------------------------------------------------------- doubles
// Shared-memory layout of one doubles vector: the pair {x,y} lives at
// circ(x,y): with d = (y-x) mod n, slot x*W + d when d < n-d (or d == n-d and
// x < y), else y*W + (x-y) mod n; W = n/2 + 2.  Reading pair {b,c} for every
// lane c (fixed b) is then conflict-free in both halves.
__device__ __forceinline__ int circ(int x, int y, int n, int W) {
    int d = y - x;
    if (d < 0) d += n;
    int e = n - d;
    if (d < e || (d == e && x < y)) return x * W + d;
    return y * W + (e == n ? 0 : e);
}

template <typename R>
__device__ __forceinline__ void rot2(typename Vec2<R>::T &x1, typename Vec2<R>::T &x2, R co, R si) {
    typedef Ar<R> A;
    typename Vec2<R>::T y1, y2;  // propagate.c:984-988
    y1.x = A::sub(A::mul(co, x1.x), A::mul(si, x2.y));
    y1.y = A::add(A::mul(co, x1.y), A::mul(si, x2.x));
    y2.x = A::sub(A::mul(co, x2.x), A::mul(si, x1.y));
    y2.y = A::add(A::mul(co, x2.y), A::mul(si, x1.x));
    x1 = y1;
    x2 = y2;
}

// 16-byte (FP32) / 32-byte (FP64) records, one vector load each
template <typename R> struct alignas(4 * sizeof(R)) Dcoef { R co, si, co2, si2; };

template <typename R>
__device__ __forceinline__ typename Vec2<R>::T make_vec2(R x, R y) {
    typename Vec2<R>::T v;
    v.x = x;
    v.y = y;
    return v;
}

// Warp per doubles vector; lane l owns columns c = l + 32*j (j < CPL).  One
// Trotter sub-step of propagate_vec_coupling_S_doubles (propagate.c:956-1045):
// half diagonal phase; for every coupling (a,b) in lexicographic order the
// rotations of the pairs (|ac>,|bc>) for all c, with the sqrt(2) angle on
// (|aa>,|ab>) then (|ab>,|bb>); half diagonal phase.  Rotations of one
// coupling touch disjoint pairs except |ab>, so lanes run them together; the
// pivot |ac> stays in a register while the first index a is unchanged.
//
// Two-level sites (es, propagate.c:1051-1181): the c == a and c == b
// rotations are absent, |ab> is rotated only with the |ac>/|bc> pairs.
template <typename R, int CPL>
__device__ void doubles_substep(typename Vec2<R>::T *F, const typename Vec2<R>::T *Uh, const Dcoef<R> *cf,
                                const int2 *pairs, int K, int n, int W, int lane, const short *__restrict__ ci,
                                bool es) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    const int slots = n * W;
    for (int e = lane; e < slots; e += 32) {  // propagate.c:959-962
        R2 z = F[e], u = Uh[e], o;
        o.x = A::sub(A::mul(z.x, u.x), A::mul(z.y, u.y));
        o.y = A::add(A::mul(z.x, u.y), A::mul(z.y, u.x));
        F[e] = o;
    }
    __syncwarp();
    int cur_a = -1;
    R2 piv[CPL];
    // the next coupling and its coefficients are loaded one step ahead
    int2 ab_next = K > 0 ? pairs[0] : make_int2(0, 0);
    Dcoef<R> q_next;
    if (K > 0) q_next = cf[0];
    for (int k = 0; k < K; k++) {
        const int a = ab_next.x, b = ab_next.y;
        const Dcoef<R> q = q_next;
        if (k + 1 < K) {
            ab_next = pairs[k + 1];
            q_next = cf[k + 1];
        }
        if (a != cur_a) {
            if (cur_a >= 0) {
#pragma unroll
                for (int j = 0; j < CPL; j++) {
                    int c = lane + 32 * j;
                    if (c < n && c != cur_a) F[ci ? ci[cur_a * n + c] : circ(cur_a, c, n, W)] = piv[j];
                }
            }
            __syncwarp();
#pragma unroll
            for (int j = 0; j < CPL; j++) {
                int c = lane + 32 * j;
                if (c < n && c != a) piv[j] = F[ci ? ci[a * n + c] : circ(a, c, n, W)];
            }
            cur_a = a;
        }
        // c == a case: (|aa>,|ab>) with the sqrt(2) angle, by the lane owning c = b
        if (!es && b - lane >= 0 && ((b - lane) & 31) == 0) {
            const int j = (b - lane) >> 5;
            const int ix = ci ? ci[a * n + a] : circ(a, a, n, W);
            R2 X = F[ix];
#pragma unroll
            for (int jj = 0; jj < CPL; jj++)
                if (jj == j) rot2<R>(X, piv[jj], q.co2, q.si2);
            F[ix] = X;
        }
        // every other lane c != a: (|ac>,|bc>); for c == b that is (|ab>,|bb>) at sqrt(2)
#pragma unroll
        for (int j = 0; j < CPL; j++) {
            const int c = lane + 32 * j;
            if (c >= n || c == a || (es && c == b)) continue;
            const bool sp = c == b;
            const int iq = ci ? ci[b * n + c] : circ(b, c, n, W);
            R2 Q = F[iq];
            rot2<R>(piv[j], Q, sp ? q.co2 : q.co, sp ? q.si2 : q.si);
            F[iq] = Q;
        }
        __syncwarp();
    }
    if (cur_a >= 0) {
#pragma unroll
        for (int j = 0; j < CPL; j++) {
            int c = lane + 32 * j;
            if (c < n && c != cur_a) F[ci ? ci[cur_a * n + c] : circ(cur_a, c, n, W)] = piv[j];
        }
    }
    __syncwarp();
    for (int e = lane; e < slots; e += 32) {  // propagate.c:1041-1044
        R2 z = F[e], u = Uh[e], o;
        o.x = A::sub(A::mul(z.x, u.x), A::mul(z.y, u.y));
        o.y = A::add(A::mul(z.x, u.y), A::mul(z.y, u.x));
        F[e] = o;
    }
    __syncwarp();
}

// Overtone dipoles: sqrt2 * mu when Anharmonicity != 0 (NISE_subs.c:490-494)
// else the Overtonedipolefile record (read_over, read_trajectory.c:402-414);
// none for two-level sites, whose dipole_double_ES / dipole_double_last_ES
// have no |aa> term (a zero operator adds only zeros there).
__device__ __forceinline__ float over_mu(const TwoD &D, long t, int x, int i) {
    if (D.es) return 0.0f;
    if (D.anh != 0.0f) return __fmul_rn(1.41421356237f, traj_mu(D.T, t, x, i));
    return D.T.over[t * (1 + 3L * D.n) + 1 + x * D.n + i];
}

// Initial doubles vector: dipole_double (NISE_subs.c:485-509) of the SE
// vector src at frame tk, component p2, into the circulant layout; element e
// of the packed order by thread tid, stride `stride`.
template <typename R>
__device__ __forceinline__ void doubles_init(const TwoD &D, typename Vec2<R>::T *F, const typename Vec2<R>::T *src,
                                             long tk, int p2, int n, int Wd, int tid, int stride) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    const int N2 = n * (n + 1) / 2;
    for (int e = tid; e < N2; e += stride) {
        // e -> (i, j) with i <= j in the packed order
        int i = 0, rem = e;
        while (rem >= n - i) { rem -= n - i; i++; }
        int j = i + rem;
        R2 f;
        if (i == j) {
            R o = (R)over_mu(D, tk, p2, i);
            R2 c = src[i];
            f.x = A::mul(o, c.x);
            f.y = A::mul(o, c.y);
        } else {
            R mi = (R)traj_mu(D.T, tk, p2, i), mj = (R)traj_mu(D.T, tk, p2, j);
            R2 ci = src[i], cj = src[j];
            f.x = A::add(A::mul(mi, cj.x), A::mul(mj, ci.x));
            f.y = A::add(A::mul(mi, cj.y), A::mul(mj, ci.y));
        }
        F[circ(i, j, n, Wd)] = f;
    }
}

// Half-step phases of frame tl (propagate.c:918-954): exp(-i (e_a+e_b-Delta)
// f/2) for every packed pair, from the frame's diagonal dg; all threads of
// the CTA.
template <typename R>
__device__ __forceinline__ void doubles_half_phases(const TwoD &D, typename Vec2<R>::T *Uh, const float *dg, long tl,
                                                    int n, int Wd) {
    typedef typename Vec2<R>::T R2;
    const int N2 = n * (n + 1) / 2;
    for (int e = threadIdx.x; e < N2; e += blockDim.x) {
        int i = 0, rem = e;
        while (rem >= n - i) { rem -= n - i; i++; }
        int j = i + rem;
        R2 u;
        if (sizeof(R) == 4) {
            float hf = __fadd_rn(dg[i], dg[j]);
            if (i == j && !D.es) hf = __fsub_rn(hf, D.anh != 0.0f ? D.anh : D.T.anh[tl * (1L + n) + 1 + i]);
            float arg = __fmul_rn(__fmul_rn(0.5f, hf), D.f32_dsub);
            u.x = (R)(float)cos((double)arg);
            u.y = (R)(-(float)sin((double)arg));
        } else {
            double hd = (double)dg[i] + (double)dg[j];
            if (i == j && !D.es) hd -= D.anh != 0.0f ? (double)D.anh : (double)D.T.anh[tl * (1L + n) + 1 + i];
            double arg = 0.5 * hd * D.f64_dsub;
            u.x = (R)cos(arg);
            u.y = (R)(-sin(arg));
        }
        Uh[circ(i, j, n, Wd)] = u;
    }
}

// CTA = W warps = W doubles vectors of one start point, all at the same t3.
template <typename R, int CPL>
__global__ void __launch_bounds__(512, 1) k2d_doubles(TwoD D, int vec_per_sample, Dcoef<R> *cf_static, int use_tab) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = D.n, N2 = n * (n + 1) / 2, Wd = n / 2 + 2, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const int slots = n * Wd;  // circulant storage (>= N2)
    R2 *Uh = (R2 *)smem_raw;                          // [N2] half phases, circulant order
    R2 *F = Uh + slots + (size_t)warp * slots;        // this warp's vector
    float *mu = (float *)(Uh + slots * (1 + nwarps)); // [3][n] mu(tl), then [3][n] overtone
    float *ov = mu + 3 * n;
    float *dg = ov + 3 * n;                           // [n] diagonal energies of the frame
    short *cidx = use_tab ? (short *)(dg + n) : nullptr;  // [n][n] circ(x, y), where it fits
    const int cta_per_sample = (vec_per_sample + nwarps - 1) / nwarps;
    const int s = blockIdx.x / cta_per_sample;
    const int u = (blockIdx.x % cta_per_sample) * nwarps + warp;
    const bool active = u < vec_per_sample;
    const long tk = tk_of(D, s);
    const int NV = nvec_se(D);
    // which vector: u < 9 -> fr for (p1,p2) = (u/3, u%3); else ft1[t1] for (p0,p2)
    int kind = u < 9 ? 0 : 1, pa = 0, p2 = 0, t1 = 0;
    if (active) {
        if (kind == 0) { pa = u / 3; p2 = u % 3; }
        else { int w = u - 9, cmb = w / D.T1; t1 = w % D.T1; pa = cmb / 3; p2 = cmb % 3; }
    }
    // unused circulant slots: unit phase, zero amplitude
    for (int e = threadIdx.x; e < slots; e += blockDim.x) Uh[e] = make_vec2<R>(1, 0);
    if (cidx)
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) cidx[e] = (short)circ(e / n, e % n, n, Wd);
    for (int e = lane; e < slots; e += 32) F[e] = make_vec2<R>(0, 0);
    __syncthreads();
    // initial vector: dipole_double of the SE vector at tk
    if (active)
        doubles_init<R>(D, F, (const R2 *)D.SE + ((size_t)s * D.T3 * NV + (kind == 0 ? pa : 3 + pa * D.T1 + t1)) * n,
                        tk, p2, n, Wd, lane, 32);
    for (int t3 = 0; t3 < D.T3; t3++) {
        const long tl = tk + t3;
        __syncthreads();
        for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) {
            mu[i] = traj_mu(D.T, tl, i / n, i % n);
            ov[i] = over_mu(D, tl, i / n, i % n);
        }
        __syncthreads();
        // EA projections and dot products (calc_2DIR.c:456-488)
        if (active && D.ea) {
            for (int p3 = 0; p3 < 3; p3++) {
                // g = dipole_double_last(mu_p3, F) for this lane's sites (float sums in site order)
                R2 gq[CPL];
#pragma unroll
                for (int jc = 0; jc < CPL; jc++) {
                    int q = lane + 32 * jc;
                    R gr = 0, gi = 0;
                    if (q < n)
                        for (int j = 0; j < n; j++) {
                            R m = (R)(j == q ? ov[p3 * n + q] : mu[p3 * n + j]);
                            R2 f = F[cidx ? cidx[j * n + q] : circ(j, q, n, Wd)];
                            gr = A::add(gr, A::mul(m, f.x));
                            gi = A::add(gi, A::mul(m, f.y));
                        }
                    gq[jc].x = gr;
                    gq[jc].y = gi;
                }
                for (int m = 0; m < 21; m++) {
                    if (c_px[m][3] != p3 || c_px[m][2] != p2) continue;
                    if (kind == 0 && c_px[m][1] != pa) continue;
                    if (kind == 1 && c_px[m][0] != pa) continue;
                    if (kind == 0) {
                        // rephasing: left = g (from fr), right = conj(leftn_p0[t1] SE snapshot)
                        int p0 = c_px[m][0];
                        for (int tt = 0; tt < D.T1; tt++) {
                            const R2 *rv = (const R2 *)D.SE + (((size_t)s * D.T3 + t3) * NV + 3 + p0 * D.T1 + tt) * n;
                            double a1 = 0, a2 = 0;
#pragma unroll
                            for (int jc = 0; jc < CPL; jc++) {
                                int q = lane + 32 * jc;
                                if (q >= n) continue;
                                R2 r = rv[q];
                                R Rr = r.x, Ri = -r.y;
                                a1 += (double)A::add(A::mul(gq[jc].y, Rr), A::mul(gq[jc].x, Ri));
                                a2 += (double)A::sub(A::mul(gq[jc].x, Rr), A::mul(Ri, gq[jc].y));
                            }
                            for (int o = 16; o > 0; o >>= 1) {
                                a1 += __shfl_xor_sync(0xffffffffu, a1, o);
                                a2 += __shfl_xor_sync(0xffffffffu, a2, o);
                            }
                            if (lane == 0) D.eaI[(((size_t)s * D.T3 + t3) * 21 + m) * D.T1 + tt] = make_double2(a1, a2);
                        }
                    } else {
                        // non-rephasing: left = g (from ft1[t1]), right = conj(leftr_p1 SE snapshot)
                        int p1 = c_px[m][1];
                        const R2 *rv = (const R2 *)D.SE + (((size_t)s * D.T3 + t3) * NV + p1) * n;
                        double a1 = 0, a2 = 0;
#pragma unroll
                        for (int jc = 0; jc < CPL; jc++) {
                            int q = lane + 32 * jc;
                            if (q >= n) continue;
                            R2 r = rv[q];
                            R nr = r.x, ni = -r.y;
                            a1 += (double)A::add(A::mul(nr, gq[jc].y), A::mul(ni, gq[jc].x));
                            a2 += (double)A::sub(A::mul(nr, gq[jc].x), A::mul(ni, gq[jc].y));
                        }
                        for (int o = 16; o > 0; o >>= 1) {
                            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
                            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
                        }
                        if (lane == 0) D.eaII[(((size_t)s * D.T3 + t3) * 21 + m) * D.T1 + t1] = make_double2(a1, a2);
                    }
                }
            }
        }
        if (t3 == D.T3 - 1) break;
        // half-step phases of the frame
        for (int i = threadIdx.x; i < n; i += blockDim.x) dg[i] = traj_diag(D.T, tl, i, false);
        __syncthreads();
        doubles_half_phases<R>(D, Uh, dg, tl, n, Wd);
        __syncthreads();
        const Dcoef<R> *cf = D.rot_static ? cf_static : cf_static + (tl - D.f0) * D.K;
        if (active)
            for (int sub = 0; sub < D.ts; sub++) doubles_substep<R, CPL>(F, Uh, cf, D.pairs, D.K, n, Wd, lane, cidx, D.es != 0);
    }
}

// ------------------------------------------------ doubles, two warps per vector
// For 32 < n <= 64 a doubles vector is shared by two warps: thread c of the
// pair (c = 32 * half + lane) owns column c of |ac>, so a CTA runs twice the
// warps of k2d_doubles on the same shared memory.  Each thread performs the
// float operations k2d_doubles performs for that column, in the same order,
// so the results are bitwise those of k2d_doubles in FP32.
//
// Ordering.  The couplings run in segments of one first site a and one warp
// of second sites b (the "owner" warp: b >> 5).  Coupling (a, b) touches
// |bc> (thread c, every c != a) and |aa> (thread b).  Within a segment:
//  * two couplings (a, b), (a, b') share only |bb'> (threads b' then b) and
//    |aa> (threads b then b'), all in the owner warp: a __syncwarp per
//    coupling orders them there;
//  * a thread c of the other warp touches only |bc> with b in the owner
//    warp, elements no other thread touches in the segment: it runs its
//    rotations with no synchronisation, and loads the elements of several
//    couplings ahead of its stores.
// The pair's named barrier separates segments (and the pivot change, where
// row a is stored back by every column and the next row loaded: thread c
// loads |a c>, which thread a stored).
__device__ __forceinline__ void duo_sync(int id) { asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory"); }

// The owner warp's couplings [k0, k1) of a segment: the sqrt(2) rotation
// (|aa>,|ab>) by thread b, then (|ac>,|bc>) for every c != a ((|ab>,|bb>) at
// sqrt(2) for c == b; absent for c == b with two-level sites).
template <typename R, bool ES>
__device__ __forceinline__ void duo_owner(typename Vec2<R>::T *F, typename Vec2<R>::T &piv, const Dcoef<R> *cf,
                                          const int2 *pairs, int k0, int k1, int ix_aa, bool act, int c,
                                          const short *cic, int n, int W) {
    typedef typename Vec2<R>::T R2;
    if (k0 >= k1) return;
    int b_next = pairs[k0].y;  // the arrays hold one record past the last coupling
    Dcoef<R> q_next = cf[k0];
    for (int k = k0; k < k1; k++) {
        const int b = b_next;
        const Dcoef<R> q = q_next;
        b_next = pairs[k + 1].y;
        q_next = cf[k + 1];
        if (!ES && c == b) {
            R2 X = F[ix_aa];
            rot2<R>(X, piv, q.co2, q.si2);
            F[ix_aa] = X;
        }
        if (act && !(ES && c == b)) {
            const bool sp = c == b;
            const int iq = cic ? cic[b * n] : circ(b, c, n, W);
            R2 Q = F[iq];
            rot2<R>(piv, Q, sp ? q.co2 : q.co, sp ? q.si2 : q.si);
            F[iq] = Q;
        }
        __syncwarp();
    }
}

// The other warp's couplings [k0, k1): (|ac>,|bc>) on private elements, four
// couplings' loads ahead of their rotations.
template <typename R>
__device__ __forceinline__ void duo_free(typename Vec2<R>::T *F, typename Vec2<R>::T &piv, const Dcoef<R> *cf,
                                         const int2 *pairs, int k0, int k1, int c, const short *cic, int n, int W) {
    typedef typename Vec2<R>::T R2;
    int k = k0;
    for (; k + 4 <= k1; k += 4) {
        int iq[4];
        R2 Q[4];
        Dcoef<R> q[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int b = pairs[k + u].y;
            q[u] = cf[k + u];
            iq[u] = cic ? cic[b * n] : circ(b, c, n, W);
        }
#pragma unroll
        for (int u = 0; u < 4; u++) Q[u] = F[iq[u]];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            rot2<R>(piv, Q[u], q[u].co, q[u].si);
            F[iq[u]] = Q[u];
        }
    }
    for (; k < k1; k++) {
        const int b = pairs[k].y;
        const Dcoef<R> q = cf[k];
        const int iq = cic ? cic[b * n] : circ(b, c, n, W);
        R2 Q = F[iq];
        rot2<R>(piv, Q, q.co, q.si);
        F[iq] = Q;
    }
}

template <typename R, bool ES>
__device__ void doubles_substep_duo(typename Vec2<R>::T *F, const typename Vec2<R>::T *Uh, const Dcoef<R> *cf,
                                    const int2 *pairs, const int4 *segs, int nsegs, int n, int W, int t64, int half,
                                    const short *__restrict__ ci, int bar) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    const int slots = n * W, c = t64;
    const bool col = c < n;
    const short *cic = ci ? ci + c : nullptr;  // column c of the slot table
    for (int e = t64; e < slots; e += 64) {  // propagate.c:959-962
        R2 z = F[e], u = Uh[e], o;
        o.x = A::sub(A::mul(z.x, u.x), A::mul(z.y, u.y));
        o.y = A::add(A::mul(z.x, u.y), A::mul(z.y, u.x));
        F[e] = o;
    }
    duo_sync(bar);
    int cur_a = -1, ix_aa = 0;
    R2 piv = make_vec2<R>(0, 0);
    for (int g = 0; g < nsegs; g++) {
        const int4 sg = segs[g];  // (a, first coupling, end, owner warp)
        const int a = sg.x;
        if (a != cur_a) {
            if (cur_a >= 0 && col && c != cur_a) F[cic ? cic[cur_a * n] : circ(cur_a, c, n, W)] = piv;
            duo_sync(bar);
            if (col && c != a) piv = F[cic ? cic[a * n] : circ(a, c, n, W)];
            ix_aa = ci ? ci[a * n + a] : circ(a, a, n, W);
            cur_a = a;
        } else {
            duo_sync(bar);
        }
        const bool act = col && c != a;
        if (half == sg.w) duo_owner<R, ES>(F, piv, cf, pairs, sg.y, sg.z, ix_aa, act, c, cic, n, W);
        else if (act) duo_free<R>(F, piv, cf, pairs, sg.y, sg.z, c, cic, n, W);
    }
    if (cur_a >= 0 && col && c != cur_a) F[cic ? cic[cur_a * n] : circ(cur_a, c, n, W)] = piv;
    duo_sync(bar);
    for (int e = t64; e < slots; e += 64) {  // propagate.c:1041-1044
        R2 z = F[e], u = Uh[e], o;
        o.x = A::sub(A::mul(z.x, u.x), A::mul(z.y, u.y));
        o.y = A::add(A::mul(z.x, u.y), A::mul(z.y, u.x));
        F[e] = o;
    }
    duo_sync(bar);
}

// The pair's part of one EA dot product: thread c holds the float terms of
// column c; the second warp hands its terms to the first through `red`
// (two buffers, so one barrier per product), which adds them in k2d_doubles'
// order (column c, then c + 32) and reduces over the lanes.  Returns the sums
// in lane 0 of the first warp.
template <typename R>
__device__ __forceinline__ double2 duo_dot(typename Vec2<R>::T term, typename Vec2<R>::T *red, int &par, int half,
                                           int lane, int n, int bar) {
    typedef typename Vec2<R>::T R2;
    R2 *buf = red + par * 32;
    if (half == 1) buf[lane] = term;
    duo_sync(bar);
    par ^= 1;
    double a1 = 0, a2 = 0;
    if (half == 0) {  // column lane < 32 < n always exists
        a1 += (double)term.x;
        a2 += (double)term.y;
        if (lane + 32 < n) {
            const R2 o = buf[lane];
            a1 += (double)o.x;
            a2 += (double)o.y;
        }
        for (int o = 16; o > 0; o >>= 1) {
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
    }
    return make_double2(a1, a2);
}

// CTA = P pairs of warps = P doubles vectors of one start point, all at the
// same t3 (32 < n <= 64).
template <typename R>
__global__ void __launch_bounds__(768, 1) k2d_doubles_duo(TwoD D, int vec_per_sample, Dcoef<R> *cf_static,
                                                          int use_tab) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = D.n, Wd = n / 2 + 2, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int pair = warp >> 1, half = warp & 1, t64 = threadIdx.x & 63, npairs = blockDim.x >> 6;
    const int bar = 1 + pair;  // named barrier of the pair (0 is __syncthreads)
    const int slots = n * Wd;  // circulant storage (>= N2)
    R2 *Uh = (R2 *)smem_raw;                            // [N2] half phases, circulant order
    R2 *F = Uh + slots + (size_t)pair * slots;          // this pair's vector
    R2 *red = Uh + slots * (1 + npairs) + pair * 64;    // [2][32] the second warp's dot-product terms
    float *mu = (float *)(Uh + slots * (1 + npairs) + 64 * npairs);  // [3][n] mu(tl), then [3][n] overtone
    float *ov = mu + 3 * n;
    float *dg = ov + 3 * n;                             // [n] diagonal energies of the frame
    short *cidx = use_tab ? (short *)(dg + n) : nullptr;  // [n][n] circ(x, y), where it fits
    const int cta_per_sample = (vec_per_sample + npairs - 1) / npairs;
    const int s = blockIdx.x / cta_per_sample;
    const int u = (blockIdx.x % cta_per_sample) * npairs + pair;
    const bool active = u < vec_per_sample;
    const long tk = tk_of(D, s);
    const int NV = nvec_se(D);
    const int q = t64;  // this thread's column
    const bool qv = q < n;
    int par = 0;
    // which vector: u < 9 -> fr for (p1,p2) = (u/3, u%3); else ft1[t1] for (p0,p2)
    int kind = u < 9 ? 0 : 1, pa = 0, p2 = 0, t1 = 0;
    if (active) {
        if (kind == 0) { pa = u / 3; p2 = u % 3; }
        else { int w = u - 9, cmb = w / D.T1; t1 = w % D.T1; pa = cmb / 3; p2 = cmb % 3; }
    }
    for (int e = threadIdx.x; e < slots; e += blockDim.x) Uh[e] = make_vec2<R>(1, 0);
    if (cidx)
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) cidx[e] = (short)circ(e / n, e % n, n, Wd);
    for (int e = t64; e < slots; e += 64) F[e] = make_vec2<R>(0, 0);
    duo_sync(bar);
    if (active)
        doubles_init<R>(D, F, (const R2 *)D.SE + ((size_t)s * D.T3 * NV + (kind == 0 ? pa : 3 + pa * D.T1 + t1)) * n,
                        tk, p2, n, Wd, t64, 64);
    for (int t3 = 0; t3 < D.T3; t3++) {
        const long tl = tk + t3;
        __syncthreads();
        for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) {
            mu[i] = traj_mu(D.T, tl, i / n, i % n);
            ov[i] = over_mu(D, tl, i / n, i % n);
        }
        __syncthreads();
        // EA projections and dot products (calc_2DIR.c:456-488), as k2d_doubles
        if (active && D.ea) {
            for (int p3 = 0; p3 < 3; p3++) {
                R2 gq;
                {
                    R gr = 0, gi = 0;
                    if (qv)
                        for (int j = 0; j < n; j++) {
                            R m = (R)(j == q ? ov[p3 * n + q] : mu[p3 * n + j]);
                            R2 f = F[cidx ? cidx[j * n + q] : circ(j, q, n, Wd)];
                            gr = A::add(gr, A::mul(m, f.x));
                            gi = A::add(gi, A::mul(m, f.y));
                        }
                    gq.x = gr;
                    gq.y = gi;
                }
                for (int m = 0; m < 21; m++) {
                    if (c_px[m][3] != p3 || c_px[m][2] != p2) continue;
                    if (kind == 0 && c_px[m][1] != pa) continue;
                    if (kind == 1 && c_px[m][0] != pa) continue;
                    if (kind == 0) {
                        int p0 = c_px[m][0];
                        for (int tt = 0; tt < D.T1; tt++) {
                            const R2 *rv = (const R2 *)D.SE + (((size_t)s * D.T3 + t3) * NV + 3 + p0 * D.T1 + tt) * n;
                            R2 term = make_vec2<R>(0, 0);
                            if (qv) {
                                R2 r = rv[q];
                                R Rr = r.x, Ri = -r.y;
                                term.x = A::add(A::mul(gq.y, Rr), A::mul(gq.x, Ri));
                                term.y = A::sub(A::mul(gq.x, Rr), A::mul(Ri, gq.y));
                            }
                            double2 d = duo_dot<R>(term, red, par, half, lane, n, bar);
                            if (half == 0 && lane == 0) D.eaI[(((size_t)s * D.T3 + t3) * 21 + m) * D.T1 + tt] = d;
                        }
                    } else {
                        int p1 = c_px[m][1];
                        const R2 *rv = (const R2 *)D.SE + (((size_t)s * D.T3 + t3) * NV + p1) * n;
                        R2 term = make_vec2<R>(0, 0);
                        if (qv) {
                            R2 r = rv[q];
                            R nr = r.x, ni = -r.y;
                            term.x = A::add(A::mul(nr, gq.y), A::mul(ni, gq.x));
                            term.y = A::sub(A::mul(nr, gq.x), A::mul(ni, gq.y));
                        }
                        double2 d = duo_dot<R>(term, red, par, half, lane, n, bar);
                        if (half == 0 && lane == 0) D.eaII[(((size_t)s * D.T3 + t3) * 21 + m) * D.T1 + t1] = d;
                    }
                }
            }
        }
        if (t3 == D.T3 - 1) break;
        for (int i = threadIdx.x; i < n; i += blockDim.x) dg[i] = traj_diag(D.T, tl, i, false);
        __syncthreads();
        doubles_half_phases<R>(D, Uh, dg, tl, n, Wd);
        __syncthreads();
        const Dcoef<R> *cf = D.rot_static ? cf_static : cf_static + (tl - D.f0) * D.K;
        if (active)
            for (int sub = 0; sub < D.ts; sub++) {
                if (D.es) doubles_substep_duo<R, true>(F, Uh, cf, D.pairs, D.segs, D.nsegs, n, Wd, t64, half, cidx, bar);
                else doubles_substep_duo<R, false>(F, Uh, cf, D.pairs, D.segs, D.nsegs, n, Wd, t64, half, cidx, bar);
            }
    }
}

// Coupling coefficients of the doubles Trotter step for the static coupling
// frame: si = -sin(J f), co = sqrt(1-si^2), and the sqrt(2) pair
// (propagate.c:970-993), float operations as the reference in FP32.
template <typename R>
__global__ void k2d_dcoef(TwoD D, Dcoef<R> *cf, long nframes) {
    long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (g >= nframes * D.K) return;
    int k = (int)(g % D.K);
    long fi = g / D.K;
    int2 ab = D.pairs[k];
    float jv = traj_coupling(D.T, D.f0 + fi, ab.x, ab.y);
    Dcoef<R> q;
    if (!(fabsf(jv) > D.T.cut)) {
        q.co = 1; q.si = 0; q.co2 = 1; q.si2 = 0;
    } else if (sizeof(R) == 4) {
        float J = __fmul_rn(jv, D.f32_dsub);
        float si = -(float)sin((double)J);
        float co = sqrtf(__fsub_rn(1.0f, __fmul_rn(si, si)));
        float J2 = __fmul_rn(J, 1.41421356237f);
        float si2 = -(float)sin((double)J2);
        float co2 = sqrtf(__fsub_rn(1.0f, __fmul_rn(si2, si2)));
        q.co = co; q.si = si; q.co2 = co2; q.si2 = si2;
    } else {
        double J = (double)jv * D.f64_dsub;
        double si = -sin(J), si2 = -sin(J * (double)1.41421356237f);
        q.co = (R)sqrt(1.0 - si * si); q.si = (R)si; q.co2 = (R)sqrt(1.0 - si2 * si2); q.si2 = (R)si2;
    }
    cf[g] = q;
}


// ---------------------------------------------------------------- doubles, RK4
// propagate_vec_RK4_doubles (propagate.c:376-590): thread per doubles vector,
// in the reference's sequential order (stage sums accumulate element by
// element in the order of its loops), state and stage vectors in global
// memory in packed order.  The EA projections and dot products per t3 are
// those of k2d_doubles, summed in site order.
template <typename R> struct Rk4D;
template <> struct Rk4D<float> {
    // k += H * (c + k' * 0.5) * factor, evaluated in double like the reference
    static __device__ __forceinline__ float half(float k, float h, float c, float kp, float fac, bool minus) {
        double y = __dmul_rn(__dmul_rn((double)h, __dadd_rn((double)c, __dmul_rn((double)kp, 0.5))), (double)fac);
        return (float)(minus ? __dsub_rn((double)k, y) : __dadd_rn((double)k, y));
    }
    static __device__ __forceinline__ float full(float k, float h, float c, float kp, float fac, bool minus) {
        float y = __fmul_rn(__fmul_rn(h, __fadd_rn(c, kp)), fac);
        return minus ? __fsub_rn(k, y) : __fadd_rn(k, y);
    }
    static __device__ __forceinline__ float first(float k, float h, float c, float fac, bool minus) {
        float y = __fmul_rn(__fmul_rn(h, c), fac);
        return minus ? __fsub_rn(k, y) : __fadd_rn(k, y);
    }
    static __device__ __forceinline__ float update(float c, float k1, float k2, float k3, float k4) {
        double sum = __dadd_rn(__dadd_rn(__dadd_rn((double)k1, __dmul_rn(2.0, (double)k2)), __dmul_rn(2.0, (double)k3)),
                               (double)k4);
        return (float)__dadd_rn((double)c, __ddiv_rn(sum, 6.0));
    }
};
template <> struct Rk4D<double> {
    static __device__ __forceinline__ double half(double k, double h, double c, double kp, double fac, bool minus) {
        double y = h * (c + kp * 0.5) * fac;
        return minus ? k - y : k + y;
    }
    static __device__ __forceinline__ double full(double k, double h, double c, double kp, double fac, bool minus) {
        double y = h * (c + kp) * fac;
        return minus ? k - y : k + y;
    }
    static __device__ __forceinline__ double first(double k, double h, double c, double fac, bool minus) {
        double y = h * c * fac;
        return minus ? k - y : k + y;
    }
    static __device__ __forceinline__ double update(double c, double k1, double k2, double k3, double k4) {
        return c + (k1 + 2.0 * k2 + 2.0 * k3 + k4) / 6.0;
    }
};

template <typename R>
__device__ void rk4_doubles_step(const TwoD &D, long t, typename Vec2<R>::T *F, typename Vec2<R>::T *Kq, R *hd) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    typedef Rk4D<R> O;
    const int n = D.n, N2 = n * (n + 1) / 2;
    const R f = sizeof(R) == 4 ? (R)D.f32_dsub : (R)D.f64_dsub;
    const R sq2 = (R)1.41421356237f;
    R2 *K1 = Kq, *K2 = K1 + N2, *K3 = K2 + N2, *K4 = K3 + N2;
    for (int a = 0; a < n; a++) {  // HD (propagate.c:427-442)
        R ea = (R)traj_diag(D.T, t, a, false);
        for (int b = a; b < n; b++) {
            R hsum = A::add(ea, (R)traj_diag(D.T, t, b, false));
            R h = A::mul(f, hsum);
            if (a == b && !D.es) {
                R an = D.anh != 0.0f ? (R)D.anh : (R)D.T.anh[t * (1L + n) + 1 + a];
                h = A::sub(h, A::mul(an, f));
            }
            hd[sindex(a, b, n)] = h;
        }
    }
    for (int sub = 0; sub < D.ts; sub++) {
        for (int e = 0; e < 4 * N2; e++) { Kq[e].x = 0; Kq[e].y = 0; }
        for (int stage = 0; stage < 4; stage++) {
            R2 *Kn = stage == 0 ? K1 : stage == 1 ? K2 : stage == 2 ? K3 : K4;
            const R2 *Kp = stage == 1 ? K1 : stage == 2 ? K2 : K3;
            for (int e = 0; e < N2; e++) {
                R2 c = F[e], k = Kn[e];
                R h = hd[e];
                if (stage == 0) { k.x = O::first(k.x, h, c.y, (R)1, false); k.y = O::first(k.y, h, c.x, (R)1, true); }
                else if (stage < 3) { k.x = O::half(k.x, h, c.y, Kp[e].y, (R)1, false); k.y = O::half(k.y, h, c.x, Kp[e].x, (R)1, true); }
                else { k.x = O::full(k.x, h, c.y, Kp[e].y, (R)1, false); k.y = O::full(k.y, h, c.x, Kp[e].x, (R)1, true); }
                Kn[e] = k;
            }
            for (int kk = 0; kk < D.K; kk++) {
                int2 ab = D.pairs[kk];
                int a = ab.x, b = ab.y;
                float jv = traj_coupling(D.T, t, a, b);
                R h0 = fabsf(jv) > D.T.cut ? A::mul(f, (R)jv) : (R)0;
                for (int c = 0; c < n; c++) {
                    // two-level sites exclude |aa> and |bb> (propagate.c:648-662)
                    if (D.es && (c == a || c == b)) continue;
                    int i1 = sindex(a, c, n), i2 = sindex(b, c, n);
                    R fac = (c == a || c == b) ? sq2 : (R)1;
                    R2 c1 = F[i1], c2 = F[i2], k1 = Kn[i1];
                    if (stage == 0) {
                        k1.x = O::first(k1.x, h0, c2.y, fac, false); k1.y = O::first(k1.y, h0, c2.x, fac, true);
                    } else if (stage < 3) {
                        k1.x = O::half(k1.x, h0, c2.y, Kp[i2].y, fac, false);
                        k1.y = O::half(k1.y, h0, c2.x, Kp[i2].x, fac, true);
                    } else {
                        k1.x = O::full(k1.x, h0, c2.y, Kp[i2].y, fac, false);
                        k1.y = O::full(k1.y, h0, c2.x, Kp[i2].x, fac, true);
                    }
                    Kn[i1] = k1;
                    R2 k2 = Kn[i2];
                    if (stage == 0) {
                        k2.x = O::first(k2.x, h0, c1.y, fac, false); k2.y = O::first(k2.y, h0, c1.x, fac, true);
                    } else if (stage < 3) {
                        k2.x = O::half(k2.x, h0, c1.y, Kp[i1].y, fac, false);
                        k2.y = O::half(k2.y, h0, c1.x, Kp[i1].x, fac, true);
                    } else {
                        k2.x = O::full(k2.x, h0, c1.y, Kp[i1].y, fac, false);
                        k2.y = O::full(k2.y, h0, c1.x, Kp[i1].x, fac, true);
                    }
                    Kn[i2] = k2;
                }
            }
        }
        R norm = 0;  // find_norm / re_normalize (NISE_subs.c:125-148)
        for (int e = 0; e < N2; e++) norm = A::add(norm, A::add(A::mul(F[e].x, F[e].x), A::mul(F[e].y, F[e].y)));
        for (int e = 0; e < N2; e++) {
            R2 z = F[e];
            z.x = O::update(z.x, K1[e].x, K2[e].x, K3[e].x, K4[e].x);
            z.y = O::update(z.y, K1[e].y, K2[e].y, K3[e].y, K4[e].y);
            F[e] = z;
        }
        R nn = 0;
        for (int e = 0; e < N2; e++) nn = A::add(nn, A::add(A::mul(F[e].x, F[e].x), A::mul(F[e].y, F[e].y)));
        if (norm != nn) {
            R factor = (R)sqrt((double)(norm / nn));
            for (int e = 0; e < N2; e++) { F[e].x = A::mul(F[e].x, factor); F[e].y = A::mul(F[e].y, factor); }
        }
    }
}

// propagate_double_sparce (propagate.c:1304-1394) through frame t: ts times
// an anharmonic half phase on |aa>, the symmetrised U (x) U update over the
// element pairs of the truncated substep propagator (time_evolution_mat,
// propagate.c:1241-1299, called with its row and column lists exchanged,
// propagate.c:1496), and the second half phase.  Elements are enumerated in
// time_evolution_mat's order (row a outer, column b inner); zero (truncated)
// elements are not in the list.  V is the temporary of the update.
template <typename R>
__device__ void sparse_doubles_step(const TwoD &D, long t, typename Vec2<R>::T *F, typename Vec2<R>::T *V) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    const int n = D.n, N2 = n * (n + 1) / 2, nn = n * n;
    const R2 *Us = (const R2 *)D.Us + (t - D.f0) * nn;
    const R sq2 = (R)1.41421356237f;
    // fm = f * 0.5 / m with f = deltat*icm2ifs*twoPi (float), the product in double
    const R fm = sizeof(R) == 4 ? (R)(float)((double)D.f32_full * 0.5 / D.ts) : (R)(D.f64_full * 0.5 / D.ts);
    for (int sub = 0; sub < D.ts; sub++) {
        for (int half = 0; half < 2; half++) {
            if (half == 1)
                for (int e = 0; e < N2; e++) F[e] = V[e];
            else
                for (int e = 0; e < N2; e++) V[e] = F[e];
            for (int a = 0; a < n; a++) {
                if (D.es) {  // propagate.c:1422-1426, 1465-1469: plain copies
                    int ia = sindex(a, a, n);
                    F[ia] = V[ia];
                    continue;
                }
                R an = D.anh != 0.0f ? (R)D.anh : (R)D.T.anh[t * (1L + n) + 1 + a];
                R arg = A::mul(fm, an);
                R co = (R)cos((double)arg), si = (R)sin((double)arg);
                int ia = sindex(a, a, n);
                R2 v = V[ia], o;
                o.x = A::sub(A::mul(co, v.x), A::mul(si, v.y));
                o.y = A::add(A::mul(co, v.y), A::mul(si, v.x));
                F[ia] = o;
            }
            if (half == 1) break;
            for (int e = 0; e < N2; e++) V[e].x = V[e].y = 0;
            for (int ea = 0; ea < nn; ea++) {
                R2 ua = Us[ea];
                if (ua.x == (R)0 && ua.y == (R)0) continue;
                const int sA = ea % n, tA = ea / n;  // R = column, C = row (exchanged lists)
                for (int eb = 0; eb <= ea; eb++) {
                    R2 ub = Us[eb];
                    if (ub.x == (R)0 && ub.y == (R)0) continue;
                    const int u = eb % n, v = eb / n;
                    R g = 1;
                    if (sA != u) g = sq2;
                    if (v != tA) g = sq2;
                    if (sA != u && v != tA) g = 1;
                    // two-level sites: g = 0 when exactly one index differs
                    // (propagate.c:1448-1450); those terms add only zeros
                    if (D.es && g != (R)1) continue;
                    const int iA = sindex(sA, u, n), iB = sindex(tA, v, n);
                    R pr = A::sub(A::mul(ua.x, ub.x), A::mul(ua.y, ub.y));
                    R pi = A::add(A::mul(ua.y, ub.x), A::mul(ua.x, ub.y));
                    R2 fb = F[iB], acc = V[iA];
                    acc.x = A::add(acc.x, A::mul(A::mul(pr, fb.x), g));
                    acc.x = A::sub(acc.x, A::mul(A::mul(pi, fb.y), g));
                    acc.y = A::add(acc.y, A::mul(A::mul(pr, fb.y), g));
                    acc.y = A::add(acc.y, A::mul(A::mul(pi, fb.x), g));
                    V[iA] = acc;
                }
            }
        }
    }
}

// Thread per doubles vector: dipole_double at tk, then per t3 the EA
// projections (dipole_double_last) and dot products, then one doubles step
// (RK4, or the Sparse/Diagonal U (x) U step).
template <typename R>
__global__ void k2d_doubles_seq(TwoD D, int vec_per_sample, void *Fbuf, void *Kbuf, void *hdbuf) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= D.S * vec_per_sample) return;
    const int s = g / vec_per_sample, u = g % vec_per_sample, n = D.n, N2 = n * (n + 1) / 2, NV = nvec_se(D);
    R2 *F = (R2 *)Fbuf + (size_t)g * N2, *Kq = (R2 *)Kbuf + (size_t)g * 4 * N2;
    R *hd = (R *)hdbuf + (size_t)g * N2;
    const long tk = tk_of(D, s);
    int kind = u < 9 ? 0 : 1, pa, p2, t1 = 0;
    if (kind == 0) { pa = u / 3; p2 = u % 3; }
    else { int w = u - 9, cmb = w / D.T1; t1 = w % D.T1; pa = cmb / 3; p2 = cmb % 3; }
    const R2 *src = (const R2 *)D.SE + ((size_t)s * D.T3 * NV + (kind == 0 ? pa : 3 + pa * D.T1 + t1)) * n;
    for (int i = 0; i < n; i++)
        for (int j = i; j < n; j++) {
            R2 f;
            if (i == j) {
                R o = (R)over_mu(D, tk, p2, i);
                f.x = A::mul(o, src[i].x);
                f.y = A::mul(o, src[i].y);
            } else {
                R mi = (R)traj_mu(D.T, tk, p2, i), mj = (R)traj_mu(D.T, tk, p2, j);
                f.x = A::add(A::mul(mi, src[j].x), A::mul(mj, src[i].x));
                f.y = A::add(A::mul(mi, src[j].y), A::mul(mj, src[i].y));
            }
            F[sindex(i, j, n)] = f;
        }
    for (int t3 = 0; t3 < D.T3; t3++) {
        const long tl = tk + t3;
        if (D.ea)
            for (int p3 = 0; p3 < 3; p3++)
                for (int m = 0; m < 21; m++) {
                    if (c_px[m][3] != p3 || c_px[m][2] != p2) continue;
                    if (kind == 0 && c_px[m][1] != pa) continue;
                    if (kind == 1 && c_px[m][0] != pa) continue;
                    const int p0 = c_px[m][0], p1 = c_px[m][1];
                    int tt0 = kind == 0 ? 0 : t1, tt1 = kind == 0 ? D.T1 : t1 + 1;
                    for (int tt = tt0; tt < tt1; tt++) {
                        const R2 *rv = (const R2 *)D.SE +
                                       (((size_t)s * D.T3 + t3) * NV + (kind == 0 ? 3 + p0 * D.T1 + tt : p1)) * n;
                        double a1 = 0, a2 = 0;
                        for (int q = 0; q < n; q++) {
                            R gr = 0, gi = 0;  // dipole_double_last for site q
                            for (int j = 0; j < n; j++) {
                                R mm = (R)(j == q ? over_mu(D, tl, p3, q) : traj_mu(D.T, tl, p3, j));
                                R2 ff = F[sindex(j, q, n)];
                                gr = A::add(gr, A::mul(mm, ff.x));
                                gi = A::add(gi, A::mul(mm, ff.y));
                            }
                            R rr = rv[q].x, ri = -rv[q].y;
                            if (kind == 0) {
                                a1 += (double)A::add(A::mul(gi, rr), A::mul(gr, ri));
                                a2 += (double)A::sub(A::mul(gr, rr), A::mul(ri, gi));
                            } else {
                                a1 += (double)A::add(A::mul(rr, gi), A::mul(ri, gr));
                                a2 += (double)A::sub(A::mul(rr, gr), A::mul(ri, gi));
                            }
                        }
                        size_t o = (((size_t)s * D.T3 + t3) * 21 + m) * D.T1 + tt;
                        if (kind == 0) D.eaI[o] = make_double2(a1, a2);
                        else D.eaII[o] = make_double2(a1, a2);
                    }
                }
        if (t3 == D.T3 - 1) break;
        if (is_eigen_scheme(D.prop)) sparse_doubles_step<R>(D, tl, F, Kq);
        else rk4_doubles_step<R>(D, tl, F, Kq, hd);
    }
}

// ---------------------------------------------------------------- response
// Thread per (start point, t3, t1): GB (calc_2DIR.c:270-286), SE (:395-411)
// and EA (:473-487) contributions of all 21 molecular polarisations.
template <typename R>
__global__ void k2d_response(TwoD D) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (g >= (long)D.S * D.T3 * D.T1) return;
    int s = (int)(g / ((long)D.T3 * D.T1)), rem = (int)(g % ((long)D.T3 * D.T1)), t3 = rem / D.T1, t1 = rem % D.T1;
    const int n = D.n, NV = nvec_se(D);
    const long tk = tk_of(D, s), tl = tk + t3;
    double acc[12];
    for (int q = 0; q < 12; q++) acc[q] = 0;
    const R2 *SE0 = (const R2 *)D.SE + (size_t)s * D.T3 * NV * n;           // snapshots at tk
    const R2 *SEt = (const R2 *)D.SE + ((size_t)s * D.T3 + t3) * NV * n;    // snapshots at tl
    float lw = D.lt[t3 * D.T1 + t1];
    for (int m = 0; m < 21; m++) {
        int p0 = c_px[m][0], p1 = c_px[m][1], p2 = c_px[m][2], p3 = c_px[m][3];
        double pw[3];
        for (int q = 0; q < 3; q++) pw[q] = (double)__fmul_rn(c_w[q][m], lw);
        if (D.gb) {
            double2 a = D.gbt1[(((size_t)s * 3 + p0) * 3 + p1) * D.T1 + t1];  // t1nr, t1ni
            double2 b = D.gbt3[(((size_t)s * 3 + p2) * 3 + p3) * D.T3 + t3];  // t3nr, t3ni
            for (int q = 0; q < 3; q++) {
                acc[4 * q + 0] -= (b.y * a.x - b.x * a.y) * pw[q];
                acc[4 * q + 1] -= (b.x * a.x + b.y * a.y) * pw[q];
                acc[4 * q + 2] -= (b.y * a.x + b.x * a.y) * pw[q];
                acc[4 * q + 3] -= (b.x * a.x - b.y * a.y) * pw[q];
            }
        }
        if (D.se) {
            // t3nr/t3ni: leftr_p1(tk) . mu_p2(tk), imaginary part negated (:353-357)
            // t1rr/t1ri: leftn_p0[t1](tk) . mu_p2(tk), imaginary negated (:363-369)
            // t3rr/t3ri: mu_p3(tl) . leftr_p1(tl) (:377-381)
            // t1nr/t1ni: leftn_p0[t1](tl) . mu_p3(tl) (:384-390)
            double t3nr = 0, t3ni = 0, t1rr = 0, t1ri = 0, t3rr = 0, t3ri = 0, t1nr = 0, t1ni = 0;
            const R2 *lr0 = SE0 + (size_t)p1 * n, *ln0 = SE0 + (size_t)(3 + p0 * D.T1 + t1) * n;
            const R2 *lrt = SEt + (size_t)p1 * n, *lnt = SEt + (size_t)(3 + p0 * D.T1 + t1) * n;
            for (int i = 0; i < n; i++) {
                R m2 = (R)traj_mu(D.T, tk, p2, i), m3 = (R)traj_mu(D.T, tl, p3, i);
                R2 a = lr0[i], b = ln0[i], c = lrt[i], d = lnt[i];
                t3nr += (double)A::mul(a.x, m2);
                t3ni -= (double)A::mul(a.y, m2);
                t1rr += (double)A::mul(b.x, m2);
                t1ri -= (double)A::mul(b.y, m2);
                t3rr += (double)A::mul(m3, c.x);
                t3ri += (double)A::mul(m3, c.y);
                t1nr += (double)A::mul(d.x, m3);
                t1ni += (double)A::mul(d.y, m3);
            }
            for (int q = 0; q < 3; q++) {
                acc[4 * q + 0] -= (t3rr * t1ri + t3ri * t1rr) * pw[q];
                acc[4 * q + 1] -= (t3rr * t1rr - t3ri * t1ri) * pw[q];
                acc[4 * q + 2] -= (t3ni * t1nr + t3nr * t1ni) * pw[q];
                acc[4 * q + 3] -= (t3nr * t1nr - t3ni * t1ni) * pw[q];
            }
        }
        if (D.ea) {
            double2 I = D.eaI[(((size_t)s * D.T3 + t3) * 21 + m) * D.T1 + t1];
            double2 II = D.eaII[(((size_t)s * D.T3 + t3) * 21 + m) * D.T1 + t1];
            for (int q = 0; q < 3; q++) {
                acc[4 * q + 0] += I.x * pw[q];
                acc[4 * q + 1] += I.y * pw[q];
                acc[4 * q + 2] += II.x * pw[q];
                acc[4 * q + 3] += II.y * pw[q];
            }
        }
    }
    for (int q = 0; q < 12; q++) D.Rs[(((size_t)s * 12 + q) * D.T3 + t3) * D.T1 + t1] = acc[q];
}

__global__ void k2d_reduce(const double *Rs, int S, size_t plane, double *R, int first) {
    size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (e >= plane) return;
    double a = first ? 0.0 : R[e];
    for (int s = 0; s < S; s++) a += Rs[(size_t)s * plane + e];
    R[e] = a;
}

// Doubles RK4 (propagate_vec_RK4_doubles, propagate.c:376-590) and sparse
// (time_evolution_mat + propagate_double_sparce) schemes are not provided by
// this engine build; see nise_2dir's status message.

template <typename R>
__global__ void k2d_leftr(TwoD D) {
    typedef typename Vec2<R>::T R2;
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= D.S * 3 * D.n) return;
    int s = g / (3 * D.n), rem = g % (3 * D.n), x = rem / D.n, i = rem % D.n;
    R2 z;
    z.x = (R)traj_mu(D.T, tj_of(D, s), x, i);
    z.y = 0;
    ((R2 *)D.Lr)[((size_t)s * 3 + x) * D.n + i] = z;
}
int launch_2d_leftr(const TwoD &D, int prec, cudaStream_t s) {
    int tot = D.S * 3 * D.n;
    if (prec == NISE_FP32) k2d_leftr<float><<<(tot + 255) / 256, 256, 0, s>>>(D);
    else k2d_leftr<double><<<(tot + 255) / 256, 256, 0, s>>>(D);
    return (int)cudaGetLastError();
}


template <typename K>
int smem_attr(K kernel, size_t bytes) {
    if (bytes > 48 * 1024)
        return (int)cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return 0;
}

int lanes_for2(size_t bytes_per_lane, int want) {
    int b = want;
    while (b > 1 && (size_t)b * bytes_per_lane > 200 * 1024) b >>= 1;
    return b;
}

template <typename R>
int run_chunk(nise_ctx *c, TwoD &D, Dcoef<R> *cf) {
    typedef typename Vec2<R>::T R2;
    cudaStream_t st = c->stream;
    int e;
    size_t lane_b = (D.prop == NISE_PROP_RK4 ? 5 : is_eigen_scheme(D.prop) ? 2 : 1) * (size_t)D.n * sizeof(R2);
    int B = lanes_for2(lane_b, 64);
    size_t sm = lane_b * B;
    const int P = (D.T1 + 1) / 2;
    if ((e = smem_attr(k2d_gb1<R>, sm))) return e;
    if ((e = smem_attr(k2d_gb3<R>, sm))) return e;
    if ((e = smem_attr(k2d_se<R>, sm))) return e;
    k2d_gb1<R><<<(D.S * 3 * P + B - 1) / B, B, sm, st>>>(D);
    c->launches++;
    if (D.gb) {
        k2d_gb3<R><<<(D.S * 3 + B - 1) / B, B, sm, st>>>(D);
        c->launches++;
    }
    if (D.se || D.ea) {
        if (D.T2 > 0) {
            size_t lb2 = 2 * (size_t)D.n * sizeof(R2);
            int B2 = lanes_for2(lb2, 64);
            if ((e = smem_attr(k2d_t2<R>, lb2 * B2))) return e;
            int nv = D.S * (3 + 3 * D.T1);
            k2d_t2<R><<<(nv + B2 - 1) / B2, B2, lb2 * B2, st>>>(D);
            c->launches++;
        }
        int nv = D.S * (3 + 3 * D.T1);
        k2d_se<R><<<(nv + B - 1) / B, B, sm, st>>>(D);
        c->launches++;
    }
    if (D.ea && (D.prop == NISE_PROP_RK4 || is_eigen_scheme(D.prop))) {
        int vps = 9 + 9 * D.T1, tot = D.S * vps, N2 = D.n * (D.n + 1) / 2;
        void *Fb = nullptr, *Kb = nullptr, *Hb = nullptr;
        if ((e = (int)cudaMallocAsync(&Fb, sizeof(R2) * (size_t)tot * N2, st))) return e;
        if ((e = (int)cudaMallocAsync(&Kb, sizeof(R2) * (size_t)tot * 4 * N2, st))) return e;
        if ((e = (int)cudaMallocAsync(&Hb, sizeof(R) * (size_t)tot * N2, st))) return e;
        k2d_doubles_seq<R><<<(tot + 63) / 64, 64, 0, st>>>(D, vps, Fb, Kb, Hb);
        c->launches++;
        cudaFreeAsync(Fb, st);
        cudaFreeAsync(Kb, st);
        cudaFreeAsync(Hb, st);
    } else if (D.ea) {
        int W = D.n / 2 + 2, slots = D.n * W;
        // as many vectors (warps) as fit next to the phase table in shared memory;
        // the n x n slot-index table only where
        // it costs no warp
        auto bytes = [&](int w, bool tab) {
            return sizeof(R2) * (size_t)slots * (1 + w) + sizeof(float) * 7 * D.n +
                   (tab ? sizeof(short) * D.n * D.n : 0);
        };
        auto fit = [&](bool tab) {
            int w = 16;
            while (bytes(w, tab) > 220 * 1024 && w > 1) w--;
            return w;
        };
        int nwarps = fit(false);
        const int use_tab = fit(true) == nwarps && bytes(nwarps, true) <= 220 * 1024;
        size_t dsm = bytes(nwarps, use_tab);
        if (dsm > 220 * 1024) return (int)cudaErrorNotSupported;
        int vps = 9 + 9 * D.T1, cps = (vps + nwarps - 1) / nwarps;
        // two warps per vector (k2d_doubles_duo, the same float operations)
        // unless kernel_config 1 asks for one
        auto bytes_duo = [&](int pairs, bool tab) {
            return sizeof(R2) * ((size_t)slots * (1 + pairs) + 64 * (size_t)pairs) + sizeof(float) * 7 * D.n +
                   (tab ? sizeof(short) * D.n * D.n : 0);
        };
        if (D.n > 32 && D.n <= 64 && c->p.kernel_config != 1) {
            int np = 11;  // 704 threads at most; named barriers 1..11
            while (np > 1 && bytes_duo(np, false) > 220 * 1024) np--;
            const int tab = bytes_duo(np, true) <= 220 * 1024;
            const size_t dsm2 = bytes_duo(np, tab);
            if (dsm2 > 220 * 1024) return (int)cudaErrorNotSupported;
            const int cps2 = (vps + np - 1) / np;
            if ((e = smem_attr(k2d_doubles_duo<R>, dsm2))) return e;
            k2d_doubles_duo<R><<<D.S * cps2, 64 * np, dsm2, st>>>(D, vps, cf, tab);
        } else if (D.n <= 32) {
            if ((e = smem_attr(k2d_doubles<R, 1>, dsm))) return e;
            k2d_doubles<R, 1><<<D.S * cps, 32 * nwarps, dsm, st>>>(D, vps, cf, use_tab);
        } else if (D.n <= 64) {
            if ((e = smem_attr(k2d_doubles<R, 2>, dsm))) return e;
            k2d_doubles<R, 2><<<D.S * cps, 32 * nwarps, dsm, st>>>(D, vps, cf, use_tab);
        } else {
            if ((e = smem_attr(k2d_doubles<R, 4>, dsm))) return e;
            k2d_doubles<R, 4><<<D.S * cps, 32 * nwarps, dsm, st>>>(D, vps, cf, use_tab);
        }
        c->launches++;
    }
    long tot = (long)D.S * D.T3 * D.T1;
    k2d_response<R><<<(tot + 255) / 256, 256, 0, st>>>(D);
    c->launches++;
    return (int)cudaGetLastError();
}

}  // namespace

extern "C" int nise_2dir(nise_ctx *c, double *R, int *sample_count) {
    if (!c || !R || !sample_count) return nise_fail(c, NISE_ERR_ARG, "null argument");
    if (!c->loaded) return nise_fail(c, NISE_ERR_STATE, "no trajectory loaded");
    cudaSetDevice(c->p.device);
    nise_wait_all_frames(c, c->stream);  // energy records still in flight from the host
    const nise_params &p = c->p;
    const int N = c->n, T1 = p.tmax1, T2 = p.tmax2, T3 = p.tmax3, prec = p.precision;
    int tech = p.technique;
    if (tech < NISE_TECH_2DIR || tech > NISE_TECH_NOEAUVVIS)
        return nise_fail(c, NISE_ERR_ARG, "technique is not in the 2DIR or 2DUVvis family");
    // calc_2DES.c:244-245, 377-378, 315, 420: the same selections by name
    const bool es = tech >= NISE_TECH_2DUVVIS;
    if (es) tech -= NISE_TECH_2DUVVIS - NISE_TECH_2DIR;
    const bool eig_scheme = p.propagation == NISE_PROP_SPARSE || p.propagation == NISE_PROP_DIAGONAL;
    if (eig_scheme && N > NISE_EIG_MAX_N)
        return nise_fail(c, NISE_ERR_UNSUPPORTED, "2DIR with Propagation Sparse/Diagonal is limited to 120 sites");
    bool gb = tech == NISE_TECH_2DIR || tech == NISE_TECH_GBIR || tech == NISE_TECH_NOEAIR;
    bool se = tech == NISE_TECH_2DIR || tech == NISE_TECH_SEIR || tech == NISE_TECH_NOEAIR;
    bool ea = tech == NISE_TECH_2DIR || tech == NISE_TECH_EAIR;
    if (ea && N > 128) return nise_fail(c, NISE_ERR_UNSUPPORTED, "doubles manifold limited to 128 sites");
    if (T2 > 0 && N > NISE_EIG_MAX_N)
        return nise_fail(c, NISE_ERR_UNSUPPORTED, "t2 eigen step limited to 120 sites");
    if (ea && !es && p.anharmonicity == 0 && (!c->d_anh || !c->d_over))
        return nise_fail(c, NISE_ERR_IO, "Anharmonicity 0 needs Anharmonicfile and Overtonedipolefile");
    // calculateWorkset (MPI_subs.c:36-110)
    int total = (p.length - T1 - T2 - T3 - 1) / p.sample + 1;
    if (total <= 0) return nise_fail(c, NISE_ERR_ARG, "Insufficient data to calculate spectrum.");
    int end = p.end == 0 ? total : p.end, begin = p.begin;
    if (end > total || begin < 0 || begin > end) return nise_fail(c, NISE_ERR_ARG, "bad BeginPoint/EndPoint");
    int count = end - begin;
    *sample_count = count == 0 ? 1 : count;
    size_t plane = (size_t)T3 * T1;
    if (count == 0) {
        memset(R, 0, sizeof(double) * 12 * plane);
        return NISE_OK;
    }
    long fmin = (long)begin * p.sample + 1, fmax = (long)(end - 1) * p.sample + T1 + T2 + T3 - 1;
    int rc;
    if ((rc = nise_check_frames(c, fmax))) return rc;
    if (ea && !es && p.anharmonicity == 0 && (fmax >= c->a_frames || fmax >= c->o_frames))
        return nise_fail(c, NISE_ERR_IO, "Anharmonicity/overtone trajectory file to short");
    c->launches = 0;
    cudaEventRecord(c->ev0, c->stream);
    // polarisation weights as float values of polar.c:12-33
    {
        const float ith = 1.0f / 30;
        float w[3][21];
        for (int x = 0; x < 21; x++) {
            w[0][x] = x <= 2 ? 6 * ith : 2 * ith;
            w[1][x] = x <= 2 ? 2 * ith : (x <= 8 ? 4 * ith : -1 * ith);
            w[2][x] = x <= 8 ? 0.0f : (x <= 14 ? 2.5f * ith : -2.5f * ith);
        }
        cudaMemcpyToSymbolAsync(c_w, w, sizeof(w), 0, cudaMemcpyHostToDevice, c->stream);
    }
    // lifetime factors (calc_2DIR.c:105-115)
    std::vector<float> lt(plane);
    for (int t1 = 0; t1 < T1; t1++)
        for (int t3 = 0; t3 < T3; t3++)
            lt[(size_t)t3 * T1 + t1] = p.lifetime > 0
                                           ? (float)exp(-(double)(t1 + t3) * p.deltat / (2 * p.lifetime))
                                           : 1.0f;
    DevBuf<float> dlt;
    if ((rc = dlt.alloc(c, plane))) return rc;
    cudaMemcpyAsync(dlt.p, lt.data(), sizeof(float) * plane, cudaMemcpyHostToDevice, c->stream);

    DevTraj T = nise_devtraj(c);
    T.shift_ptr = nullptr;  // calc_2DIR reads frames with read_He: no SingleShift
    T.nshift = 0;
    size_t rsz = prec == NISE_FP32 ? sizeof(float) : sizeof(double), r2 = 2 * rsz;
    // singles coefficient tables over all frames of the job
    long nf = fmax - fmin + 1;
    TwoD D{};
    SinglesBufs SB;
    if ((rc = nise_singles_tables(c, T, fmin, nf, 0, ea, D, SB))) return rc;
    D.T = T;
    D.T1 = T1; D.T2 = T2; D.T3 = T3; D.sample = p.sample;
    D.gb = gb; D.se = se; D.ea = ea;
    D.es = es;
    D.anh = p.anharmonicity;
    D.f32_full = nise_f32(p, 1, 1);
    D.f64_full = nise_f64(p, 1, 1);
    D.f32_dsub = nise_f32(p, 1, p.ts);
    D.f64_dsub = nise_f64(p, 1, p.ts);
    D.Us = SB.Us;
    DevBuf<char> dcoef;
    D.rot_static = p.hamiltonian == NISE_HAM_COUPLING;
    if (ea) {  // doubles coupling coefficients: once (static couplings) or per frame
        long ncf = D.rot_static ? 1 : nf;
        if ((rc = dcoef.alloc(c, 4 * rsz * ((size_t)ncf * D.K + 1)))) return rc;  // one record past the last
        long tot = ncf * D.K;
        if (tot > 0) {
            if (prec == NISE_FP32)
                k2d_dcoef<float><<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(D, (Dcoef<float> *)dcoef.p, ncf);
            else
                k2d_dcoef<double><<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(D, (Dcoef<double> *)dcoef.p, ncf);
            c->launches++;
        }
    }
    // t2 eigendecompositions of every frame in [begin*sample+T1, (end-1)*sample+T1+T2)
    DevBuf<double> eV, ew;
    DevBuf<long> eframes;
    if (T2 > 0 && (se || ea)) {
        long e0 = (long)begin * p.sample + T1, e1 = (long)(end - 1) * p.sample + T1 + T2;
        std::vector<long> fr;
        for (long t = e0; t < e1; t++) fr.push_back(t);
        if ((rc = eframes.upload(c, fr)) || (rc = eV.alloc(c, fr.size() * (size_t)N * N)) ||
            (rc = ew.alloc(c, fr.size() * (size_t)N)))
            return rc;
        EigJob EJ;
        EJ.T = T; EJ.n = N; EJ.singleshift = 0;
        if ((rc = nise_cuda(c, launch_eig(EJ, eframes.p, (long)fr.size(), eV.p, ew.p, c->stream), "t2 eigensolver")))
            return rc;
        c->launches++;
        D.e0 = e0; D.eV = eV.p; D.ew = ew.p;
    }
    // chunks of start points sized to ~1.5 GB of per-chunk buffers
    const int NV = 3 + 3 * T1;
    size_t per_sample = r2 * ((size_t)3 * T1 * N + 3 * N + (size_t)T3 * NV * N) + sizeof(double2) * (9 * (size_t)T1 + 9 * T3) +
                        2 * sizeof(double2) * (size_t)T3 * 21 * T1 + sizeof(double) * 12 * plane;
    if (D.ea && (D.prop == NISE_PROP_RK4 || is_eigen_scheme(D.prop)))  // sequential doubles: state, 4 stages, diagonal
        per_sample += (9 + 9 * (size_t)T1) * (size_t)N * (N + 1) / 2 * (5 * r2 + r2 / 2);
    size_t budget = (size_t)1536 << 20;
    int chunk = (int)(budget / (per_sample > 0 ? per_sample : 1));
    if (chunk < 1) chunk = 1;
    if (chunk > count) chunk = count;
    if (p.launch_mode == NISE_PLAIN) chunk = 1;  // one start point per launch of every kernel
    DevBuf<char> L, Lr, SE, gbt1, gbt3, eaI, eaII, Rs;
    DevBuf<double> dR;
    if ((rc = L.alloc(c, r2 * (size_t)chunk * 3 * T1 * N)) || (rc = Lr.alloc(c, r2 * (size_t)chunk * 3 * N)) ||
        (rc = SE.alloc(c, r2 * (size_t)chunk * T3 * NV * N)) ||
        (rc = gbt1.alloc(c, sizeof(double2) * (size_t)chunk * 9 * T1)) ||
        (rc = gbt3.alloc(c, sizeof(double2) * (size_t)chunk * 9 * T3)) ||
        (rc = eaI.alloc(c, sizeof(double2) * (size_t)chunk * T3 * 21 * T1)) ||
        (rc = eaII.alloc(c, sizeof(double2) * (size_t)chunk * T3 * 21 * T1)) ||
        (rc = Rs.alloc(c, sizeof(double) * (size_t)chunk * 12 * plane)) || (rc = dR.alloc(c, 12 * plane)))
        return rc;
    cudaMemsetAsync(eaI.p, 0, sizeof(double2) * (size_t)chunk * T3 * 21 * T1, c->stream);
    cudaMemsetAsync(eaII.p, 0, sizeof(double2) * (size_t)chunk * T3 * 21 * T1, c->stream);
    D.L = L.p; D.Lr = Lr.p; D.SE = SE.p;
    D.gbt1 = (double2 *)gbt1.p; D.gbt3 = (double2 *)gbt3.p;
    D.eaI = (double2 *)eaI.p; D.eaII = (double2 *)eaII.p;
    D.Rs = (double *)Rs.p; D.lt = dlt.p;
    cudaEventRecord(c->evk0, c->stream);
    for (int s0 = begin; s0 < end; s0 += chunk) {
        D.s0 = s0;
        D.S = (end - s0) < chunk ? (end - s0) : chunk;
        // leftr_x = mu_x(tj) (calc_2DIR.c:303-304): host-free fill via a tiny copy kernel
        if ((rc = nise_cuda(c, launch_2d_leftr(D, prec, c->stream), "2DIR leftr"))) return rc;
        c->launches++;
        int e = prec == NISE_FP32 ? run_chunk<float>(c, D, (Dcoef<float> *)dcoef.p)
                                  : run_chunk<double>(c, D, (Dcoef<double> *)dcoef.p);
        if ((rc = nise_cuda(c, e, "2DIR kernels"))) return rc;
        k2d_reduce<<<(unsigned)((12 * plane + 255) / 256), 256, 0, c->stream>>>((const double *)Rs.p, D.S, 12 * plane,
                                                                               dR.p, s0 == begin);
        c->launches++;
    }
    cudaEventRecord(c->evk1, c->stream);
    cudaEventRecord(c->ev1, c->stream);
    cudaMemcpyAsync(R, dR.p, sizeof(double) * 12 * plane, cudaMemcpyDeviceToHost, c->stream);
    if ((rc = nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "2DIR"))) return rc;
    nise_collect_timing(c);
    // doubles Trotter work: vectors * steps * ts * (K rotations * (n-2) * 12 + 2 * N2 phases * 6)
    double N2 = (double)N * (N + 1) / 2;
    c->last_flops = ea ? (double)count * (9.0 + 9.0 * T1) * (T3 - 1) * p.ts * (12.0 * D.K * N + 12.0 * N2) : 0;
    c->last_bytes = (double)(fmax - fmin + 1) * 4 * (p.hamiltonian == NISE_HAM_COUPLING ? N : c->nn2);
    return NISE_OK;
}

extern "C" int nise_propagate_doubles(nise_ctx *c, const float *H, void *re, void *im, int nvec, const float *anh) {
    (void)H; (void)re; (void)im; (void)nvec; (void)anh;
    return nise_fail(c, NISE_ERR_UNSUPPORTED, "single doubles steps are not exposed by this engine build");
}
