// Device implementations of the singles propagation schemes, shared by the
// absorption and 2DIR kernels.  Each applies one full time step to the
// vector held in column `lane` of a [site][lane] shared-memory array, with
// the operand order and rounding of the reference (see Ar<> in common.cuh).
#pragma once
#include "common.cuh"
#include "nise_b200.h"

template <typename R> struct Cst;
template <> struct Cst<float> {
    static __device__ __forceinline__ float2 rot(float j, float fsub, float cut) {
        // propagate.c:853 (list keeps |J| > cut), :880-882
        if (!(fabsf(j) > cut)) return make_float2(1.0f, 0.0f);
        float J = __fmul_rn(j, fsub);
        float si = (float)(-sin((double)J));
        float co = sqrtf(__fsub_rn(1.0f, __fmul_rn(si, si)));
        return make_float2(co, si);
    }
};
template <> struct Cst<double> {
    static __device__ __forceinline__ double2 rot(float j, double fsub, float cut) {
        if (!(fabsf(j) > cut)) return make_double2(1.0, 0.0);
        double J = (double)j * fsub;
        double si = -sin(J);
        return make_double2(sqrt(1.0 - si * si), si);
    }
};

// One Trotter step (m sub-steps) of the vector held in column `lane` of S.
template <typename R>
__device__ __forceinline__ void trotter_apply(typename Vec2<R>::T *S, int B, int lane, int n, int K,
                                             const int2 *__restrict__ pairs,
                                             const typename Vec2<R>::T *__restrict__ Uf,
                                             const typename Vec2<R>::T *__restrict__ Rf, int m) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    for (int sub = 0; sub < m; sub++) {
        for (int a = 0; a < n; a++) {  // propagate.c:870-873
            R2 z = S[a * B + lane], u = Uf[a], o;
            o.x = A::sub(A::mul(z.x, u.x), A::mul(z.y, u.y));
            o.y = A::add(A::mul(z.y, u.x), A::mul(z.x, u.y));
            S[a * B + lane] = o;
        }
        for (int k = 0; k < K; k++) {  // propagate.c:876-888
            int2 ab = pairs[k];
            R2 cs = Rf[k];
            R2 xa = S[ab.x * B + lane], xb = S[ab.y * B + lane], ya, yb;
            ya.x = A::sub(A::mul(cs.x, xa.x), A::mul(cs.y, xb.y));
            ya.y = A::add(A::mul(cs.x, xa.y), A::mul(cs.y, xb.x));
            yb.x = A::sub(A::mul(cs.x, xb.x), A::mul(cs.y, xa.y));
            yb.y = A::add(A::mul(cs.x, xb.y), A::mul(cs.y, xa.x));
            S[ab.x * B + lane] = ya;
            S[ab.y * B + lane] = yb;
        }
        for (int a = 0; a < n; a++) {  // propagate.c:891-894
            R2 z = S[a * B + lane], u = Uf[a], o;
            o.x = A::sub(A::mul(z.x, u.x), A::mul(z.y, u.y));
            o.y = A::add(A::mul(z.y, u.x), A::mul(z.x, u.y));
            S[a * B + lane] = o;
        }
    }
}

// k_q accumulation with the operand types of propagate.c:323-357: the first
// and last stages are float, the two middle stages are evaluated in double
// (the literal 0.5 promotes them) and rounded back to float.
template <typename R> struct Rk4Ops;
template <> struct Rk4Ops<float> {
    static __device__ __forceinline__ float half(float acc, float h, float c, float k, bool minus) {
        double y = __dmul_rn((double)h, __dadd_rn((double)c, __dmul_rn((double)k, 0.5)));
        return (float)(minus ? __dsub_rn((double)acc, y) : __dadd_rn((double)acc, y));
    }
    static __device__ __forceinline__ float full(float acc, float h, float c, float k, bool minus) {
        float y = __fmul_rn(h, __fadd_rn(c, k));
        return minus ? __fsub_rn(acc, y) : __fadd_rn(acc, y);
    }
    static __device__ __forceinline__ float first(float acc, float h, float c, bool minus) {
        float y = __fmul_rn(h, c);
        return minus ? __fsub_rn(acc, y) : __fadd_rn(acc, y);
    }
    static __device__ __forceinline__ float update(float c, float k1, float k2, float k3, float k4) {
        float sum = __fadd_rn(__fadd_rn(__fadd_rn(k1, __fmul_rn(2.0f, k2)), __fmul_rn(2.0f, k3)), k4);
        return (float)__dadd_rn((double)c, __ddiv_rn((double)sum, 6.0));
    }
};
template <> struct Rk4Ops<double> {
    static __device__ __forceinline__ double half(double acc, double h, double c, double k, bool minus) {
        double y = h * (c + k * 0.5);
        return minus ? acc - y : acc + y;
    }
    static __device__ __forceinline__ double full(double acc, double h, double c, double k, bool minus) {
        double y = h * (c + k);
        return minus ? acc - y : acc + y;
    }
    static __device__ __forceinline__ double first(double acc, double h, double c, bool minus) {
        double y = h * c;
        return minus ? acc - y : acc + y;
    }
    static __device__ __forceinline__ double update(double c, double k1, double k2, double k3, double k4) {
        return c + (k1 + 2.0 * k2 + 2.0 * k3 + k4) / 6.0;
    }
};

template <typename R>
__device__ __forceinline__ R norm_of(const typename Vec2<R>::T *C, int B, int lane, int n) {
    R s = 0;
    for (int a = 0; a < n; a++) {  // find_norm, NISE_subs.c:125-133
        typename Vec2<R>::T z = C[a * B + lane];
        s = Ar<R>::add(s, Ar<R>::add(Ar<R>::mul(z.x, z.x), Ar<R>::mul(z.y, z.y)));
    }
    return s;
}

// One RK4 step (m sub-steps), propagate.c:311-366.  S holds the state and
// K1..K4 follow it in shared memory, all [site][lane].
template <typename R>
__device__ __forceinline__ void rk4_apply(typename Vec2<R>::T *S, int B, int lane, int n, int K,
                                         const int2 *__restrict__ ent, const R *__restrict__ val, int m) {
    typedef typename Vec2<R>::T R2;
    typedef Rk4Ops<R> O;
    R2 *K1 = S + (size_t)n * B, *K2 = K1 + (size_t)n * B, *K3 = K2 + (size_t)n * B, *K4 = K3 + (size_t)n * B;
    for (int sub = 0; sub < m; sub++) {
        for (int a = 0; a < n; a++) {
            R2 z;
            z.x = 0;
            z.y = 0;
            K1[a * B + lane] = z; K2[a * B + lane] = z; K3[a * B + lane] = z; K4[a * B + lane] = z;
        }
        for (int k = 0; k < K; k++) {
            int2 e = ent[k];
            R h = val[k];
            int c = e.x, r = e.y;
            R2 sr = S[r * B + lane], kc = K1[c * B + lane];
            kc.x = O::first(kc.x, h, sr.y, false);
            kc.y = O::first(kc.y, h, sr.x, true);
            K1[c * B + lane] = kc;
            if (r != c) {
                R2 sc = S[c * B + lane], kr = K1[r * B + lane];
                kr.x = O::first(kr.x, h, sc.y, false);
                kr.y = O::first(kr.y, h, sc.x, true);
                K1[r * B + lane] = kr;
            }
        }
        for (int stage = 1; stage < 4; stage++) {
            R2 *Kp = stage == 1 ? K1 : (stage == 2 ? K2 : K3);
            R2 *Kn = stage == 1 ? K2 : (stage == 2 ? K3 : K4);
            for (int k = 0; k < K; k++) {
                int2 e = ent[k];
                R h = val[k];
                int c = e.x, r = e.y;
                R2 sr = S[r * B + lane], pr = Kp[r * B + lane], kc = Kn[c * B + lane];
                if (stage < 3) {
                    kc.x = O::half(kc.x, h, sr.y, pr.y, false);
                    kc.y = O::half(kc.y, h, sr.x, pr.x, true);
                } else {
                    kc.x = O::full(kc.x, h, sr.y, pr.y, false);
                    kc.y = O::full(kc.y, h, sr.x, pr.x, true);
                }
                Kn[c * B + lane] = kc;
                if (r != c) {
                    R2 sc = S[c * B + lane], pc = Kp[c * B + lane], kr = Kn[r * B + lane];
                    if (stage < 3) {
                        kr.x = O::half(kr.x, h, sc.y, pc.y, false);
                        kr.y = O::half(kr.y, h, sc.x, pc.x, true);
                    } else {
                        kr.x = O::full(kr.x, h, sc.y, pc.y, false);
                        kr.y = O::full(kr.y, h, sc.x, pc.x, true);
                    }
                    Kn[r * B + lane] = kr;
                }
            }
        }
        R norm = norm_of<R>(S, B, lane, n);
        for (int a = 0; a < n; a++) {
            R2 z = S[a * B + lane], k1 = K1[a * B + lane], k2 = K2[a * B + lane], k3 = K3[a * B + lane],
               k4 = K4[a * B + lane];
            z.x = O::update(z.x, k1.x, k2.x, k3.x, k4.x);
            z.y = O::update(z.y, k1.y, k2.y, k3.y, k4.y);
            S[a * B + lane] = z;
        }
        R nn = norm_of<R>(S, B, lane, n);  // re_normalize, NISE_subs.c:136-148
        if (norm != nn) {
            R factor = (R)sqrt((double)(norm / nn));
            for (int a = 0; a < n; a++) {
                R2 z = S[a * B + lane];
                z.x = Ar<R>::mul(z.x, factor);
                z.y = Ar<R>::mul(z.y, factor);
                S[a * B + lane] = z;
            }
        }
    }
}

// Response of one vector at one time: sum_i mu_i * psi_i.  In FP32 the
// product is rounded to float before the FP64 sum, as calc_S1
// (absorption.c:205-212) does with a double accumulator.  The FP64 sum runs
// in one fixed order that a thread and a warp can both produce: a partial
// sum per site residue r = i mod 32 (ascending sites), then the 32 partials
// in residue order.  It differs from the site order of the reference only by
// FP64 rounding, and every kernel that uses it (a thread per vector here, a
// warp per vector in resp_sum_warp) gives bitwise the same responses.
// Residues r >= n have no sites: their partial is +0, which leaves a sum
// that starts at +0 unchanged, so they are skipped.
template <typename R>
__device__ __forceinline__ double2 dot_mu(const DevTraj &T, long t, int x, const typename Vec2<R>::T *S, int B,
                                          int lane, int n) {
    double re = 0, im = 0;
    for (int r = 0; r < 32 && r < n; r++) {
        double pr = 0, pi = 0;
        for (int i = r; i < n; i += 32) {
            R m = (R)traj_mu(T, t, x, i);
            typename Vec2<R>::T z = S[i * B + lane];
            pr += (double)Ar<R>::mul(m, z.x);
            pi += (double)Ar<R>::mul(m, z.y);
        }
        re += pr;
        im += pi;
    }
    return make_double2(re, im);
}

// The residue-order sum of dot_mu across a warp: lane r holds the partial
// sum of sites r, r+32, ... (ascending); every lane gets the total.
__device__ __forceinline__ double2 resp_sum_warp(double pr, double pi, int n) {
    double re = 0, im = 0;
    for (int r = 0; r < 32 && r < n; r++) {
        re += __shfl_sync(0xffffffffu, pr, r);
        im += __shfl_sync(0xffffffffu, pi, r);
    }
    return make_double2(re, im);
}

__host__ __device__ __forceinline__ bool is_eigen_scheme(int prop) {
    return prop == NISE_PROP_SPARSE || prop == NISE_PROP_DIAGONAL;
}

// propagate_vec_DIA / propagate_vec_DIA_S (propagate.c:60-125, 185-258) on
// one vector of the [site][lane] layout: c_a <- sum_b U_ab c_b, accumulated
// in b order (float operations in FP32 mode); truncated elements of U are
// zero.  The temporary is the second half of the lane's shared memory.
template <typename R>
__device__ __forceinline__ void dia_apply(typename Vec2<R>::T *S, int B, int lane, int n,
                                          const typename Vec2<R>::T *U) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    R2 *Tm = S + (size_t)n * B;
    for (int a = 0; a < n; a++) {
        R2 acc;
        acc.x = acc.y = 0;
        for (int b = 0; b < n; b++) {
            R2 u = U[(size_t)a * n + b], z = S[b * B + lane];
            acc.x = A::add(acc.x, A::sub(A::mul(u.x, z.x), A::mul(u.y, z.y)));
            acc.y = A::add(acc.y, A::add(A::mul(u.x, z.y), A::mul(u.y, z.x)));
        }
        Tm[a * B + lane] = acc;
    }
    for (int a = 0; a < n; a++) S[a * B + lane] = Tm[a * B + lane];
}

// One singles time step (propagate_vector, propagate.c:20-39) of the
// configured scheme through frame t, from the job's coefficient tables.
template <typename R>
__device__ __forceinline__ void singles_step(const SinglesTab &D, typename Vec2<R>::T *S, int B, int lane, long t) {
    typedef typename Vec2<R>::T R2;
    long fi = t - D.f0;
    if (is_eigen_scheme(D.prop)) {
        dia_apply<R>(S, B, lane, D.n, (const R2 *)D.Ud + fi * D.n * D.n);
    } else if (D.prop == NISE_PROP_RK4) {
        rk4_apply<R>(S, B, lane, D.n, D.Kr, D.ent, (const R *)D.rkval + fi * D.Kr, D.ts);
    } else {
        const R2 *Uf = (const R2 *)D.U + fi * D.n;
        const R2 *Rf = D.rot_static ? (const R2 *)D.rot : (const R2 *)D.rot + fi * D.K;
        trotter_apply<R>(S, B, lane, D.n, D.K, D.pairs, Uf, Rf, D.ts);
    }
}

// Shared memory one lane of singles_step needs: the vector, plus a
// temporary vector (eigen route) or the four RK4 stages.
template <typename R>
__host__ __device__ __forceinline__ size_t singles_lane_bytes(int n, int prop) {
    return (prop == NISE_PROP_RK4 ? 5 : is_eigen_scheme(prop) ? 2 : 1) * (size_t)n * sizeof(typename Vec2<R>::T);
}
