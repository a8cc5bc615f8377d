// Adjoint of linear absorption (no reference counterpart; the reference has
// no derivatives).  The differentiable model is the Trotter "Coupling"
// absorption of propagate_vec_coupling_S (propagate.c:821-899) and
// absorption.c:119-145 in FP64 (and, further below, the RK4 scheme of
// propagate_vec_RK4 and the exact propagator of propagate_vec_DIA), with
// three parameters:
//   b_a  per-site energy shifts added to the shifted diagonal (the b of a
//        SingleShift with a = 1, hamshift.c:59-66),
//   s    a global scale of every coupling (after the read cut),
//   T1   the Lifetime of the 1D transform (1DFFT.c:178-181).
// Rotations are applied for every nonzero coupling of the pattern (the
// read cut removes |J| < Couplingcut), so the model is smooth in s.
//
// Forward (k_adj_fwd): thread per vector (start point, polarisation), the
// state in shared memory ([site][lane]); the response is recorded and the
// state is stored every K steps (checkpoints) and at the last step.
// Backward (k_adj_bwd): reverse-time propagation from the last state, each
// Trotter operation undone in reverse order (they are unitary, the inverse
// is the conjugate operation) while the adjoint state is carried back through
// the same operations; the state is reset from the checkpoint whenever the
// reverse sweep reaches one, which bounds the drift of the reconstruction.
// Per operation the derivative terms are accumulated:
//   half phase  y_a = exp(-i h_a f/2) x_a:   dL/db_a += (f/2) Im(conj(l_a) y_a)
//   rotation    y = R(theta) x, theta = s J f:  dL/ds += J f Re(l . dR/dtheta x)
// and the response gradient G(t1) is injected as l_a += mu_a(t) G(t1).
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace {

// FP64 tables for frames [f0, f0+nf): U[t][a] = (cos(h f/2), -sin(h f/2)),
// rot[t][k] = (co, si) with si = -sin(s J f), co = sqrt(1 - si^2), and
// jf[t][k] = J f (the derivative of the angle with respect to s).
__global__ void k_adj_prep(DevTraj T, AdjPlan P) {
    long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long nU = P.nf * P.n, nR = P.nf * P.k;
    if (g < nU) {
        long t = g / P.n;
        int a = (int)(g % P.n);
        double h = (double)traj_diag_raw(T, P.f0 + t, a) + P.shift[a];
        double s, c;
        sincos(0.5 * h * P.f, &s, &c);
        P.U[g] = make_double2(c, -s);
        return;
    }
    g -= nU;
    if (g < nR) {
        long t = g / P.k;
        int k = (int)(g % P.k);
        int2 ab = P.pairs[k];
        double jf = (double)traj_coupling(T, P.f0 + t, ab.x, ab.y) * P.f;
        double si = -sin(P.scale * jf);
        P.rot[g] = make_double2(sqrt(1.0 - si * si), si);
        P.jf[g] = jf;
    }
}

__device__ __forceinline__ void adj_phase(double2 *X, int B, int lane, int n, const double2 *U) {
    for (int a = 0; a < n; a++) {
        double2 u = U[a], z = X[a * B + lane];
        X[a * B + lane] = make_double2(z.x * u.x - z.y * u.y, z.y * u.x + z.x * u.y);
    }
}

// One forward Trotter step through frame table row fi (ts sub-steps).
__device__ void adj_step(double2 *X, int B, int lane, const AdjPlan &P, long fi) {
    const double2 *U = P.U + fi * P.n, *Rt = P.rot + fi * P.k;
    for (int sub = 0; sub < P.ts; sub++) {
        adj_phase(X, B, lane, P.n, U);
        for (int k = 0; k < P.k; k++) {
            int2 ab = P.pairs[k];
            double2 cs = Rt[k], xa = X[ab.x * B + lane], xb = X[ab.y * B + lane];
            // ya = co xa + i si xb, yb = co xb + i si xa
            X[ab.x * B + lane] = make_double2(cs.x * xa.x - cs.y * xb.y, cs.x * xa.y + cs.y * xb.x);
            X[ab.y * B + lane] = make_double2(cs.x * xb.x - cs.y * xa.y, cs.x * xb.y + cs.y * xa.x);
        }
        adj_phase(X, B, lane, P.n, U);
    }
}

__global__ void k_adj_fwd(DevTraj T, AdjPlan P, AbsJob J, double2 *resp, double2 *ckpt) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *X = (double2 *)smem_raw;
    const int B = blockDim.x, lane = threadIdx.x, n = P.n;
    const int v = blockIdx.x * B + lane;
    if (v >= 3 * J.nsamp) return;
    const int x = v % 3;
    const long ti = (long)(J.begin + v / 3) * J.sample;
    for (int a = 0; a < n; a++) X[a * B + lane] = make_double2((double)traj_mu(T, ti, x, a), 0.0);
    double2 *ck = ckpt + (size_t)v * P.nck * n;
    for (int t1 = 0; t1 < J.tmax; t1++) {
        const long t = ti + t1;
        double re = 0, im = 0;
        for (int a = 0; a < n; a++) {
            double m = (double)traj_mu(T, t, x, a);
            double2 z = X[a * B + lane];
            re += m * z.x;
            im += m * z.y;
        }
        resp[(size_t)v * J.tmax + t1] = make_double2(re, im);
        if (t1 % P.K == 0)
            for (int a = 0; a < n; a++) ck[(size_t)(t1 / P.K) * n + a] = X[a * B + lane];
        if (t1 == J.tmax - 1) {
            for (int a = 0; a < n; a++) ck[(size_t)(P.nck - 1) * n + a] = X[a * B + lane];
            break;
        }
        adj_step(X, B, lane, P, t - P.f0);
    }
}

// Undo a half phase (x = conj(u) y) and carry the adjoint back (l <- conj(u) l);
// the derivative of y_a with respect to b_a is (-i f/2) y_a, whose pairing
// with the adjoint is Re(conj(l_a) (-i f/2) y_a) = (f/2)(l.x y.y - l.y y.x).
__device__ __forceinline__ void adj_phase_back(double2 *X, double2 *L, double *gs, int B, int lane, int n,
                                               const double2 *U, double hf) {
    for (int a = 0; a < n; a++) {
        double2 u = U[a], y = X[a * B + lane], l = L[a * B + lane];
        gs[a * B + lane] += hf * (l.x * y.y - l.y * y.x);
        X[a * B + lane] = make_double2(y.x * u.x + y.y * u.y, y.y * u.x - y.x * u.y);
        L[a * B + lane] = make_double2(l.x * u.x + l.y * u.y, l.y * u.x - l.x * u.y);
    }
}

__global__ void k_adj_bwd(DevTraj T, AdjPlan P, AbsJob J, const double2 *G, const double2 *ckpt, double *gshift,
                          double *gscale) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int B = blockDim.x, lane = threadIdx.x, n = P.n;
    double2 *X = (double2 *)smem_raw, *L = X + (size_t)n * B;
    double *gs = (double *)(L + (size_t)n * B);
    const int v = blockIdx.x * B + lane;
    if (v >= 3 * J.nsamp) return;
    const int x = v % 3;
    const long ti = (long)(J.begin + v / 3) * J.sample;
    const double2 *ck = ckpt + (size_t)v * P.nck * n;
    const double hf = 0.5 * P.f;
    double gsc = 0;
    {
        const long t = ti + J.tmax - 1;
        const double2 g = G[J.tmax - 1];
        for (int a = 0; a < n; a++) {
            double m = (double)traj_mu(T, t, x, a);
            X[a * B + lane] = ck[(size_t)(P.nck - 1) * n + a];
            L[a * B + lane] = make_double2(m * g.x, m * g.y);
            gs[a * B + lane] = 0;
        }
    }
    for (int t1 = J.tmax - 2; t1 >= 0; t1--) {
        const long t = ti + t1, fi = t - P.f0;
        const double2 *U = P.U + fi * n, *Rt = P.rot + fi * P.k;
        const double *Jf = P.jf + fi * P.k;
        for (int sub = P.ts - 1; sub >= 0; sub--) {
            adj_phase_back(X, L, gs, B, lane, n, U, hf);
            for (int k = P.k - 1; k >= 0; k--) {
                int2 ab = P.pairs[k];
                double co = Rt[k].x, si = Rt[k].y;
                double2 ya = X[ab.x * B + lane], yb = X[ab.y * B + lane];
                double2 la = L[ab.x * B + lane], lb = L[ab.y * B + lane];
                // inputs: xa = co ya - i si yb, xb = co yb - i si ya
                double2 xa = make_double2(co * ya.x + si * yb.y, co * ya.y - si * yb.x);
                double2 xb = make_double2(co * yb.x + si * ya.y, co * yb.y - si * ya.x);
                // dy/dtheta with sin(theta) = -si, cos(theta) = co:
                // dya = si xa - i co xb, dyb = si xb - i co xa
                double2 da = make_double2(si * xa.x + co * xb.y, si * xa.y - co * xb.x);
                double2 db = make_double2(si * xb.x + co * xa.y, si * xb.y - co * xa.x);
                gsc += Jf[k] * (la.x * da.x + la.y * da.y + lb.x * db.x + lb.y * db.y);
                X[ab.x * B + lane] = xa;
                X[ab.y * B + lane] = xb;
                L[ab.x * B + lane] = make_double2(co * la.x + si * lb.y, co * la.y - si * lb.x);
                L[ab.y * B + lane] = make_double2(co * lb.x + si * la.y, co * lb.y - si * la.x);
            }
            adj_phase_back(X, L, gs, B, lane, n, U, hf);
        }
        if (t1 % P.K == 0)
            for (int a = 0; a < n; a++) X[a * B + lane] = ck[(size_t)(t1 / P.K) * n + a];
        const double2 g = G[t1];
        for (int a = 0; a < n; a++) {
            double m = (double)traj_mu(T, t, x, a);
            double2 l = L[a * B + lane];
            L[a * B + lane] = make_double2(l.x + m * g.x, l.y + m * g.y);
        }
    }
    for (int a = 0; a < n; a++) gshift[(size_t)v * n + a] = gs[a * B + lane];
    gscale[v] = gsc;
}

// Deterministic sums over vectors: g[a] = sum_v part[v][a] (a < n), in v order.
__global__ void k_adj_reduce(const double *part, int nvec, int n, double *g) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    double s = 0;
    for (int v = 0; v < nvec; v++) s += part[(size_t)v * n + a];
    g[a] = s;
}

int lanes_adj(size_t lane_bytes) {
    int B = 64;
    while (B > 1 && lane_bytes * B > 200 * 1024) B >>= 1;
    return B;
}

// ------------------------------------------------- RK4 and the exact step
// Models whose step is a Taylor polynomial of A = -i H f/m, applied m times
// per frame: y = P(A) x, P(A) = sum_(j<=deg) A^j / j!.
//  * RK4 (propagate_vec_RK4, propagate.c:261-373): deg 4 (RK4 for a
//    constant H is its fourth-order Taylor polynomial), m = Trotter
//    sub-steps, then x' = y |x| / |y| (re_normalize to the pre-step norm).
//  * The exact propagator exp(-i H f) of propagate_vec_DIA
//    (propagate.c:60-125; Propagation Sparse with Threshold 0, or Diagonal):
//    deg 18 and m = ceil(f ||H||) over the job's frames (||H|| bounded by
//    max |h_a + b_a| + |s| ||J||_F), so ||A|| <= 1 and the series' remainder
//    is below 1/19! * e = 2e-17 relative; no renormalisation.
// H = diag(h + b) + s J over every nonzero coupling of the pattern (as the
// Trotter model, so that it is smooth in s).  Vectors live in global scratch,
// slot q of vector v at base + (q n + a) nvec + v (a warp's lanes read
// consecutive addresses).
//
// Adjoint of one sub-step, l the gradient with respect to x':
//   renormalised: c = Re(l . y), l_y = r l - c |x| y / |y|^3 (r = |x|/|y|),
//   and the norm's own term c x / (|x| |y|) goes to l_x; otherwise l_y = l;
//   l_x += P(A)^+ l_y = sum_p w_p / p!, w_p = (A^+)^p l_y, A^+ = +i H f/m;
//   dL = Re sum_{p+q<=deg-1} w_p^+ dA u_q / (p+q+1)!, u_q = A^q x,
//   dA = -i dH f/m: the shift b_a gets (f/m) sum Im(conj(v_q,a) u_q,a) and
//   the scale s gets (f/m) sum_k J_k [Im(conj(v_q,a) u_q,b) +
//   Im(conj(v_q,b) u_q,a)], with v_q = sum_{p<=deg-1-q} w_p / (p+q+1)!.
// The backward sweep recomputes the frame states of each checkpoint block,
// then each frame's sub-step inputs, from the forward checkpoints.
constexpr int kPolyMaxDeg = 18;

struct Rk4Adj {
    int n, k, m, K, nck, nvec;
    int deg, renorm;  // polynomial degree; renormalise each sub-step (RK4)
    const int2 *pairs;
    long f0, nf;
    const double *D, *Jc, *jf;  // [nf][n] (h + b) f/m, [nf][k] s J f/m, [nf][k] J f/m
    double2 *scr;               // [slots][n][nvec]
    double fm;
};

__global__ void k_adj_rk4_prep(DevTraj T, AdjPlan P, double fm, double *D, double *Jc, double *jf) {
    long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long nU = P.nf * P.n, nR = P.nf * P.k;
    if (g < nU) {
        long t = g / P.n;
        int a = (int)(g % P.n);
        D[g] = ((double)traj_diag_raw(T, P.f0 + t, a) + P.shift[a]) * fm;
        return;
    }
    g -= nU;
    if (g < nR) {
        long t = g / P.k;
        int k = (int)(g % P.k);
        int2 ab = P.pairs[k];
        const double J = (double)traj_coupling(T, P.f0 + t, ab.x, ab.y) * fm;
        jf[g] = J;
        Jc[g] = P.scale * J;
    }
}

// Per frame an upper bound of ||A|| for m = 1, from the tables built with
// fm = f: max_a |D_a| + sqrt(2 sum_k Jc_k^2) (the Frobenius norm of the
// couplings); bnd[0] gets the maximum over the frames.
__global__ void k_adj_bound(const double *D, const double *Jc, int n, int k, long nf, double *bnd) {
    __shared__ double red[256];
    double mx = 0;
    for (long t = threadIdx.x; t < nf; t += blockDim.x) {
        double d = 0, j2 = 0;
        for (int a = 0; a < n; a++) d = fmax(d, fabs(D[t * n + a]));
        for (int q = 0; q < k; q++) j2 += Jc[t * k + q] * Jc[t * k + q];
        mx = fmax(mx, d + sqrt(2 * j2));
    }
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) bnd[0] = red[0];
}

struct Slot {
    double2 *p;
    int nvec;
    __device__ double2 &operator[](int a) const { return p[(size_t)a * nvec]; }
};

__device__ __forceinline__ Slot slot(const Rk4Adj &R, int q, int v) {
    return Slot{R.scr + (size_t)q * R.n * R.nvec + v, R.nvec};
}

// y = H0 x (H0 = H f/m, real symmetric), frame row fi.
__device__ void rk4_h(const Rk4Adj &R, long fi, Slot x, Slot y) {
    const double *D = R.D + fi * R.n, *Jc = R.Jc + fi * R.k;
    for (int a = 0; a < R.n; a++) {
        const double2 z = x[a];
        y[a] = make_double2(D[a] * z.x, D[a] * z.y);
    }
    for (int k = 0; k < R.k; k++) {
        const int2 ab = R.pairs[k];
        const double j = Jc[k];
        const double2 xa = x[ab.x], xb = x[ab.y], ya = y[ab.x], yb = y[ab.y];
        y[ab.x] = make_double2(ya.x + j * xb.x, ya.y + j * xb.y);
        y[ab.y] = make_double2(yb.x + j * xa.x, yb.y + j * xa.y);
    }
}

// y = A x (adj = false, A = -i H0) or y = A^+ x (adj = true, +i H0).
__device__ void rk4_a(const Rk4Adj &R, long fi, Slot x, Slot y, bool adj) {
    rk4_h(R, fi, x, y);
    for (int a = 0; a < R.n; a++) {
        const double2 h = y[a];
        y[a] = adj ? make_double2(-h.y, h.x) : make_double2(h.y, -h.x);
    }
}

__device__ double rk4_norm2(const Rk4Adj &R, Slot x) {
    double s = 0;
    for (int a = 0; a < R.n; a++) {
        const double2 z = x[a];
        s += z.x * z.x + z.y * z.y;
    }
    return s;
}

// y = P(A) x by Horner's rule (t <- x + A t / j, j = deg .. 1); tmp is scratch.
__device__ void rk4_poly(const Rk4Adj &R, long fi, Slot x, Slot y, Slot tmp) {
    for (int a = 0; a < R.n; a++) y[a] = x[a];
    for (int j = R.deg; j >= 1; j--) {
        rk4_a(R, fi, y, tmp, false);
        const double c = 1.0 / j;
        for (int a = 0; a < R.n; a++) {
            const double2 z = x[a], u = tmp[a];
            y[a] = make_double2(z.x + c * u.x, z.y + c * u.y);
        }
    }
}

// One frame: m sub-steps x <- P(A) x (|x| / |P(A) x| when renormalised), in
// place (y, tmp scratch).
__device__ void rk4_frame(const Rk4Adj &R, long fi, Slot x, Slot y, Slot tmp) {
    for (int sub = 0; sub < R.m; sub++) {
        const double n0 = R.renorm ? rk4_norm2(R, x) : 1.0;
        rk4_poly(R, fi, x, y, tmp);
        const double sc = R.renorm ? sqrt(n0 / rk4_norm2(R, y)) : 1.0;
        for (int a = 0; a < R.n; a++) {
            const double2 z = y[a];
            x[a] = make_double2(z.x * sc, z.y * sc);
        }
    }
}

// slots of the forward kernel: 0 state, 1 y, 2 tmp
__global__ void k_adj_rk4_fwd(DevTraj T, Rk4Adj R, AbsJob J, double2 *resp, double2 *ckpt) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= R.nvec) return;
    const int x = v % 3, n = R.n;
    const long ti = (long)(J.begin + v / 3) * J.sample;
    Slot X = slot(R, 0, v), Y = slot(R, 1, v), Tm = slot(R, 2, v);
    for (int a = 0; a < n; a++) X[a] = make_double2((double)traj_mu(T, ti, x, a), 0.0);
    for (int t1 = 0; t1 < J.tmax; t1++) {
        const long t = ti + t1;
        double re = 0, im = 0;
        for (int a = 0; a < n; a++) {
            const double mu = (double)traj_mu(T, t, x, a);
            const double2 z = X[a];
            re += mu * z.x;
            im += mu * z.y;
        }
        resp[(size_t)v * J.tmax + t1] = make_double2(re, im);
        if (t1 == J.tmax - 1) break;
        if (t1 % R.K == 0)
            for (int a = 0; a < n; a++) ckpt[((size_t)v * R.nck + t1 / R.K) * n + a] = X[a];
        rk4_frame(R, t - R.f0, X, Y, Tm);
    }
}

// slots of the backward kernel: 0 l, 1 y, 2 tmp, 3 l_new, 4 w, 5 w',
// 6 .. 6+deg-1 u_q, then deg slots v_q, then the block's frame states (K),
// then the frame's sub-step inputs (m)
__global__ void k_adj_rk4_bwd(DevTraj T, Rk4Adj R, AbsJob J, const double2 *G, const double2 *ckpt, double *gshift,
                              double *gscale) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= R.nvec) return;
    const int x = v % 3, n = R.n;
    const long ti = (long)(J.begin + v / 3) * J.sample;
    Slot L = slot(R, 0, v), Y = slot(R, 1, v), Tm = slot(R, 2, v), Ln = slot(R, 3, v), W = slot(R, 4, v),
         W2 = slot(R, 5, v);
    double *gs = gshift + (size_t)v * n;
    for (int a = 0; a < n; a++) gs[a] = 0;
    double gsc = 0;
    {
        const double2 g = G[J.tmax - 1];
        for (int a = 0; a < n; a++) {
            const double mu = (double)traj_mu(T, ti + J.tmax - 1, x, a);
            L[a] = make_double2(mu * g.x, mu * g.y);
        }
    }
    const int D = R.deg, su = 6, sv = 6 + D, ss = 6 + 2 * D, si = ss + R.K;  // slot bases
    double c_pq[kPolyMaxDeg + 1];  // 1/j!
    c_pq[0] = 1.0;
    for (int j = 1; j <= D; j++) c_pq[j] = c_pq[j - 1] / j;
    for (int cb = R.nck - 1; cb >= 0; cb--) {
        const int tb0 = cb * R.K, tb1 = min(tb0 + R.K, J.tmax - 1);  // frames [tb0, tb1) propagate
        // the block's frame states from its checkpoint
        Slot S0 = slot(R, ss, v);
        for (int a = 0; a < n; a++) S0[a] = ckpt[((size_t)v * R.nck + cb) * n + a];
        for (int j = 1; j < tb1 - tb0; j++) {
            Slot Sp = slot(R, ss + j - 1, v), Sj = slot(R, ss + j, v);
            for (int a = 0; a < n; a++) Sj[a] = Sp[a];
            rk4_frame(R, ti + tb0 + j - 1 - R.f0, Sj, Y, Tm);
        }
        for (int t1 = tb1 - 1; t1 >= tb0; t1--) {
            const long fi = ti + t1 - R.f0;
            // the frame's sub-step inputs
            for (int a = 0; a < n; a++) slot(R, si, v)[a] = slot(R, ss + t1 - tb0, v)[a];
            for (int s = 1; s < R.m; s++) {
                Slot Ip = slot(R, si + s - 1, v), Is = slot(R, si + s, v);
                for (int a = 0; a < n; a++) Is[a] = Ip[a];
                const double n0 = R.renorm ? rk4_norm2(R, Is) : 1.0;
                rk4_poly(R, fi, Is, Y, Tm);
                const double sc = R.renorm ? sqrt(n0 / rk4_norm2(R, Y)) : 1.0;
                for (int a = 0; a < n; a++) {
                    const double2 z = Y[a];
                    Is[a] = make_double2(z.x * sc, z.y * sc);
                }
            }
            for (int s = R.m - 1; s >= 0; s--) {
                Slot X = slot(R, si + s, v);
                // forward powers u_q = A^q x (u_0 = x)
                for (int a = 0; a < n; a++) slot(R, su, v)[a] = X[a];
                for (int q = 1; q < D; q++) rk4_a(R, fi, slot(R, su + q - 1, v), slot(R, su + q, v), false);
                // the renormalisation: y = P(A) x
                double r = 1.0, cy = 0.0, cx = 0.0;
                if (R.renorm) {
                    rk4_poly(R, fi, X, Y, Tm);
                    const double nx = sqrt(rk4_norm2(R, X)), ny = sqrt(rk4_norm2(R, Y));
                    double c = 0;
                    for (int a = 0; a < n; a++) {
                        const double2 l = L[a], y = Y[a];
                        c += l.x * y.x + l.y * y.y;
                    }
                    r = nx / ny;
                    cy = c * nx / (ny * ny * ny);
                    cx = c / (nx * ny);
                }
                // w_0 = l_y; l_new = norm term + w_0; v_q = w_0 / (q+1)!
                for (int a = 0; a < n; a++) {
                    const double2 l = L[a], z = X[a];
                    const double2 y = R.renorm ? Y[a] : make_double2(0.0, 0.0);
                    const double2 w = make_double2(r * l.x - cy * y.x, r * l.y - cy * y.y);
                    W[a] = w;
                    Ln[a] = make_double2(cx * z.x + w.x, cx * z.y + w.y);
                    for (int q = 0; q < D; q++) slot(R, sv + q, v)[a] = make_double2(w.x * c_pq[q + 1], w.y * c_pq[q + 1]);
                }
                for (int p = 1; p <= D; p++) {  // w_p = A^+ w_(p-1)
                    rk4_a(R, fi, p % 2 ? W : W2, p % 2 ? W2 : W, true);
                    Slot Wp = p % 2 ? W2 : W;
                    for (int a = 0; a < n; a++) {
                        const double2 w = Wp[a];
                        const double2 ln = Ln[a];
                        Ln[a] = make_double2(ln.x + c_pq[p] * w.x, ln.y + c_pq[p] * w.y);
                        for (int q = 0; q + p <= D - 1; q++) {
                            const double2 vq = slot(R, sv + q, v)[a];
                            const double cf = c_pq[p + q + 1];
                            slot(R, sv + q, v)[a] = make_double2(vq.x + cf * w.x, vq.y + cf * w.y);
                        }
                    }
                }
                // parameter gradients: Im(conj(v) u) = v.x u.y - v.y u.x
                const double *jf = R.jf + fi * R.k;
                for (int q = 0; q < D; q++) {
                    Slot Vq = slot(R, sv + q, v), Uq = slot(R, su + q, v);
                    for (int a = 0; a < n; a++) {
                        const double2 vv = Vq[a], uu = Uq[a];
                        gs[a] += R.fm * (vv.x * uu.y - vv.y * uu.x);
                    }
                    for (int k = 0; k < R.k; k++) {
                        const int2 ab = R.pairs[k];
                        const double2 va = Vq[ab.x], vb = Vq[ab.y], ua = Uq[ab.x], ub = Uq[ab.y];
                        gsc += jf[k] * ((va.x * ub.y - va.y * ub.x) + (vb.x * ua.y - vb.y * ua.x));
                    }
                }
                for (int a = 0; a < n; a++) L[a] = Ln[a];
            }
            const double2 g = G[t1];
            for (int a = 0; a < n; a++) {
                const double mu = (double)traj_mu(T, ti + t1, x, a);
                const double2 l = L[a];
                L[a] = make_double2(l.x + mu * g.x, l.y + mu * g.y);
            }
        }
    }
    gscale[v] = gsc;
}

}  // namespace

int launch_adj_prep(const DevTraj &T, const AdjPlan &P, cudaStream_t s) {
    long tot = P.nf * P.n + P.nf * P.k;
    if (tot <= 0) return 0;
    k_adj_prep<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(T, P);
    return (int)cudaGetLastError();
}

int launch_adj_fwd(const DevTraj &T, const AdjPlan &P, const AbsJob &J, double2 *resp, double2 *ckpt,
                   cudaStream_t s) {
    const int nvec = 3 * J.nsamp;
    const size_t lb = sizeof(double2) * P.n;
    const int B = lanes_adj(lb);
    const size_t sm = lb * B;
    cudaError_t e = cudaFuncSetAttribute(k_adj_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e) return (int)e;
    k_adj_fwd<<<(nvec + B - 1) / B, B, sm, s>>>(T, P, J, resp, ckpt);
    return (int)cudaGetLastError();
}

int launch_adj_bwd(const DevTraj &T, const AdjPlan &P, const AbsJob &J, const double2 *G, const double2 *ckpt,
                   double *gshift_part, double *gscale_part, double *gshift, double *gscale, cudaStream_t s) {
    const int nvec = 3 * J.nsamp;
    const size_t lb = (2 * sizeof(double2) + sizeof(double)) * P.n;
    const int B = lanes_adj(lb);
    const size_t sm = lb * B;
    cudaError_t e = cudaFuncSetAttribute(k_adj_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e) return (int)e;
    k_adj_bwd<<<(nvec + B - 1) / B, B, sm, s>>>(T, P, J, G, ckpt, gshift_part, gscale_part);
    k_adj_reduce<<<(P.n + 127) / 128, 128, 0, s>>>(gshift_part, nvec, P.n, gshift);
    k_adj_reduce<<<1, 1, 0, s>>>(gscale_part, nvec, 1, gscale);
    return (int)cudaGetLastError();
}

int launch_adj_rk4(const DevTraj &T, const AdjPlan &P, const Rk4Adj &R, const AbsJob &J, const double2 *G,
                   double2 *resp, double2 *ckpt, double *gshift_part, double *gscale_part, double *gshift,
                   double *gscale, cudaStream_t s) {
    if (!G) {
        k_adj_rk4_fwd<<<(R.nvec + 63) / 64, 64, 0, s>>>(T, R, J, resp, ckpt);
        return (int)cudaGetLastError();
    }
    k_adj_rk4_bwd<<<(R.nvec + 63) / 64, 64, 0, s>>>(T, R, J, G, ckpt, gshift_part, gscale_part);
    k_adj_reduce<<<(P.n + 127) / 128, 128, 0, s>>>(gshift_part, R.nvec, P.n, gshift);
    k_adj_reduce<<<1, 1, 0, s>>>(gscale_part, R.nvec, 1, gscale);
    return (int)cudaGetLastError();
}

// Tables D, Jc, jf of the polynomial models for the step f/m (fm); with bnd,
// also the bound of ||A|| over the frames (meaningful for fm = f).
int launch_adj_poly_prep(const DevTraj &T, const AdjPlan &P, double fm, double *D, double *Jc, double *jf,
                         double *bnd, cudaStream_t s) {
    const long tot = P.nf * P.n + P.nf * P.k;
    if (tot > 0) k_adj_rk4_prep<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(T, P, fm, D, Jc, jf);
    if (bnd) k_adj_bound<<<1, 256, 0, s>>>(D, Jc, P.n, P.k, P.nf, bnd);
    return (int)cudaGetLastError();
}

// ------------------------------------------------------------------ host
#include <cmath>
#include <cstring>

#include "nise_internal.h"

namespace {

const float kCv32 = 2.99792458e-5f;
const float kTwoPi32 = (float)(2 * 3.14159265359);

struct AdjRun {
    int begin = 0, end = 0, nsamp = 0;
    long f0 = 0, nf = 0;
    std::vector<double2> S;  // response sums (tmax)
};

// FP64 forward of the model; leaves the tables and checkpoints in the
// caller's buffers for the backward sweep.
int adj_forward(nise_ctx *c, const double *shift, double scale, int K, AdjRun &R, DevBuf<double> &dshift,
                DevBuf<int2> &dpairs, DevBuf<double2> &U, DevBuf<double2> &rot, DevBuf<double> &jf,
                DevBuf<double2> &ckpt, AdjPlan &P, AbsJob &J) {
    const nise_params &p = c->p;
    if (!c->loaded) return nise_fail(c, NISE_ERR_STATE, "no trajectory loaded");
    if (!shift || !(scale == scale)) return nise_fail(c, NISE_ERR_ARG, "null shifts or invalid scale");
    const int N = c->n, tmax = p.tmax1;
    int n_samples = (p.length - p.tmax1 - 1) / p.sample + 1;
    if (n_samples <= 0) return nise_fail(c, NISE_ERR_ARG, "Insufficient data to calculate spectrum.");
    R.end = p.end == 0 ? n_samples : p.end;
    R.begin = p.begin;
    if (R.end > n_samples || R.begin < 0 || R.begin >= R.end) return nise_fail(c, NISE_ERR_ARG, "bad BeginPoint/EndPoint");
    R.nsamp = R.end - R.begin;
    R.f0 = (long)R.begin * p.sample;
    long f1 = (long)(R.end - 1) * p.sample + tmax - 1;
    int rc;
    if ((rc = nise_check_frames(c, f1))) return rc;
    R.nf = f1 - R.f0 > 0 ? f1 - R.f0 : 1;
    std::vector<int2> pairs;
    if ((rc = nise_pattern(c, R.f0, R.nf, pairs))) return rc;
    const int nvec = 3 * R.nsamp;
    memset(&P, 0, sizeof(P));
    P.n = N;
    P.k = (int)pairs.size();
    P.ts = p.ts;
    P.K = K;
    P.nck = (tmax - 1) / K + 2;
    P.f0 = R.f0;
    P.nf = R.nf;
    P.scale = scale;
    P.f = nise_f64(p, 1, p.ts);
    std::vector<double> hs(shift, shift + N);
    if ((rc = dshift.upload(c, hs)) || (rc = dpairs.upload(c, pairs.empty() ? std::vector<int2>(1) : pairs)) ||
        (rc = U.alloc(c, (size_t)R.nf * N)) || (rc = rot.alloc(c, (size_t)R.nf * (P.k ? P.k : 1))) ||
        (rc = jf.alloc(c, (size_t)R.nf * (P.k ? P.k : 1))) || (rc = ckpt.alloc(c, (size_t)nvec * P.nck * N)))
        return rc;
    P.shift = dshift.p;
    P.pairs = dpairs.p;
    P.U = U.p;
    P.rot = rot.p;
    P.jf = jf.p;
    memset(&J, 0, sizeof(J));
    J.begin = R.begin;
    J.nsamp = R.nsamp;
    J.sample = p.sample;
    J.tmax = tmax;
    J.ts = p.ts;
    DevTraj T = nise_devtraj(c);
    DevBuf<double2> resp, out;
    if ((rc = resp.alloc(c, (size_t)nvec * tmax)) || (rc = out.alloc(c, tmax))) return rc;
    c->launches = 0;
    cudaEventRecord(c->ev0, c->stream);
    cudaEventRecord(c->evk0, c->stream);
    if ((rc = nise_cuda(c, launch_adj_prep(T, P, c->stream), "adjoint tables"))) return rc;
    if ((rc = nise_cuda(c, launch_adj_fwd(T, P, J, resp.p, ckpt.p, c->stream), "adjoint forward"))) return rc;
    if ((rc = nise_cuda(c, launch_reduce_resp(resp.p, nvec, tmax, out.p, c->stream), "response reduction")))
        return rc;
    c->launches += 3;
    R.S.resize(tmax);
    cudaMemcpyAsync(R.S.data(), out.p, sizeof(double2) * tmax, cudaMemcpyDeviceToHost, c->stream);
    return nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "adjoint forward");
}

// The polynomial models (Propagation RK4, or the exact propagator): forward
// responses, tables and checkpoints left in W for the backward sweep.
struct Rk4Work {
    DevBuf<double> dshift, D, Jc, jf, bnd;
    DevBuf<int2> dpairs;
    DevBuf<double2> scr, ckpt;
    AdjPlan P;
    Rk4Adj A;
    AbsJob J;
};

int adj_rk4_forward(nise_ctx *c, const double *shift, double scale, int K, bool exact, AdjRun &R, Rk4Work &W) {
    const nise_params &p = c->p;
    if (!c->loaded) return nise_fail(c, NISE_ERR_STATE, "no trajectory loaded");
    if (!shift || !(scale == scale)) return nise_fail(c, NISE_ERR_ARG, "null shifts or invalid scale");
    const int N = c->n, tmax = p.tmax1;
    int n_samples = (p.length - p.tmax1 - 1) / p.sample + 1;
    if (n_samples <= 0) return nise_fail(c, NISE_ERR_ARG, "Insufficient data to calculate spectrum.");
    R.end = p.end == 0 ? n_samples : p.end;
    R.begin = p.begin;
    if (R.end > n_samples || R.begin < 0 || R.begin >= R.end) return nise_fail(c, NISE_ERR_ARG, "bad BeginPoint/EndPoint");
    R.nsamp = R.end - R.begin;
    R.f0 = (long)R.begin * p.sample;
    long f1 = (long)(R.end - 1) * p.sample + tmax - 1;
    int rc;
    if ((rc = nise_check_frames(c, f1))) return rc;
    R.nf = f1 - R.f0 > 0 ? f1 - R.f0 : 1;
    std::vector<int2> pairs;
    if ((rc = nise_pattern(c, R.f0, R.nf, pairs))) return rc;
    const int nvec = 3 * R.nsamp;
    AdjPlan &P = W.P;
    memset(&P, 0, sizeof(P));
    P.n = N;
    P.k = (int)pairs.size();
    P.f0 = R.f0;
    P.nf = R.nf;
    P.scale = scale;
    std::vector<double> hs(shift, shift + N);
    if ((rc = W.dshift.upload(c, hs)) || (rc = W.dpairs.upload(c, pairs.empty() ? std::vector<int2>(1) : pairs)) ||
        (rc = W.D.alloc(c, (size_t)R.nf * N)) || (rc = W.Jc.alloc(c, (size_t)R.nf * (P.k ? P.k : 1))) ||
        (rc = W.jf.alloc(c, (size_t)R.nf * (P.k ? P.k : 1))) || (rc = W.bnd.alloc(c, 1)))
        return rc;
    P.shift = W.dshift.p;
    P.pairs = W.dpairs.p;
    DevTraj T = nise_devtraj(c);
    c->launches = 0;
    cudaEventRecord(c->ev0, c->stream);
    cudaEventRecord(c->evk0, c->stream);
    // RK4: degree 4, m = Trotter sub-steps, renormalised; the exact step:
    // degree 18, m = ceil(f ||H||) so that every sub-step has ||A|| <= 1
    int m = p.ts, deg = 4;
    if (exact) {
        deg = kPolyMaxDeg;
        double hb = 0;
        if ((rc = nise_cuda(c, launch_adj_poly_prep(T, P, nise_f64(p, 1, 1), W.D.p, W.Jc.p, W.jf.p, W.bnd.p, c->stream),
                            "adjoint tables")))
            return rc;
        cudaMemcpyAsync(&hb, W.bnd.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
        if ((rc = nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "adjoint norm bound"))) return rc;
        if (!(hb >= 0 && hb < 1e6)) return nise_fail(c, NISE_ERR_ARG, "exact-propagator adjoint: |H| f = %g", hb);
        m = hb > 1 ? (int)ceil(hb) : 1;
        c->launches += 2;
    }
    P.ts = m;
    Rk4Adj &A = W.A;
    memset(&A, 0, sizeof(A));
    A.n = N;
    A.k = P.k;
    A.m = m;
    A.deg = deg;
    A.renorm = exact ? 0 : 1;
    A.K = K;
    A.nck = (tmax - 1 + K - 1) / K;
    A.nvec = nvec;
    A.f0 = R.f0;
    A.nf = R.nf;
    A.fm = nise_f64(p, 1, m);
    const size_t slots = 6 + 2 * (size_t)deg + K + m;
    if ((size_t)nvec * N * slots * sizeof(double2) > ((size_t)8 << 30))
        return nise_fail(c, NISE_ERR_NOMEM, "adjoint: %zu bytes of scratch", (size_t)nvec * N * slots * 16);
    if ((rc = W.scr.alloc(c, slots * N * nvec)) || (rc = W.ckpt.alloc(c, (size_t)nvec * (A.nck ? A.nck : 1) * N)))
        return rc;
    A.pairs = W.dpairs.p;
    A.D = W.D.p;
    A.Jc = W.Jc.p;
    A.jf = W.jf.p;
    A.scr = W.scr.p;
    if (!exact || m > 1) {
        if ((rc = nise_cuda(c, launch_adj_poly_prep(T, P, A.fm, W.D.p, W.Jc.p, W.jf.p, nullptr, c->stream),
                            "adjoint tables")))
            return rc;
        c->launches++;
    }
    AbsJob &J = W.J;
    memset(&J, 0, sizeof(J));
    J.begin = R.begin;
    J.nsamp = R.nsamp;
    J.sample = p.sample;
    J.tmax = tmax;
    J.ts = m;
    DevBuf<double2> resp, out;
    if ((rc = resp.alloc(c, (size_t)nvec * tmax)) || (rc = out.alloc(c, tmax))) return rc;
    if ((rc = nise_cuda(c, launch_adj_rk4(T, P, A, J, nullptr, resp.p, W.ckpt.p, nullptr, nullptr, nullptr, nullptr,
                                          c->stream),
                        "adjoint forward")) ||
        (rc = nise_cuda(c, launch_reduce_resp(resp.p, nvec, tmax, out.p, c->stream), "response reduction")))
        return rc;
    c->launches += 2;
    R.S.resize(tmax);
    cudaMemcpyAsync(R.S.data(), out.p, sizeof(double2) * tmax, cudaMemcpyDeviceToHost, c->stream);
    return nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "adjoint forward");
}

// Which model differentiates the context's propagation: 0 the Trotter
// model, 1 RK4, 2 the exact propagator (Sparse with Threshold 0 or above 1,
// Diagonal); -1 none (Sparse with a truncating Threshold, propagate_vec_DIA_S).
int adj_model(const nise_ctx *c) {
    switch (c->p.propagation) {
    case NISE_PROP_COUPLING: return 0;
    case NISE_PROP_RK4: return 1;
    case NISE_PROP_SPARSE:
    case NISE_PROP_DIAGONAL: return c->thres != 0 && !(c->thres > 1) ? -1 : 2;
    default: return -1;
    }
}

int adj_unsupported(nise_ctx *c) {
    return nise_fail(c, NISE_ERR_UNSUPPORTED,
                     "the absorption adjoint differentiates Propagation Coupling, RK4, Diagonal and Sparse with "
                     "Threshold 0 (not the truncated propagator)");
}

// The FP64 branch of the 1D transform input factors (1DFFT.c:170-200) for
// point j, lifetime given explicitly.
double fft_factor(const nise_params &p, int j, double lifetime) {
    double d = 1;
    if (lifetime > 0) d *= exp(-j * (double)p.deltat / (2 * lifetime));
    if (p.homogen > 0) d *= exp(-j * (double)p.deltat / (2 * (double)p.homogen));
    if (p.inhomogen > 0)
        d *= exp(-j * (double)p.deltat * j * (double)p.deltat / (2 * (double)p.inhomogen * p.inhomogen));
    if (p.window == 1) {
        double a = j * (double)kTwoPi32 / (4 * p.tmax1 - 4);
        d *= cos(a) * cos(a);
    }
    if (j == 0) d *= 0.5;
    return d;
}

// Rows of Absorption.dat in FP64 (1DFFT.c:208-228): FFT index and frequency.
void fft_rows(const nise_ctx *c, int fft, std::vector<int> &idx, std::vector<double> &w) {
    const nise_params &p = c->p;
    auto emit = [&](int i, int num) {
        double x = -((double)num / p.deltat / (double)kCv32 / fft - (double)c->shifte);
        if (!(x > p.min1 && x < p.max1)) return;
        idx.push_back(i);
        w.push_back(x);
    };
    for (int i = fft / 2; i <= fft - 1; i++) emit(i, fft - i);
    for (int i = 0; i <= fft / 2 - 1; i++) emit(i, -i);
}

// Spectrum rows of the response S in FP64 on the host (direct DFT at the
// emitted indices): spec = (Im Out, Re Out) * 2 dt c_v.
void model_spectrum(const nise_ctx *c, const std::vector<double2> &S, int samples, double lifetime,
                    const std::vector<int> &idx, std::vector<double> &sr, std::vector<double> &si) {
    const nise_params &p = c->p;
    const int tmax = p.tmax1, fft = p.fft < tmax ? tmax : p.fft;
    std::vector<double2> in(tmax);
    for (int j = 0; j < tmax; j++) {
        double d = fft_factor(p, j, lifetime);
        in[j] = make_double2(S[j].y / samples * d, S[j].x / samples * d);
    }
    const double scale = 2.0 * (double)p.deltat * (double)kCv32;
    sr.assign(idx.size(), 0);
    si.assign(idx.size(), 0);
    for (size_t r = 0; r < idx.size(); r++) {
        double ore = 0, oim = 0;
        for (int j = 0; j < tmax; j++) {
            long m = ((long)j * idx[r]) % fft;
            double ang = -2.0 * M_PI * (double)m / fft, cs = cos(ang), sn = sin(ang);
            ore += in[j].x * cs - in[j].y * sn;
            oim += in[j].x * sn + in[j].y * cs;
        }
        sr[r] = oim * scale;
        si[r] = ore * scale;
    }
}

}  // namespace

extern "C" int nise_absorption_model(nise_ctx *c, const double *site_shift, double coupling_scale, double lifetime,
                                     double *freq, double *spec_re, double *spec_im, int max_rows, int *rows) {
    if (!c || !freq || !spec_re || !spec_im || !rows) return nise_fail(c, NISE_ERR_ARG, "null argument");
    cudaSetDevice(c->p.device);
    nise_wait_all_frames(c, c->stream);  // energy records still in flight from the host
    AdjRun R;
    DevBuf<double> dshift, jf;
    DevBuf<int2> dpairs;
    DevBuf<double2> U, rot, ckpt;
    AdjPlan P;
    AbsJob J;
    Rk4Work W;
    const int model = adj_model(c);
    if (model < 0) return adj_unsupported(c);
    int rc = model ? adj_rk4_forward(c, site_shift, coupling_scale, 32, model == 2, R, W)
                   : adj_forward(c, site_shift, coupling_scale, c->p.tmax1, R, dshift, dpairs, U, rot, jf, ckpt, P, J);
    if (rc) return rc;
    cudaEventRecord(c->evk1, c->stream);
    cudaEventRecord(c->ev1, c->stream);
    cudaStreamSynchronize(c->stream);
    nise_collect_timing(c);
    const int fft = c->p.fft < c->p.tmax1 ? c->p.tmax1 : c->p.fft;
    std::vector<int> idx;
    std::vector<double> w, sr, si;
    fft_rows(c, fft, idx, w);
    model_spectrum(c, R.S, R.end, lifetime, idx, sr, si);
    int n = (int)idx.size() < max_rows ? (int)idx.size() : max_rows;
    for (int r = 0; r < n; r++) {
        freq[r] = w[r];
        spec_re[r] = sr[r];
        spec_im[r] = si[r];
    }
    *rows = n;
    return NISE_OK;
}

extern "C" int nise_backward_absorption(nise_ctx *c, const double *site_shift, double coupling_scale,
                                        double lifetime, const double *dL_dspec_re, const double *dL_dspec_im,
                                        int rows, double *g_shift, double *g_scale, double *g_lifetime) {
    if (!c || !dL_dspec_re || !dL_dspec_im || !g_shift || !g_scale || !g_lifetime)
        return nise_fail(c, NISE_ERR_ARG, "null argument");
    cudaSetDevice(c->p.device);
    nise_wait_all_frames(c, c->stream);  // energy records still in flight from the host
    const nise_params &p = c->p;
    const int fft = p.fft < p.tmax1 ? p.tmax1 : p.fft, tmax = p.tmax1, N = c->n;
    std::vector<int> idx;
    std::vector<double> w;
    fft_rows(c, fft, idx, w);
    if (rows != (int)idx.size())
        return nise_fail(c, NISE_ERR_SHAPE, "dL/dspec has %d rows, the spectrum has %d", rows, (int)idx.size());
    AdjRun R;
    DevBuf<double> dshift, jf;
    DevBuf<int2> dpairs;
    DevBuf<double2> U, rot, ckpt;
    AdjPlan P;
    AbsJob J;
    const int K = 32;  // checkpoint interval (steps)
    const int model = adj_model(c);
    if (model < 0) return adj_unsupported(c);
    const bool rk4 = model > 0;  // a polynomial model
    Rk4Work W;
    int rc = rk4 ? adj_rk4_forward(c, site_shift, coupling_scale, K, model == 2, R, W)
                 : adj_forward(c, site_shift, coupling_scale, K, R, dshift, dpairs, U, rot, jf, ckpt, P, J);
    if (rc) return rc;
    // adjoint of the transform: dL/dOut_k = (dL/dspec_im + i dL/dspec_re) * 2 dt c_v,
    // dL/din_j = sum_k exp(+2 pi i jk/fft) dL/dOut_k, then through the input factors
    const double scale = 2.0 * (double)p.deltat * (double)kCv32;
    std::vector<double2> G(tmax);
    double gl = 0;
    for (int j = 0; j < tmax; j++) {
        double gr = 0, gi = 0;
        for (size_t r = 0; r < idx.size(); r++) {
            long m = ((long)j * idx[r]) % fft;
            double ang = 2.0 * M_PI * (double)m / fft, cs = cos(ang), sn = sin(ang);
            double orr = dL_dspec_im[r] * scale, oii = dL_dspec_re[r] * scale;
            gr += cs * orr - sn * oii;
            gi += sn * orr + cs * oii;
        }
        double d = fft_factor(p, j, lifetime);
        // in_j = d * (Im S_j + i Re S_j) / samples
        G[j] = make_double2(gi * d / R.end, gr * d / R.end);
        if (lifetime > 0) {
            double inr = R.S[j].y / R.end * d, ini = R.S[j].x / R.end * d;
            gl += (gr * inr + gi * ini) * (j * (double)p.deltat / (2 * lifetime * lifetime));
        }
    }
    DevBuf<double2> dG;
    DevBuf<double> gsp, gcp, gs, gc;
    const int nvec = 3 * R.nsamp;
    if ((rc = dG.upload(c, G)) || (rc = gsp.alloc(c, (size_t)nvec * N)) || (rc = gcp.alloc(c, nvec)) ||
        (rc = gs.alloc(c, N)) || (rc = gc.alloc(c, 1)))
        return rc;
    DevTraj T = nise_devtraj(c);
    if (rk4)
        rc = nise_cuda(c, launch_adj_rk4(T, W.P, W.A, W.J, dG.p, nullptr, W.ckpt.p, gsp.p, gcp.p, gs.p, gc.p, c->stream),
                       "polynomial adjoint backward");
    else
        rc = nise_cuda(c, launch_adj_bwd(T, P, J, dG.p, ckpt.p, gsp.p, gcp.p, gs.p, gc.p, c->stream),
                       "adjoint backward");
    if (rc) return rc;
    c->launches += 3;
    cudaEventRecord(c->evk1, c->stream);
    std::vector<double> hs(N);
    double hc = 0;
    cudaMemcpyAsync(hs.data(), gs.p, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(&hc, gc.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    cudaEventRecord(c->ev1, c->stream);
    if ((rc = nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "adjoint backward"))) return rc;
    nise_collect_timing(c);
    for (int a = 0; a < N; a++) g_shift[a] = hs[a];
    *g_scale = hc;
    *g_lifetime = gl;
    return NISE_OK;
}
