// Coefficient tables of the singles propagation schemes over the frames of
// one job, shared by the 2D and linear-technique drivers.
//
// The reference rebuilds the propagator of a frame for every vector it
// propagates through that frame (propagate_vector, propagate.c:20-39).  Here
// each frame's coefficients are computed once per job and read by every
// vector: Trotter half phases and rotation coefficients (k_prep_trotter), the
// RK4 Hamiltonian entries (k_prep_rk4), or, for Sparse/Diagonal, the one-step
// propagator U = V exp(-i e f) V^T from the batched eigensolver (eigen.cu,
// diag.cu).  With doubles, the eigen route also builds the truncated sub-step
// propagator of time_evolution_mat (propagate.c:1241-1299).
#include <algorithm>
#include <vector>

#include "eigen.h"
#include "engine.h"
#include "nise_internal.h"

int nise_singles_tables(nise_ctx *c, const DevTraj &T, long fmin, long nf, int singleshift, bool doubles_u,
                        SinglesTab &S, SinglesBufs &B) {
    const nise_params &p = c->p;
    const int N = c->n, prec = p.precision;
    const size_t rsz = prec == NISE_FP32 ? sizeof(float) : sizeof(double), r2 = 2 * rsz;
    int rc;
    std::vector<int2> pairs;
    if ((rc = nise_pattern(c, fmin, nf, pairs))) return rc;
    const int K = (int)pairs.size();
    // segments of one first site and one warp (b >> 5) of second sites, for
    // the doubles kernel that shares a vector between two warps
    std::vector<int4> segs;
    for (int k = 0; k < K;) {
        const int a = pairs[k].x, w = pairs[k].y >> 5, k0 = k;
        while (k < K && pairs[k].x == a && (pairs[k].y >> 5) == w) k++;
        segs.push_back(make_int4(a, k0, k, w));
    }
    if (segs.empty()) segs.push_back(make_int4(0, 0, 0, 0));
    pairs.push_back(make_int2(0, 0));  // one record past the last: read ahead without a bound check
    if ((rc = B.pairs.upload(c, pairs)) || (rc = B.segs.upload(c, segs))) return rc;
    S.n = N;
    S.ts = p.ts;
    S.prop = p.propagation;
    S.f0 = fmin;
    S.pairs = B.pairs.p;
    S.K = K;
    S.segs = B.segs.p;
    S.nsegs = K ? (int)segs.size() : 0;
    S.U = S.rot = S.rkval = S.Ud = nullptr;
    S.ent = nullptr;
    S.Kr = 0;
    S.rot_static = p.hamiltonian == NISE_HAM_COUPLING;
    B.Us = nullptr;
    if (p.propagation == NISE_PROP_COUPLING) {
        TrotterPlan P;
        P.n = N; P.k = S.K; P.pairs = B.pairs.p; P.f0 = fmin; P.nf = nf;
        P.rot_static = S.rot_static;
        P.singleshift = singleshift;
        if ((rc = B.U.alloc(c, r2 * (size_t)nf * N))) return rc;
        if ((rc = B.rot.alloc(c, r2 * (size_t)(P.rot_static ? 1 : nf) * (P.k ? P.k : 1)))) return rc;
        P.U = B.U.p;
        P.rot = B.rot.p;
        if ((rc = nise_cuda(c, launch_prep_trotter(prec, T, P, nise_f64(p, 1, p.ts), nise_f32(p, 1, p.ts), c->stream),
                            "Trotter prep")))
            return rc;
        c->launches += 1 + P.rot_static;
        S.U = B.U.p;
        S.rot = B.rot.p;
    } else if (p.propagation == NISE_PROP_SPARSE || p.propagation == NISE_PROP_DIAGONAL) {
        // propagate_vector's Sparse scheme (DIA, or DIA_S when 0 < Threshold
        // <= 1) and time_evolution_mat's truncated sub-step propagator for the
        // doubles (Threshold always applied); Diagonal is the untruncated
        // exact propagator.
        if (N > 1024)
            return nise_fail(c, NISE_ERR_UNSUPPORTED, "Propagation Sparse/Diagonal on per-frame tables is limited to "
                             "1024 sites");
        const float thr = p.propagation == NISE_PROP_DIAGONAL ? 0.0f : c->thres;
        const bool trunc_singles = thr != 0 && !(thr > 1);
        const long FC = std::max(1L, std::min(nf, (long)(((size_t)512 << 20) / (sizeof(double) * (size_t)N * N))));
        std::vector<long> frs(nf);
        for (long t = 0; t < nf; t++) frs[t] = fmin + t;
        DevBuf<long> dfr;
        DevBuf<double> V, w, Aws;
        DevBuf<int> st;
        if ((rc = dfr.upload(c, frs)) || (rc = V.alloc(c, (size_t)FC * N * N)) || (rc = w.alloc(c, (size_t)FC * N)) ||
            (rc = Aws.alloc(c, eig_any_ws_doubles(N, FC))) || (rc = st.alloc(c, 1)) ||
            (rc = B.U.alloc(c, r2 * (size_t)nf * N * N)))
            return rc;
        cudaMemsetAsync(st.p, 0, sizeof(int), c->stream);
        if (doubles_u && (rc = B.rot.alloc(c, r2 * (size_t)nf * N * N))) return rc;
        EigJob EJ;
        EJ.T = T; EJ.n = N; EJ.singleshift = singleshift;
        const int pr = prec == NISE_FP32 ? 0 : 1;
        const double ffull = prec == NISE_FP32 ? (double)nise_f32(p, 1, 1) : nise_f64(p, 1, 1);
        const double fsub = prec == NISE_FP32 ? (double)nise_f32(p, 1, p.ts) : nise_f64(p, 1, p.ts);
        for (long q = 0; q < nf; q += FC) {
            long m = std::min(FC, nf - q);
            if ((rc = nise_cuda(c, launch_eig_any(EJ, dfr.p + q, m, V.p, w.p, Aws.p, st.p, c->stream), "eigensolver")))
                return rc;
            if ((rc = nise_cuda(c, launch_build_u_any(pr, V.p, w.p, m, N, ffull, thr, trunc_singles,
                                                  B.U.p + r2 * (size_t)q * N * N, c->stream), "propagator build")))
                return rc;
            c->launches += 2;
            if (doubles_u) {
                if ((rc = nise_cuda(c, launch_build_u_any(pr, V.p, w.p, m, N, fsub, thr, 1, B.rot.p + r2 * (size_t)q * N * N,
                                                      c->stream), "doubles propagator build")))
                    return rc;
                c->launches++;
            }
        }
        int hst = 0;
        if ((rc = nise_cuda(c, (int)cudaMemcpyAsync(&hst, st.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
                            "eigensolver status")) ||
            (rc = nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "eigensolver")))
            return rc;
        if (hst) return nise_fail(c, NISE_ERR_DEVICE, "the eigensolver did not converge on a frame");
        S.Ud = B.U.p;
        if (doubles_u) B.Us = B.rot.p;
    } else {
        std::vector<int2> ent;
        size_t q = 0;
        for (int a = 0; a < N; a++) {
            ent.push_back(make_int2(a, a));
            while (q < (size_t)K && pairs[q].x == a) ent.push_back(pairs[q++]);
        }
        if ((rc = B.ent.upload(c, ent))) return rc;
        Rk4Plan P;
        P.n = N; P.k = (int)ent.size(); P.entries = B.ent.p; P.f0 = fmin; P.nf = nf; P.singleshift = singleshift;
        if ((rc = B.rkval.alloc(c, rsz * (size_t)nf * P.k))) return rc;
        P.val = B.rkval.p;
        if ((rc = nise_cuda(c, launch_prep_rk4(prec, T, P, nise_f64(p, 1, p.ts), nise_f32(p, 1, p.ts), c->stream),
                            "RK4 prep")))
            return rc;
        c->launches++;
        S.ent = B.ent.p;
        S.Kr = P.k;
        S.rkval = B.rkval.p;
    }
    return NISE_OK;
}
