// Linear absorption jobs (absorption.c:18-202): planning, enqueueing and
// collection of one context's job, the launch autotuner, and the batch API
// that runs many contexts' jobs as one CUDA graph.
//
// A job is split so that everything that allocates or synchronises happens
// in plan() (validation, coupling pattern, CSR/ELL tables, rotation levels,
// device buffers, autotuning) and enqueue() only launches kernels on a given
// stream.  nise_absorption runs plan/enqueue/collect on the context's stream;
// nise_batch_create plans every job, then captures all enqueues, each on its
// own forked stream, into one graph that nise_batch_run launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "eigen.h"
#include "engine.h"
#include "nise_b200.h"
#include "nise_internal.h"

namespace {

enum Scheme { SCHEME_TROTTER, SCHEME_RK4, SCHEME_TAYLOR, SCHEME_EIGEN };

// Launch configurations the autotuner chooses from.
//   Trotter: 0 = thread per vector (k_abs_trotter), T = 64/128/256 =
//            level-scheduled rotations with T threads per start point
//            (k_abs_trotter_lv); 32 / 33 = warp per vector
//            (k_abs_trotter_wv) with the rotation table in shared / global
//            memory; all bitwise identical.
//   Taylor:  3 = k_abs_taylor2 with 4 vectors per CTA, 8 = the sliced-ELL
//            kernel with 8 (k_abs_taylor2 with 8 where it does not fit),
//            -8 = k_abs_taylor2 with 8, 10 = the FP32 sliced-ELL kernel with
//            the Chebyshev expansion of the step (k_abs_cheb3), 12 = the FP32
//            sliced-ELL kernel with 4 vectors per CTA (k_abs_taylor4).
typedef std::tuple<int, int, int, int, int> TuneKey;  // scheme, precision, sites, couplings, static
std::map<TuneKey, int> g_tuned;
std::mutex g_tune_mu;

// Trotter: the warp-per-vector kernel where the levels are wide (lattices:
// ~20 rotations per level) or the job has too few vectors to fill warps of
// threads (a warp per vector then has the shorter critical path); thread per
// vector for chains (one rotation per level) with many vectors.
int default_config(int scheme, int N, bool plain, bool cheb, int K, int nchk, int nvec, bool has4, bool rv,
                   bool rot_static) {
    if (scheme == SCHEME_TROTTER) {
        // a warp per two vectors once there are 8 or more vectors per SM (static
        // couplings; 1024-site lattice, 1185 vectors: 39.3 against 43.9 ms),
        // else a warp per vector (C4's 585-vector jobs: 18.6 against 25.5 ms at
        // 1875 sites)
        if (K > 0 && rot_static && nvec >= 8 * sm_count()) return 34;
        if (K > 0 && (K >= 4 * nchk || nvec < 1024)) return 32;
        return N >= 96 ? 128 : 0;
    }
    // one start point per launch (3 vectors): the sliced-ELL kernel, which
    // gives every vector its own CTA when there are fewer vectors than SMs
    if (plain) return 8;
    (void)cheb;           // the Chebyshev kernel is a tuned alternative: fewer terms, more work per term
    // less than one wave of 8-vector CTAs: 4 vectors per CTA reach twice the
    // SMs.  C4 jobs (585 vectors): the FP32 sliced-ELL kernel with 4 vectors
    // up to 1024 sites (295 sites 1.96 against 2.31 ms for k_abs_taylor2 and
    // 2.32 for the default), k_abs_taylor2 with 4 above (1440 sites 12.1
    // against 15.8 and 25.0 ms)
    if (nvec < 8 * sm_count()) return has4 && N <= 1024 ? 12 : 3;
    // whole waves of 8-vector CTAs: the row-owner kernel with the Chebyshev
    // expansion (FP32 lattices up to 1024 sites; on the 1024-site lattice,
    // 100 000 frames: 52.0 ms against 55.8 with the Taylor series and 69.7 on
    // the 8-vector sliced-ELL kernel)
    if (rv && cheb) return 15;
    return 8;
}

// Rotation levels of the lexicographic coupling list: perm holds the
// rotation indices ordered by (level, index), lvptr the level boundaries.
// Two rotations that share a site keep their order (the later one has the
// higher level), so applying the rotations in perm order performs the same
// floating-point operations on every site as the lexicographic order of
// propagate.c:876-888.
void rotation_levels(const std::vector<int2> &pairs, int n, std::vector<int> &perm, std::vector<int> &lvptr) {
    std::vector<int> last(n, 0), lv(pairs.size());
    int nlev = 0;
    for (size_t k = 0; k < pairs.size(); k++) {
        int l = std::max(last[pairs[k].x], last[pairs[k].y]) + 1;
        last[pairs[k].x] = last[pairs[k].y] = l;
        lv[k] = l - 1;
        nlev = std::max(nlev, l);
    }
    lvptr.assign(nlev + 1, 0);
    for (int l : lv) lvptr[l + 1]++;
    for (int l = 0; l < nlev; l++) lvptr[l + 1] += lvptr[l];
    perm.assign(pairs.size(), 0);
    std::vector<int> fill(lvptr.begin(), lvptr.end() - 1);
    for (size_t k = 0; k < pairs.size(); k++) perm[fill[lv[k]]++] = (int)k;
}

// The levels split into chunks of at most 32 rotations (one warp step of
// the warp-per-vector kernel each): chk holds the chunk boundaries.
void rotation_chunks(const std::vector<int> &lvptr, std::vector<int> &chk) {
    chk.assign(1, 0);
    for (size_t l = 0; l + 1 < lvptr.size(); l++)
        for (int q = lvptr[l]; q < lvptr[l + 1]; q += 32) chk.push_back(std::min(q + 32, lvptr[l + 1]));
}

// Bank order within each chunk.  The warp kernels give lane l of a chunk the
// chunk's l-th rotation and load its two sites with one shared-memory load
// each (idle lanes: the spare site n + ((start + l - K) & 31)).  A load is
// served in groups of lanes (a site of 8 bytes: half-warps, the site's bank
// pair given by site mod 16; of 16 bytes, the two-vector kernel: quarter-warps,
// site mod 8), and sites of one group with the same residue conflict.  The
// rotations of a chunk are disjoint and the 2x2 rotation is symmetric in its
// two sites, so any order within the chunk and either site first give the same
// float operations on every site; a local search (fixed seed) picks the order
// and the orientation with the fewest conflicting wavefronts over both
// layouts.  flip[q] = 1: rotation perm[q] is applied as (b, a).
void bank_order(const std::vector<int2> &pairs, int n, const std::vector<int> &chk, std::vector<int> &perm,
                std::vector<char> &flip) {
    const int K = (int)pairs.size();
    flip.assign(perm.size(), 0);
    uint32_t st = 0x9e3779b9u;
    auto rnd = [&]() {
        st ^= st << 13;
        st ^= st >> 17;
        st ^= st << 5;
        return st;
    };
    for (size_t c = 0; c + 1 < chk.size(); c++) {
        const int c0 = chk[c], m = chk[c + 1] - c0;
        if (m < 2) continue;
        int sa[32], sb[32];
        auto load = [&]() {
            for (int l = 0; l < 32; l++) {
                if (l < m) {
                    const int2 p = pairs[perm[c0 + l]];
                    sa[l] = flip[c0 + l] ? p.y : p.x;
                    sb[l] = flip[c0 + l] ? p.x : p.y;
                } else {
                    sa[l] = sb[l] = n + ((c0 + l - K) & 31);
                }
            }
        };
        auto cost = [&]() {
            int tot = 0;
            for (int lay = 0; lay < 2; lay++) {
                const int w = lay ? 8 : 16, g = lay ? 8 : 16;
                for (int l0 = 0; l0 < 32; l0 += w)
                    for (const int *s : {sa, sb}) {
                        int cnt[16] = {0}, mx = 0;
                        for (int l = l0; l < l0 + w; l++) mx = std::max(mx, ++cnt[s[l] % g]);
                        tot += mx;
                    }
            }
            return tot;
        };
        // greedy start: lane by lane the rotation and orientation whose sites
        // collide least with the sites already in the lane's groups (the idle
        // lanes' spare sites included)
        {
            int ca8[2][16] = {{0}}, cb8[2][16] = {{0}}, ca16[4][8] = {{0}}, cb16[4][8] = {{0}};
            for (int l = m; l < 32; l++) {
                const int s = n + ((c0 + l - K) & 31);
                ca8[l >> 4][s % 16]++;
                cb8[l >> 4][s % 16]++;
                ca16[l >> 3][s % 8]++;
                cb16[l >> 3][s % 8]++;
            }
            std::vector<int> rest(perm.begin() + c0, perm.begin() + c0 + m);
            for (int l = 0; l < m; l++) {
                int bi = 0, bo = 0, bc = 1 << 30;
                for (int i = 0; i < (int)rest.size(); i++)
                    for (int o = 0; o < 2; o++) {
                        const int2 p = pairs[rest[i]];
                        const int a = o ? p.y : p.x, b = o ? p.x : p.y;
                        const int cc = ca8[l >> 4][a % 16] + cb8[l >> 4][b % 16] + ca16[l >> 3][a % 8] +
                                       cb16[l >> 3][b % 8];
                        if (cc < bc) bc = cc, bi = i, bo = o;
                    }
                const int2 p = pairs[rest[bi]];
                const int a = bo ? p.y : p.x, b = bo ? p.x : p.y;
                ca8[l >> 4][a % 16]++;
                cb8[l >> 4][b % 16]++;
                ca16[l >> 3][a % 8]++;
                cb16[l >> 3][b % 8]++;
                perm[c0 + l] = rest[bi];
                flip[c0 + l] = (char)bo;
                rest.erase(rest.begin() + bi);
            }
        }
        load();
        int best = cost();
        for (int it = 0; it < 24 * m; it++) {
            const int i = (int)(rnd() % m);
            if (rnd() % 10 < 3) {
                flip[c0 + i] ^= 1;
                load();
                const int t = cost();
                if (t <= best) best = t;
                else flip[c0 + i] ^= 1;
            } else {
                const int j = (int)(rnd() % m);
                if (i == j) continue;
                std::swap(perm[c0 + i], perm[c0 + j]);
                std::swap(flip[c0 + i], flip[c0 + j]);
                load();
                const int t = cost();
                if (t <= best) best = t;
                else {
                    std::swap(perm[c0 + i], perm[c0 + j]);
                    std::swap(flip[c0 + i], flip[c0 + j]);
                }
            }
        }
    }
}

}  // namespace

extern "C" int nise_rotation_schedule(const int *ab, int k, int n, int *perm, int *lvptr, int *nlev, int *chkptr,
                                      int *nchk, int *flip) {
    if (k < 0 || n < 1 || (k && (!ab || !perm)) || !lvptr || !nlev || !chkptr || !nchk) {
        nise_set_global_error("bad rotation schedule arguments");
        return NISE_ERR_ARG;
    }
    std::vector<int2> pairs(k);
    for (int q = 0; q < k; q++) {
        pairs[q] = make_int2(ab[2 * q], ab[2 * q + 1]);
        if (pairs[q].x < 0 || pairs[q].x >= n || pairs[q].y < 0 || pairs[q].y >= n || pairs[q].x == pairs[q].y) {
            nise_set_global_error("rotation pair out of range");
            return NISE_ERR_ARG;
        }
    }
    std::vector<int> hperm, hlv, hchk;
    rotation_levels(pairs, n, hperm, hlv);
    rotation_chunks(hlv, hchk);
    std::vector<char> hflip;
    bank_order(pairs, n, hchk, hperm, hflip);
    std::copy(hperm.begin(), hperm.end(), perm);
    if (flip) std::copy(hflip.begin(), hflip.end(), flip);
    std::copy(hlv.begin(), hlv.end(), lvptr);
    std::copy(hchk.begin(), hchk.end(), chkptr);
    *nlev = (int)hlv.size() - 1;
    *nchk = (int)hchk.size() - 1;
    return NISE_OK;
}

struct AbsRun {
    nise_ctx *c = nullptr;
    int N = 0, tmax = 0, prec = 0, begin = 0, end = 0, nsamp = 0, nvec = 0;
    long f0 = 0, nf = 0;
    bool plain = false;
    int scheme = SCHEME_TROTTER;
    int config = 0;
    DevTraj T;
    AbsJob J;
    DevBuf<double2> resp, out;
    // Trotter
    DevBuf<int2> dpairs;
    DevBuf<char> U, rot;
    DevBuf<int> lvptr, lvchk;  // level bounds; the same split into chunks of at most 32
    int nlev = 0, nchk = 0;
    TrotterPlan TP;
    // RK4
    DevBuf<int2> dent;
    DevBuf<char> rkval;
    Rk4Plan RP;
    // Taylor
    DevBuf<int> drp, dcol, dorder, dsptr, dcorder, drows, dsptr4, drows4;
    DevBuf<int2> dell4;
    int ell4_nslices = 0, ell4_nent = 0;
    DevBuf<float4> dtri8;  // row-owner layout (k_abs_taylor_rv)
    DevBuf<int> dtptr8, drows8, dwsl8[2], derr;
    int ell8_nslices = 0, ell8_ntg = 0, ell8_it[2] = {0, 0};
    DevBuf<char> dval, dell;
    DevBuf<float> dinvr, dcen;
    DevBuf<float2> dcoef;
    TaylorPlan XP;
    double rowabs = 0;
    bool cheb = false;  // Chebyshev tables allocated (FP32, sliced ELL fits)
    // eigen route
    DevBuf<char> Ue;
    DevBuf<long> efr;
    DevBuf<double> eV, ew, eA;  // eigenvectors, eigenvalues, QR workspace (above the Jacobi's size)
    DevBuf<int> estatus;
    DevBuf<float> tcX;           // state columns of the tensor-core apply
    bool use_tc = false;
    bool stream_u = false;  // propagators built and applied chunk by chunk (tensor cores, batched)
    long FC = 1;
    bool truncated = false;
    double fe = 0;
    // work accounting
    std::vector<long> cross;
    long vec_steps = 0;
    double alg_bytes = 0;  // every frame read once (diagonal or full record) and the dipoles

    int plan(nise_ctx *ctx, bool autotune);
    int enqueue(cudaStream_t s, bool events);
    // The static-coupling series kernels wave by wave, each wave after the
    // energy chunk holding its last frame (and the series tables of the
    // frames up to there): the copy from the host overlaps the propagation.
    int enqueue_waves(cudaStream_t s);
    bool waves_apply() const;
    // the side stream of enqueue_waves' 1-vector CTAs, created on first use
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    ~AbsRun() {
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (side) cudaStreamDestroy(side);
    }
    // A plan reused by a later call: the trajectory pointers may have moved
    // and the error flags start clear.
    void refresh() {
        T = nise_devtraj(c);
        if (derr.p) cudaMemsetAsync(derr.p, 0, sizeof(int), c->stream);
        if (estatus.p) cudaMemsetAsync(estatus.p, 0, sizeof(int), c->stream);
    }
    // after the job: a kernel whose bounded wait for a staged frame gave up
    // leaves its flag set (NISE_ERR_TIMEOUT)
    int check_err() {
        int h = 0;
        if (derr.p) {
            if (cudaMemcpy(&h, derr.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
                return nise_fail(c, NISE_ERR_DEVICE, "error flag read failed");
            if (h) return nise_fail(c, NISE_ERR_TIMEOUT, "a bounded wait for a staged frame gave up");
        }
        if (estatus.p) {
            if (cudaMemcpy(&h, estatus.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
                return nise_fail(c, NISE_ERR_DEVICE, "eigensolver status read failed");
            if (h) return nise_fail(c, NISE_ERR_DEVICE, "the eigensolver did not converge on a frame");
        }
        return NISE_OK;
    }
    int run_main(cudaStream_t s, int cfg, double2 *dst);
    double flops() const;
    int tune();
};

int AbsRun::plan(nise_ctx *ctx, bool autotune) {
    c = ctx;
    if (!c->loaded) return nise_fail(c, NISE_ERR_STATE, "no trajectory loaded");
    const nise_params &p = c->p;
    N = c->n;
    tmax = p.tmax1;
    prec = p.precision;
    // determine_samples (NISE_subs.c:197-221)
    int n_samples = (p.length - p.tmax1 - 1) / p.sample + 1;
    if (n_samples <= 0) return nise_fail(c, NISE_ERR_ARG, "Insufficient data to calculate spectrum.");
    end = p.end == 0 ? n_samples : p.end;
    if (end > n_samples) return nise_fail(c, NISE_ERR_ARG, "Endpoint larger than number of samples was specified.");
    begin = p.begin;
    if (begin < 0 || begin >= end) return nise_fail(c, NISE_ERR_ARG, "BeginPoint must be below EndPoint");
    nsamp = end - begin;
    nvec = 3 * nsamp;
    f0 = (long)begin * p.sample;
    long f1 = (long)(end - 1) * p.sample + tmax - 1;  // last frame read
    int rc;
    if ((rc = nise_check_frames(c, f1))) return rc;
    nf = f1 - f0;  // frames propagated through: [f0, f1)
    if (nf < 1) nf = 1;
    T = nise_devtraj(c);
    memset(&J, 0, sizeof(J));
    J.begin = begin;
    J.nsamp = nsamp;
    J.sample = p.sample;
    J.tmax = tmax;
    J.ts = p.ts;
    J.f = nise_f64(p, 1, 1);
    J.f32_sub = nise_f32(p, 1, p.ts);
    J.f64_sub = nise_f64(p, 1, p.ts);
    J.f32_full = nise_f32(p, 1, 1);
    plain = p.launch_mode == NISE_PLAIN;
    if ((rc = resp.alloc(c, (size_t)nvec * tmax)) || (rc = out.alloc(c, tmax))) return rc;
    cross.assign(nf, 0);
    for (int s = 0; s < nsamp; s++) {
        long a = (long)(begin + s) * p.sample - f0;
        for (int t = 0; t < tmax - 1; t++) cross[a + t] += 3;
    }
    vec_steps = 3L * nsamp * (tmax - 1);
    alg_bytes = (double)nf * 4 * (p.hamiltonian == NISE_HAM_COUPLING ? N : c->nn2) +
                    (double)(p.hamiltonian == NISE_HAM_COUPLING ? 3 * N : (nf + 1) * 3L * N) * 4;
    const size_t rsz = prec == NISE_FP32 ? sizeof(float) : sizeof(double), r2 = 2 * rsz;

    if (p.propagation == NISE_PROP_COUPLING) {
        scheme = SCHEME_TROTTER;
        std::vector<int2> pairs;
        if ((rc = nise_pattern(c, f0, nf, pairs))) return rc;
        memset(&TP, 0, sizeof(TP));
        TP.n = N;
        TP.k = (int)pairs.size();
        TP.f0 = f0;
        TP.nf = nf;
        TP.rot_static = p.hamiltonian == NISE_HAM_COUPLING;
        TP.singleshift = c->nshift > 0;
        // the pairs (and so the rotation tables) in level order
        std::vector<int> hperm, hlv;
        rotation_levels(pairs, N, hperm, hlv);
        nlev = (int)hlv.size() - 1;
        std::vector<int> hchk;
        rotation_chunks(hlv, hchk);
        nchk = (int)hchk.size() - 1;
        std::vector<char> hflip;
        bank_order(pairs, N, hchk, hperm, hflip);
        std::vector<int2> lpairs(pairs.size());
        for (size_t q = 0; q < pairs.size(); q++) {
            const int2 ab = pairs[hperm[q]];
            lpairs[q] = hflip[q] ? make_int2(ab.y, ab.x) : ab;
        }
        if ((rc = dpairs.upload(c, lpairs.empty() ? std::vector<int2>(1) : lpairs)) ||
            (rc = U.alloc(c, r2 * (size_t)nf * N)) ||
            (rc = rot.alloc(c, r2 * (size_t)(TP.rot_static ? 1 : nf) * (TP.k ? TP.k : 1))) ||
            (rc = lvptr.upload(c, hlv)))
            return rc;
        if ((rc = lvchk.upload(c, hchk))) return rc;
        TP.pairs = dpairs.p;
        TP.U = U.p;
        TP.rot = rot.p;
    } else if (p.propagation == NISE_PROP_RK4) {
        scheme = SCHEME_RK4;
        std::vector<int2> pairs, ent;
        if ((rc = nise_pattern(c, f0, nf, pairs))) return rc;
        size_t q = 0;
        for (int a = 0; a < N; a++) {  // propagate.c:294-305 order: (a,a) then (a,b>a)
            ent.push_back(make_int2(a, a));
            while (q < pairs.size() && pairs[q].x == a) ent.push_back(pairs[q++]);
        }
        memset(&RP, 0, sizeof(RP));
        RP.n = N;
        RP.k = (int)ent.size();
        RP.f0 = f0;
        RP.nf = nf;
        RP.singleshift = c->nshift > 0;
        if ((rc = dent.upload(c, ent)) || (rc = rkval.alloc(c, rsz * (size_t)nf * RP.k))) return rc;
        RP.entries = dent.p;
        RP.val = rkval.p;
    } else {
        // Sparse / Diagonal: the exact propagator exp(-i H dt) (propagate_vec_DIA,
        // propagate.c:60-125).  Threshold > 0 keeps only large elements of U
        // (propagate_vec_DIA_S, propagate.c:185-258) and needs the explicit
        // eigen propagator, as do per-frame couplings (HamiltonianType Full).
        // Otherwise the static couplings go through the sparse Taylor series,
        // for Sparse and Diagonal alike (the same exact propagator; on the
        // 103-site lattice of the mixed batch 0.9 ms instead of 79 ms);
        // kernel_config 2 asks for the eigen route anyway.
        truncated = c->thres != 0 && !(c->thres > 1);
        const bool eigen_route = truncated || p.hamiltonian != NISE_HAM_COUPLING || p.kernel_config == 2;
        if (eigen_route) {
            scheme = SCHEME_EIGEN;
            // FP32 above the Jacobi's size: U applied on the tensor cores
            // (kernel_config 16: the per-start-point kernel, 17: the tensor
            // cores at any size).  Batched, the tensor-core apply runs frame
            // by frame, so the propagators are built and applied in chunks
            // and only a chunk of them is held: up to 2048 sites (the
            // eigensolver's shared memory), else every frame's U is held.
            AbsJob Jt = J;
            if (plain) Jt.nsamp = 1;
            use_tc = prec == NISE_FP32 && tc_dia_fits(Jt, N) &&
                     (p.kernel_config == 17 || (N > NISE_EIG_MAX_N && p.kernel_config != 16));
            stream_u = use_tc && !plain;
            if (N > (stream_u ? 2048 : 1024))
                return nise_fail(c, NISE_ERR_UNSUPPORTED,
                                 "the eigen route (Threshold > 0, per-frame couplings, kernel_config 2) is limited to "
                                 "%d sites here (2048 with the tensor-core apply of a batched FP32 job)",
                                 stream_u ? 2048 : 1024);
            // frames per eigensolver launch (one CTA per frame): a wave of
            // the 148 SMs, or as many as 1 GB of eigenvectors, QR workspace
            // (and streamed U) holds, at most 16 GB
            const size_t per_frame = sizeof(double) * (size_t)N * N * (N > NISE_EIG_MAX_N ? 2 : 1) +
                                     (stream_u ? r2 * (size_t)N * N : 0);
            FC = std::max(148L, (long)(((size_t)1 << 30) / per_frame));
            FC = std::max(1L, std::min(std::min(nf, FC), (long)(((size_t)16 << 30) / per_frame)));
            const size_t ubytes = r2 * (size_t)(stream_u ? FC : nf) * N * N;
            if (ubytes > ((size_t)64 << 30))
                return nise_fail(c, NISE_ERR_NOMEM,
                                 "eigen route: %ld frames of %d sites need more than 64 GB of propagators", nf, N);
            std::vector<long> frames(nf);
            for (long t = 0; t < nf; t++) frames[t] = f0 + t;
            if ((rc = Ue.alloc(c, ubytes)) || (rc = efr.upload(c, frames)) || (rc = eV.alloc(c, (size_t)FC * N * N)) ||
                (rc = ew.alloc(c, (size_t)FC * N)) || (rc = eA.alloc(c, eig_any_ws_doubles(N, FC))) ||
                (rc = estatus.alloc(c, 1)))
                return rc;
            cudaMemsetAsync(estatus.p, 0, sizeof(int), c->stream);
            // propagate_vec_DIA: f = deltat*icm2ifs*twoPi*sign in float, one full step
            fe = prec == NISE_FP32 ? (double)J.f32_full : J.f;
            if (use_tc && ((rc = tcX.alloc(c, (size_t)4 * tc_dia_columns(Jt) * N)) || (rc = derr.alloc(c, 1))))
                return rc;
            if (use_tc) cudaMemsetAsync(derr.p, 0, sizeof(int), c->stream);
        } else {
            scheme = SCHEME_TAYLOR;
            // CSR of the static couplings (read cut applied, |J| >= cut kept)
            std::vector<int> rp(N + 1, 0), col;
            std::vector<double> vd;
            for (int i = 0; i < N; i++) {
                double rs = 0;
                for (int j = 0; j < N; j++) {
                    if (j == i) continue;
                    int a = i < j ? i : j, b = i < j ? j : i;
                    float v = c->h_hc[b + (long)a * ((N << 1) - a - 1) / 2];
                    if (v != 0.0f) {
                        col.push_back(j);
                        vd.push_back(v);
                        rs += fabs(v);
                    }
                }
                rp[i + 1] = (int)col.size();
                rowabs = rs > rowabs ? rs : rowabs;
            }
            if ((rc = drp.upload(c, rp)) || (rc = dcol.upload(c, col.empty() ? std::vector<int>(1, 0) : col)))
                return rc;
            if (prec == NISE_FP32) {
                std::vector<float> vf(vd.begin(), vd.end());
                if (vf.empty()) vf.push_back(0);
                if ((rc = dval.alloc(c, sizeof(float) * vf.size()))) return rc;
                cudaMemcpyAsync(dval.p, vf.data(), sizeof(float) * vf.size(), cudaMemcpyHostToDevice, c->stream);
            } else {
                std::vector<double> v2 = vd;
                if (v2.empty()) v2.push_back(0);
                if ((rc = dval.alloc(c, sizeof(double) * v2.size()))) return rc;
                cudaMemcpyAsync(dval.p, v2.data(), sizeof(double) * v2.size(), cudaMemcpyHostToDevice, c->stream);
            }
            if ((rc = dorder.alloc(c, (size_t)nf))) return rc;
            // sliced ELL (4-row slices, [slot][row]) of the same couplings for the
            // shared-memory kernel; entry offsets are byte offsets of rows of
            // NISE_T3_ROW complex numbers.  Each row lists its neighbours of the other
            // parity first: the four rows of a slice alternate in parity, so a
            // slot whose rows all pick the same relative parity gathers two even
            // and two odd rows, which share no shared-memory banks (FP32).
            std::vector<int> ecol(col.size());
            std::vector<double> evd(col.size());
            for (int i = 0; i < N; i++) {
                int w = rp[i];
                for (int pass = 0; pass < 2; pass++)
                    for (int q = rp[i]; q < rp[i + 1]; q++)
                        if ((((col[q] ^ i) & 1) == 1) == (pass == 0)) {
                            ecol[w] = col[q];
                            evd[w] = vd[q];
                            w++;
                        }
            }
            // Rows of each slice: the sites of each parity, ordered by neighbour
            // count, interleaved even/odd, so the 4 rows of a slice keep the
            // alternating parity and have nearly equal lengths (little ELL padding).
            const int nsl = (N + 3) / 4;
            std::vector<int> srow(4 * (size_t)nsl, N);
            {
                std::vector<int> cls[2];
                for (int i = 0; i < N; i++) cls[i & 1].push_back(i);
                for (int k = 0; k < 2; k++)
                    std::stable_sort(cls[k].begin(), cls[k].end(), [&](int a, int b) {
                        return rp[a + 1] - rp[a] > rp[b + 1] - rp[b];
                    });
                size_t take[2] = {0, 0};
                for (int pos = 0; pos < 4 * nsl; pos++) {
                    int want = pos & 1;
                    if (take[want] >= cls[want].size()) want ^= 1;
                    if (take[want] < cls[want].size()) srow[pos] = cls[want][take[want]++];
                }
            }
            std::vector<int> sptr(nsl + 1, 0);
            for (int sl = 0; sl < nsl; sl++) {
                int L = 0;
                for (int r = 0; r < 4; r++) {
                    int row = srow[4 * sl + r];
                    if (row < N) L = std::max(L, rp[row + 1] - rp[row]);
                }
                sptr[sl + 1] = sptr[sl] + 4 * L;
            }
            const int nent = sptr[nsl];
            const size_t esz = prec == NISE_FP32 ? 8 : 16;
            std::vector<unsigned char> ell((size_t)(nent > 0 ? nent : 1) * esz, 0);
            for (int sl = 0; sl < nsl; sl++) {
                int L = (sptr[sl + 1] - sptr[sl]) / 4;
                for (int slot = 0; slot < L; slot++)
                    for (int r = 0; r < 4; r++) {
                        int row = srow[4 * sl + r], e = sptr[sl] + slot * 4 + r;
                        const int rowb = NISE_T3_ROW * (prec == NISE_FP32 ? 8 : 16);  // bytes per state row
                        int off = (row < N ? row : 0) * rowb;
                        double v = 0;
                        if (row < N && slot < rp[row + 1] - rp[row]) {
                            off = ecol[rp[row] + slot] * rowb;
                            v = evd[rp[row] + slot];
                        }
                        unsigned char *dst = ell.data() + (size_t)e * esz;
                        memcpy(dst, &off, 4);
                        if (prec == NISE_FP32) {
                            float fv = (float)v;
                            memcpy(dst + 4, &fv, 4);
                        } else {
                            memcpy(dst + 8, &v, 8);
                        }
                    }
            }
            if ((rc = drows.upload(c, srow))) return rc;
            if (prec == NISE_FP32) {
                // 4-vector variant: 8-row slices covering the residues of the site
                // index mod 4 twice (rows of 32 bytes: each residue owns a quarter
                // of the banks), neighbours ordered by residue difference, each
                // residue class sorted by neighbour count.
                const int ns4 = (N + 7) / 8;
                std::vector<int> r4(8 * (size_t)ns4, N);
                std::vector<int> cls[4];
                for (int i = 0; i < N; i++) cls[i & 3].push_back(i);
                for (int k = 0; k < 4; k++)
                    std::stable_sort(cls[k].begin(), cls[k].end(), [&](int a, int b) {
                        return rp[a + 1] - rp[a] > rp[b + 1] - rp[b];
                    });
                size_t take[4] = {0, 0, 0, 0};
                for (int pos = 0; pos < 8 * ns4; pos++) {
                    for (int d = 0; d < 4; d++) {
                        int k = (pos + d) & 3;
                        if (take[k] < cls[k].size()) {
                            r4[pos] = cls[k][take[k]++];
                            break;
                        }
                    }
                }
                std::vector<int> c4(col.size());
                std::vector<float> v4(col.size());
                for (int i = 0; i < N; i++) {
                    int w = rp[i];
                    for (int d = 0; d < 4; d++)
                        for (int q = rp[i]; q < rp[i + 1]; q++)
                            if (((col[q] - i) & 3) == d) {
                                c4[w] = col[q];
                                v4[w] = (float)vd[q];
                                w++;
                            }
                }
                std::vector<int> sp4(ns4 + 1, 0);
                for (int sl = 0; sl < ns4; sl++) {
                    int L = 0;
                    for (int r = 0; r < 8; r++) {
                        int row = r4[8 * sl + r];
                        if (row < N) L = std::max(L, rp[row + 1] - rp[row]);
                    }
                    sp4[sl + 1] = sp4[sl] + 8 * L;
                }
                std::vector<int2> e4(sp4[ns4] > 0 ? sp4[ns4] : 1, make_int2(0, 0));
                for (int sl = 0; sl < ns4; sl++) {
                    int L = (sp4[sl + 1] - sp4[sl]) / 8;
                    for (int slot = 0; slot < L; slot++)
                        for (int r = 0; r < 8; r++) {
                            int row = r4[8 * sl + r], e = sp4[sl] + slot * 8 + r;
                            int off = (row < N ? row : 0) * 4;
                            float v = 0.f;
                            if (row < N && slot < rp[row + 1] - rp[row]) {
                                off = c4[rp[row] + slot] * 4;
                                v = v4[rp[row] + slot];
                            }
                            int vb;
                            memcpy(&vb, &v, 4);
                            e4[e] = make_int2(off, vb);
                        }
                }
                if ((rc = dell4.upload(c, e4)) || (rc = dsptr4.upload(c, sp4)) || (rc = drows4.upload(c, r4)))
                    return rc;
                ell4_nslices = ns4;
                ell4_nent = sp4[ns4];
            }
            if (prec == NISE_FP32) {
                // row-owner layout: 8-row slices whose rows alternate in parity (the
                // same degree-sorted interleave as above), neighbours other parity
                // first (ecol); padding slots point at a row of the other parity
                // with weight 0
                const int ns8 = (N + 7) / 8;
                std::vector<int> r8(8 * (size_t)ns8, N);
                {
                    std::vector<int> cls[2];
                    for (int i = 0; i < N; i++) cls[i & 1].push_back(i);
                    for (int k = 0; k < 2; k++)
                        std::stable_sort(cls[k].begin(), cls[k].end(), [&](int a, int b) {
                            return rp[a + 1] - rp[a] > rp[b + 1] - rp[b];
                        });
                    size_t take[2] = {0, 0};
                    for (int pos = 0; pos < 8 * ns8; pos++) {
                        int want = pos & 1;
                        if (take[want] >= cls[want].size()) want ^= 1;
                        if (take[want] < cls[want].size()) r8[pos] = cls[want][take[want]++];
                    }
                }
                std::vector<int> sp8(ns8 + 1, 0);
                for (int sl = 0; sl < ns8; sl++) {
                    int Lm = 0;
                    for (int r = 0; r < 8; r++) {
                        int row = r8[8 * sl + r];
                        if (row < N) Lm = std::max(Lm, rp[row + 1] - rp[row]);
                    }
                    sp8[sl + 1] = sp8[sl] + 8 * Lm;
                }
                // slot triples: [group][row] float4 of three weights and the
                // three neighbours' row indices (10 bits each; a slot count not
                // divisible by 3 padded with weight-0 slots)
                std::vector<int> pp8(ns8 + 1, 0);
                for (int sl = 0; sl < ns8; sl++) pp8[sl + 1] = pp8[sl] + ((sp8[sl + 1] - sp8[sl]) / 8 + 2) / 3;
                const int ntg = pp8[ns8];
                std::vector<float4> t8(8 * (size_t)std::max(ntg, 1), make_float4(0.f, 0.f, 0.f, 0.f));
                std::vector<uint32_t> tix(t8.size(), 0);
                for (int sl = 0; sl < ns8; sl++) {
                    const int Lm = (sp8[sl + 1] - sp8[sl]) / 8;
                    for (int slot = 0; slot < 3 * (pp8[sl + 1] - pp8[sl]); slot++)
                        for (int r = 0; r < 8; r++) {
                            int row = r8[8 * sl + r];
                            int pad = row < N ? (row ^ 1) : 1;
                            if (pad >= N) pad = N > 1 ? N - 2 : 0;
                            uint32_t col = (uint32_t)pad;
                            float v = 0.f;
                            if (row < N && slot < Lm && slot < rp[row + 1] - rp[row]) {
                                col = (uint32_t)ecol[rp[row] + slot];
                                v = (float)evd[rp[row] + slot];
                            }
                            const size_t e = 8 * (size_t)(pp8[sl] + slot / 3) + r;
                            (slot % 3 == 0 ? t8[e].x : slot % 3 == 1 ? t8[e].y : t8[e].z) = v;
                            tix[e] |= col << (10 * (slot % 3));
                        }
                }
                for (size_t e = 0; e < t8.size(); e++) memcpy(&t8[e].w, &tix[e], 4);
                // slices dealt to the warps longest first, each to the warp with
                // the fewest slots so far (24 and 32 warps)
                const int shapes[2] = {24, 32};
                for (int sh = 0; sh < 2; sh++) {
                    const int nw = shapes[sh];
                    std::vector<int> order(ns8), load(nw, 0), cnt(nw, 0), wl(nw * 8, -1);
                    for (int sl = 0; sl < ns8; sl++) order[sl] = sl;
                    std::stable_sort(order.begin(), order.end(),
                                     [&](int a, int b) { return pp8[a + 1] - pp8[a] > pp8[b + 1] - pp8[b]; });
                    bool ok = true;
                    for (int sl : order) {
                        int w = 0;
                        for (int q = 1; q < nw; q++)
                            if (load[q] < load[w] || (load[q] == load[w] && cnt[q] < cnt[w])) w = q;
                        if (cnt[w] >= 8) { ok = false; break; }
                        wl[w * 8 + cnt[w]++] = sl;
                        load[w] += pp8[sl + 1] - pp8[sl];
                    }
                    if (!ok) continue;
                    // each warp's slices in slice order (neighbouring rows together)
                    for (int w = 0; w < nw; w++) std::sort(wl.begin() + w * 8, wl.begin() + w * 8 + cnt[w]);
                    ell8_it[sh] = *std::max_element(cnt.begin(), cnt.end());
                    if ((rc = dwsl8[sh].upload(c, wl))) return rc;
                }
                if ((rc = dtri8.upload(c, t8)) || (rc = dtptr8.upload(c, pp8)) || (rc = drows8.upload(c, r8))) return rc;
                ell8_nslices = ns8;
                ell8_ntg = ntg;
            }
            if ((rc = derr.alloc(c, 1))) return rc;
            cudaMemsetAsync(derr.p, 0, sizeof(int), c->stream);
            if ((rc = dell.alloc(c, ell.size()))) return rc;
            cudaMemcpyAsync(dell.p, ell.data(), ell.size(), cudaMemcpyHostToDevice, c->stream);
            if ((rc = dsptr.upload(c, sptr))) return rc;
            memset(&XP, 0, sizeof(XP));
            XP.n = N;
            XP.nnz = (int)col.size();
            XP.row_ptr = drp.p;
            XP.col = dcol.p;
            XP.val = dval.p;
            XP.static_j = 1;
            XP.ell = dell.p;
            XP.ell_sptr = dsptr.p;
            XP.ell_rows = drows.p;
            if (dell4.p) {
                XP.ell4 = dell4.p;
                XP.ell4_sptr = dsptr4.p;
                XP.ell4_rows = drows4.p;
                XP.ell4_nslices = ell4_nslices;
                XP.ell4_nent = ell4_nent;
            }
            XP.ell_nslices = nsl;
            XP.ell_nent = nent;
            if (dtri8.p) {
                XP.ell8_tri = dtri8.p;
                XP.ell8_tptr = dtptr8.p;
                XP.ell8_rows = drows8.p;
                XP.ell8_nslices = ell8_nslices;
                XP.ell8_ntg = ell8_ntg;
                for (int sh = 0; sh < 2; sh++) {
                    XP.ell8_wsl[sh] = dwsl8[sh].p;
                    XP.ell8_it[sh] = ell8_it[sh];
                }
            }
            XP.err = derr.p;
            XP.f0 = f0;
            XP.nf = nf;
            XP.singleshift = c->nshift > 0;
            // Chebyshev kernel: FP32, its shared-memory footprint (state, diagonal, ELL)
            const size_t csm = (size_t)N * NISE_T3_ROW * 8 + (size_t)N * 32 + (size_t)nent * 8 + 4 * (5 * nsl + 1) + 4096;
            cheb = prec == NISE_FP32 && ((csm <= 227 * 1024 && (nsl + 15) / 16 <= 32) || dtri8.p);
            if (cheb && ((rc = dcorder.alloc(c, (size_t)nf)) || (rc = dinvr.alloc(c, (size_t)nf)) || (rc = dcen.alloc(c, (size_t)nf)) ||
                         (rc = dcoef.alloc(c, (size_t)nf * (NISE_CHEB_KMAX + 1)))))
                return rc;
        }
    }
    config = default_config(scheme, N, plain, cheb, TP.k, nchk, plain ? 3 : nvec, dell4.p != nullptr,
                            scheme == SCHEME_TAYLOR && taylor_rv_fits(T, XP),
                            scheme == SCHEME_TROTTER && TP.rot_static);
    if (p.kernel_config != 0) {  // forced by the caller
        const int k = p.kernel_config;
        if (scheme == SCHEME_EIGEN && (k == 2 || k == 16 || k == 17)) return NISE_OK;
        if (scheme == SCHEME_TROTTER &&
            (k == 1 || k == 32 || k == 33 || (k == 34 && TP.rot_static) || k == 64 || k == 128 || k == 256))
            config = k == 1 ? 0 : k;
        else if (scheme == SCHEME_TAYLOR &&
                 (k == 3 || k == 8 || k == 9 || (k == 10 && cheb) || (k == 12 && dell4.p) || k == 13 || k == 14 ||
                  (k == 15 && cheb && dtri8.p)))
            config = k == 9 ? -8 : k;
        else return nise_fail(c, NISE_ERR_ARG, "kernel_config %d does not apply to this scheme", k);
        return NISE_OK;
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(TuneKey(scheme, prec, N, scheme == SCHEME_TROTTER ? TP.k : 0,
                                       scheme == SCHEME_TROTTER ? TP.rot_static : 0));
        if (it != g_tuned.end()) config = it->second;
    }
    if (autotune && (scheme == SCHEME_TROTTER || scheme == SCHEME_TAYLOR) && !plain)
        if ((rc = tune())) return rc;
    return NISE_OK;
}

// The propagation kernel(s) of the job with launch configuration cfg.
int AbsRun::run_main(cudaStream_t s, int cfg, double2 *dst) {
    const int pr = prec == NISE_FP32 ? 0 : 1;
    int e = 0, kernels = 1;
    auto one = [&](const AbsJob &Js, double2 *r) -> int {
        kernels = 1;
        switch (scheme) {
        case SCHEME_TROTTER:
            if (cfg == 32 || cfg == 33) return launch_abs_trotter_wv(pr, T, TP, Js, r, lvchk.p, nchk, cfg == 32, s);
            if (cfg == 34) return launch_abs_trotter_wv2(pr, T, TP, Js, r, lvchk.p, nchk, s);
            if (cfg > 0) return launch_abs_trotter_lv(pr, T, TP, Js, r, lvptr.p, nlev, cfg, s);
            return launch_abs_trotter(pr, T, TP, Js, r, s);
        case SCHEME_RK4:
            return launch_abs_rk4(pr, T, RP, Js, r, s);
        case SCHEME_TAYLOR: {
            TaylorPlan P = XP;
            P.only_v2 = cfg < 0;
            P.use_v4 = cfg == 12;
            P.no_rv = cfg == 13;
            if (cfg == 10 || cfg == 15) {
                P.order = dcorder.p;
                P.cheb_inv_r = dinvr.p;
                P.cheb_center = dcen.p;
                P.cheb_coef = dcoef.p;
                P.rv_cheb = cfg == 15;
                P.order_taylor = dorder.p;
            } else {
                P.order = dorder.p;
                P.cheb_inv_r = nullptr;
                P.cheb_center = nullptr;
                P.cheb_coef = nullptr;
            }
            P.rv_shape = cfg == 14 ? 1 : 0;
            return launch_abs_taylor(pr, T, P, Js, r, cfg == 10 || cfg >= 13 ? 8 : cfg < 0 ? -cfg : cfg, s, &kernels);
        }
        default:
            if (stream_u) {
                // chunks of FC frames: eigendecompositions, propagators, then
                // the tensor-core steps of those frames
                EigJob EJ;
                EJ.T = T;
                EJ.n = N;
                EJ.singleshift = c->nshift > 0;
                int er = 0;
                for (long q = 0; q < nf && !er; q += FC) {
                    const long m = std::min(FC, nf - q);
                    if ((er = launch_eig_any(EJ, efr.p + q, m, eV.p, ew.p, eA.p, estatus.p, s))) break;
                    if ((er = launch_build_u_any(pr, eV.p, ew.p, m, N, fe, c->thres, truncated, Ue.p, s))) break;
                    // the last chunk runs on to the last response frame, which needs no propagator
                    const long tb = q + m >= nf ? tc_dia_last_frame(Js) : f0 + q + m - 1;
                    er = launch_abs_dia_tc_frames(T, Ue.p, f0 + q, N, Js, r, tcX.p, derr.p, f0 + q, tb, s);
                    kernels += 2;
                }
                return er;
            }
            if (use_tc) return launch_abs_dia_tc(T, Ue.p, f0, N, Js, r, tcX.p, derr.p, s);
            return launch_abs_dia(pr, T, Ue.p, f0, N, Js, r, s);
        }
    };
    if (plain) {
        for (int q = 0; q < nsamp && !e; q++) {
            AbsJob Js = J;
            Js.begin = begin + q;
            Js.nsamp = 1;
            e = one(Js, dst + (size_t)3 * q * tmax);
            c->launches += kernels;
        }
    } else {
        e = one(J, dst);
        c->launches += kernels;
    }
    return e;
}

// Time every candidate configuration on the job itself (into the response
// buffer, which enqueue() overwrites) and keep the fastest.
int AbsRun::tune() {
    std::vector<int> cand;
    if (scheme == SCHEME_TROTTER) {
        cand = {0, 32, 33, 64, 128, 256};
        if (TP.rot_static) cand.push_back(34);
    } else {
        cand = {3, -8, 8, 13, 14};
        if (cheb) cand.push_back(10);
        if (cheb && dtri8.p) cand.push_back(15);
        if (dell4.p) cand.push_back(12);
    }
    // the tables the kernels read (both series for the Taylor route)
    int rc;
    if ((rc = enqueue(c->stream, false))) return rc;
    if (scheme == SCHEME_TAYLOR) {
        TaylorPlan P = XP;
        if ((rc = nise_cuda(c, launch_prep_taylor(prec, T, P, rowabs, J.f, dorder.p, c->stream), "Taylor prep")))
            return rc;
        if (cheb && (rc = nise_cuda(c, launch_prep_cheb(T, P, rowabs, J.f, dcorder.p, dinvr.p, dcen.p, dcoef.p, c->stream),
                                    "Chebyshev prep")))
            return rc;
    }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    int best_cfg = config;
    for (int cfg : cand) {
        cudaEventRecord(a, c->stream);
        int e = run_main(c->stream, cfg, resp.p);
        cudaEventRecord(b, c->stream);
        if (e) continue;  // a configuration that cannot launch (shared memory) is skipped
        if (cudaEventSynchronize(b) != cudaSuccess) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best) {
            best = ms;
            best_cfg = cfg;
        }
    }
    cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    config = best_cfg;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[TuneKey(scheme, prec, N, scheme == SCHEME_TROTTER ? TP.k : 0,
                    scheme == SCHEME_TROTTER ? TP.rot_static : 0)] = best_cfg;
    return nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "autotuner");
}

// Kernels of the job on stream s: tables, propagation, response sum.
bool AbsRun::waves_apply() const {
    return c->nchunks > 0 && scheme == SCHEME_TAYLOR && !plain && (config == 15 || config == 8) &&
           prec == NISE_FP32 && taylor_rv_fits(T, XP) && nvec > sm_count();
}

int AbsRun::enqueue_waves(cudaStream_t s) {
    TaylorPlan P = XP;
    P.rv_shape = 0;
    if (config == 15) {
        P.order = dcorder.p;
        P.cheb_inv_r = dinvr.p;
        P.cheb_center = dcen.p;
        P.cheb_coef = dcoef.p;
        P.rv_cheb = 1;
        P.order_taylor = dorder.p;
    } else {
        P.order = dorder.p;
    }
    // whole waves of 8-vector CTAs, the rest on 1-vector CTAs (as launch_abs_taylor).
    // Here the 1-vector CTAs take the FIRST vectors, whose frames arrive first:
    // they run on a side stream while the rest of the trajectory is copied, and
    // the waves (the job's length either way: 1-vector CTAs then five waves on
    // their SMs) start as their frames land.
    const int nsm = sm_count(), ctas = (nvec + 7) / 8;
    int main = nvec;
    if (ctas % nsm != 0 && ctas % nsm < nsm / 2 && ctas >= nsm) main = (ctas / nsm) * nsm * 8;
    const int ntail = nvec - main;
    long prepped = f0;  // frames [f0, prepped) have their series tables
    int rc = 0;
    auto prep_to = [&](long last) -> int {
        if (last < prepped) return 0;
        nise_wait_frames(c, s, last);
        TaylorPlan Q = XP;
        Q.f0 = prepped;
        Q.nf = last + 1 - prepped;
        const long o = prepped - f0;
        int e = 0;
        if (config == 15) {
            e = nise_cuda(c, launch_prep_cheb(T, Q, rowabs, J.f, dcorder.p + o, dinvr.p + o, dcen.p + o,
                                              dcoef.p + o * (NISE_CHEB_KMAX + 1), s), "Chebyshev prep");
            c->launches++;
        }
        if (!e && config != 15) {  // config 15 runs the Chebyshev series on every CTA
            e = nise_cuda(c, launch_prep_taylor(prec, T, Q, rowabs, J.f, dorder.p + o, s), "Taylor prep");
            c->launches++;
        }
        prepped = last + 1;
        return e;
    };
    // the last frame any of vectors [.., ve) steps through
    auto last_frame = [&](int ve) { return (long)(J.begin + (ve - 1) / 3) * J.sample + J.tmax - 2; };
    if (ntail > 0) {
        if (!side) {
            if ((rc = nise_cuda(c, (int)cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking), "side stream")) ||
                (rc = nise_cuda(c, (int)cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming), "event")) ||
                (rc = nise_cuda(c, (int)cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming), "event")))
                return rc;
        }
        if ((rc = prep_to(last_frame(ntail)))) return rc;
        cudaEventRecord(ev_fork, s);
        cudaStreamWaitEvent(side, ev_fork, 0);
        rc = nise_cuda(c, launch_abs_taylor_part(T, P, J, resp.p, 0, ntail, true, side), "propagation");
        c->launches++;
        cudaEventRecord(ev_join, side);
    }
    for (int v = ntail; v < nvec && !rc; v += 8 * nsm) {
        const int ve = std::min(v + 8 * nsm, nvec);
        if ((rc = prep_to(last_frame(ve)))) break;
        rc = nise_cuda(c, launch_abs_taylor_part(T, P, J, resp.p, v, ve - v, false, s), "propagation");
        c->launches++;
    }
    if (ntail > 0) cudaStreamWaitEvent(s, ev_join, 0);  // joined on every path
    return rc;
}

int AbsRun::enqueue(cudaStream_t s, bool events) {
    const int pr = prec == NISE_FP32 ? 0 : 1;
    int rc;
    const bool waves = waves_apply();
    if (c->nchunks > 0 && !waves) nise_wait_all_frames(c, s);
    if (events) cudaEventRecord(c->evk0, s);
    if (waves) {
        if ((rc = enqueue_waves(s))) return rc;
        if (events) cudaEventRecord(c->evk1, s);
        if ((rc = nise_cuda(c, launch_reduce_resp(resp.p, nvec, tmax, out.p, s), "response reduction"))) return rc;
        c->launches++;
        return NISE_OK;
    }
    switch (scheme) {
    case SCHEME_TROTTER:
        if ((rc = nise_cuda(c, launch_prep_trotter(prec, T, TP, J.f64_sub, J.f32_sub, s), "Trotter prep"))) return rc;
        c->launches += 1 + (TP.rot_static ? 1 : 0);
        break;
    case SCHEME_RK4:
        if ((rc = nise_cuda(c, launch_prep_rk4(prec, T, RP, J.f64_sub, J.f32_sub, s), "RK4 prep"))) return rc;
        c->launches++;
        break;
    case SCHEME_TAYLOR: {
        TaylorPlan P = XP;
        if (config == 10 || config == 15) {
            rc = nise_cuda(c, launch_prep_cheb(T, P, rowabs, J.f, dcorder.p, dinvr.p, dcen.p, dcoef.p, s), "Chebyshev prep");
            c->launches++;
        }
        if (!rc && config != 10 && config != 15) {
            rc = nise_cuda(c, launch_prep_taylor(prec, T, P, rowabs, J.f, dorder.p, s), "Taylor prep");
            c->launches++;
        }
        if (rc) return rc;
        break;
    }
    default: {
        EigJob EJ;
        EJ.T = T;
        EJ.n = N;
        EJ.singleshift = c->nshift > 0;
        const size_t r2 = prec == NISE_FP32 ? sizeof(float2) : sizeof(double2);
        for (long q = 0; q < nf && !stream_u; q += FC) {  // streamed: built inside the propagation
            long m = std::min(FC, nf - q);
            if ((rc = nise_cuda(c, launch_eig_any(EJ, efr.p + q, m, eV.p, ew.p, eA.p, estatus.p, s), "eigensolver")))
                return rc;
            if ((rc = nise_cuda(c, launch_build_u_any(pr, eV.p, ew.p, m, N, fe, c->thres, truncated,
                                                  Ue.p + r2 * (size_t)q * N * N, s),
                                "propagator build")))
                return rc;
            c->launches += 2;
        }
    }
    }
    if ((rc = nise_cuda(c, run_main(s, config, resp.p), "propagation"))) return rc;
    if (events) cudaEventRecord(c->evk1, s);
    if ((rc = nise_cuda(c, launch_reduce_resp(resp.p, nvec, tmax, out.p, s), "response reduction"))) return rc;
    c->launches++;
    return NISE_OK;
}

// Algorithmic flops of the propagation (after the job ran: the Taylor orders
// are read back from the device).
double AbsRun::flops() const {
    const nise_params &p = c->p;
    switch (scheme) {
    case SCHEME_TROTTER:
        // per vector step: ts * (K rotations * 12 flops + 2 N half-phases * 6 flops)
        return (double)vec_steps * p.ts * (12.0 * TP.k + 12.0 * N);
    case SCHEME_RK4:
        // per sub-step: 4 stages over the list (off-diagonal entries twice) + update and norms
        return (double)vec_steps * p.ts * (4.0 * 4.0 * (2.0 * RP.k - N) + 20.0 * N);
    case SCHEME_TAYLOR: {
        // per vector step and Taylor order: nnz complex*real products (4 flops)
        // and the diagonal, scaling and accumulation (6 flops per site)
        // (Chebyshev: the same products per term plus the recurrence, 10 flops per site)
        std::vector<int> order(nf);
        const bool ch = config == 10 || config == 15;
        cudaMemcpy(order.data(), ch ? dcorder.p : dorder.p, sizeof(int) * nf, cudaMemcpyDeviceToHost);
        double orders = 0;
        for (long t = 0; t < nf; t++) orders += (double)order[t] * cross[t];
        return orders * (4.0 * XP.nnz + (ch ? 10.0 : 6.0) * N);
    }
    default:
        return (double)nf * 6.7 * N * (double)N * N + (double)vec_steps * 8.0 * N * N;
    }
}

extern "C" int nise_absorption(nise_ctx *c, double *re_S, double *im_S, int *samples) {
    if (!c || !re_S || !im_S || !samples) return nise_fail(c, NISE_ERR_ARG, "null argument");
    cudaSetDevice(c->p.device);
    c->launches = 0;
    c->last_flops = c->last_bytes = 0;
    int rc;
    AbsRun *Rp = nullptr;
    if (c->abs_plan && c->abs_plan_epoch == c->plan_epoch) {
        Rp = (AbsRun *)c->abs_plan.get();  // same layout, couplings, SingleShift and stream
        Rp->refresh();
    } else {
        c->abs_plan.reset();
        if (c->p.hamiltonian != NISE_HAM_COUPLING) nise_wait_all_frames(c, c->stream);  // the pattern scan reads frames
        std::unique_ptr<AbsRun> fresh(new AbsRun);
        if ((rc = fresh->plan(c, false))) return rc;
        Rp = fresh.release();
        c->abs_plan = std::shared_ptr<void>(Rp, [](void *q) { delete (AbsRun *)q; });
        c->abs_plan_epoch = c->plan_epoch;
    }
    AbsRun &R = *Rp;
    cudaEventRecord(c->ev0, c->stream);
    if ((rc = R.enqueue(c->stream, true))) return rc;
    cudaEventRecord(c->ev1, c->stream);
    std::vector<double2> h(R.tmax);
    cudaMemcpyAsync(h.data(), R.out.p, sizeof(double2) * R.tmax, cudaMemcpyDeviceToHost, c->stream);
    if ((rc = nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "absorption"))) return rc;
    if ((rc = R.check_err())) return rc;
    nise_collect_timing(c);
    c->last_flops = R.flops();
    c->last_bytes = R.alg_bytes;
    for (int t = 0; t < R.tmax; t++) {
        re_S[t] = h[t].x;
        im_S[t] = h[t].y;
    }
    *samples = R.end;  // absorption.c:185 divides by `samples`, which equals end after the loop
    return NISE_OK;
}

extern "C" int nise_absorption_tune(nise_ctx *c) {
    if (!c) return nise_fail(nullptr, NISE_ERR_ARG, "null context");
    cudaSetDevice(c->p.device);
    c->abs_plan.reset();
    c->plan_epoch++;
    nise_wait_all_frames(c, c->stream);
    AbsRun R;
    c->launches = 0;
    return R.plan(c, true);
}

// ------------------------------------------------------------------ batch
struct nise_batch {
    std::vector<nise_ctx *> ctx;
    std::vector<std::unique_ptr<AbsRun>> runs;
    std::vector<std::unique_ptr<DevBuf<double2>>> spec, fftin;
    std::vector<FftJob> fj;
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> done;
    cudaStream_t master = nullptr;
    cudaEvent_t start = nullptr, stop = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<std::vector<double2>> host_out, host_spec;
    double last_ms = 0;
    std::vector<double> job_ms;
    int device = 0;
    std::string err;
};

static int batch_fail(nise_batch *b, int code, const std::string &msg) {
    b->err = msg;
    nise_set_global_error(msg.c_str());
    return code;
}

extern "C" void nise_batch_destroy(nise_batch *b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->master) cudaStreamSynchronize(b->master);
    for (auto s : b->side) cudaStreamDestroy(s);
    for (auto e : b->done) cudaEventDestroy(e);
    if (b->start) cudaEventDestroy(b->start);
    if (b->stop) cudaEventDestroy(b->stop);
    b->spec.clear();
    b->fftin.clear();
    b->runs.clear();
    if (b->master) cudaStreamDestroy(b->master);
    delete b;
}

extern "C" int nise_batch_create(nise_ctx *const *ctxs, int n, int autotune, nise_batch **out) {
    if (!ctxs || n <= 0 || !out) return nise_fail(nullptr, NISE_ERR_ARG, "nise_batch_create: bad arguments");
    *out = nullptr;
    nise_batch *b = new nise_batch();
    b->device = ctxs[0]->p.device;
    cudaSetDevice(b->device);
    for (int i = 0; i < n; i++) {
        nise_ctx *c = ctxs[i];
        if (!c || c->p.device != b->device) {
            nise_batch_destroy(b);
            return nise_fail(nullptr, NISE_ERR_ARG, "nise_batch_create: all contexts must be valid and on one device");
        }
        b->ctx.push_back(c);
        b->runs.emplace_back(new AbsRun());
        c->launches = 0;
        // the graph below captures kernels only: energy records still in
        // flight from the host land first
        if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
        c->nchunks = 0;
        int rc = b->runs.back()->plan(c, autotune != 0);
        if (rc) {
            std::string m = "job " + std::to_string(i) + ": " + c->err;
            nise_batch_destroy(b);
            return nise_fail(nullptr, rc, "%s", m.c_str());
        }
        const nise_params &p = c->p;
        FftJob J;
        J.tmax = p.tmax1;
        J.fft = p.fft < p.tmax1 ? p.tmax1 : p.fft;
        J.samples = b->runs.back()->end;
        J.window = p.window;
        J.fp32 = p.precision == NISE_FP32;
        J.deltat = p.deltat;
        J.lifetime = p.lifetime;
        J.homogen = p.homogen;
        J.inhomogen = p.inhomogen;
        b->fj.push_back(J);
        b->spec.emplace_back(new DevBuf<double2>());
        b->fftin.emplace_back(new DevBuf<double2>());
        if ((rc = b->spec.back()->alloc(c, J.fft)) || (rc = b->fftin.back()->alloc(c, J.fft))) {
            nise_batch_destroy(b);
            return rc;
        }
    }
    for (auto c : b->ctx) cudaStreamSynchronize(c->stream);  // tables and buffers in place
    if (cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking) || cudaEventCreate(&b->start) ||
        cudaEventCreate(&b->stop)) {
        nise_batch_destroy(b);
        return nise_fail(nullptr, NISE_ERR_DEVICE, "nise_batch_create: stream/event creation failed");
    }
    b->side.resize(n);
    b->done.resize(n);
    for (int i = 0; i < n; i++)
        if (cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking) || cudaEventCreate(&b->done[i])) {
            nise_batch_destroy(b);
            return nise_fail(nullptr, NISE_ERR_DEVICE, "nise_batch_create: stream/event creation failed");
        }
    // capture: fork every job onto its own stream, join them back
    cudaEvent_t fork;
    cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
    int rc = NISE_OK;
    if (cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaEventDestroy(fork);
        nise_batch_destroy(b);
        return nise_fail(nullptr, NISE_ERR_DEVICE, "nise_batch_create: stream capture failed to begin");
    }
    cudaEventRecord(fork, b->master);
    for (int i = 0; i < n && rc == NISE_OK; i++) {
        cudaStreamWaitEvent(b->side[i], fork, 0);
        rc = b->runs[i]->enqueue(b->side[i], false);
        if (rc == NISE_OK)
            rc = nise_cuda(b->ctx[i], launch_fft1d_buf(b->fj[i], b->runs[i]->out.p, b->spec[i]->p, b->fftin[i]->p,
                                                       b->side[i]),
                           "1D FFT");
        cudaEventRecord(b->done[i], b->side[i]);
        cudaStreamWaitEvent(b->master, b->done[i], 0);
    }
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(b->master, &g);
    cudaEventDestroy(fork);
    if (rc != NISE_OK || ce != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        std::string m = rc ? "capture: job kernels failed to enqueue" : cudaGetErrorString(ce);
        nise_batch_destroy(b);
        return nise_fail(nullptr, rc ? rc : NISE_ERR_DEVICE, "nise_batch_create: %s", m.c_str());
    }
    b->graph = g;
    if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) {
        nise_batch_destroy(b);
        return nise_fail(nullptr, NISE_ERR_DEVICE, "nise_batch_create: graph instantiation failed");
    }
    b->host_out.resize(n);
    b->host_spec.resize(n);
    b->job_ms.assign(n, 0);
    *out = b;
    return NISE_OK;
}

extern "C" int nise_batch_run(nise_batch *b) {
    if (!b) return nise_fail(nullptr, NISE_ERR_ARG, "null batch");
    cudaSetDevice(b->device);
    cudaEventRecord(b->start, b->master);
    if (cudaGraphLaunch(b->exec, b->master) != cudaSuccess)
        return batch_fail(b, NISE_ERR_DEVICE, "nise_batch_run: graph launch failed");
    cudaEventRecord(b->stop, b->master);
    const int n = (int)b->runs.size();
    for (int i = 0; i < n; i++) {
        AbsRun &R = *b->runs[i];
        b->host_out[i].resize(R.tmax);
        b->host_spec[i].resize(b->fj[i].fft);
        cudaMemcpyAsync(b->host_out[i].data(), R.out.p, sizeof(double2) * R.tmax, cudaMemcpyDeviceToHost, b->master);
        cudaMemcpyAsync(b->host_spec[i].data(), b->spec[i]->p, sizeof(double2) * b->fj[i].fft,
                        cudaMemcpyDeviceToHost, b->master);
    }
    cudaError_t e = cudaStreamSynchronize(b->master);
    if (e != cudaSuccess) return batch_fail(b, NISE_ERR_DEVICE, std::string("nise_batch_run: ") + cudaGetErrorString(e));
    for (int i = 0; i < n; i++)
        if (b->runs[i]->check_err())
            return batch_fail(b, NISE_ERR_TIMEOUT, "nise_batch_run: a bounded wait for a staged frame gave up");
    float ms = 0;
    cudaEventElapsedTime(&ms, b->start, b->stop);
    b->last_ms = ms;
    return NISE_OK;
}

extern "C" int nise_batch_result(nise_batch *b, int i, double *re_S, double *im_S, int *samples) {
    if (!b || i < 0 || i >= (int)b->runs.size() || !re_S || !im_S || !samples)
        return nise_fail(nullptr, NISE_ERR_ARG, "nise_batch_result: bad arguments");
    const auto &h = b->host_out[i];
    if (h.empty()) return batch_fail(b, NISE_ERR_STATE, "nise_batch_result: the batch has not run");
    for (size_t t = 0; t < h.size(); t++) {
        re_S[t] = h[t].x;
        im_S[t] = h[t].y;
    }
    *samples = b->runs[i]->end;
    return NISE_OK;
}

extern "C" int nise_batch_spectrum(nise_batch *b, int i, double *freq, double *spec_re, double *spec_im, int max_rows,
                                   int *rows) {
    if (!b || i < 0 || i >= (int)b->runs.size() || !freq || !spec_re || !spec_im || !rows)
        return nise_fail(nullptr, NISE_ERR_ARG, "nise_batch_spectrum: bad arguments");
    if (b->host_spec[i].empty()) return batch_fail(b, NISE_ERR_STATE, "nise_batch_spectrum: the batch has not run");
    *rows = nise_spectrum_rows(b->ctx[i], b->host_spec[i].data(), b->fj[i].fft, freq, spec_re, spec_im, max_rows);
    return NISE_OK;
}

extern "C" int nise_batch_timing(const nise_batch *b, double *ms, long *kernel_launches) {
    if (!b) return NISE_ERR_ARG;
    if (ms) *ms = b->last_ms;
    if (kernel_launches) {
        long n = 0;
        for (auto c : b->ctx) n += c->launches;
        *kernel_launches = n + (long)b->runs.size() * 2;  // + the two transform kernels per job
    }
    return NISE_OK;
}

extern "C" const char *nise_batch_error(const nise_batch *b) { return b ? b->err.c_str() : nise_global_error(); }
