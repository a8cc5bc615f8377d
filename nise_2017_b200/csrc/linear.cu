// Linear techniques besides absorption on one GPU: linear dichroism
// (calc_LD.c:15-283), Raman (raman.c:15-290), SFG (sfg.c:15-278), density of
// states (calc_DOS.c:15-222) and circular dichroism (calc_CD.c:15-377).
//
// Each is the absorption loop (absorption.c:18-202) over start points
// ti = sample * s with other initial vectors and other read-outs:
//
//   LD     3 vectors mu_x(ti); read-out mu_x(tj), channel -0.5 xx - 0.5 yy + zz
//   Raman  6 vectors alpha_x(ti) (Alphafile); read-out alpha_x(tj);
//          VV = components 0, 3, 5; VH = 2 x components 1, 2, 4
//   SFG    the vector mu_z(ti) (the reference also propagates mu_x and mu_y,
//          which no read-out uses); read-outs alpha_5 (PPP) and
//          (alpha_0 + alpha_3) / 2 (SSP) at tj
//   DOS    N unit vectors e_i; read-out component i (the trace of U)
//   CD     3N vectors mu_x(ti)_j e_j; read-outs, for the two y != x,
//          sum_i sign(x,y) (r_z,i - r_z,j) mu_y,i psi_i with z = 3 - x - y
//
// One thread propagates one vector (the [site][lane] shared-memory layout and
// the singles_step of the 2D kernels, so every vector sees the reference's
// single-precision operations in FP32 mode) and writes its read-outs of every
// t1 to a per-vector array; a second kernel sums them per channel in a fixed
// order (FP64 sums, as the absorption path).  Products keep the reference's
// float operand order; the scalings by -0.5, 2 and 1/2 are exact.
//
// SingleShift enters through read_Hamiltonian only, which of these SFG
// calls (sfg.c:172); LD, Raman, DOS and CD read frames with read_He/read_Dia.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "nise_internal.h"
#include "schemes.cuh"

namespace {

struct LinJob : SinglesTab {
    DevTraj T;
    int tech, begin, S, sample, tmax;  // S start points from `begin`
    int nvec, nread;                   // vectors per start point, read-outs per vector
    const float *alpha;                // polarisability records [frame][1 + 6n] (read_alpha)
    long al_words;
    const float *pos;                  // CD position records [frame][1 + 3n] (read_mue layout)
    long pos_words;
    double2 *part;                     // [S][nvec][nread][tmax]
};

struct LinSpec {
    int nvec_fixed, nvec_per_site, nread, nch, singleshift, dipoles, alpha, pos;
};

// Vectors, read-outs and channels of each technique, and what it reads.
LinSpec lin_spec(int tech) {
    switch (tech) {
    case NISE_TECH_LD: return {3, 0, 1, 1, 0, 1, 0, 0};
    case NISE_TECH_RAMAN: return {6, 0, 1, 2, 0, 0, 1, 0};
    case NISE_TECH_SFG: return {1, 0, 3, 2, 1, 1, 1, 0};
    case NISE_TECH_DOS: return {0, 1, 1, 1, 0, 0, 0, 0};
    case NISE_TECH_CD: return {0, 3, 2, 1, 0, 1, 0, 1};
    default: return {0, 0, 0, 0, 0, 0, 0, 0};
    }
}

__device__ __forceinline__ float lin_alpha(const LinJob &J, long t, int x, int i) {
    return J.alpha[t * J.al_words + 1 + (long)x * J.n + i];
}

// CD positions (calc_CD.c:164-170, 254-262): frame t, or frame 0 for
// HamiltonianType Coupling.
__device__ __forceinline__ float lin_pos(const LinJob &J, long t, int z, int i) {
    if (J.T.mu_static) t = 0;
    return J.pos[t * J.pos_words + 1 + (long)z * J.n + i];
}

// The two polarisations y != x of a CD read-out r, in the reference's loop
// order, and the sign of its (x, y, z) term (calc_CD.c:264-274).
__device__ __forceinline__ int cd_y(int x, int r) { return r == 0 ? (x == 0 ? 1 : 0) : (x == 2 ? 1 : 2); }
__device__ __forceinline__ float cd_sign(int x, int y) {
    // +1 for (x,y) = (2,1), (1,0), (0,2); -1 for (1,2), (2,0), (0,1)
    return ((y - x + 3) % 3 == 2) ? 1.0f : -1.0f;
}

// Initial value of site i of vector v at the start frame ti.
__device__ __forceinline__ float lin_init(const LinJob &J, int v, long ti, int i) {
    const int n = J.n;
    switch (J.tech) {
    case NISE_TECH_LD: return traj_mu(J.T, ti, v, i);
    case NISE_TECH_RAMAN: return lin_alpha(J, ti, v, i);
    case NISE_TECH_SFG: return traj_mu(J.T, ti, 2, i);
    case NISE_TECH_DOS: return i == v ? 1.0f : 0.0f;
    default: {  // CD: mu_x(ti)_j on site j
        const int x = v / n, j = v % n;
        return i == j ? traj_mu(J.T, ti, x, j) : 0.0f;
    }
    }
}

// Read-out r of vector v at frame t: sum_i w_i psi_i with float products in
// FP32 mode and an FP64 sum in site order.
template <typename R>
__device__ double2 lin_read(const LinJob &J, int v, int r, long t, const typename Vec2<R>::T *S, int B, int lane) {
    typedef typename Vec2<R>::T R2;
    typedef Ar<R> A;
    const int n = J.n;
    double re = 0, im = 0;
    if (J.tech == NISE_TECH_DOS) {
        R2 z = S[v * B + lane];
        return make_double2((double)z.x, (double)z.y);
    }
    if (J.tech == NISE_TECH_CD) {
        const int x = v / n, j = v % n, y = cd_y(x, r), z = 3 - x - y;
        // static dipoles: the reference copies component x here (calc_CD.c:250)
        const int ym = J.T.mu_static ? x : y;
        // the operator sign * (r_i - r_j) * mu_i is formed in float, as the
        // reference's float operands are, in both precisions
        const float sg = cd_sign(x, y), pj = lin_pos(J, t, z, j);
        for (int i = 0; i < n; i++) {
            R w = (R)__fmul_rn(__fmul_rn(sg, __fsub_rn(lin_pos(J, t, z, i), pj)), traj_mu(J.T, t, ym, i));
            R2 c = S[i * B + lane];
            re += (double)A::mul(w, c.x);
            im += (double)A::mul(w, c.y);
        }
        return make_double2(re, im);
    }
    for (int i = 0; i < n; i++) {
        float m;
        if (J.tech == NISE_TECH_LD) m = traj_mu(J.T, t, v, i);
        else if (J.tech == NISE_TECH_RAMAN) m = lin_alpha(J, t, v, i);
        else m = lin_alpha(J, t, r == 0 ? 5 : (r == 1 ? 0 : 3), i);  // SFG: PPP, then SSP xx, yy
        R2 c = S[i * B + lane];
        re += (double)A::mul((R)m, c.x);
        im += (double)A::mul((R)m, c.y);
    }
    return make_double2(re, im);
}

// Thread per (start point, vector): read-outs before each step, as the
// reference's t1 loop (the step after the last read-out is not needed).
template <typename R>
__global__ void k_lin(LinJob J) {
    typedef typename Vec2<R>::T R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *S = (R2 *)smem_raw;
    const int B = blockDim.x, lane = threadIdx.x, n = J.n;
    const long g = blockIdx.x * (long)B + lane;
    if (g >= (long)J.S * J.nvec) return;
    const int s = (int)(g / J.nvec), v = (int)(g % J.nvec);
    const long ti = (long)(J.begin + s) * J.sample;
    for (int i = 0; i < n; i++) {
        R2 z;
        z.x = (R)lin_init(J, v, ti, i);
        z.y = 0;
        S[i * B + lane] = z;
    }
    double2 *out = J.part + ((size_t)s * J.nvec + v) * J.nread * J.tmax;
    for (int t1 = 0; t1 < J.tmax; t1++) {
        const long tj = ti + t1;
        for (int r = 0; r < J.nread; r++) out[(size_t)r * J.tmax + t1] = lin_read<R>(J, v, r, tj, S, B, lane);
        if (t1 < J.tmax - 1) singles_step<R>(J, S, B, lane, tj);
    }
}

// Weight of read-out r of vector v in channel ch.
__device__ __forceinline__ double lin_weight(int tech, int ch, int v, int r) {
    switch (tech) {
    case NISE_TECH_LD: return v == 2 ? 1.0 : -0.5;                  // calc_LD.c:286-290
    case NISE_TECH_RAMAN:                                             // raman.c:181-182, 293-307
        if (ch == 0) return (v == 0 || v == 3 || v == 5) ? 1.0 : 0.0;
        return (v == 1 || v == 2 || v == 4) ? 2.0 : 0.0;
    case NISE_TECH_SFG:                                               // sfg.c:183-184, 281-297
        if (ch == 0) return r == 0 ? 1.0 : 0.0;
        return r == 0 ? 0.0 : 0.5;
    default: return 1.0;
    }
}

// out[ch][t1] (+)= sum over start points, vectors and read-outs, in order.
__global__ void k_lin_reduce(const double2 *part, int S, int nvec, int nread, int tmax, int tech, int nch,
                             double2 *out, int first) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nch * tmax) return;
    const int ch = g / tmax, t1 = g % tmax;
    double re = 0, im = 0;
    for (int s = 0; s < S; s++)
        for (int v = 0; v < nvec; v++)
            for (int r = 0; r < nread; r++) {
                const double w = lin_weight(tech, ch, v, r);
                if (w == 0.0) continue;
                double2 z = part[(((size_t)s * nvec + v) * nread + r) * tmax + t1];
                re += w * z.x;
                im += w * z.y;
            }
    if (first) out[g] = make_double2(re, im);
    else out[g] = make_double2(out[g].x + re, out[g].y + im);
}

template <typename R>
int run_lin(const LinJob &J, double2 *out, int nch, int first, cudaStream_t st) {
    size_t lane_b = singles_lane_bytes<R>(J.n, J.prop);
    int B = 64;
    while (B > 1 && (size_t)B * lane_b > 200 * 1024) B >>= 1;
    size_t sm = lane_b * B;
    int e;
    if (sm > 48 * 1024 &&
        (e = (int)cudaFuncSetAttribute(k_lin<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)))
        return e;
    long nv = (long)J.S * J.nvec;
    k_lin<R><<<(unsigned)((nv + B - 1) / B), B, sm, st>>>(J);
    int tot = nch * J.tmax;
    k_lin_reduce<<<(tot + 127) / 128, 128, 0, st>>>(J.part, J.S, J.nvec, J.nread, J.tmax, J.tech, nch, out, first);
    return (int)cudaGetLastError();
}

struct LinFiles {
    const char *td, *spec;
};

// Output files of each channel (calc_LD.c:265-278, raman.c:263-287,
// sfg.c:253-277, calc_DOS.c:206-214, calc_CD.c:359-372).
const LinFiles *lin_files(int tech, int *nch) {
    static const LinFiles ld[] = {{"TD_LD.dat", "LD.dat"}};
    static const LinFiles raman[] = {{"TD_Raman_VV.dat", "Raman_VV.dat"}, {"TD_Raman_VH.dat", "Raman_VH.dat"}};
    static const LinFiles sfg[] = {{"TD_SFG_PPP.dat", "SFG_PPP.dat"}, {"TD_SFG_SSP.dat", "SFG_SSP.dat"}};
    static const LinFiles dos[] = {{"TD_DOS.dat", "DOS.dat"}};
    static const LinFiles cd[] = {{"TD_CD.dat", "CD.dat"}};
    switch (tech) {
    case NISE_TECH_LD: *nch = 1; return ld;
    case NISE_TECH_RAMAN: *nch = 2; return raman;
    case NISE_TECH_SFG: *nch = 2; return sfg;
    case NISE_TECH_DOS: *nch = 1; return dos;
    case NISE_TECH_CD: *nch = 1; return cd;
    default: *nch = 0; return nullptr;
    }
}

}  // namespace

extern "C" const char *nise_linear_file(int technique, int channel, int td) {
    int nch = 0;
    const LinFiles *f = lin_files(technique, &nch);
    if (!f || channel < 0 || channel >= nch) return nullptr;
    return td ? f[channel].td : f[channel].spec;
}

extern "C" int nise_linear(nise_ctx *c, double *re_S, double *im_S, int max_channels, int *channels, int *samples) {
    if (!c || !re_S || !im_S || !channels || !samples) return nise_fail(c, NISE_ERR_ARG, "null argument");
    if (!c->loaded) return nise_fail(c, NISE_ERR_STATE, "no trajectory loaded");
    cudaSetDevice(c->p.device);
    nise_wait_all_frames(c, c->stream);  // energy records still in flight from the host
    const nise_params &p = c->p;
    const int tech = p.technique, N = c->n, tmax = p.tmax1;
    const LinSpec L = lin_spec(tech);
    if (L.nch == 0) return nise_fail(c, NISE_ERR_ARG, "technique is not one of LD, Raman, SFG, DOS, CD");
    if (max_channels < L.nch) return nise_fail(c, NISE_ERR_ARG, "%d response channels needed", L.nch);
    if (L.alpha && !c->d_alpha) return nise_fail(c, NISE_ERR_IO, "Raman/SFG need the Alphafile records");
    if (L.pos && !c->d_pos) return nise_fail(c, NISE_ERR_IO, "CD needs the Positionfile records");
    if (L.alpha && p.doubles != 0)  // read_alpha (read_trajectory.c:385-397)
        return nise_fail(c, NISE_ERR_UNSUPPORTED, "Doubles not equal to zero, Raman 1D does not support double excited states");
    // determine_samples (NISE_subs.c:197-221) and the end checks of the technique files
    int n_samples = (p.length - tmax - 1) / p.sample + 1;
    if (n_samples <= 0) return nise_fail(c, NISE_ERR_ARG, "Insufficient data to calculate spectrum.");
    int end = p.end == 0 ? n_samples : p.end, begin = p.begin;
    if (end > n_samples) return nise_fail(c, NISE_ERR_ARG, "Endpoint larger than number of samples was specified.");
    if (begin < 0 || begin >= end) return nise_fail(c, NISE_ERR_ARG, "BeginPoint must be below EndPoint");
    const int count = end - begin;
    *channels = L.nch;
    *samples = end;  // every technique file divides by `samples`, which equals end after its loop
    const long fmin = (long)begin * p.sample, fmax = (long)(end - 1) * p.sample + tmax - 1;
    int rc;
    if (fmax >= c->e_frames)
        return nise_fail(c, NISE_ERR_IO, "Hamiltonian trajectory file to short, could not fill buffer!!!");
    if (L.dipoles && (rc = nise_check_frames(c, fmax))) return rc;
    if (L.alpha && fmax >= c->al_frames)
        return nise_fail(c, NISE_ERR_IO, "Polarizability trajectory file to short, could not fill buffer!!!");
    if (L.pos && p.hamiltonian != NISE_HAM_COUPLING && fmax >= c->pos_frames)
        return nise_fail(c, NISE_ERR_IO, "Position trajectory file to short, could not fill buffer!!!");
    c->launches = 0;
    cudaEventRecord(c->ev0, c->stream);
    DevTraj T = nise_devtraj(c);
    if (!L.singleshift) {  // read_He / read_Dia: no SingleShift
        T.shift_ptr = nullptr;
        T.nshift = 0;
    }
    LinJob J{};
    SinglesBufs SB;
    const long nf = std::max(1L, fmax - fmin);  // frames propagated through: [fmin, fmax)
    if ((rc = nise_singles_tables(c, T, fmin, nf, L.singleshift, false, J, SB))) return rc;
    J.T = T;
    J.tech = tech;
    J.sample = p.sample;
    J.tmax = tmax;
    J.nvec = L.nvec_fixed + L.nvec_per_site * N;
    J.nread = L.nread;
    J.alpha = c->d_alpha;
    J.al_words = 1 + 6L * N;
    J.pos = c->d_pos;
    J.pos_words = 1 + 3L * N + 3L * N * p.doubles;
    // start points per launch: the per-vector read-outs within ~1 GB
    const size_t per_sample = sizeof(double2) * (size_t)J.nvec * J.nread * tmax;
    int chunk = (int)std::max<size_t>(1, ((size_t)1 << 30) / per_sample);
    if (chunk > count) chunk = count;
    if (p.launch_mode == NISE_PLAIN) chunk = 1;
    DevBuf<double2> part, out;
    if ((rc = part.alloc(c, per_sample / sizeof(double2) * chunk)) || (rc = out.alloc(c, (size_t)L.nch * tmax)))
        return rc;
    J.part = part.p;
    cudaEventRecord(c->evk0, c->stream);
    for (int s0 = begin; s0 < end; s0 += chunk) {
        J.begin = s0;
        J.S = std::min(chunk, end - s0);
        int e = p.precision == NISE_FP32 ? run_lin<float>(J, out.p, L.nch, s0 == begin, c->stream)
                                         : run_lin<double>(J, out.p, L.nch, s0 == begin, c->stream);
        if ((rc = nise_cuda(c, e, "linear technique kernels"))) return rc;
        c->launches += 2;
    }
    cudaEventRecord(c->evk1, c->stream);
    std::vector<double2> h((size_t)L.nch * tmax);
    cudaMemcpyAsync(h.data(), out.p, sizeof(double2) * h.size(), cudaMemcpyDeviceToHost, c->stream);
    cudaEventRecord(c->ev1, c->stream);
    if ((rc = nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "linear technique"))) return rc;
    nise_collect_timing(c);
    for (size_t k = 0; k < h.size(); k++) {
        re_S[k] = h[k].x;
        im_S[k] = h[k].y;
    }
    c->last_flops = 0;
    c->last_bytes = (double)(fmax - fmin + 1) * 4 * (p.hamiltonian == NISE_HAM_COUPLING ? N : c->nn2);
    return NISE_OK;
}
