// Linear techniques besides absorption on one GPU: linear dichroism
// (calc_LD.c:15-283), Raman (raman.c:15-290), SFG (sfg.c:15-278), density of
// states (calc_DOS.c:15-222), circular dichroism (calc_CD.c:15-377) and
// luminescence (luminescence.c:17-240).
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
//   Lum    3 vectors rho mu_x(ti), rho the equilibrium density matrix at the
//          Temperature (below); read-out mu_x(tj); channels total, x, y, z
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
#include "eigen.h"
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
    const double *init;                // Lum: weighted initial vectors [sample - init_begin][3][n]
    int init_begin;
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
    case NISE_TECH_LUM: return {3, 0, 1, 4, 1, 1, 0, 0};  // read_Hamiltonian: SingleShift applies
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

// Initial value of site i of vector v of start point s (chunk-relative) at
// the start frame ti.
__device__ __forceinline__ double lin_init(const LinJob &J, int s, int v, long ti, int i) {
    const int n = J.n;
    switch (J.tech) {
    case NISE_TECH_LUM: return J.init[((size_t)(J.begin + s - J.init_begin) * 3 + v) * n + i];
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
        if (J.tech == NISE_TECH_LD || J.tech == NISE_TECH_LUM) m = traj_mu(J.T, t, v, i);
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
        z.x = (R)lin_init(J, s, v, ti, i);
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
    case NISE_TECH_LUM:                                               // luminescence.c:166-169
        return ch == 0 || ch == v + 1 ? 1.0 : 0.0;
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

// ---------------------------------------------------------------- luminescence
// The reference weights mu_x(ti) by the equilibrium density matrix before the
// propagation (luminescence.c:140-146), with the Hamiltonian the program read
// last: for component 0 of a start point the last frame of the previous start
// point (ti - Samplerate + tmax1 - 1), for components 1 and 2 the last frame
// of this one (ti + tmax1 - 1), and before the first read the coupling frame of
// HamiltonianType Coupling (read_coupling) or zeros.  A work item names the
// start point, the component and where its Hamiltonian comes from.
struct LumItem {
    int s, x;  // start point (absolute), dipole component
    long q;    // eigen slot (exact) or frame (imaginary time); -1 the initial Hamiltonian, -2 zeros
};

// Fixed-order sum over the CTA (every thread gets the total).
__device__ double lum_block_sum(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0;
    for (int w = 0; w < nw; w++) t += red[w];
    return t;
}

// Exact weights (bltz_weight, luminescence.c:246-314): rho mu = V c V^T mu / Q
// with c_k = exp(-e_k / kT) from the FP64 eigendecomposition of the item's
// Hamiltonian (V in launch_eig_any's layout: [a][k] up to NISE_EIG_MAX_N
// sites, [k][a] above), Q = sum_k c_k.  The weights are formed relative to the
// lowest eigenvalue (the same ratios, no overflow); Q is summed from zero (the
// reference leaves it uninitialised).  One CTA per item; out in FP64.
template <bool LARGE>
__global__ void k_lum_exact(DevTraj T, int n, int sample, int begin, const double *V, const double *w,
                            const LumItem *items, float kBT, double *init) {
    extern __shared__ double lsh[];
    double *proj = lsh, *c = lsh + n, *red = c + n;
    const LumItem it = items[blockIdx.x];
    const long ti = (long)it.s * sample;
    double *out = init + ((size_t)(it.s - begin) * 3 + it.x) * n;
    if (it.q == -2) {  // no Hamiltonian read yet: all weights 1, rho = I / n
        for (int a = threadIdx.x; a < n; a += blockDim.x) out[a] = (double)traj_mu(T, ti, it.x, a) / n;
        return;
    }
    const size_t slot = it.q < 0 ? 0 : (size_t)it.q;
    const double *e = w + slot * n, *Vs = V + slot * n * n;
    auto Vak = [&](int a, int k) { return LARGE ? Vs[(size_t)k * n + a] : Vs[(size_t)a * n + k]; };
    double emin = 1e300;
    for (int k = threadIdx.x; k < n; k += blockDim.x) emin = fmin(emin, e[k]);
    for (int o = 16; o > 0; o >>= 1) emin = fmin(emin, __shfl_xor_sync(0xffffffffu, emin, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = emin;
    __syncthreads();
    emin = red[0];
    for (int q = 1; q < (int)(blockDim.x >> 5); q++) emin = fmin(emin, red[q]);
    double part = 0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        c[k] = exp(-(e[k] - emin) / (double)kBT);
        double pk = 0;
        for (int a = 0; a < n; a++) pk += Vak(a, k) * (double)traj_mu(T, ti, it.x, a);
        proj[k] = pk;
    }
    for (int k = threadIdx.x; k < n; k += blockDim.x) part += c[k];
    const double Q = lum_block_sum(part, red + 32);
    __syncthreads();
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
        double acc = 0;
        for (int k = 0; k < n; k++) acc += Vak(a, k) * c[k] * proj[k];
        out[a] = acc / Q;
    }
}

// Imaginary-time weights (bltz_weight_itime, luminescence.c:318-409), the
// reference's float and double operations in FP32 mode: per step the
// diagonal half-factors exp(-H_aa f / 2), the couplings |J| > Couplingcut in
// lexicographic order as pairs (cosh, -sinh)(J f), the half-factors again,
// f = 1 / (m kT); the result scaled back to the initial norm.  Thread per
// item, two rows of n scratch values each.
template <typename R>
__global__ void k_lum_itime(DevTraj T, DevTraj T0, int n, int sample, int begin, int m, float kBT, int singleshift,
                            const LumItem *items, int nitems, R *scratch, double *init) {
    typedef Ar<R> A;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nitems) return;
    const LumItem it = items[g];
    const long ti = (long)it.s * sample;
    R *cr = scratch + (size_t)g * 2 * n, *reU = cr + n;
    const bool zero = it.q == -2;
    const DevTraj &H = it.q == -1 ? T0 : T;
    const long q = it.q < 0 ? 0 : it.q;
    const bool ss = it.q >= 0 && singleshift;
    const R f = (R)(1.0 / (double)((float)m * kBT));
    R norm = 0;
    for (int a = 0; a < n; a++) {
        cr[a] = (R)traj_mu(T, ti, it.x, a);
        norm = A::add(norm, A::mul(cr[a], cr[a]));
        const double h = zero ? 0.0 : (double)traj_diag(H, q, a, ss);
        reU[a] = (R)exp(-0.5 * h * (double)f);
    }
    for (int i = 0; i < m; i++) {
        for (int a = 0; a < n; a++) cr[a] = A::mul(cr[a], reU[a]);
        if (!zero)
            for (int a = 0; a < n; a++)
                for (int b = a + 1; b < n; b++) {
                    R J = (R)traj_coupling(H, q, a, b);
                    if (!(fabs((double)J) > (double)H.cut)) continue;
                    J = A::mul(-J, f);
                    const R eJ = (R)(exp((double)J) * 0.5), emJ = (R)(exp(-(double)J) * 0.5);
                    const R sih = A::sub(eJ, emJ), coh = A::add(eJ, emJ);
                    const R c1 = A::add(A::mul(coh, cr[a]), A::mul(sih, cr[b]));
                    const R c2 = A::add(A::mul(coh, cr[b]), A::mul(sih, cr[a]));
                    cr[a] = c1;
                    cr[b] = c2;
                }
        for (int a = 0; a < n; a++) cr[a] = A::mul(cr[a], reU[a]);
    }
    R Q = 0;
    for (int a = 0; a < n; a++) Q = A::add(Q, A::mul(cr[a], cr[a]));
    const R iQ = (R)sqrt((double)(norm / Q));
    double *out = init + ((size_t)(it.s - begin) * 3 + it.x) * n;
    for (int a = 0; a < n; a++) out[a] = (double)A::mul(cr[a], iQ);
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

// The weighted initial vectors of start points [begin, end) of a
// luminescence job: init[s - begin][x][n] (FP64).
int lum_weights(nise_ctx *c, const DevTraj &T, int begin, int end, int singleshift, DevBuf<double> &init) {
    const nise_params &p = c->p;
    const int N = c->n, tmax = p.tmax1, count = end - begin;
    if (!(p.temperature > 0)) return nise_fail(c, NISE_ERR_ARG, "Temperature must be positive");
    if (p.imag_steps < 0) return nise_fail(c, NISE_ERR_ARG, "ImaginaryTimesteps must not be negative");
    const float kBT = p.temperature * 0.695;  // Kelvin to cm^-1, in float (luminescence.c:256)
    int rc;
    if ((rc = init.alloc(c, (size_t)count * 3 * N))) return rc;
    cudaStream_t st = c->stream;
    // the Hamiltonian before the first read: the coupling frame of HamiltonianType
    // Coupling as one Full record (its diagonal is shifted already), else zeros
    const bool coup = p.hamiltonian == NISE_HAM_COUPLING;
    DevBuf<float> h0;
    DevTraj T0 = T;
    if (coup) {
        if ((rc = h0.alloc(c, 1 + (size_t)c->nn2))) return rc;
        cudaMemsetAsync(h0.p, 0, sizeof(float), st);
        cudaMemcpyAsync(h0.p + 1, c->d_hc, sizeof(float) * c->nn2, cudaMemcpyDeviceToDevice, st);
        T0.energy = h0.p;
        T0.e_words = 1 + c->nn2;
        T0.e_frames = 1;
        T0.full = 1;
        T0.shifte = 0;
        T0.shift_ptr = nullptr;
        T0.nshift = 0;
    }
    auto last_frame = [&](int s) { return (long)s * p.sample + tmax - 1; };
    const long initial = coup ? -1 : -2;
    if (p.imag_steps > 0) {
        std::vector<LumItem> items;
        for (int s = begin; s < end; s++)
            for (int x = 0; x < 3; x++)
                items.push_back({s, x, x == 0 ? (s == begin ? initial : last_frame(s - 1)) : last_frame(s)});
        DevBuf<LumItem> dit;
        DevBuf<char> scr;
        const size_t rsz = p.precision == NISE_FP32 ? sizeof(float) : sizeof(double);
        if ((rc = dit.upload(c, items)) || (rc = scr.alloc(c, rsz * 2 * (size_t)N * items.size()))) return rc;
        const int ni = (int)items.size(), B = 64;
        if (p.precision == NISE_FP32)
            k_lum_itime<float><<<(ni + B - 1) / B, B, 0, st>>>(T, T0, N, p.sample, begin, p.imag_steps, kBT,
                                                              singleshift, dit.p, ni, (float *)scr.p, init.p);
        else
            k_lum_itime<double><<<(ni + B - 1) / B, B, 0, st>>>(T, T0, N, p.sample, begin, p.imag_steps, kBT,
                                                               singleshift, dit.p, ni, (double *)scr.p, init.p);
        c->launches++;
        return nise_cuda(c, (int)cudaGetLastError(), "luminescence weights");
    }
    // exact weights: eigendecompositions of the frames last_frame(s), chunk by chunk
    const size_t per = sizeof(double) * (size_t)N * N * (N > NISE_EIG_MAX_N ? 2 : 1);
    const long FC = std::max(1L, std::min((long)count, (long)(((size_t)1 << 30) / per)));
    std::vector<long> frames(count);
    for (int i = 0; i < count; i++) frames[i] = last_frame(begin + i);
    // items in chunk order: for the start point of slot i, components 1 and 2;
    // for the next start point, component 0
    std::vector<LumItem> items;
    std::vector<int> chunk_at;
    for (long q0 = 0; q0 < count; q0 += FC) {
        chunk_at.push_back((int)items.size());
        for (long i = 0; i < std::min(FC, count - q0); i++) {
            const int s = begin + (int)(q0 + i);
            items.push_back({s, 1, i});
            items.push_back({s, 2, i});
            if (s + 1 < end) items.push_back({s + 1, 0, i});
        }
    }
    chunk_at.push_back((int)items.size());
    items.push_back({begin, 0, coup ? 0 : -2});  // the first start point's component 0
    DevBuf<double> V, w, A;
    DevBuf<int> status;
    DevBuf<long> fr, fr0;
    DevBuf<LumItem> dit;
    if ((rc = fr.upload(c, frames)) || (rc = fr0.upload(c, std::vector<long>(1, 0))) || (rc = dit.upload(c, items)) ||
        (rc = V.alloc(c, (size_t)FC * N * N)) || (rc = w.alloc(c, (size_t)FC * N)) ||
        (rc = A.alloc(c, eig_any_ws_doubles(N, FC))) || (rc = status.alloc(c, 1)))
        return rc;
    cudaMemsetAsync(status.p, 0, sizeof(int), st);
    const bool large = N > NISE_EIG_MAX_N;
    const size_t sm = sizeof(double) * (2 * (size_t)N + 64);
    auto weigh = [&](int i0, int i1) -> int {
        if (i1 <= i0) return 0;
        if (large) {
            cudaFuncSetAttribute(k_lum_exact<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_lum_exact<true><<<i1 - i0, 256, sm, st>>>(T, N, p.sample, begin, V.p, w.p, dit.p + i0, kBT, init.p);
        } else {
            cudaFuncSetAttribute(k_lum_exact<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_lum_exact<false><<<i1 - i0, 256, sm, st>>>(T, N, p.sample, begin, V.p, w.p, dit.p + i0, kBT, init.p);
        }
        c->launches++;
        return (int)cudaGetLastError();
    };
    EigJob EJ;
    EJ.T = T;
    EJ.n = N;
    EJ.singleshift = singleshift && c->nshift > 0;
    for (size_t k = 0; k + 1 < chunk_at.size(); k++) {
        const long q0 = (long)k * FC, m = std::min(FC, count - q0);
        if ((rc = nise_cuda(c, launch_eig_any(EJ, fr.p + q0, m, V.p, w.p, A.p, status.p, st), "eigensolver")) ||
            (rc = nise_cuda(c, weigh(chunk_at[k], chunk_at[k + 1]), "luminescence weights")))
            return rc;
        c->launches++;
    }
    if (coup) {  // the coupling frame, diagonalised like a frame of its own
        EigJob E0 = EJ;
        E0.T = T0;
        E0.singleshift = 0;
        if ((rc = nise_cuda(c, launch_eig_any(E0, fr0.p, 1, V.p, w.p, A.p, status.p, st), "eigensolver")))
            return rc;
        c->launches++;
    }
    if ((rc = nise_cuda(c, weigh((int)items.size() - 1, (int)items.size()), "luminescence weights"))) return rc;
    int hst = 0;
    cudaMemcpyAsync(&hst, status.p, sizeof(int), cudaMemcpyDeviceToHost, st);
    if ((rc = nise_cuda(c, (int)cudaStreamSynchronize(st), "luminescence weights"))) return rc;
    if (hst) return nise_fail(c, NISE_ERR_DEVICE, "the eigensolver did not converge on a frame");
    return NISE_OK;
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
    // luminescence.c:223-234: a time-domain file for the total only
    static const LinFiles lum[] = {{"TD_Lum.dat", "Luminescence.dat"},
                                   {nullptr, "Luminescence_x.dat"},
                                   {nullptr, "Luminescence_y.dat"},
                                   {nullptr, "Luminescence_z.dat"}};
    switch (tech) {
    case NISE_TECH_LD: *nch = 1; return ld;
    case NISE_TECH_RAMAN: *nch = 2; return raman;
    case NISE_TECH_SFG: *nch = 2; return sfg;
    case NISE_TECH_DOS: *nch = 1; return dos;
    case NISE_TECH_CD: *nch = 1; return cd;
    case NISE_TECH_LUM: *nch = 4; return lum;
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
    if (L.nch == 0)
        return nise_fail(c, NISE_ERR_ARG, "technique is not one of LD, Raman, SFG, DOS, CD, Luminescence");
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
    // SingleShift only where the technique reads through read_Hamiltonian and a
    // SingleShiftfile was given (without one there is no per-site table to read)
    const int singleshift = L.singleshift && c->nshift > 0;
    if ((rc = nise_singles_tables(c, T, fmin, nf, singleshift, false, J, SB))) return rc;
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
    DevBuf<double> linit;
    if (tech == NISE_TECH_LUM) {
        if ((rc = lum_weights(c, T, begin, end, singleshift, linit))) return rc;
        J.init = linit.p;
        J.init_begin = begin;
    }
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
