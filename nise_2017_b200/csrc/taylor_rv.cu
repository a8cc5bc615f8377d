// Linear absorption with the exact propagator exp(-i H f) for static
// couplings (HamiltonianType Coupling with Propagation Sparse, Threshold 0,
// or Diagonal; the reference's propagate_vec_DIA, propagate.c:60-125, called
// from the sample loop of absorption.c:119-145), FP32, as a sparse Taylor
// series.  Row-owner layout:
//
//  - a CTA propagates 8 vectors (consecutive (start point, polarisation)
//    pairs) through all their steps; their state lives in shared memory as
//    rows of 8 complex numbers (64 bytes per site), in two buffers: Taylor
//    term k is gathered from one and written to the other, so a term costs
//    one CTA barrier;
//  - a lane owns one site row and two of the vectors (lane = 4 * r + c: row r
//    of an 8-row slice, vectors 2c and 2c+1), so one coupling entry and one
//    16-byte gather feed four FMAs;
//  - the 8 rows of a slice alternate in parity and every row lists its
//    other-parity neighbours first, so the two rows of a quarter-warp gather
//    rows of opposite parity, which sit on opposite halves of the banks;
//  - couplings are stored in slot triples, one 16-byte entry per row: the
//    three weights and the three neighbours' 10-bit row indices, so one
//    load (8 rows: one shared-memory wavefront) serves three slots;
//  - the slices are dealt to the warps longest first (each warp's total
//    slot count nearly equal: the CTA barrier waits for the slowest warp);
//  - the diagonal records of the frames the CTA's vectors need next are
//    staged into shared memory with bulk copies (cp.async.bulk, completion on
//    an mbarrier) one step ahead; the dipoles are static (read_coupling,
//    read_trajectory.c:61-67) and read through the L1 cache.
//
// Series order per frame from k_prep_taylor (remainder below FP32 unit
// roundoff).
#include <cstdint>

#include "common.cuh"
#include "engine.h"

namespace {

constexpr int kRvG = 8;           // vectors per CTA
constexpr int kRvSlots = 4;       // 8 consecutive vectors span at most 4 start points
constexpr int kRvMaxIT = 8;       // slices per warp
constexpr unsigned kRvSpin = 1u << 20;  // bound on the mbarrier waits

struct RvLayout {
    size_t cur, tri, tptr, rows, wsl, dg, red, mbar, total;
    int dgw;  // words per staged diagonal record (16-byte multiple)
};

__host__ __device__ inline size_t rv_al(size_t x) { return (x + 15) & ~(size_t)15; }

// Shared-memory layout for n sites, ntg slot-triple groups (8 rows each), nsl
// slices and nw warps.
__host__ __device__ inline RvLayout rv_layout(int n, int ntg, int nsl, int nw) {
    RvLayout L;
    size_t o = 0;
    L.cur = o;
    o = rv_al(o + (size_t)2 * n * 64);
    L.tri = o;
    o = rv_al(o + (size_t)(ntg + 1) * 8 * 16);  // + one group of slack for the prefetch
    L.tptr = o;
    o = rv_al(o + (size_t)(nsl + 1) * 4);
    L.rows = o;
    o = rv_al(o + (size_t)nsl * 8 * 4);
    L.wsl = o;
    o = rv_al(o + (size_t)nw * kRvMaxIT * 4);
    L.dgw = (n + 6) & ~3;  // a record shifted by up to 3 words, rounded up to 4 words
    L.dg = o;
    o = rv_al(o + (size_t)kRvSlots * L.dgw * 4);
    L.red = o;
    o = rv_al(o + (size_t)nw * kRvG * 2 * 8);
    L.mbar = o;
    o = rv_al(o + 16);
    L.total = o;
    return L;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *m, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *m, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *m, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(m)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of an mbarrier.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *m, uint32_t parity) {
    for (unsigned it = 0; it < kRvSpin; it++)
        if (mbar_try_wait(m, parity)) return true;
    return false;
}

// Bulk copy global -> this CTA's shared memory, completion counted on m.
// Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *m) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(m))
                 : "memory");
}

// First word (16-byte aligned) and lead of the diagonal record of frame t:
// the record's data start at word t * e_words + 1 of the energy image.
__device__ __forceinline__ long rv_rec_word(const DevTraj &T, long t, int *lead) {
    const long w0 = t * T.e_words + 1, a = w0 & ~3L;
    *lead = (int)(w0 - a);
    return a;
}

// Stage the diagonal records of the CTA's start points at step t1 (one
// thread).
__device__ __forceinline__ void rv_stage(const DevTraj &T, const AbsJob &J, int sfirst, int nslot, int t1, int n,
                                         float *dgbuf, int dgw, uint64_t *m) {
    uint32_t bytes = 0;
    for (int k = 0; k < nslot; k++) {
        int lead;
        rv_rec_word(T, (long)(J.begin + sfirst + k) * J.sample + t1, &lead);
        bytes += (uint32_t)(((lead + n) + 3) & ~3) * 4;
    }
    // the buffer was last read through the generic proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(m, bytes);
    for (int k = 0; k < nslot; k++) {
        int lead;
        const long a = rv_rec_word(T, (long)(J.begin + sfirst + k) * J.sample + t1, &lead);
        bulk_g2s(dgbuf + (size_t)k * dgw, T.energy + a, (uint32_t)(((lead + n) + 3) & ~3) * 4, m);
    }
}

// CHEB: the Chebyshev expansion of exp(-i H f) instead of the Taylor series
// (tables from k_prep_cheb: per frame the centre c of the diagonal range,
// 1/R with R >= ||H - c||_2 by Gershgorin, and the coefficients
// c_0 = J_0(fR), c_k = 2 (-i)^k J_k(fR), times the phase exp(-i f c); order by
// the tail of the Bessel coefficients).  With H' = (H - c)/R: T_0 = psi,
// T_1 = H' psi, T_k = 2 H' T_(k-1) - T_(k-2); the result is sum_k c_k T_k.
// Each vector uses its own frame's c, R and coefficients.
template <int IT, int NT, bool CHEB>
__global__ void __launch_bounds__(NT, 1)
    k_abs_taylor_rv(DevTraj T, TaylorPlan P, AbsJob J, double2 *resp, int v0, int nvec, const int *__restrict__ wsl_g) {
    constexpr int NW = NT / 32;
    extern __shared__ __align__(16) unsigned char sm[];
    const int n = P.n, nsl = P.ell8_nslices, ntg = P.ell8_ntg;
    const RvLayout L = rv_layout(n, ntg, nsl, NW);
    float4 *cur = (float4 *)(sm + L.cur);  // [2][n][4]
    float4 *tri = (float4 *)(sm + L.tri);
    int *tptr = (int *)(sm + L.tptr);
    int *rows = (int *)(sm + L.rows);
    int *wsl = (int *)(sm + L.wsl);
    float *dg = (float *)(sm + L.dg);
    double *red = (double *)(sm + L.red);
    uint64_t *mbar = (uint64_t *)(sm + L.mbar);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r = lane >> 2, c = lane & 3;

    for (int e = tid; e < 8 * ntg; e += NT) tri[e] = P.ell8_tri[e];
    for (int e = tid; e < 8; e += NT) tri[8 * ntg + e] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int e = tid; e <= nsl; e += NT) tptr[e] = P.ell8_tptr[e];
    for (int e = tid; e < 8 * nsl; e += NT) rows[e] = P.ell8_rows[e];
    for (int e = tid; e < NW * kRvMaxIT; e += NT) wsl[e] = wsl_g[e];
    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }

    // the CTA's vectors: vv = v0 + vb + g, start point J.begin + vv / 3, polarisation vv % 3
    const int vb = blockIdx.x * kRvG;
    const int sfirst = (v0 + vb) / 3;
    const int nslot = (v0 + min(vb + kRvG, nvec) - 1) / 3 - sfirst + 1;
    int x0, x1, s0, s1;
    {
        int v = vb + 2 * c;
        int vv = v0 + (v < nvec ? v : vb);
        x0 = vv % 3;
        s0 = vv / 3 - sfirst;
        v = vb + 2 * c + 1;
        vv = v0 + (v < nvec ? v : vb);
        x1 = vv % 3;
        s1 = vv / 3 - sfirst;
    }
    const float *mu0 = T.mu_static + x0 * n, *mu1 = T.mu_static + x1 * n;

    float4 psi[IT];
    float d0[IT], d1[IT];
    __syncthreads();
    // site of this lane's row in its it-th slice (n: none)
    auto site = [&](int it) {
        const int sl = wsl[warp * kRvMaxIT + it];
        return sl >= 0 ? rows[8 * sl + r] : n;
    };
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const int i = site(it);
        psi[it] = i < n ? make_float4(__ldg(mu0 + i), 0.f, __ldg(mu1 + i), 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
        d0[it] = d1[it] = 0.f;
    }
    if (tid == 0 && J.tmax > 1) rv_stage(T, J, sfirst, nslot, 0, n, dg, L.dgw, &mbar[0]);

    for (int t1 = 0; t1 < J.tmax; t1++) {
        // response of step t1 (absorption.c:128-131): mu(tj) . psi, FP32
        // products summed in FP64 (rows in slice order, then lanes, then warps)
        double re0 = 0, im0 = 0, re1 = 0, im1 = 0;
#pragma unroll
        for (int it = 0; it < IT; it++) {
            const int i = site(it);
            if (i < n) {
                const float m0 = __ldg(mu0 + i), m1 = __ldg(mu1 + i);
                re0 += (double)(m0 * psi[it].x);
                im0 += (double)(m0 * psi[it].y);
                re1 += (double)(m1 * psi[it].z);
                im1 += (double)(m1 * psi[it].w);
            }
        }
        for (int o = 4; o < 32; o <<= 1) {
            re0 += __shfl_xor_sync(0xffffffffu, re0, o);
            im0 += __shfl_xor_sync(0xffffffffu, im0, o);
            re1 += __shfl_xor_sync(0xffffffffu, re1, o);
            im1 += __shfl_xor_sync(0xffffffffu, im1, o);
        }
        if (r == 0) {
            double *q = red + (size_t)(warp * kRvG + 2 * c) * 2;
            q[0] = re0;
            q[1] = im0;
            q[2] = re1;
            q[3] = im1;
        }
        __syncthreads();
        if (tid < kRvG && vb + tid < nvec) {
            double sr = 0, si = 0;
            for (int w = 0; w < NW; w++) {
                sr += red[(size_t)(w * kRvG + tid) * 2];
                si += red[(size_t)(w * kRvG + tid) * 2 + 1];
            }
            resp[(size_t)(v0 + vb + tid) * J.tmax + t1] = make_double2(sr, si);
        }
        if (t1 == J.tmax - 1) break;

        // the frame's diagonal, staged one step ahead (use t1 of the barrier)
        const bool ok = mbar_wait_bounded(&mbar[0], t1 & 1);
        if (!__syncthreads_and(ok)) {
            if (tid == 0) atomicExch(P.err, 1);
            mbar_wait_bounded(&mbar[0], t1 & 1);  // let the copy in flight land
            return;
        }
        {
            int lead0, lead1;
            rv_rec_word(T, (long)(J.begin + sfirst + s0) * J.sample + t1, &lead0);
            rv_rec_word(T, (long)(J.begin + sfirst + s1) * J.sample + t1, &lead1);
            const float *r0 = dg + (size_t)s0 * L.dgw + lead0, *r1 = dg + (size_t)s1 * L.dgw + lead1;
            // Chebyshev: the diagonal relative to each frame's centre c_t
            float c0 = 0.f, c1 = 0.f;
            if constexpr (CHEB) {
                c0 = __ldg(P.cheb_center + (long)(J.begin + sfirst + s0) * J.sample + t1 - P.f0);
                c1 = __ldg(P.cheb_center + (long)(J.begin + sfirst + s1) * J.sample + t1 - P.f0);
            }
#pragma unroll
            for (int it = 0; it < IT; it++) {
                const int i = site(it);
                if (i < n) {
                    float h0 = __fsub_rn(r0[i], T.shifte), h1 = __fsub_rn(r1[i], T.shifte);
                    if (P.singleshift) {  // read_Hamiltonian -> apply_singleshift (hamshift.c:59-66)
                        for (int e = T.shift_ptr[i]; e < T.shift_ptr[i + 1]; e++) {
                            h0 = __fadd_rn(__fmul_rn(h0, T.shift_ab[2 * e]), T.shift_ab[2 * e + 1]);
                            h1 = __fadd_rn(__fmul_rn(h1, T.shift_ab[2 * e]), T.shift_ab[2 * e + 1]);
                        }
                    }
                    d0[it] = CHEB ? __fsub_rn(h0, c0) : h0;
                    d1[it] = CHEB ? __fsub_rn(h1, c1) : h1;
                    cur[(size_t)i * 4 + c] = psi[it];  // term 0 into buffer 0
                }
            }
        }
        int K = 1;
        for (int k = 0; k < nslot; k++) K = max(K, P.order[(long)(J.begin + sfirst + k) * J.sample + t1 - P.f0]);
        // Chebyshev: each vector's frame scale and coefficients; the result
        // starts at c_0 T_0
        const long fr0 = (long)(J.begin + sfirst + s0) * J.sample + t1 - P.f0;
        const long fr1 = (long)(J.begin + sfirst + s1) * J.sample + t1 - P.f0;
        float ir0 = 0.f, ir1 = 0.f;
        const float2 *cc0 = nullptr, *cc1 = nullptr;
        if constexpr (CHEB) {
            ir0 = __ldg(P.cheb_inv_r + fr0);
            ir1 = __ldg(P.cheb_inv_r + fr1);
            cc0 = P.cheb_coef + fr0 * (NISE_CHEB_KMAX + 1);
            cc1 = P.cheb_coef + fr1 * (NISE_CHEB_KMAX + 1);
            const float2 q0 = __ldg(cc0), q1 = __ldg(cc1);
#pragma unroll
            for (int it = 0; it < IT; it++) {
                const float4 z = psi[it];
                psi[it] = make_float4(q0.x * z.x - q0.y * z.y, q0.x * z.y + q0.y * z.x, q1.x * z.z - q1.y * z.w,
                                      q1.x * z.w + q1.y * z.z);
            }
        }
        __syncthreads();  // term 0 written; the staged records and the response partials read
        if (tid == 0 && t1 + 1 < J.tmax - 1) rv_stage(T, J, sfirst, nslot, t1 + 1, n, dg, L.dgw, &mbar[0]);
        for (int k = 1; k <= K; k++) {
            const float cf = (float)(J.f / k);
            float2 q0 = make_float2(0.f, 0.f), q1 = q0;
            if constexpr (CHEB) {
                q0 = __ldg(cc0 + k);
                q1 = __ldg(cc1 + k);
            }
            const float4 *src = cur + (size_t)((k - 1) & 1) * n * 4;
            float4 *dst = cur + (size_t)(k & 1) * n * 4;
            const char *srcc = (const char *)(src + c);
#pragma unroll
            for (int it = 0; it < IT; it++) {
                const int sl = wsl[warp * kRvMaxIT + it];
                if (sl < 0) continue;
                const int i = rows[8 * sl + r];
                const float4 own = i < n ? src[(size_t)i * 4 + c] : make_float4(0.f, 0.f, 0.f, 0.f);
                float a0 = d0[it] * own.x, b0 = d0[it] * own.y;
                float a1 = d1[it] * own.z, b1 = d1[it] * own.w;
                // slot triples; the next triple is loaded one iteration ahead
                // (past the slice it is unused; one group of slack)
                const int p1 = tptr[sl + 1];
                int p = tptr[sl];
                float4 w = tri[8 * p + r];
                for (; p < p1; p++) {
                    const float4 nw = tri[8 * (p + 1) + r];
                    const uint32_t ix = __float_as_uint(w.w);
                    const float4 za = *(const float4 *)(srcc + ((ix & 0x3ffu) << 6));
                    const float4 zb = *(const float4 *)(srcc + (((ix >> 10) & 0x3ffu) << 6));
                    const float4 zc = *(const float4 *)(srcc + ((ix >> 20) << 6));
                    a0 += w.x * za.x;
                    b0 += w.x * za.y;
                    a1 += w.x * za.z;
                    b1 += w.x * za.w;
                    a0 += w.y * zb.x;
                    b0 += w.y * zb.y;
                    a1 += w.y * zb.z;
                    b1 += w.y * zb.w;
                    a0 += w.z * zc.x;
                    b0 += w.z * zc.y;
                    a1 += w.z * zc.z;
                    b1 += w.z * zc.w;
                    w = nw;
                }
                if (i < n) {
                    if constexpr (CHEB) {
                        // T_k = 2 (H/R) T_(k-1) - T_(k-2) (T_1 = (H/R) T_0); T_(k-2)
                        // of this row is in the buffer T_k replaces
                        float4 nx;
                        if (k == 1) {
                            nx = make_float4(ir0 * a0, ir0 * b0, ir1 * a1, ir1 * b1);
                        } else {
                            const float4 pv = dst[(size_t)i * 4 + c];
                            const float s0r = 2.f * ir0, s1r = 2.f * ir1;
                            nx = make_float4(s0r * a0 - pv.x, s0r * b0 - pv.y, s1r * a1 - pv.z, s1r * b1 - pv.w);
                        }
                        dst[(size_t)i * 4 + c] = nx;
                        psi[it].x += q0.x * nx.x - q0.y * nx.y;
                        psi[it].y += q0.x * nx.y + q0.y * nx.x;
                        psi[it].z += q1.x * nx.z - q1.y * nx.w;
                        psi[it].w += q1.x * nx.w + q1.y * nx.z;
                    } else {
                        // (-i)(f/k)(H t): the next term
                        const float4 nx = make_float4(cf * b0, -cf * a0, cf * b1, -cf * a1);
                        dst[(size_t)i * 4 + c] = nx;
                        psi[it].x += nx.x;
                        psi[it].y += nx.y;
                        psi[it].z += nx.z;
                        psi[it].w += nx.w;
                    }
                }
            }
            __syncthreads();
        }
    }
}

template <int IT, int NT, bool CHEB>
int run_rv1(const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp, int v0, int nvec, const int *wsl,
            cudaStream_t s) {
    const size_t smem = rv_layout(P.n, P.ell8_ntg, P.ell8_nslices, NT / 32).total;
    cudaError_t e =
        cudaFuncSetAttribute(k_abs_taylor_rv<IT, NT, CHEB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    k_abs_taylor_rv<IT, NT, CHEB><<<(nvec + kRvG - 1) / kRvG, NT, smem, s>>>(T, P, J, resp, v0, nvec, wsl);
    return (int)cudaGetLastError();
}

template <int IT, int NT>
int run_rv(const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp, int v0, int nvec, const int *wsl,
           cudaStream_t s) {
    if (P.cheb_coef) return run_rv1<IT, NT, true>(T, P, J, resp, v0, nvec, wsl, s);
    return run_rv1<IT, NT, false>(T, P, J, resp, v0, nvec, wsl, s);
}

}  // namespace

// Warps of the row-owner kernel's two launch shapes (768 and 1024 threads);
// the host deals the slices to each shape's warps.
const int kRvWarps[2] = {24, 32};

bool taylor_rv_fits(const DevTraj &T, const TaylorPlan &P) {
    if (!P.ell8_tri || !P.err || !T.mu_static || T.full || !P.static_j || P.n > 1024) return false;
    const int sh = P.rv_shape;
    if (sh < 0 || sh > 1 || !P.ell8_wsl[sh] || P.ell8_it[sh] > kRvMaxIT) return false;
    return rv_layout(P.n, P.ell8_ntg, P.ell8_nslices, kRvWarps[sh]).total <= 227 * 1024;
}

int launch_abs_taylor_rv(const DevTraj &T, const TaylorPlan &P, const AbsJob &J, double2 *resp, int v0, int nvec,
                         cudaStream_t s) {
    if (nvec <= 0) return 0;
    if (!taylor_rv_fits(T, P)) return (int)cudaErrorNotSupported;
    const int sh = P.rv_shape, it = P.ell8_it[sh];
    const int *wsl = P.ell8_wsl[sh];
    if (sh == 0) {
        if (it <= 4) return run_rv<4, 768>(T, P, J, resp, v0, nvec, wsl, s);
        if (it <= 6) return run_rv<6, 768>(T, P, J, resp, v0, nvec, wsl, s);
        return run_rv<8, 768>(T, P, J, resp, v0, nvec, wsl, s);
    }
    if (it <= 4) return run_rv<4, 1024>(T, P, J, resp, v0, nvec, wsl, s);
    if (it <= 6) return run_rv<6, 1024>(T, P, J, resp, v0, nvec, wsl, s);
    return run_rv<8, 1024>(T, P, J, resp, v0, nvec, wsl, s);
}
