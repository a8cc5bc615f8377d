// Eigen-route linear absorption with the one-step propagators applied on the
// tensor cores (FP32 mode).
//
// The reference applies U = V exp(-i e f) V^T to one vector at a time
// (propagate_vec_DIA, propagate.c:109-119) inside the sample loop of
// absorption.c:119-145.  Here the loop runs over frames (time-major): every
// vector in flight on frame t -- start points s with s*Samplerate <= t <
// s*Samplerate + tmax1, three polarisations each -- is a column of one state
// matrix X, and the step is one complex product Y = U_t X:
//
//   Y_r = U_r X_r - U_i X_i,   Y_i = U_i X_r + U_r X_i.
//
// k_tc_apply computes it with tcgen05.mma (kind::tf32) from shared-memory
// tiles: a CTA owns 128 rows of Y, its two accumulators (Y_r, Y_i) live in
// tensor memory, and the sites are taken 32 at a time (128-byte rows,
// 128-byte swizzle, K-major operands).  FP32 accuracy comes from splitting
// every operand into three tf32 pieces, x = x0 + x1 + x2 (11 significant bits
// each), and keeping the six products down to 2^-22 (x0y0, x0y1, x1y0, x1y1,
// x0y2, x2y0): the dropped terms are below 2^-33.  The tensor core adds the
// products of one instruction after aligning them and rounds toward zero, so
// the leading products of U_r X_r, U_i X_i, U_i X_r and U_r X_i each get an
// accumulator (no cancellation of large terms inside it), and the five
// correction products of Y_r and of Y_i two more, rounded at their own
// 2^-11 smaller scale; the six are combined in registers.  Measured against
// the per-start-point FP32 kernel: 1.2e-6 of the response over 48 steps
// (with everything in two accumulators 5e-6).  The -U_i X_i correction
// terms use the instruction descriptor's negate-A bit.  k_tc_resp starts the new vectors of
// frame t (X = mu_x(t)) and takes every active vector's response mu_x(t) . X
// (absorption.c:128-131: float products, FP64 sum in a fixed order).
// Start point s uses columns 3*(s mod S) .. +2, S = floor((tmax-1)/Samplerate)
// + 1 slots: a slot is free again before its next start point begins.
#include <algorithm>
#include <cstdint>

#include "common.cuh"
#include "engine.h"

namespace {

constexpr int kTcThreads = 256;
constexpr int kTcRows = 128;     // rows of Y per CTA (MMA M)
constexpr int kTcK = 32;         // sites per stage (one 128-byte row of tf32)
constexpr unsigned kTcSpin = 1u << 22;

// Tensor-memory columns for six accumulators of nc columns (a power of 2, >= 32).
__host__ __device__ constexpr uint32_t tmem_cols(int nc) {
    return 6 * nc <= 32 ? 32u : 6 * nc <= 64 ? 64u : 6 * nc <= 128 ? 128u : 6 * nc <= 256 ? 256u : 512u;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// x = p[0] + p[1] + p[2], each a tf32 value (round to nearest): 33
// significant bits, so the sum is x to well below FP32 rounding.
__device__ __forceinline__ void split3(float x, float p[3]) {
    p[0] = to_tf32(x);
    const float r = x - p[0];
    p[1] = to_tf32(r);
    p[2] = to_tf32(r - p[1]);
}

// 16 consecutive accumulator columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t v[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}

// Byte offset of element (row r, k) of a K-major tile with 128-byte rows and
// the 128-byte swizzle (16-byte chunk index XOR row mod 8); tiles start on
// 1024-byte boundaries.
__device__ __forceinline__ uint32_t sw128(int r, int k) {
    return (uint32_t)(r * 128 + ((((k >> 2) ^ (r & 7)) & 7) << 4) + ((k & 3) << 2));
}

// Shared-memory matrix descriptor (tcgen05): K-major, 128-byte swizzle,
// stride between 8-row groups 1024 bytes, leading offset 16 bytes (unused
// for swizzled K-major), descriptor version 1.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;              // leading byte offset 16 B (>> 4)
    d |= (uint64_t)(1024 >> 4) << 32;    // stride byte offset
    d |= (uint64_t)1 << 46;              // version
    d |= (uint64_t)2 << 61;              // 128-byte swizzle
    return d;
}

// Instruction descriptor: D f32, A and B tf32, both K-major, M = 128, N.
__host__ __device__ constexpr uint32_t make_idesc(int n, bool neg_a) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((neg_a ? 1u : 0u) << 13) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
        "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ bool mbar_try(uint64_t *m, uint32_t parity) {
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

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *m, uint32_t parity) {
    for (unsigned it = 0; it < kTcSpin; it++)
        if (mbar_try(m, parity)) return true;
    return false;
}

// Per-frame start and response: CTA per column of X (block 256 threads).
// X planes: xr, xi [cols][n].
__global__ void __launch_bounds__(256) k_tc_resp(DevTraj T, AbsJob J, int n, long t, int slots, float *xr, float *xi,
                                                 double2 *resp) {
    __shared__ double red[2][8];
    const int col = blockIdx.x, slot = col / 3, x = col % 3;
    // the start point of this slot active on frame t, if any
    const long tfirst = (long)J.begin * J.sample;
    const long rel = t - tfirst;                 // frames since the first start
    long q = rel / J.sample;                     // latest start point (relative) at or before t
    q -= ((q % slots) - slot + slots) % slots;   // the latest one using this slot
    if (q < 0 || q >= J.nsamp) return;
    const long t1 = rel - q * J.sample;
    if (t1 < 0 || t1 >= J.tmax) return;
    float *pr = xr + (size_t)col * n, *pi = xi + (size_t)col * n;
    double re = 0, im = 0;
    for (int a = threadIdx.x; a < n; a += 256) {
        const float m = traj_mu(T, t, x, a);
        if (t1 == 0) {  // absorption.c:107-117: the vector starts as mu_x(ti)
            pr[a] = m;
            pi[a] = 0.f;
        }
        re += (double)(m * pr[a]);
        im += (double)(m * pi[a]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        red[0][warp] = re;
        red[1][warp] = im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sr = 0, si = 0;
        for (int w = 0; w < 8; w++) {
            sr += red[0][w];
            si += red[1][w];
        }
        resp[(size_t)(3 * q + x) * J.tmax + t1] = make_double2(sr, si);
    }
}

// Y = U_t X for 128 rows per CTA; NC columns (a multiple of 16, <= 64).
// Shared-memory tiles (1024-byte aligned, 128-byte swizzled rows of 32
// tf32): A[c][p] = piece p of U_c (c = 0 real, 1 imaginary) for the CTA's 128
// rows, B[c][p] = piece p of X_c for the NC columns, sites c0 .. c0 + 31.
template <int NC>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_tc_apply(const float2 *__restrict__ U, int n, const float *__restrict__ xr, const float *__restrict__ xi,
               float *__restrict__ yr, float *__restrict__ yi, int *err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    constexpr size_t kA = (size_t)kTcRows * 128, kB = (size_t)NC * 128;
    unsigned char *aT[2][3], *bT[2][3];
    for (int c = 0; c < 2; c++)
        for (int q = 0; q < 3; q++) {
            aT[c][q] = base + (size_t)(3 * c + q) * kA;
            bT[c][q] = base + 6 * kA + (size_t)(3 * c + q) * kB;
        }
    uint64_t *mbar = (uint64_t *)(base + 6 * kA + 6 * kB);
    uint32_t *tslot = (uint32_t *)(mbar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int a0 = blockIdx.x * kTcRows;

    if (warp == 0) {  // two accumulators of NC columns each
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(tmem_cols(NC)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // Accumulators: the leading products x0 y0 of U_r X_r, U_i X_i, U_i X_r
    // and U_r X_i each in its own (no cancellation between large terms inside
    // the tensor core, whose additions round toward zero), the five
    // correction products of Y_r and of Y_i in two more, at their own (2^-11
    // smaller) scale; combined in registers with round-to-nearest
    const uint32_t tmem = *tslot;
    const uint32_t m_rr = tmem, m_ii = tmem + NC, m_ir = tmem + 2 * NC, m_ri = tmem + 3 * NC;
    const uint32_t c_r = tmem + 4 * NC, c_i = tmem + 5 * NC;
    const uint32_t id_pos = make_idesc(NC, false), id_neg = make_idesc(NC, true);

    const int nk = (n + kTcK - 1) / kTcK;
    bool ok = true;
    int kfail = 0;
    for (int kc = 0; kc < nk && ok; kc++) {
        kfail = kc;
        const int c0 = kc * kTcK;
        // A: U[a0 + r][c0 .. c0 + 31], two complex per thread-iteration
        for (int q = tid; q < kTcRows * (kTcK / 2); q += kTcThreads) {
            const int r = q / (kTcK / 2), k = (q % (kTcK / 2)) * 2, a = a0 + r, c = c0 + k;
            float2 u0 = make_float2(0.f, 0.f), u1 = u0;
            if (a < n && c < n) {  // rows of odd n are only 8-byte aligned
                u0 = U[(size_t)a * n + c];
                if (c + 1 < n) u1 = U[(size_t)a * n + c + 1];
            }
            const uint32_t off = sw128(r, k);
            float pr0[3], pr1[3], pi0[3], pi1[3];
            split3(u0.x, pr0);
            split3(u1.x, pr1);
            split3(u0.y, pi0);
            split3(u1.y, pi1);
#pragma unroll
            for (int p = 0; p < 3; p++) {
                *(float2 *)(aT[0][p] + off) = make_float2(pr0[p], pr1[p]);
                *(float2 *)(aT[1][p] + off) = make_float2(pi0[p], pi1[p]);
            }
        }
        // B: X[m][c0 .. c0 + 31], four sites per thread-iteration
        for (int q = tid; q < NC * (kTcK / 4); q += kTcThreads) {
            const int m = q / (kTcK / 4), k = (q % (kTcK / 4)) * 4, c = c0 + k;
            float vr[4][3], vi[4][3];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                split3(c + j < n ? xr[(size_t)m * n + c + j] : 0.f, vr[j]);
                split3(c + j < n ? xi[(size_t)m * n + c + j] : 0.f, vi[j]);
            }
            const uint32_t off = sw128(m, k);
#pragma unroll
            for (int p = 0; p < 3; p++) {
                *(float4 *)(bT[0][p] + off) = make_float4(vr[0][p], vr[1][p], vr[2][p], vr[3][p]);
                *(float4 *)(bT[1][p] + off) = make_float4(vi[0][p], vi[1][p], vi[2][p], vi[3][p]);
            }
        }
        // the tiles written by the threads become operands of the tensor core
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint64_t A[2][3], B[2][3];
            for (int c = 0; c < 2; c++)
                for (int q = 0; q < 3; q++) {
                    A[c][q] = make_desc(smem_u32(aT[c][q]));
                    B[c][q] = make_desc(smem_u32(bT[c][q]));
                }
            // piece pairs (i, j) with i + j <= 2 except (2, 0)/(0, 2) counted once each
            constexpr int PI[6] = {0, 0, 1, 1, 0, 2}, PJ[6] = {0, 1, 0, 1, 2, 0};
#pragma unroll
            for (int s = 0; s < kTcK / 8; s++) {  // K = 8 tf32 (32 bytes) per instruction
                const uint64_t dk = (uint64_t)((s * 32) >> 4);
                const uint32_t first = (kc == 0 && s == 0) ? 0u : 1u;
                mma_tf32(m_rr, A[0][0] + dk, B[0][0] + dk, id_pos, first);
                mma_tf32(m_ii, A[1][0] + dk, B[1][0] + dk, id_pos, first);
                mma_tf32(m_ir, A[1][0] + dk, B[0][0] + dk, id_pos, first);
                mma_tf32(m_ri, A[0][0] + dk, B[1][0] + dk, id_pos, first);
#pragma unroll
                for (int t = 1; t < 6; t++) {
                    const uint32_t acc = (kc == 0 && s == 0 && t == 1) ? 0u : 1u;
                    // Y_r += U_r X_r - U_i X_i;  Y_i += U_i X_r + U_r X_i
                    mma_tf32(c_r, A[0][PI[t]] + dk, B[0][PJ[t]] + dk, id_pos, acc);
                    mma_tf32(c_r, A[1][PI[t]] + dk, B[1][PJ[t]] + dk, id_neg, 1);
                    mma_tf32(c_i, A[1][PI[t]] + dk, B[0][PJ[t]] + dk, id_pos, acc);
                    mma_tf32(c_i, A[0][PI[t]] + dk, B[1][PJ[t]] + dk, id_pos, 1);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(mbar))
                         : "memory");
        }
        // the tiles are reused by the next stage once the MMAs have read them
        ok = __syncthreads_and(mbar_wait_bounded(mbar, kc & 1));
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
        mbar_wait_bounded(mbar, kfail & 1);  // let MMAs in flight finish before the memory is freed
    } else {
        // warp w reads tensor-memory lanes 32 (w % 4) ..: warps 0-3 Y_r, warps 4-7 Y_i
        const int row = 32 * (warp & 3) + lane, a = a0 + row;
        const uint32_t lanes = (uint32_t)(32 * (warp & 3)) << 16;
        const bool re = warp < 4;  // Y_r = m_rr - m_ii + c_r,  Y_i = m_ir + m_ri + c_i
        const uint32_t p0 = (re ? m_rr : m_ir) + lanes, p1 = (re ? m_ii : m_ri) + lanes, pc = (re ? c_r : c_i) + lanes;
        const float sg = re ? -1.f : 1.f;
        float *y = re ? yr : yi;
#pragma unroll
        for (int c16 = 0; c16 < NC; c16 += 16) {
            uint32_t v0[16], v1[16], w[16];
            tmem_ld16(p0 + (uint32_t)c16, v0);
            tmem_ld16(p1 + (uint32_t)c16, v1);
            tmem_ld16(pc + (uint32_t)c16, w);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (a < n)
#pragma unroll
                for (int j = 0; j < 16; j++)
                    y[(size_t)(c16 + j) * n + a] =
                        (__uint_as_float(v0[j]) + sg * __uint_as_float(v1[j])) + __uint_as_float(w[j]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                                "r"(tmem_cols(NC)));
}

template <int NC>
size_t tc_apply_smem() {
    return 1024 + (size_t)6 * kTcRows * 128 + (size_t)6 * NC * 128 + 64;
}

template <int NC>
int run_tc_apply(const float2 *U, int n, const float *xr, const float *xi, float *yr, float *yi, int *err,
                 cudaStream_t s) {
    const size_t sm = tc_apply_smem<NC>();
    cudaError_t e = cudaFuncSetAttribute(k_tc_apply<NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return (int)e;
    k_tc_apply<NC><<<(n + kTcRows - 1) / kTcRows, kTcThreads, sm, s>>>(U, n, xr, xi, yr, yi, err);
    return (int)cudaGetLastError();
}

}  // namespace

int tc_dia_columns(const AbsJob &J) {
    const int slots = (J.tmax - 1) / J.sample + 1;
    const int cols = 3 * std::min(slots, J.nsamp);
    return (cols + 15) / 16 * 16;
}

bool tc_dia_fits(const AbsJob &J, int n) { return n >= 1 && tc_dia_columns(J) <= 64; }

long tc_dia_first_frame(const AbsJob &J) { return (long)J.begin * J.sample; }
long tc_dia_last_frame(const AbsJob &J) { return (long)(J.begin + J.nsamp - 1) * J.sample + J.tmax - 1; }

// Frames ta..tb of the job in order: starts and responses on frame t, then the
// step with U_t (at U + (t - ufirst) n^2) for every frame some vector still
// propagates through.  X holds 4 planes of cols x n floats (two ping-pong
// state buffers, real and imaginary); it is cleared when ta is the job's
// first frame, and frame t's state is in the first pair of planes when
// t - first frame is even.
int launch_abs_dia_tc_frames(const DevTraj &T, const void *U, long ufirst, int n, const AbsJob &J, double2 *resp,
                             float *X, int *err, long ta, long tb, cudaStream_t s) {
    if (J.nsamp <= 0) return 0;
    const int cols = tc_dia_columns(J);
    if (cols > 64) return (int)cudaErrorNotSupported;
    const int slots = (J.tmax - 1) / J.sample + 1;
    const long tfirst = tc_dia_first_frame(J), tlast = tc_dia_last_frame(J);
    ta = std::max(ta, tfirst);
    tb = std::min(tb, tlast);
    if (ta > tb) return 0;
    if (ta == tfirst) {
        cudaError_t e = cudaMemsetAsync(X, 0, sizeof(float) * 4 * (size_t)cols * n, s);
        if (e != cudaSuccess) return (int)e;
    }
    float *cr = X, *ci = X + (size_t)cols * n, *nr = ci + (size_t)cols * n, *ni = nr + (size_t)cols * n;
    if ((ta - tfirst) & 1) {
        std::swap(cr, nr);
        std::swap(ci, ni);
    }
    const int ncol = 3 * std::min(slots, J.nsamp);
    for (long t = ta; t <= tb; t++) {
        k_tc_resp<<<ncol, 256, 0, s>>>(T, J, n, t, slots, cr, ci, resp);
        if (t == tlast) break;
        const float2 *Ut = (const float2 *)U + (size_t)(t - ufirst) * n * n;
        int rc;
        switch (cols) {
        case 16: rc = run_tc_apply<16>(Ut, n, cr, ci, nr, ni, err, s); break;
        case 32: rc = run_tc_apply<32>(Ut, n, cr, ci, nr, ni, err, s); break;
        case 48: rc = run_tc_apply<48>(Ut, n, cr, ci, nr, ni, err, s); break;
        default: rc = run_tc_apply<64>(Ut, n, cr, ci, nr, ni, err, s); break;
        }
        if (rc) return rc;
        std::swap(cr, nr);
        std::swap(ci, ni);
    }
    return (int)cudaGetLastError();
}

// Every frame of the job, the propagators of frames f0.. all in U.
int launch_abs_dia_tc(const DevTraj &T, const void *U, long f0, int n, const AbsJob &J, double2 *resp, float *X,
                      int *err, cudaStream_t s) {
    return launch_abs_dia_tc_frames(T, U, f0, n, J, resp, X, err, tc_dia_first_frame(J), tc_dia_last_frame(J), s);
}
