// Linear absorption (Trotter "Coupling" scheme) for callers that cannot let
// the library allocate device memory.
//
// Who needs this: applications that own every byte of device memory through
// their own pool or arena allocator and hand out fixed buffers, and code that
// must not trigger the device-wide synchronisation a cudaMalloc/cudaFree can
// cause in the middle of their own stream work.  Such callers pass their
// device buffers; this entry point takes every intermediate table from one
// file-scope device array, g_noalloc_scratch, and calls no cudaMalloc,
// cudaFree or other allocating routine.
//
// Limits and sharing: the array holds NISE_NOALLOC_SCRATCH_BYTES (32 MiB) on
// every GPU that loads the library, for the life of the process.  Jobs whose
// tables do not fit are rejected with NISE_ERR_SHAPE.  All calls share the
// array: calls whose device work overlaps in time (different streams, or
// different host threads on one device) race on it and must be serialised by
// the caller.  Each call rewrites every table it reads, so nothing from a
// previous call leaks into a result.
//
// Set-up: the device address of the array is looked up once per device with
// cudaGetSymbolAddress (host code cannot use the symbol itself as a device
// pointer) on the first call made with that device current; make that first
// call before any stream capture begins.
#include <cstdint>
#include <cstring>

#include "common.cuh"
#include "engine.h"
#include "nise_b200.h"

#define NISE_NOALLOC_SCRATCH_BYTES (32u << 20)
#define NISE_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_noalloc_scratch[NISE_NOALLOC_SCRATCH_BYTES];

namespace {

void *g_scratch_addr[NISE_NOALLOC_MAX_DEVICES];  // device address per device ordinal

// Compact the flagged packed off-diagonals into the lexicographic pair list.
__global__ void k_na_compact(const int *flag, int n, int2 *pairs, int *count) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int k = 0;
    for (int a = 0; a < n; a++)
        for (int b = a + 1; b < n; b++)
            if (flag[sindex(a, b, n)]) pairs[k++] = make_int2(a, b);
    *count = k;
}

// Sum the per-vector responses in order and split them into re/im outputs.
__global__ void k_na_reduce(const double2 *resp, int nvec, int tmax, double *re, double *im) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tmax) return;
    double a = 0, b = 0;
    for (int v = 0; v < nvec; v++) {
        double2 z = resp[(size_t)v * tmax + t];
        a += z.x;
        b += z.y;
    }
    re[t] = a;
    im[t] = b;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" void nise_set_global_error(const char *msg);

// f = deltat * icm2ifs * twoPi / m, left to right in float (propagate.c:836).
static float f32_sub(const nise_params *p) {
    float f = p->deltat * 2.99792458e-5f;
    f = f * (float)(2 * 3.14159265359);
    return f / (float)p->ts;
}

extern "C" int nise_absorption_noalloc(const nise_params *p, const void *d_energy, size_t energy_bytes,
                                       const void *d_dipole, size_t dipole_bytes, double *d_re_S, double *d_im_S,
                                       int *samples, void *stream) {
    if (!p || !d_energy || !d_dipole || !d_re_S || !d_im_S || !samples) {
        nise_set_global_error("nise_absorption_noalloc: null argument");
        return NISE_ERR_ARG;
    }
    if (p->propagation != NISE_PROP_COUPLING || p->hamiltonian != NISE_HAM_FULL ||
        p->technique != NISE_TECH_ABSORPTION) {
        nise_set_global_error("nise_absorption_noalloc: needs Technique Absorption, Propagation Coupling and "
                              "HamiltonianType Full");
        return NISE_ERR_UNSUPPORTED;
    }
    if (p->singles <= 0 || p->sample <= 0 || p->ts <= 0 || !(p->deltat > 0) || p->tmax1 <= 0 ||
        (p->precision != NISE_FP32 && p->precision != NISE_FP64)) {
        nise_set_global_error("nise_absorption_noalloc: invalid parameters");
        return NISE_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NISE_NOALLOC_MAX_DEVICES) {
        nise_set_global_error("nise_absorption_noalloc: no usable current device");
        return NISE_ERR_DEVICE;
    }
    if (!g_scratch_addr[dev]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) {
            nise_set_global_error(cudaGetErrorString(e));
            return NISE_ERR_DEVICE;
        }
        g_scratch_addr[dev] = ptr;
    }
    unsigned char *base = (unsigned char *)g_scratch_addr[dev];
    cudaStream_t st = (cudaStream_t)stream;
    const int n = p->singles, tmax = p->tmax1, prec = p->precision;
    // determine_samples (NISE_subs.c:197-221)
    int n_samples = (p->length - p->tmax1 - 1) / p->sample + 1;
    int end = p->end == 0 ? n_samples : p->end;
    if (n_samples <= 0 || end > n_samples || p->begin < 0 || p->begin >= end) {
        nise_set_global_error("nise_absorption_noalloc: no samples (Length, RunTimes, BeginPoint, EndPoint)");
        return NISE_ERR_ARG;
    }
    const int nsamp = end - p->begin, nvec = 3 * nsamp;
    long nn2 = (long)n * (n + 1) / 2;
    long e_words = 1 + nn2 + (long)p->doubles * (p->doubles + 1) / 2, d_words = 1 + 3L * n + 3L * n * p->doubles;
    long e_frames = (long)(energy_bytes / (4 * (size_t)e_words)), d_frames = (long)(dipole_bytes / (4 * (size_t)d_words));
    long f0 = (long)p->begin * p->sample, f1 = (long)(end - 1) * p->sample + tmax - 1;
    if (f1 >= e_frames || f1 >= d_frames) {
        nise_set_global_error("nise_absorption_noalloc: trajectory to short for the requested samples");
        return NISE_ERR_IO;
    }
    long nf = f1 - f0 > 0 ? f1 - f0 : 1;
    size_t r2 = prec == NISE_FP32 ? sizeof(float2) : sizeof(double2);
    // scratch layout; the pair table is sized for every off-diagonal
    size_t o_flag = 0, o_cnt = align256(o_flag + sizeof(int) * nn2), o_pairs = align256(o_cnt + sizeof(int));
    size_t o_U = align256(o_pairs + sizeof(int2) * (nn2 > n ? nn2 - n : 1));
    size_t o_rot = align256(o_U + r2 * (size_t)nf * n);
    size_t o_resp = align256(o_rot + r2 * (size_t)nf * (nn2 > n ? nn2 - n : 1));
    size_t need = o_resp + sizeof(double2) * (size_t)nvec * tmax;
    if (need > NISE_NOALLOC_SCRATCH_BYTES) {
        nise_set_global_error("nise_absorption_noalloc: job needs more than the 32 MiB static scratch "
                              "(fewer frames, sites or start points per call)");
        return NISE_ERR_SHAPE;
    }
    DevTraj T;
    memset(&T, 0, sizeof(T));
    T.energy = (const float *)d_energy;
    T.e_words = e_words;
    T.e_frames = e_frames;
    T.full = 1;
    T.dipole = (const float *)d_dipole;
    T.d_words = d_words;
    T.d_frames = d_frames;
    T.n = n;
    T.shifte = (p->max1 + p->min1) / 2;
    T.cut = p->couplingcut;
    int *flag = (int *)(base + o_flag), *cnt = (int *)(base + o_cnt);
    int2 *pairs = (int2 *)(base + o_pairs);
    // the flag table starts at zero on every call
    if (cudaMemsetAsync(flag, 0, sizeof(int) * nn2, st) != cudaSuccess) goto dev_fail;
    if (launch_pattern_scan(T, f0, nf, flag, st)) goto dev_fail;
    k_na_compact<<<1, 1, 0, st>>>(flag, n, pairs, cnt);
    int K;
    if (cudaMemcpyAsync(&K, cnt, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) goto dev_fail;
    if (cudaStreamSynchronize(st) != cudaSuccess) goto dev_fail;
    {
        TrotterPlan P;
        P.n = n;
        P.k = K;
        P.pairs = pairs;
        P.f0 = f0;
        P.nf = nf;
        P.U = base + o_U;
        P.rot = base + o_rot;
        P.rot_static = 0;
        P.singleshift = 0;
        double fsub = (double)p->deltat * (double)2.99792458e-5f * (double)(float)(2 * 3.14159265359) / p->ts;
        if (launch_prep_trotter(prec, T, P, fsub, f32_sub(p), st)) goto dev_fail;
        AbsJob J;
        memset(&J, 0, sizeof(J));
        J.begin = p->begin;
        J.nsamp = nsamp;
        J.sample = p->sample;
        J.tmax = tmax;
        J.ts = p->ts;
        double2 *resp = (double2 *)(base + o_resp);
        if (launch_abs_trotter(prec, T, P, J, resp, st)) goto dev_fail;
        k_na_reduce<<<(tmax + 127) / 128, 128, 0, st>>>(resp, nvec, tmax, d_re_S, d_im_S);
        if (cudaGetLastError() != cudaSuccess) goto dev_fail;
        if (cudaStreamSynchronize(st) != cudaSuccess) goto dev_fail;
    }
    *samples = end;  // absorption.c:185
    return NISE_OK;
dev_fail:
    nise_set_global_error(cudaGetErrorString(cudaGetLastError()));
    return NISE_ERR_DEVICE;
}
