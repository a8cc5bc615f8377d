// C ABI of the engine (include/nise_b200.h): context, trajectory loading,
// job planning and the output writers.  No exit() on any path: every failure
// is a status code plus a message.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "eigen.h"
#include "engine.h"
#include "nise_b200.h"
#include "nise_internal.h"

namespace {
thread_local std::string g_error;

// Physical constants of the reference (src/types.h:5-12), declared float there.
const float kIcm2ifs = 2.99792458e-5f;
const float kTwoPi = (float)(2 * 3.14159265359);
const float kCv = 2.99792458e-5f;

bool read_file(const char *path, std::vector<char> &out) {
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    out.resize(n > 0 ? (size_t)n : 0);
    bool ok = n <= 0 || fread(out.data(), 1, (size_t)n, f) == (size_t)n;
    fclose(f);
    return ok;
}
}  // namespace

extern "C" void nise_set_global_error(const char *msg) { g_error = msg ? msg : ""; }
extern "C" const char *nise_global_error(void) { return g_error.c_str(); }

int nise_fail(nise_ctx *c, int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    g_error = buf;
    return code;
}

int nise_cuda(nise_ctx *c, int e, const char *what) {
    if (e == 0) return NISE_OK;
    return nise_fail(c, NISE_ERR_DEVICE, "%s: %s", what, cudaGetErrorString((cudaError_t)e));
}

// f = deltat * icm2ifs * twoPi * sign / m evaluated left to right in float,
// as propagate.c:836 does.
float nise_f32(const nise_params &p, int sign, int m) {
    float f = p.deltat * kIcm2ifs;
    f = f * kTwoPi;
    f = f * (float)sign;
    return f / (float)m;
}
double nise_f64(const nise_params &p, int sign, int m) {
    return (double)p.deltat * (double)kIcm2ifs * (double)kTwoPi * sign / m;
}

extern "C" int nise_create(const nise_params *p, nise_ctx **out) {
    if (!p || !out) return nise_fail(nullptr, NISE_ERR_ARG, "null argument");
    *out = nullptr;
    if (p->singles <= 0) return nise_fail(nullptr, NISE_ERR_ARG, "Singles must be positive");
    if (p->sample <= 0) return nise_fail(nullptr, NISE_ERR_ARG, "Samplerate must be positive");
    if (!(p->deltat > 0)) return nise_fail(nullptr, NISE_ERR_ARG, "Timestep must be positive");
    if (p->ts <= 0) return nise_fail(nullptr, NISE_ERR_ARG, "Trotter must be positive");
    if (p->tmax1 <= 0) return nise_fail(nullptr, NISE_ERR_ARG, "First runtime variable is zero");
    if (p->precision != NISE_FP32 && p->precision != NISE_FP64)
        return nise_fail(nullptr, NISE_ERR_ARG, "precision must be NISE_FP32 or NISE_FP64");
    nise_ctx *c = new nise_ctx();
    c->p = *p;
    c->n = p->singles;
    c->nn2 = (long)p->singles * (p->singles + 1) / 2;
    // readinput.c:264-271: Threshold rescaled by (dt*icm2ifs*2pi/ts)^2 in float
    c->thres = p->thres;
    if (p->propagation == NISE_PROP_SPARSE || p->propagation == NISE_PROP_DIAGONAL) {
        float s = nise_f32(*p, 1, p->ts);
        c->thres = p->thres * (s * s);
        if (c->thres > 0.1f) {
            delete c;
            return nise_fail(nullptr, NISE_ERR_ARG, "Unrealistic value for threshold");
        }
    }
    c->shifte = (p->max1 + p->min1) / 2;
    int e = (int)cudaSetDevice(p->device);
    if (!e) e = (int)cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    c->stream = c->own_stream;
    if (!e) e = (int)cudaEventCreate(&c->ev0);
    if (!e) e = (int)cudaEventCreate(&c->ev1);
    if (!e) e = (int)cudaEventCreate(&c->evk0);
    if (!e) e = (int)cudaEventCreate(&c->evk1);
    if (e) {
        int rc = nise_cuda(nullptr, e, "device setup");
        delete c;
        return rc;
    }
    *out = c;
    return NISE_OK;
}

void nise_free_traj(nise_ctx *c) {
    void *ptrs[] = {c->d_energy, c->d_dipole, c->d_hc, c->d_mu_static, c->d_anh, c->d_over, c->d_shift_site,
                    c->d_shift_ab};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    c->d_energy = c->d_dipole = c->d_hc = c->d_mu_static = c->d_anh = c->d_over = c->d_shift_ab = nullptr;
    c->d_shift_site = nullptr;
    c->cap_energy = c->cap_dipole = c->cap_anh = c->cap_over = c->cap_hc = c->cap_mu = c->cap_ab = 0;
    c->loaded = false;
}

extern "C" void nise_destroy(nise_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->p.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->stream = c->own_stream;
    nise_free_traj(c);
    cudaEvent_t evs[] = {c->ev0, c->ev1, c->evk0, c->evk1};
    for (cudaEvent_t ev : evs)
        if (ev) cudaEventDestroy(ev);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

extern "C" const char *nise_last_error(const nise_ctx *c) { return c ? c->err.c_str() : g_error.c_str(); }

// Copy host bytes to a context buffer, keeping the allocation when it is
// already large enough (repeated uploads of same-sized trajectories allocate
// nothing).
static int upload(nise_ctx *c, float **dst, size_t *cap, const void *src, size_t bytes) {
    if (!src || !bytes) {
        if (*dst) cudaFree(*dst);
        *dst = nullptr;
        *cap = 0;
        return NISE_OK;
    }
    if (bytes > *cap) {
        if (*dst) cudaFree(*dst);
        *dst = nullptr;
        *cap = 0;
        if (cudaMalloc((void **)dst, bytes) != cudaSuccess)
            return nise_fail(c, NISE_ERR_NOMEM, "device allocation of %zu bytes failed", bytes);
        *cap = bytes;
    }
    int e = (int)cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
    return nise_cuda(c, e, "trajectory upload");
}

extern "C" int nise_set_trajectory(nise_ctx *c, const void *energy, size_t energy_bytes, const void *dipole,
                                   size_t dipole_bytes, const void *coupling, size_t coupling_bytes,
                                   const void *anharm, size_t anharm_bytes, const void *overtone,
                                   size_t overtone_bytes) {
    if (!c) return nise_fail(nullptr, NISE_ERR_ARG, "null context");
    if (!energy || !dipole) return nise_fail(c, NISE_ERR_ARG, "energy and dipole records are required");
    cudaSetDevice(c->p.device);
    const nise_params &p = c->p;
    int N = c->n;
    bool coupling_type = p.hamiltonian == NISE_HAM_COUPLING;
    long full_words = 1 + c->nn2 + (long)p.doubles * (p.doubles + 1) / 2;
    c->e_words = coupling_type ? 1 + N : full_words;
    c->e_frames = (long)(energy_bytes / (4 * (size_t)c->e_words));
    c->d_words = 1 + 3L * N + 3L * N * p.doubles;
    c->d_frames = (long)(dipole_bytes / (4 * (size_t)c->d_words));
    if (c->e_frames < 1) return nise_fail(c, NISE_ERR_IO, "Hamiltonian trajectory file to short");
    if (c->d_frames < 1) return nise_fail(c, NISE_ERR_IO, "Dipole trajectory file to short");
    int rc;
    if ((rc = upload(c, &c->d_energy, &c->cap_energy, energy, (size_t)c->e_frames * 4 * c->e_words))) return rc;
    if ((rc = upload(c, &c->d_dipole, &c->cap_dipole, dipole, (size_t)c->d_frames * 4 * c->d_words))) return rc;
    c->a_frames = anharm ? (long)(anharm_bytes / (4 * (size_t)(1 + N))) : 0;
    c->o_frames = overtone ? (long)(overtone_bytes / (4 * (size_t)(1 + 3L * N))) : 0;
    if ((rc = upload(c, &c->d_anh, &c->cap_anh, anharm, (size_t)c->a_frames * 4 * (1 + N)))) return rc;
    if ((rc = upload(c, &c->d_over, &c->cap_over, overtone, (size_t)c->o_frames * 4 * (1 + 3L * N)))) return rc;
    c->h_hc.clear();
    c->h_mu_static.clear();
    if (coupling_type) {
        // read_coupling (read_trajectory.c:47-70): one Full record at position 0
        // with the read cut, and the dipoles of frame 0.
        if (!coupling || coupling_bytes < 4 * (size_t)full_words)
            return nise_fail(c, NISE_ERR_IO, "Coupling trajectory file to short");
        c->h_hc.assign((const float *)coupling + 1, (const float *)coupling + 1 + c->nn2);
        for (int i = 0; i < N; i++) c->h_hc[(size_t)i * N + i - (size_t)i * (i + 1) / 2] -= c->shifte;
        for (int i = 0; i < N; i++)
            for (int j = i + 1; j < N; j++) {
                long idx = j + (long)i * ((N << 1) - i - 1) / 2;
                if (fabs(c->h_hc[idx]) < p.couplingcut) c->h_hc[idx] = 0;
            }
        const float *m = (const float *)dipole + 1;
        c->h_mu_static.assign(m, m + 3L * N);
        if ((rc = upload(c, &c->d_hc, &c->cap_hc, c->h_hc.data(), sizeof(float) * c->nn2))) return rc;
        if ((rc = upload(c, &c->d_mu_static, &c->cap_mu, c->h_mu_static.data(), sizeof(float) * 3 * N))) return rc;
    } else {
        if ((rc = upload(c, &c->d_hc, &c->cap_hc, nullptr, 0))) return rc;
        if ((rc = upload(c, &c->d_mu_static, &c->cap_mu, nullptr, 0))) return rc;
    }
    int e = (int)cudaStreamSynchronize(c->stream);
    if (e) return nise_cuda(c, e, "trajectory upload");
    c->loaded = true;
    return NISE_OK;
}

extern "C" int nise_set_singleshift(nise_ctx *c, int n, const int *sites, const float *a, const float *b) {
    if (!c || n < 0) return nise_fail(c, NISE_ERR_ARG, "bad SingleShift arguments");
    cudaSetDevice(c->p.device);
    std::vector<float> ab(2 * (size_t)n);
    for (int i = 0; i < n; i++) {
        if (sites[i] < 0 || sites[i] >= c->n) return nise_fail(c, NISE_ERR_ARG, "SingleShift site out of range");
        ab[2 * i] = a[i];
        ab[2 * i + 1] = b[i];
    }
    if (c->d_shift_site) cudaFree(c->d_shift_site);
    c->d_shift_site = nullptr;
    c->nshift = n;
    int rc;
    if (n) {
        if (cudaMalloc((void **)&c->d_shift_site, sizeof(int) * n))
            return nise_fail(c, NISE_ERR_NOMEM, "device allocation failed");
        cudaMemcpyAsync(c->d_shift_site, sites, sizeof(int) * n, cudaMemcpyHostToDevice, c->stream);
    }
    if ((rc = upload(c, &c->d_shift_ab, &c->cap_ab, n ? ab.data() : nullptr, sizeof(float) * 2 * n))) return rc;
    return nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "SingleShift upload");
}

extern "C" int nise_load_files(nise_ctx *c) {
    if (!c) return nise_fail(nullptr, NISE_ERR_ARG, "null context");
    const nise_params &p = c->p;
    std::vector<char> E, D, C, A, O;
    if (!read_file(p.energyFName, E)) return nise_fail(c, NISE_ERR_IO, "Hamiltonian file not found!");
    if (!read_file(p.dipoleFName, D)) return nise_fail(c, NISE_ERR_IO, "Dipole file %s not found!", p.dipoleFName);
    if (p.hamiltonian == NISE_HAM_COUPLING && !read_file(p.couplingFName, C))
        return nise_fail(c, NISE_ERR_IO, "Coupling file not found!");
    bool two_d = p.technique >= NISE_TECH_2DIR && p.technique <= NISE_TECH_NOEAIR;
    if (two_d && p.anharmonicity == 0) {
        if (!read_file(p.anharFName, A))
            return nise_fail(c, NISE_ERR_IO, "Anharmonicity file %s not found!", p.anharFName);
        if (!read_file(p.overdipFName, O))
            return nise_fail(c, NISE_ERR_IO, "Overtone dipole file %s not found!", p.overdipFName);
    }
    int rc = nise_set_trajectory(c, E.data(), E.size(), D.data(), D.size(), C.empty() ? nullptr : C.data(),
                                 C.size(), A.empty() ? nullptr : A.data(), A.size(), O.empty() ? nullptr : O.data(),
                                 O.size());
    if (rc) return rc;
    // read_shift (hamshift.c:13-47); a missing file is reported and ignored there.
    if (p.singleShiftFName[0]) {
        FILE *f = fopen(p.singleShiftFName, "r");
        if (f) {
            int n = 0;
            if (fscanf(f, "%d", &n) != 1 || n < 0) {
                fclose(f);
                return nise_fail(c, NISE_ERR_IO, "Could not read number of single shifts site from %s",
                                 p.singleShiftFName);
            }
            std::vector<int> s(n);
            std::vector<float> a(n), b(n);
            for (int i = 0; i < n; i++)
                if (fscanf(f, "%d %f %f", &s[i], &a[i], &b[i]) != 3) {
                    fclose(f);
                    return nise_fail(c, NISE_ERR_IO, "bad SingleShift file %s", p.singleShiftFName);
                }
            fclose(f);
            return nise_set_singleshift(c, n, s.data(), a.data(), b.data());
        }
    }
    return NISE_OK;
}

DevTraj nise_devtraj(const nise_ctx *c) {
    DevTraj T;
    memset(&T, 0, sizeof(T));
    T.energy = c->d_energy;
    T.e_words = c->e_words;
    T.e_frames = c->e_frames;
    T.full = c->p.hamiltonian == NISE_HAM_FULL;
    T.dipole = c->d_dipole;
    T.d_words = c->d_words;
    T.d_frames = c->d_frames;
    T.mu_static = c->d_mu_static;
    T.hc = c->d_hc;
    T.anh = c->d_anh;
    T.a_frames = c->a_frames;
    T.over = c->d_over;
    T.o_frames = c->o_frames;
    T.shift_site = c->d_shift_site;
    T.shift_ab = c->d_shift_ab;
    T.nshift = c->nshift;
    T.n = c->n;
    T.shifte = c->shifte;
    T.cut = c->p.couplingcut;
    return T;
}

// Off-diagonal coupling pattern (a < b, lexicographic) with |J| > cut in any
// frame of [f0, f0 + nf): from the static coupling frame or a device scan.
int nise_pattern(nise_ctx *c, long f0, long nf, std::vector<int2> &pairs) {
    int N = c->n;
    pairs.clear();
    if (c->p.hamiltonian == NISE_HAM_COUPLING) {
        for (int a = 0; a < N; a++)
            for (int b = a + 1; b < N; b++)
                if (fabsf(c->h_hc[b + (long)a * ((N << 1) - a - 1) / 2]) > c->p.couplingcut)
                    pairs.push_back(make_int2(a, b));
        return NISE_OK;
    }
    DevBuf<int> flag;
    int rc = flag.alloc(c, c->nn2);
    if (rc) return rc;
    cudaMemsetAsync(flag.p, 0, sizeof(int) * c->nn2, c->stream);
    DevTraj T = nise_devtraj(c);
    if ((rc = nise_cuda(c, launch_pattern_scan(T, f0, nf, flag.p, c->stream), "pattern scan"))) return rc;
    c->launches++;
    std::vector<int> h(c->nn2);
    cudaMemcpyAsync(h.data(), flag.p, sizeof(int) * c->nn2, cudaMemcpyDeviceToHost, c->stream);
    if ((rc = nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "pattern scan"))) return rc;
    for (int a = 0; a < N; a++)
        for (int b = a + 1; b < N; b++)
            if (h[b + (long)a * ((N << 1) - a - 1) / 2]) pairs.push_back(make_int2(a, b));
    return NISE_OK;
}

int nise_check_frames(nise_ctx *c, long last_frame) {
    if (last_frame >= c->e_frames)
        return nise_fail(c, NISE_ERR_IO, "Hamiltonian trajectory file to short, could not fill buffer!!! (frame %ld)",
                         last_frame);
    if (c->p.hamiltonian != NISE_HAM_COUPLING && last_frame >= c->d_frames)
        return nise_fail(c, NISE_ERR_IO, "Dipole trajectory file to short, could not fill buffer!!! (frame %ld)",
                         last_frame);
    return NISE_OK;
}

// ------------------------------------------------------------ absorption
// Eigen route of the exact propagators (diag.cu): every frame of [f0, f0+nf)
// is diagonalised in FP64 (chunks of frames), its one-step propagator U is
// built (truncated when a Threshold is active) and applied to every start
// point crossing it.  Records evk0/evk1 around the device work.
static int abs_eigen(nise_ctx *c, const DevTraj &T, const AbsJob &J, long f0, long nf, double2 *resp, bool plain,
                     bool truncated) {
    const int N = c->n, prec = c->p.precision;
    const size_t r2 = prec == NISE_FP32 ? sizeof(float2) : sizeof(double2);
    const size_t ubytes = r2 * (size_t)nf * N * N;
    if (ubytes > ((size_t)64 << 30))
        return nise_fail(c, NISE_ERR_NOMEM, "eigen route: %ld frames of %d sites need more than 64 GB of propagators",
                         nf, N);
    int rc;
    DevBuf<char> U;
    DevBuf<long> fr;
    DevBuf<double> V, w;
    std::vector<long> frames(nf);
    for (long t = 0; t < nf; t++) frames[t] = f0 + t;
    const long FC = std::max(1L, std::min(nf, (long)(((size_t)512 << 20) / (sizeof(double) * (size_t)N * N))));
    if ((rc = U.alloc(c, ubytes)) || (rc = fr.upload(c, frames)) || (rc = V.alloc(c, (size_t)FC * N * N)) ||
        (rc = w.alloc(c, (size_t)FC * N)))
        return rc;
    EigJob EJ;
    EJ.T = T;
    EJ.n = N;
    EJ.singleshift = c->nshift > 0;
    // propagate_vec_DIA: f = deltat*icm2ifs*twoPi*sign in float, one full step
    const double f = prec == NISE_FP32 ? (double)J.f32_full : J.f;
    cudaEventRecord(c->evk0, c->stream);
    for (long q = 0; q < nf; q += FC) {
        long m = std::min(FC, nf - q);
        if ((rc = nise_cuda(c, launch_eig(EJ, fr.p + q, m, V.p, w.p, c->stream), "eigensolver"))) return rc;
        if ((rc = nise_cuda(c, launch_build_u(prec == NISE_FP32 ? 0 : 1, V.p, w.p, m, N, f, c->thres, truncated,
                                              U.p + r2 * (size_t)q * N * N, c->stream),
                            "propagator build")))
            return rc;
        c->launches += 2;
    }
    if (plain) {
        for (int s = 0; s < J.nsamp; s++) {
            AbsJob Js = J;
            Js.begin = J.begin + s;
            Js.nsamp = 1;
            if ((rc = nise_cuda(c, launch_abs_dia(prec == NISE_FP32 ? 0 : 1, T, U.p, f0, N, Js,
                                                  resp + (size_t)3 * s * J.tmax, c->stream),
                                "eigen propagation")))
                return rc;
            c->launches++;
        }
    } else {
        if ((rc = nise_cuda(c, launch_abs_dia(prec == NISE_FP32 ? 0 : 1, T, U.p, f0, N, J, resp, c->stream),
                            "eigen propagation")))
            return rc;
        c->launches++;
    }
    cudaEventRecord(c->evk1, c->stream);
    return NISE_OK;
}

extern "C" int nise_absorption(nise_ctx *c, double *re_S, double *im_S, int *samples) {
    if (!c || !re_S || !im_S || !samples) return nise_fail(c, NISE_ERR_ARG, "null argument");
    if (!c->loaded) return nise_fail(c, NISE_ERR_STATE, "no trajectory loaded");
    cudaSetDevice(c->p.device);
    const nise_params &p = c->p;
    int N = c->n, tmax = p.tmax1, prec = p.precision;
    // determine_samples (NISE_subs.c:197-221)
    int n_samples = (p.length - p.tmax1 - 1) / p.sample + 1;
    if (n_samples <= 0) return nise_fail(c, NISE_ERR_ARG, "Insufficient data to calculate spectrum.");
    int end = p.end == 0 ? n_samples : p.end;
    if (end > n_samples) return nise_fail(c, NISE_ERR_ARG, "Endpoint larger than number of samples was specified.");
    int begin = p.begin;
    if (begin < 0 || begin >= end) return nise_fail(c, NISE_ERR_ARG, "BeginPoint must be below EndPoint");
    int nsamp = end - begin, nvec = 3 * nsamp;
    long f0 = (long)begin * p.sample;
    long f1 = (long)(end - 1) * p.sample + tmax - 1;  // last frame read
    int rc;
    if ((rc = nise_check_frames(c, f1))) return rc;
    long nf = f1 - f0;  // frames that are propagated through: [f0, f1)
    if (nf < 1) nf = 1;
    DevTraj T = nise_devtraj(c);
    AbsJob J;
    J.begin = begin;
    J.nsamp = nsamp;
    J.sample = p.sample;
    J.tmax = tmax;
    J.ts = p.ts;
    J.f = nise_f64(p, 1, 1);
    J.f32_sub = nise_f32(p, 1, p.ts);
    J.f64_sub = nise_f64(p, 1, p.ts);
    J.f32_full = nise_f32(p, 1, 1);
    DevBuf<double2> resp, out;
    if ((rc = resp.alloc(c, (size_t)nvec * tmax)) || (rc = out.alloc(c, tmax))) return rc;
    c->launches = 0;
    c->last_flops = c->last_bytes = 0;
    const bool plain = p.launch_mode == NISE_PLAIN;
    size_t rsz = prec == NISE_FP32 ? sizeof(float) : sizeof(double);
    cudaEventRecord(c->ev0, c->stream);
    // Vectors crossing each propagated frame: used for the algorithmic work.
    std::vector<long> cross(nf, 0);
    for (int s = 0; s < nsamp; s++) {
        long a = (long)(begin + s) * p.sample - f0;
        for (int t = 0; t < tmax - 1; t++) cross[a + t] += 3;
    }
    long vec_steps = 3L * nsamp * (tmax - 1);
    // bytes: every frame read once (diagonal or full record) and the dipoles
    c->last_bytes = (double)nf * 4 * (p.hamiltonian == NISE_HAM_COUPLING ? N : c->nn2) +
                    (double)(p.hamiltonian == NISE_HAM_COUPLING ? 3 * N : (nf + 1) * 3L * N) * 4;

    if (p.propagation == NISE_PROP_COUPLING) {
        std::vector<int2> pairs;
        if ((rc = nise_pattern(c, f0, nf, pairs))) return rc;
        DevBuf<int2> dpairs;
        DevBuf<char> U, rot;
        TrotterPlan P;
        P.n = N;
        P.k = (int)pairs.size();
        P.f0 = f0;
        P.nf = nf;
        P.rot_static = p.hamiltonian == NISE_HAM_COUPLING;
        P.singleshift = c->nshift > 0;
        if ((rc = dpairs.upload(c, pairs))) return rc;
        if ((rc = U.alloc(c, 2 * rsz * (size_t)nf * N))) return rc;
        if ((rc = rot.alloc(c, 2 * rsz * (size_t)(P.rot_static ? 1 : nf) * (P.k ? P.k : 1)))) return rc;
        P.pairs = dpairs.p;
        P.U = U.p;
        P.rot = rot.p;
        // per vector step: ts * (K rotations * 12 flops + 2 N half-phases * 6 flops)
        c->last_flops = (double)vec_steps * p.ts * (12.0 * P.k + 12.0 * N);
        if ((rc = nise_cuda(c, launch_prep_trotter(prec, T, P, J.f64_sub, J.f32_sub, c->stream), "Trotter prep")))
            return rc;
        c->launches += 1 + (P.rot_static ? 1 : 0);
        cudaEventRecord(c->evk0, c->stream);
        if (plain) {
            for (int s = 0; s < nsamp; s++) {
                AbsJob Js = J;
                Js.begin = begin + s;
                Js.nsamp = 1;
                if ((rc = nise_cuda(c, launch_abs_trotter(prec, T, P, Js, resp.p + (size_t)3 * s * tmax, c->stream),
                                    "Trotter propagation")))
                    return rc;
                c->launches++;
            }
        } else {
            if ((rc = nise_cuda(c, launch_abs_trotter(prec, T, P, J, resp.p, c->stream), "Trotter propagation")))
                return rc;
            c->launches++;
        }
        cudaEventRecord(c->evk1, c->stream);
    } else if (p.propagation == NISE_PROP_RK4) {
        std::vector<int2> pairs, ent;
        if ((rc = nise_pattern(c, f0, nf, pairs))) return rc;
        size_t q = 0;
        for (int a = 0; a < N; a++) {  // propagate.c:294-305 order: (a,a) then (a,b>a)
            ent.push_back(make_int2(a, a));
            while (q < pairs.size() && pairs[q].x == a) ent.push_back(pairs[q++]);
        }
        DevBuf<int2> dent;
        DevBuf<char> val;
        Rk4Plan P;
        P.n = N;
        P.k = (int)ent.size();
        P.f0 = f0;
        P.nf = nf;
        P.singleshift = c->nshift > 0;
        if ((rc = dent.upload(c, ent))) return rc;
        if ((rc = val.alloc(c, rsz * (size_t)nf * P.k))) return rc;
        P.entries = dent.p;
        P.val = val.p;
        // per sub-step: 4 stages over the list (off-diagonal entries twice) + update and norms
        c->last_flops = (double)vec_steps * p.ts * (4.0 * 4.0 * (2.0 * P.k - N) + 20.0 * N);
        if ((rc = nise_cuda(c, launch_prep_rk4(prec, T, P, J.f64_sub, J.f32_sub, c->stream), "RK4 prep"))) return rc;
        c->launches++;
        cudaEventRecord(c->evk0, c->stream);
        if (plain) {
            for (int s = 0; s < nsamp; s++) {
                AbsJob Js = J;
                Js.begin = begin + s;
                Js.nsamp = 1;
                if ((rc = nise_cuda(c, launch_abs_rk4(prec, T, P, Js, resp.p + (size_t)3 * s * tmax, c->stream),
                                    "RK4 propagation")))
                    return rc;
                c->launches++;
            }
        } else {
            if ((rc = nise_cuda(c, launch_abs_rk4(prec, T, P, J, resp.p, c->stream), "RK4 propagation"))) return rc;
            c->launches++;
        }
        cudaEventRecord(c->evk1, c->stream);
    } else {
        // Sparse / Diagonal: exact propagator exp(-i H dt) (propagate_vec_DIA,
        // propagate.c:60-125).  Threshold > 0 keeps only large elements of U
        // (propagate_vec_DIA_S, propagate.c:185-258) and needs the explicit
        // eigen propagator, as do per-frame couplings (HamiltonianType Full)
        // and the Diagonal scheme up to NISE_EIG_MAX_N sites.  Otherwise the
        // static couplings go through the sparse Taylor series below.
        const bool truncated = c->thres != 0 && !(c->thres > 1);
        const bool eigen_route = truncated || p.hamiltonian != NISE_HAM_COUPLING ||
                                 (p.propagation == NISE_PROP_DIAGONAL && N <= NISE_EIG_MAX_N);
        if (eigen_route) {
            if (N > NISE_EIG_MAX_N)
                return nise_fail(c, NISE_ERR_UNSUPPORTED,
                                 truncated ? "Sparse with Threshold > 0 is limited to 120 sites (eigen route)"
                                           : "exact propagation of per-frame couplings (HamiltonianType Full) is "
                                             "limited to 120 sites (eigen route)");
            if ((rc = abs_eigen(c, T, J, f0, nf, resp.p, plain, truncated))) return rc;
            c->last_flops = (double)nf * 6.7 * N * (double)N * N + (double)vec_steps * 8.0 * N * N;
        } else {
        // CSR of the static couplings (read cut applied, |J| >= cut kept)
        std::vector<int> rp(N + 1, 0), col;
        std::vector<double> vd;
        double rowabs = 0;
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
        DevBuf<int> drp, dcol, dorder;
        DevBuf<char> dval;
        if ((rc = drp.upload(c, rp)) || (rc = dcol.upload(c, col.empty() ? std::vector<int>(1, 0) : col))) return rc;
        if (prec == NISE_FP32) {
            std::vector<float> vf(vd.begin(), vd.end());
            if (vf.empty()) vf.push_back(0);
            if ((rc = dval.alloc(c, sizeof(float) * vf.size()))) return rc;
            cudaMemcpyAsync(dval.p, vf.data(), sizeof(float) * vf.size(), cudaMemcpyHostToDevice, c->stream);
        } else {
            if (vd.empty()) vd.push_back(0);
            if ((rc = dval.alloc(c, sizeof(double) * vd.size()))) return rc;
            cudaMemcpyAsync(dval.p, vd.data(), sizeof(double) * vd.size(), cudaMemcpyHostToDevice, c->stream);
        }
        if ((rc = dorder.alloc(c, (size_t)nf))) return rc;
        // sliced ELL (4-row slices, [slot][row]) of the same couplings for the
        // shared-memory kernel; entry offsets address rows of 10 complex numbers
        const int nsl = (N + 3) / 4;
        std::vector<int> sptr(nsl + 1, 0);
        for (int sl = 0; sl < nsl; sl++) {
            int L = 0;
            for (int r = 0; r < 4; r++) {
                int row = 4 * sl + r;
                if (row < N) L = std::max(L, rp[row + 1] - rp[row]);
            }
            sptr[sl + 1] = sptr[sl] + 4 * L;
        }
        const int nent = sptr[nsl];
        DevBuf<char> dell;
        DevBuf<int> dsptr;
        {
            size_t esz = prec == NISE_FP32 ? 8 : 16;
            std::vector<unsigned char> ell((size_t)(nent > 0 ? nent : 1) * esz, 0);
            for (int sl = 0; sl < nsl; sl++) {
                int L = (sptr[sl + 1] - sptr[sl]) / 4;
                for (int slot = 0; slot < L; slot++)
                    for (int r = 0; r < 4; r++) {
                        int row = 4 * sl + r, e = sptr[sl] + slot * 4 + r;
                        int off = (row < N ? row : 0) * 10;
                        double v = 0;
                        if (row < N && slot < rp[row + 1] - rp[row]) {
                            off = col[rp[row] + slot] * 10;
                            v = vd.empty() ? 0 : vd[rp[row] + slot];
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
            if ((rc = dell.alloc(c, ell.size()))) return rc;
            cudaMemcpyAsync(dell.p, ell.data(), ell.size(), cudaMemcpyHostToDevice, c->stream);
            if ((rc = dsptr.upload(c, sptr))) return rc;
        }
        TaylorPlan P;
        memset(&P, 0, sizeof(P));
        P.n = N;
        P.nnz = (int)col.size();
        P.row_ptr = drp.p;
        P.col = dcol.p;
        P.val = dval.p;
        P.static_j = 1;
        P.ell = dell.p;
        P.ell_sptr = dsptr.p;
        P.ell_nslices = nsl;
        P.ell_nent = nent;
        P.f0 = f0;
        P.nf = nf;
        P.singleshift = c->nshift > 0;
        if ((rc = nise_cuda(c, launch_prep_taylor(prec, T, P, rowabs, J.f, dorder.p, c->stream), "Taylor prep")))
            return rc;
        c->launches++;
        // per vector step and Taylor order: nnz complex*real products (4 flops)
        // and the diagonal, scaling and accumulation (6 flops per site)
        std::vector<int> order(nf);
        cudaMemcpyAsync(order.data(), dorder.p, sizeof(int) * nf, cudaMemcpyDeviceToHost, c->stream);
        if ((rc = nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "Taylor prep"))) return rc;
        double orders = 0;
        for (long t = 0; t < nf; t++) orders += (double)order[t] * cross[t];
        c->last_flops = orders * (4.0 * P.nnz + 6.0 * N);
        cudaEventRecord(c->evk0, c->stream);
        if (plain) {
            for (int s = 0; s < nsamp; s++) {
                AbsJob Js = J;
                Js.begin = begin + s;
                Js.nsamp = 1;
                if ((rc = nise_cuda(c, launch_abs_taylor(prec, T, P, Js, resp.p + (size_t)3 * s * tmax, 3, c->stream),
                                    "Taylor propagation")))
                    return rc;
                c->launches++;
            }
        } else {
            if ((rc = nise_cuda(c, launch_abs_taylor(prec, T, P, J, resp.p, 8, c->stream), "Taylor propagation")))
                return rc;
            c->launches++;
        }
        cudaEventRecord(c->evk1, c->stream);
        }
    }
    if ((rc = nise_cuda(c, launch_reduce_resp(resp.p, nvec, tmax, out.p, c->stream), "response reduction")))
        return rc;
    c->launches++;
    cudaEventRecord(c->ev1, c->stream);
    std::vector<double2> h(tmax);
    cudaMemcpyAsync(h.data(), out.p, sizeof(double2) * tmax, cudaMemcpyDeviceToHost, c->stream);
    if ((rc = nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "absorption"))) return rc;
    nise_collect_timing(c);
    for (int t = 0; t < tmax; t++) {
        re_S[t] = h[t].x;
        im_S[t] = h[t].y;
    }
    *samples = end;  // absorption.c:185 divides by `samples`, which equals end after the loop
    return NISE_OK;
}

// do_1DFFT (1DFFT.c:144-228): transform on the device, axis and window on the host.
extern "C" int nise_absorption_fft(nise_ctx *c, const double *re_S, const double *im_S, int samples, double *freq,
                                   double *spec_re, double *spec_im, int max_rows, int *rows) {
    if (!c || !re_S || !im_S || !freq || !spec_re || !spec_im || !rows)
        return nise_fail(c, NISE_ERR_ARG, "null argument");
    if (samples <= 0) return nise_fail(c, NISE_ERR_ARG, "samples must be positive");
    cudaSetDevice(c->p.device);
    const nise_params &p = c->p;
    int fft = p.fft < p.tmax1 ? p.tmax1 : p.fft;
    FftJob J;
    J.tmax = p.tmax1;
    J.fft = fft;
    J.samples = samples;
    J.window = p.window;
    J.fp32 = p.precision == NISE_FP32;
    J.deltat = p.deltat;
    J.lifetime = p.lifetime;
    J.homogen = p.homogen;
    J.inhomogen = p.inhomogen;
    std::vector<double2> h(p.tmax1);
    for (int i = 0; i < p.tmax1; i++) h[i] = make_double2(re_S[i], im_S[i]);
    DevBuf<double2> din, dspec;
    int rc;
    if ((rc = din.alloc(c, p.tmax1)) || (rc = dspec.alloc(c, fft))) return rc;
    cudaMemcpyAsync(din.p, h.data(), sizeof(double2) * p.tmax1, cudaMemcpyHostToDevice, c->stream);
    if ((rc = nise_cuda(c, launch_fft1d(J, din.p, dspec.p, c->stream), "1D FFT"))) return rc;
    std::vector<double2> spec(fft);
    cudaMemcpyAsync(spec.data(), dspec.p, sizeof(double2) * fft, cudaMemcpyDeviceToHost, c->stream);
    if ((rc = nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "1D FFT"))) return rc;
    const bool f32 = p.precision == NISE_FP32;
    float shift1 = c->shifte;
    int n = 0;
    auto emit = [&](int i, int num) {
        double w;
        if (f32) {
            float x = (float)num / p.deltat;
            x = x / kCv;
            x = x / (float)fft;
            x = x - shift1;
            w = -x;
            if (!((float)w > p.min1 && (float)w < p.max1)) return;
        } else {
            w = -((double)num / p.deltat / (double)kCv / fft - (double)shift1);
            if (!(w > p.min1 && w < p.max1)) return;
        }
        if (n < max_rows) {
            freq[n] = w;
            spec_re[n] = spec[i].x;
            spec_im[n] = spec[i].y;
        }
        n++;
    };
    for (int i = fft / 2; i <= fft - 1; i++) emit(i, fft - i);
    for (int i = 0; i <= fft / 2 - 1; i++) emit(i, -i);
    *rows = n < max_rows ? n : max_rows;
    return NISE_OK;
}

void nise_collect_timing(nise_ctx *c) {
    float ms = 0, kms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    cudaEventElapsedTime(&kms, c->evk0, c->evk1);
    c->last_ms = ms;
    c->last_main_ms = kms;
}

extern "C" int nise_set_stream(nise_ctx *c, void *stream) {
    if (!c) return nise_fail(nullptr, NISE_ERR_ARG, "null context");
    cudaStreamSynchronize(c->stream);
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return NISE_OK;
}

extern "C" int nise_last_timing(const nise_ctx *c, double *total_ms, double *main_kernel_ms, long *launches) {
    if (!c) return NISE_ERR_ARG;
    if (total_ms) *total_ms = c->last_ms;
    if (main_kernel_ms) *main_kernel_ms = c->last_main_ms;
    if (launches) *launches = c->launches;
    return NISE_OK;
}

extern "C" int nise_last_work(const nise_ctx *c, double *flops, double *hbm_bytes) {
    if (!c) return NISE_ERR_ARG;
    if (flops) *flops = c->last_flops;
    if (hbm_bytes) *hbm_bytes = c->last_bytes;
    return NISE_OK;
}

// ------------------------------------------------------------ single steps
extern "C" int nise_propagate(nise_ctx *c, const float *H, void *re, void *im, int nvec, int sign) {
    if (!c || !H || !re || !im || nvec <= 0 || (sign != 1 && sign != -1))
        return nise_fail(c, NISE_ERR_ARG, "bad nise_propagate arguments");
    cudaSetDevice(c->p.device);
    const nise_params &p = c->p;
    int N = c->n, prec = p.precision;
    size_t rsz = prec == NISE_FP32 ? sizeof(float) : sizeof(double);
    DevBuf<float> dH;
    DevBuf<char> dr, di;
    int rc;
    if ((rc = dH.alloc(c, (size_t)nvec * c->nn2)) || (rc = dr.alloc(c, rsz * nvec * N)) ||
        (rc = di.alloc(c, rsz * nvec * N)))
        return rc;
    cudaMemcpyAsync(dH.p, H, sizeof(float) * nvec * c->nn2, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(dr.p, re, rsz * nvec * N, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(di.p, im, rsz * nvec * N, cudaMemcpyHostToDevice, c->stream);
    int e;
    if (p.propagation == NISE_PROP_COUPLING)
        e = launch_step_coupling(prec, N, p.couplingcut, dH.p, dr.p, di.p, nvec, p.ts, nise_f64(p, sign, p.ts),
                                 nise_f32(p, sign, p.ts), c->stream);
    else if (p.propagation == NISE_PROP_RK4)
        e = launch_step_rk4(prec, N, p.couplingcut, dH.p, dr.p, di.p, nvec, p.ts, nise_f64(p, sign, p.ts),
                            nise_f32(p, sign, p.ts), c->stream);
    else {
        if (c->thres != 0 && !(c->thres > 1))
            return nise_fail(c, NISE_ERR_UNSUPPORTED, "Sparse with Threshold > 0 (truncated U) is not supported");
        e = launch_step_taylor(prec, N, dH.p, dr.p, di.p, nvec, nise_f64(p, sign, 1), c->stream);
    }
    if ((rc = nise_cuda(c, e, "propagate"))) return rc;
    cudaMemcpyAsync(re, dr.p, rsz * nvec * N, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(im, di.p, rsz * nvec * N, cudaMemcpyDeviceToHost, c->stream);
    return nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "propagate");
}

// ------------------------------------------------------------ writers
extern "C" int nise_write_td_absorption(const char *path, const nise_params *p, const double *re_S,
                                        const double *im_S, int samples) {
    if (!path || !p || !re_S || !im_S || samples <= 0) return NISE_ERR_ARG;
    FILE *f = fopen(path, "w");
    if (!f) return NISE_ERR_IO;
    for (int t1 = 0; t1 < p->tmax1; t1++) {  // absorption.c:181-189
        fprintf(f, "%f ", t1 * p->deltat);
        if (p->precision == NISE_FP32)
            fprintf(f, "%e %e ", (float)(re_S[t1] / samples), (float)(im_S[t1] / samples));
        else
            fprintf(f, "%e %e ", re_S[t1] / samples, im_S[t1] / samples);
        fprintf(f, "\n");
    }
    fclose(f);
    return NISE_OK;
}

extern "C" int nise_write_spectrum(const char *path, const double *freq, const double *spec_re,
                                   const double *spec_im, int rows) {
    if (!path || rows < 0) return NISE_ERR_ARG;
    FILE *f = fopen(path, "w");
    if (!f) return NISE_ERR_IO;
    for (int i = 0; i < rows; i++) {  // 1DFFT.c:212-216
        fprintf(f, "%f ", freq[i]);
        fprintf(f, "%e %e ", spec_re[i], spec_im[i]);
        fprintf(f, "\n");
    }
    fclose(f);
    return NISE_OK;
}

extern "C" int nise_write_2d(const char *path, const nise_params *p, const double *re, const double *im,
                             int sample_count) {
    if (!path || !p || !re || !im || sample_count <= 0) return NISE_ERR_ARG;
    FILE *f = fopen(path, "w");
    if (!f) return NISE_ERR_IO;
    for (int t1 = 0; t1 < p->tmax1; t1++) {  // print2D, MPI_subs.c:20-34
        int t2 = p->tmax2;
        for (int t3 = 0; t3 < p->tmax3; t3++) {
            double r = re[(size_t)t3 * p->tmax1 + t1] / sample_count, i = im[(size_t)t3 * p->tmax1 + t1] / sample_count;
            if (t3 == 0) r /= 2, i /= 2;
            if (p->precision == NISE_FP32) r = (float)r, i = (float)i;
            fprintf(f, "%f %f %f %e %e\n", t1 * p->deltat, t2 * p->deltat, t3 * p->deltat, r, i);
        }
    }
    fclose(f);
    return NISE_OK;
}
