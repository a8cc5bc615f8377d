// C ABI of the engine (include/nise_b200.h): context, trajectory loading,
// job planning and the output writers.  No exit() on any path: every failure
// is a status code plus a message.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdint>
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
    if (!e) {
        // Jobs allocate their tables stream-ordered from the device's default
        // pool; keep freed blocks in the pool (this process only) instead of
        // returning them to the driver at every synchronisation, so repeated
        // jobs do not remap memory.
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, p->device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
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
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    c->nchunks = 0;
    c->plan_epoch++;
    void *ptrs[] = {c->d_energy, c->d_dipole, c->d_hc, c->d_mu_static, c->d_anh, c->d_over, c->d_shift_ptr,
                    c->d_shift_ab, c->d_alpha, c->d_pos};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    c->d_energy = c->d_dipole = c->d_hc = c->d_mu_static = c->d_anh = c->d_over = c->d_shift_ab = nullptr;
    c->d_alpha = c->d_pos = nullptr;
    c->d_shift_ptr = nullptr;
    c->cap_energy = c->cap_dipole = c->cap_anh = c->cap_over = c->cap_hc = c->cap_mu = c->cap_ab = 0;
    c->cap_alpha = c->cap_pos = 0;
    c->al_frames = c->pos_frames = 0;
    c->loaded = false;
}

// Every device trajectory image carries kImageSlack bytes past its last
// record: bulk copies of a record, widened to 16-byte boundaries, stay inside
// the allocation.
static const size_t kImageSlack = 256;

extern "C" void nise_destroy(nise_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->p.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    c->abs_plan.reset();  // its buffers are freed on the stream they were allocated on
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->stream = c->own_stream;
    nise_free_traj(c);
    cudaEvent_t evs[] = {c->ev0, c->ev1, c->evk0, c->evk1, c->copy_ready};
    for (cudaEvent_t ev : evs)
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : c->chunk_ev) cudaEventDestroy(ev);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

void nise_wait_frames(nise_ctx *c, cudaStream_t s, long last_frame) {
    for (int k = 0; k < c->nchunks; k++)
        if (c->chunk_end[k] > last_frame || k == c->nchunks - 1) {
            cudaStreamWaitEvent(s, c->chunk_ev[k], 0);
            return;
        }
}

void nise_wait_all_frames(nise_ctx *c, cudaStream_t s) {
    if (c->nchunks) cudaStreamWaitEvent(s, c->chunk_ev[c->nchunks - 1], 0);
}

// Energy image from pinned host memory in chunks of about 16 MB on the copy
// stream, after the work already enqueued on the context's stream (which may
// still read the old image); the copies complete the chunk events.
static int upload_energy_chunked(nise_ctx *c, const void *src, size_t bytes) {
    if (bytes > c->cap_energy) {
        cudaStreamSynchronize(c->stream);
        if (c->d_energy) cudaFree(c->d_energy);
        c->d_energy = nullptr;
        c->cap_energy = 0;
        if (cudaMalloc((void **)&c->d_energy, bytes + kImageSlack) != cudaSuccess)
            return nise_fail(c, NISE_ERR_NOMEM, "device allocation of %zu bytes failed", bytes);
        cudaMemsetAsync((char *)c->d_energy + bytes, 0, kImageSlack, c->stream);
        c->cap_energy = bytes;
    }
    if (!c->copy_stream && cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
        return nise_fail(c, NISE_ERR_DEVICE, "copy stream creation failed");
    if (!c->copy_ready && cudaEventCreateWithFlags(&c->copy_ready, cudaEventDisableTiming) != cudaSuccess)
        return nise_fail(c, NISE_ERR_DEVICE, "event creation failed");
    cudaEventRecord(c->copy_ready, c->stream);
    cudaStreamWaitEvent(c->copy_stream, c->copy_ready, 0);
    const size_t rec = 4 * (size_t)c->e_words;
    const long per = std::max(1L, (long)(((size_t)16 << 20) / rec));
    c->nchunks = 0;
    c->chunk_end.clear();
    for (long f0 = 0; f0 < c->e_frames; f0 += per) {
        const long f1 = std::min(c->e_frames, f0 + per);
        if ((int)c->chunk_ev.size() <= c->nchunks) {
            cudaEvent_t ev;
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
                return nise_fail(c, NISE_ERR_DEVICE, "event creation failed");
            c->chunk_ev.push_back(ev);
        }
        int e = (int)cudaMemcpyAsync((char *)c->d_energy + (size_t)f0 * rec, (const char *)src + (size_t)f0 * rec,
                                     (size_t)(f1 - f0) * rec, cudaMemcpyHostToDevice, c->copy_stream);
        if (e) return nise_cuda(c, e, "trajectory upload");
        cudaEventRecord(c->chunk_ev[c->nchunks], c->copy_stream);
        c->chunk_end.push_back(f1);
        c->nchunks++;
    }
    return NISE_OK;
}

static bool pinned_host(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
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
        if (cudaMalloc((void **)dst, bytes + kImageSlack) != cudaSuccess)
            return nise_fail(c, NISE_ERR_NOMEM, "device allocation of %zu bytes failed", bytes);
        cudaMemsetAsync((char *)*dst + bytes, 0, kImageSlack, c->stream);
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
    const size_t ebytes = (size_t)c->e_frames * 4 * c->e_words;
    // the plan of the previous call stays valid for the same layout and the
    // same couplings (the diagonal records are read by the kernels, not the plan)
    const long old_frames = c->e_frames, old_words = c->e_words;
    std::vector<float> old_hc;
    old_hc.swap(c->h_hc);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);  // an earlier chunked copy
    c->nchunks = 0;
    // the small records first: a pageable copy queued behind the chunked
    // energy copy on the copy engine would hold the host until it is done
    if ((rc = upload(c, &c->d_dipole, &c->cap_dipole, dipole, (size_t)c->d_frames * 4 * c->d_words))) return rc;
    c->a_frames = anharm ? (long)(anharm_bytes / (4 * (size_t)(1 + N))) : 0;
    c->o_frames = overtone ? (long)(overtone_bytes / (4 * (size_t)(1 + 3L * N))) : 0;
    if ((rc = upload(c, &c->d_anh, &c->cap_anh, anharm, (size_t)c->a_frames * 4 * (1 + N)))) return rc;
    if ((rc = upload(c, &c->d_over, &c->cap_over, overtone, (size_t)c->o_frames * 4 * (1 + 3L * N)))) return rc;
    const std::vector<float> old_mu = c->h_mu_static;
    c->h_mu_static.clear();
    bool hc_changed = true;
    if (coupling_type) {
        // read_coupling (read_trajectory.c:47-70): one Full record at position 0
        // with the read cut, and the dipoles of frame 0.
        if (!coupling || coupling_bytes < 4 * (size_t)full_words)
            return nise_fail(c, NISE_ERR_IO, "Coupling trajectory file to short");
        const float *raw = (const float *)coupling + 1;
        const bool same = c->d_hc && old_hc.size() == (size_t)c->nn2 && c->h_hc_raw.size() == (size_t)c->nn2 &&
                          memcmp(c->h_hc_raw.data(), raw, sizeof(float) * c->nn2) == 0;
        hc_changed = !same;
        if (same) {
            c->h_hc.swap(old_hc);  // processed and on the device already
        } else {
            c->h_hc_raw.assign(raw, raw + c->nn2);
            c->h_hc.assign(raw, raw + c->nn2);
            for (int i = 0; i < N; i++) c->h_hc[(size_t)i * N + i - (size_t)i * (i + 1) / 2] -= c->shifte;
            for (int i = 0; i < N; i++)
                for (int j = i + 1; j < N; j++) {
                    long idx = j + (long)i * ((N << 1) - i - 1) / 2;
                    if (fabs(c->h_hc[idx]) < p.couplingcut) c->h_hc[idx] = 0;
                }
            if ((rc = upload(c, &c->d_hc, &c->cap_hc, c->h_hc.data(), sizeof(float) * c->nn2))) return rc;
        }
        const float *m = (const float *)dipole + 1;
        c->h_mu_static.assign(m, m + 3L * N);
        if (!(c->d_mu_static && c->h_mu_static == old_mu) &&
            (rc = upload(c, &c->d_mu_static, &c->cap_mu, c->h_mu_static.data(), sizeof(float) * 3 * N)))
            return rc;
    } else {
        c->h_hc.clear();
        c->h_hc_raw.clear();
        if ((rc = upload(c, &c->d_hc, &c->cap_hc, nullptr, 0))) return rc;
        if ((rc = upload(c, &c->d_mu_static, &c->cap_mu, nullptr, 0))) return rc;
    }
    if (ebytes >= ((size_t)64 << 20) && pinned_host(energy)) {
        if ((rc = upload_energy_chunked(c, energy, ebytes))) return rc;
    } else if ((rc = upload(c, &c->d_energy, &c->cap_energy, energy, ebytes))) {
        return rc;
    }
    int e = (int)cudaStreamSynchronize(c->stream);
    if (e) return nise_cuda(c, e, "trajectory upload");
    if (!coupling_type || c->e_frames != old_frames || c->e_words != old_words || hc_changed || !c->loaded)
        c->plan_epoch++;
    c->loaded = true;
    return NISE_OK;
}

extern "C" int nise_set_trajectory_onfly(nise_ctx *c, const void *energy, size_t energy_bytes, const void *dipole,
                                         size_t dipole_bytes, const void *position, size_t position_bytes,
                                         const void *pbc, size_t pbc_bytes, const void *anharm, size_t anharm_bytes,
                                         const void *overtone, size_t overtone_bytes) {
    if (!c) return nise_fail(nullptr, NISE_ERR_ARG, "null context");
    const nise_params &p = c->p;
    if (p.hamiltonian != NISE_HAM_TDC && p.hamiltonian != NISE_HAM_EDC)
        return nise_fail(c, NISE_ERR_ARG, "couplings on the fly need HamiltonianType TransitionDipole or ExtendedDipole");
    if (!energy || !dipole || !position) return nise_fail(c, NISE_ERR_ARG, "energy, dipole and position records are required");
    cudaSetDevice(p.device);
    const int N = c->n;
    const bool edc = p.hamiltonian == NISE_HAM_EDC;
    const long full_words = 1 + c->nn2 + (long)p.doubles * (p.doubles + 1) / 2;
    const long dip_words = 1 + 3L * N + 3L * N * p.doubles;
    long frames = (long)(energy_bytes / (4 * (size_t)(1 + N)));
    const long d_frames = (long)(dipole_bytes / (4 * (size_t)dip_words));
    const long p_frames = (long)(position_bytes / (4 * (size_t)dip_words)) / (edc ? 2 : 1);
    if (frames < 1) return nise_fail(c, NISE_ERR_IO, "Hamiltonian trajectory file to short");
    // frames whose couplings can be built: every input must hold the frame
    frames = std::min(frames, std::min(d_frames, p_frames));
    if (pbc) frames = std::min(frames, (long)(pbc_bytes / 16));
    if (frames < 1) return nise_fail(c, NISE_ERR_IO, "Dipole/Position/PBC trajectory file to short");
    int rc;
    // dipoles, anharmonicities and overtone dipoles as for a Full trajectory
    c->d_words = dip_words;
    c->d_frames = d_frames;
    if ((rc = upload(c, &c->d_dipole, &c->cap_dipole, dipole, (size_t)d_frames * 4 * dip_words))) return rc;
    c->a_frames = anharm ? (long)(anharm_bytes / (4 * (size_t)(1 + N))) : 0;
    c->o_frames = overtone ? (long)(overtone_bytes / (4 * (size_t)(1 + 3L * N))) : 0;
    if ((rc = upload(c, &c->d_anh, &c->cap_anh, anharm, (size_t)c->a_frames * 4 * (1 + N)))) return rc;
    if ((rc = upload(c, &c->d_over, &c->cap_over, overtone, (size_t)c->o_frames * 4 * (1 + 3L * N)))) return rc;
    if ((rc = upload(c, &c->d_hc, &c->cap_hc, nullptr, 0))) return rc;
    if ((rc = upload(c, &c->d_mu_static, &c->cap_mu, nullptr, 0))) return rc;
    c->h_hc.clear();
    c->h_mu_static.clear();
    // inputs of the frame builder (freed when it is done) and the built records
    const size_t rec_bytes = (size_t)frames * 4 * full_words;
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    c->nchunks = 0;
    c->plan_epoch++;
    if (rec_bytes > c->cap_energy) {
        if (c->d_energy) cudaFree(c->d_energy);
        c->d_energy = nullptr;
        c->cap_energy = 0;
        if (cudaMalloc((void **)&c->d_energy, rec_bytes + kImageSlack) != cudaSuccess)
            return nise_fail(c, NISE_ERR_NOMEM, "couplings on the fly: %zu bytes of frame records do not fit", rec_bytes);
        c->cap_energy = rec_bytes;
    }
    DevBuf<char> ddiag, dpos, dpbc;
    const size_t pos_bytes = (size_t)frames * (edc ? 2 : 1) * 4 * dip_words;
    if ((rc = ddiag.alloc(c, (size_t)frames * 4 * (1 + N))) || (rc = dpos.alloc(c, pos_bytes)) ||
        (pbc && (rc = dpbc.alloc(c, (size_t)frames * 16))))
        return rc;
    cudaMemcpyAsync(ddiag.p, energy, (size_t)frames * 4 * (1 + N), cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(dpos.p, position, pos_bytes, cudaMemcpyHostToDevice, c->stream);
    if (pbc) cudaMemcpyAsync(dpbc.p, pbc, (size_t)frames * 16, cudaMemcpyHostToDevice, c->stream);
    OnflyJob J;
    J.diag = (const float *)ddiag.p;
    J.pos = (const float *)dpos.p;
    J.dip = c->d_dipole;
    J.pbc = pbc ? (const float *)dpbc.p : nullptr;
    J.frames = frames;
    J.full_words = full_words;
    J.dip_words = dip_words;
    J.n = N;
    J.edc = edc;
    if ((rc = nise_cuda(c, launch_onfly(J, c->d_energy, c->stream), "coupling frame builder"))) return rc;
    c->e_words = full_words;
    c->e_frames = frames;
    int e = (int)cudaStreamSynchronize(c->stream);
    if (e) return nise_cuda(c, e, "coupling frame builder");
    c->loaded = true;
    return NISE_OK;
}

extern "C" int nise_set_operators(nise_ctx *c, const void *alpha, size_t alpha_bytes, const void *position,
                                  size_t position_bytes) {
    if (!c) return nise_fail(nullptr, NISE_ERR_ARG, "null context");
    cudaSetDevice(c->p.device);
    const int N = c->n;
    // read_alpha (read_trajectory.c:380-399): int tag + 6N floats per frame;
    // CD positions with read_mue's layout (:357-377): int tag + 3N floats
    c->al_frames = alpha ? (long)(alpha_bytes / (4 * (size_t)(1 + 6L * N))) : 0;
    const long pw = 1 + 3L * N + 3L * N * c->p.doubles;  // read_mue's record
    c->pos_frames = position ? (long)(position_bytes / (4 * (size_t)pw)) : 0;
    if (alpha && c->al_frames < 1) return nise_fail(c, NISE_ERR_IO, "Polarizability trajectory file to short");
    if (position && c->pos_frames < 1) return nise_fail(c, NISE_ERR_IO, "Position trajectory file to short");
    int rc;
    if ((rc = upload(c, &c->d_alpha, &c->cap_alpha, alpha, (size_t)c->al_frames * 4 * (1 + 6L * N)))) return rc;
    if ((rc = upload(c, &c->d_pos, &c->cap_pos, position, (size_t)c->pos_frames * 4 * pw))) return rc;
    return nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "operator upload");
}

extern "C" int nise_set_singleshift(nise_ctx *c, int n, const int *sites, const float *a, const float *b) {
    if (!c || n < 0) return nise_fail(c, NISE_ERR_ARG, "bad SingleShift arguments");
    cudaSetDevice(c->p.device);
    // entries grouped by site, each site's in file order (apply_singleshift,
    // hamshift.c:59-66, applies them one after another)
    std::vector<int> ptr(c->n + 1, 0);
    for (int i = 0; i < n; i++) {
        if (sites[i] < 0 || sites[i] >= c->n) return nise_fail(c, NISE_ERR_ARG, "SingleShift site out of range");
        ptr[sites[i] + 1]++;
    }
    for (int s = 0; s < c->n; s++) ptr[s + 1] += ptr[s];
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    std::vector<float> ab(2 * (size_t)n);
    for (int i = 0; i < n; i++) {
        int e = fill[sites[i]]++;
        ab[2 * e] = a[i];
        ab[2 * e + 1] = b[i];
    }
    if (c->d_shift_ptr) cudaFree(c->d_shift_ptr);
    c->d_shift_ptr = nullptr;
    c->nshift = n;
    c->plan_epoch++;
    int rc;
    if (n) {
        if (cudaMalloc((void **)&c->d_shift_ptr, sizeof(int) * (c->n + 1)))
            return nise_fail(c, NISE_ERR_NOMEM, "device allocation failed");
        cudaMemcpyAsync(c->d_shift_ptr, ptr.data(), sizeof(int) * (c->n + 1), cudaMemcpyHostToDevice, c->stream);
    }
    if ((rc = upload(c, &c->d_shift_ab, &c->cap_ab, n ? ab.data() : nullptr, sizeof(float) * 2 * n))) return rc;
    return nise_cuda(c, (int)cudaStreamSynchronize(c->stream), "SingleShift upload");
}

extern "C" int nise_load_files(nise_ctx *c) {
    if (!c) return nise_fail(nullptr, NISE_ERR_ARG, "null context");
    const nise_params &p = c->p;
    std::vector<char> E, D, C, A, O;
    if (!read_file(p.energyFName, E)) return nise_fail(c, NISE_ERR_IO, "Hamiltonian file not found!");
    const bool no_dipoles = p.technique == NISE_TECH_DOS || p.technique == NISE_TECH_RAMAN;
    if (no_dipoles && p.hamiltonian != NISE_HAM_TDC && p.hamiltonian != NISE_HAM_EDC) {
        // calc_DOS and raman.c open no dipole file: one zero record stands in for it
        if (!read_file(p.dipoleFName, D)) D.assign(4 * (1 + 3 * (size_t)c->n), 0);
    } else if (!read_file(p.dipoleFName, D)) {
        return nise_fail(c, NISE_ERR_IO, "Dipole file %s not found!", p.dipoleFName);
    }
    if (p.hamiltonian == NISE_HAM_COUPLING && !read_file(p.couplingFName, C))
        return nise_fail(c, NISE_ERR_IO, "Coupling file not found!");
    // calc_2DIR.c:130-147 opens these files; calc_2DES (UVvis) reads neither
    bool two_d_ir = p.technique >= NISE_TECH_2DIR && p.technique <= NISE_TECH_NOEAIR;
    if (two_d_ir && p.anharmonicity == 0) {
        if (!read_file(p.anharFName, A))
            return nise_fail(c, NISE_ERR_IO, "Anharmonicity file %s not found!", p.anharFName);
        if (!read_file(p.overdipFName, O))
            return nise_fail(c, NISE_ERR_IO, "Overtone dipole file %s not found!", p.overdipFName);
    }
    int rc;
    if (p.hamiltonian == NISE_HAM_TDC || p.hamiltonian == NISE_HAM_EDC) {
        std::vector<char> P, B;
        if (!read_file(p.positionFName, P))
            return nise_fail(c, NISE_ERR_IO, "Atom position file for TDC on the fly not found!");
        if (p.pbcFName[0] && !read_file(p.pbcFName, B))
            return nise_fail(c, NISE_ERR_IO, "Periodic Boundary Condition file not found!");
        rc = nise_set_trajectory_onfly(c, E.data(), E.size(), D.data(), D.size(), P.data(), P.size(),
                                       B.empty() ? nullptr : B.data(), B.size(), A.empty() ? nullptr : A.data(),
                                       A.size(), O.empty() ? nullptr : O.data(), O.size());
    } else {
        rc = nise_set_trajectory(c, E.data(), E.size(), D.data(), D.size(), C.empty() ? nullptr : C.data(), C.size(),
                                 A.empty() ? nullptr : A.data(), A.size(), O.empty() ? nullptr : O.data(), O.size());
    }
    if (rc) return rc;
    // Alphafile (raman.c:74-78, sfg.c:82-86) and the CD Positionfile (calc_CD.c:84-88)
    if (p.technique == NISE_TECH_RAMAN || p.technique == NISE_TECH_SFG || p.technique == NISE_TECH_CD) {
        std::vector<char> Al, Ps;
        if (p.technique != NISE_TECH_CD && !read_file(p.alphaFName, Al))
            return nise_fail(c, NISE_ERR_IO, "%s file %s not found!",
                             p.technique == NISE_TECH_RAMAN ? "Raman" : "Polarizability", p.alphaFName);
        if (p.technique == NISE_TECH_CD && !read_file(p.positionFName, Ps))
            return nise_fail(c, NISE_ERR_IO, "Position file %s not found!", p.positionFName);
        if ((rc = nise_set_operators(c, Al.empty() ? nullptr : Al.data(), Al.size(),
                                     Ps.empty() ? nullptr : Ps.data(), Ps.size())))
            return rc;
    }
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
    T.full = c->p.hamiltonian != NISE_HAM_COUPLING;  // Full, or records built from positions
    T.dipole = c->d_dipole;
    T.d_words = c->d_words;
    T.d_frames = c->d_frames;
    T.mu_static = c->d_mu_static;
    T.hc = c->d_hc;
    T.anh = c->d_anh;
    T.a_frames = c->a_frames;
    T.over = c->d_over;
    T.o_frames = c->o_frames;
    T.shift_ptr = c->d_shift_ptr;
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
    *rows = nise_spectrum_rows(c, spec.data(), fft, freq, spec_re, spec_im, max_rows);
    return NISE_OK;
}

// Frequency axis and window of do_1DFFT (1DFFT.c:208-228): the rows of
// Absorption.dat from the device spectrum spec[fft].
int nise_spectrum_rows(const nise_ctx *c, const double2 *spec, int fft, double *freq, double *spec_re,
                       double *spec_im, int max_rows) {
    const nise_params &p = c->p;
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
    return n < max_rows ? n : max_rows;
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
    c->plan_epoch++;
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
extern "C" int nise_write_td(const char *path, const nise_params *p, const double *re_S, const double *im_S,
                             int samples, int trailing_blank) {
    if (!path || !p || !re_S || !im_S || samples <= 0) return NISE_ERR_ARG;
    FILE *f = fopen(path, "w");
    if (!f) return NISE_ERR_IO;
    for (int t1 = 0; t1 < p->tmax1; t1++) {  // absorption.c:181-189
        fprintf(f, "%f ", t1 * p->deltat);
        const char *fmt = trailing_blank ? "%e %e " : "%e %e";
        if (p->precision == NISE_FP32)
            fprintf(f, fmt, (float)(re_S[t1] / samples), (float)(im_S[t1] / samples));
        else
            fprintf(f, fmt, re_S[t1] / samples, im_S[t1] / samples);
        fprintf(f, "\n");
    }
    fclose(f);
    return NISE_OK;
}

extern "C" int nise_write_td_absorption(const char *path, const nise_params *p, const double *re_S,
                                        const double *im_S, int samples) {
    return nise_write_td(path, p, re_S, im_S, samples, 1);
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
