// Engine-internal host definitions shared by api.cpp and the 2D driver.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "devtypes.h"
#include "nise_b200.h"

struct nise_ctx {
    nise_params p;
    std::string err;
    int n = 0;
    long nn2 = 0;
    float shifte = 0;
    float thres = 0;  // Threshold after the reference's rescaling
    cudaStream_t stream = nullptr;      // stream all work is enqueued on
    cudaStream_t own_stream = nullptr;  // the context's own stream
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evk0 = nullptr, evk1 = nullptr;
    double last_ms = 0, last_main_ms = 0;
    double last_flops = 0, last_bytes = 0;
    long launches = 0;
    bool loaded = false;
    // trajectory in device memory (record images, 4-byte words)
    float *d_energy = nullptr, *d_dipole = nullptr, *d_hc = nullptr, *d_mu_static = nullptr;
    float *d_anh = nullptr, *d_over = nullptr, *d_shift_ab = nullptr;
    int *d_shift_ptr = nullptr;  // [N+1] SingleShift entries per site
    int nshift = 0;
    long e_words = 0, e_frames = 0, d_words = 0, d_frames = 0, a_frames = 0, o_frames = 0;
    size_t cap_energy = 0, cap_dipole = 0, cap_anh = 0, cap_over = 0, cap_hc = 0, cap_mu = 0, cap_ab = 0;
    // operator records of the linear techniques: polarisabilities (Raman,
    // SFG; 6N per frame) and positions (CD; 3N per frame)
    float *d_alpha = nullptr, *d_pos = nullptr;
    long al_frames = 0, pos_frames = 0;
    size_t cap_alpha = 0, cap_pos = 0;
    std::vector<float> h_hc;        // coupling frame (HamiltonianType Coupling), shifted, cut
    std::vector<float> h_hc_raw;    // the coupling record as given (an unchanged one is not processed again)
    std::vector<float> h_mu_static; // dipoles of frame 0 (HamiltonianType Coupling)
    // Energy records copied from pinned host memory in frame chunks on
    // copy_stream: chunk k holds frames [chunk_end[k-1], chunk_end[k]) and
    // completes chunk_ev[k].  Kernels wait for the chunks they read
    // (nise_wait_frames), so the copy overlaps the propagation.
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copy_ready = nullptr;
    std::vector<cudaEvent_t> chunk_ev;
    std::vector<long> chunk_end;
    int nchunks = 0;
    // The linear-absorption plan of the last call (tables, sliced ELL, work
    // buffers), reused while plan_epoch is unchanged: every change of the
    // trajectory layout, couplings, SingleShift or stream advances it.
    long plan_epoch = 0;
    long abs_plan_epoch = -1;
    std::shared_ptr<void> abs_plan;
};

// Make stream s wait until energy frames [0, last_frame] are on the device.
void nise_wait_frames(nise_ctx *c, cudaStream_t s, long last_frame);
void nise_wait_all_frames(nise_ctx *c, cudaStream_t s);

int nise_fail(nise_ctx *c, int code, const char *fmt, ...);
int nise_cuda(nise_ctx *c, int e, const char *what);
float nise_f32(const nise_params &p, int sign, int m);
double nise_f64(const nise_params &p, int sign, int m);
DevTraj nise_devtraj(const nise_ctx *c);
int nise_pattern(nise_ctx *c, long f0, long nf, std::vector<int2> &pairs);
int nise_check_frames(nise_ctx *c, long last_frame);
// Device time between ev0/ev1 (whole call) and evk0/evk1 (main kernels).
void nise_collect_timing(nise_ctx *c);
// Rows of Absorption.dat (1DFFT.c:208-228) from a device spectrum spec[fft];
// returns the number of rows written (at most max_rows).
int nise_spectrum_rows(const nise_ctx *c, const double2 *spec, int fft, double *freq, double *spec_re,
                       double *spec_im, int max_rows);
extern "C" void nise_set_global_error(const char *msg);

// Stream-ordered device buffer owned by one call.
template <typename T> struct DevBuf {
    T *p = nullptr;
    cudaStream_t s = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    int alloc(nise_ctx *c, size_t count) {
        s = c->stream;
        if (count == 0) count = 1;
        if (cudaMallocAsync((void **)&p, sizeof(T) * count, s) != cudaSuccess) {
            p = nullptr;
            return nise_fail(c, NISE_ERR_NOMEM, "device allocation of %zu bytes failed", sizeof(T) * count);
        }
        return NISE_OK;
    }
    int upload(nise_ctx *c, const std::vector<T> &h) {
        int rc = alloc(c, h.size());
        if (rc) return rc;
        if (!h.empty()) cudaMemcpyAsync(p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s);
        return NISE_OK;
    }
    ~DevBuf() {
        if (p) cudaFreeAsync(p, s);
    }
};

// Device buffers behind a SinglesTab (and the eigen route's doubles sub-step
// propagators Us[t][n][n] when requested).
struct SinglesBufs {
    DevBuf<int2> pairs, ent;
    DevBuf<int4> segs;
    DevBuf<char> U, rot, rkval;
    const void *Us = nullptr;
};

// Build the singles scheme's coefficient tables for frames [f0, f0 + nf)
// of the context's trajectory (singleshift: apply SingleShift to the
// diagonal, as read_Hamiltonian does); doubles_u adds the eigen route's
// truncated sub-step propagators for doubles propagation.
int nise_singles_tables(nise_ctx *c, const DevTraj &T, long f0, long nf, int singleshift, bool doubles_u,
                        SinglesTab &S, SinglesBufs &B);
