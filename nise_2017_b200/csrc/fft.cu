// Final transforms on the device: the 1D absorption spectrum (1DFFT.c:144-206).
//
// The response has at most a few thousand points, so the transform is a
// direct DFT in FP64 with exact twiddle indices ((j*k) mod n), one output per
// thread: O(n^2) work that finishes in microseconds and matches FFTW to
// rounding for any n, including the non-power-of-two sizes NISE allows.
#include "common.cuh"
#include "engine.h"

namespace {

__device__ __forceinline__ float c_v32() { return 2.99792458e-5f; }
__device__ __forceinline__ float twopi32() { return (float)(2 * 3.14159265359); }

// fftIn of do_1DFFT: swapped (Im, Re)/samples, decays, Hann window, first
// point halved (1DFFT.c:170-200).  In FP32 mode the decay exponents are
// formed in single precision like the reference; the products are double.
__global__ void k_fft_input(FftJob J, const double2 *S, double2 *in) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= J.fft) return;
    double2 z = make_double2(0.0, 0.0);
    if (i < J.tmax) {
        z.x = S[i].y / J.samples;
        z.y = S[i].x / J.samples;
        if (J.fp32) {
            float dt = (float)J.deltat, fi = (float)(-i);
            if (J.lifetime > 0.0) {
                double d = exp((double)__fdiv_rn(__fmul_rn(fi, dt), __fmul_rn(2.0f, (float)J.lifetime)));
                z.x *= d; z.y *= d;
            }
            if (J.homogen > 0.0) {
                double d = exp((double)__fdiv_rn(__fmul_rn(fi, dt), __fmul_rn(2.0f, (float)J.homogen)));
                z.x *= d; z.y *= d;
            }
            if (J.inhomogen > 0.0) {
                float num = __fmul_rn(__fmul_rn(__fmul_rn(fi, dt), (float)i), dt);
                float den = __fmul_rn(__fmul_rn(2.0f, (float)J.inhomogen), (float)J.inhomogen);
                double d = exp((double)__fdiv_rn(num, den));
                z.x *= d; z.y *= d;
            }
            if (J.window == 1) {
                float a = __fdiv_rn(__fmul_rn((float)i, twopi32()), (float)(4 * J.tmax - 4));
                double w = cos((double)a) * cos((double)a);
                z.x *= w; z.y *= w;
            }
        } else {
            double twopi = (double)twopi32();
            if (J.lifetime > 0.0) { double d = exp(-i * J.deltat / (2 * J.lifetime)); z.x *= d; z.y *= d; }
            if (J.homogen > 0.0) { double d = exp(-i * J.deltat / (2 * J.homogen)); z.x *= d; z.y *= d; }
            if (J.inhomogen > 0.0) {
                double d = exp(-i * J.deltat * i * J.deltat / (2 * J.inhomogen * J.inhomogen));
                z.x *= d; z.y *= d;
            }
            if (J.window == 1) {
                double a = i * twopi / (4 * J.tmax - 4);
                double w = cos(a) * cos(a);
                z.x *= w; z.y *= w;
            }
        }
        if (i == 0) { z.x *= 0.5; z.y *= 0.5; }
    }
    in[i] = z;
}

// Forward DFT out[k] = sum_j in[j] exp(-2 pi i jk/n) followed by the output
// scaling of 1DFFT.c:203-206 (spec = (Out.im, Out.re) * 2 dt c_v, stored as
// float in FP32 mode as the reference's spec arrays are).
__global__ void k_dft_spec(FftJob J, const double2 *in, double2 *spec) {
    extern __shared__ double2 tile[];
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    int n = J.fft;
    double sr = 0, si = 0;
    for (int base = 0; base < n; base += blockDim.x) {
        int j = base + threadIdx.x;
        tile[threadIdx.x] = j < n ? in[j] : make_double2(0.0, 0.0);
        __syncthreads();
        int lim = min((int)blockDim.x, n - base);
        if (k < n)
            for (int q = 0; q < lim; q++) {
                long m = ((long)(base + q) * k) % n;
                double s, c;
                sincospi(-2.0 * (double)m / n, &s, &c);
                double2 z = tile[q];
                sr += z.x * c - z.y * s;
                si += z.x * s + z.y * c;
            }
        __syncthreads();
    }
    if (k >= n) return;
    double scale = 2.0 * J.deltat * (double)c_v32();
    double2 o = make_double2(si * scale, sr * scale);
    if (J.fp32) {
        o.x = (double)(float)(si * 2 * (double)(float)J.deltat * (double)c_v32());
        o.y = (double)(float)(sr * 2 * (double)(float)J.deltat * (double)c_v32());
    }
    spec[k] = o;
}

}  // namespace

int launch_fft1d_buf(const FftJob &J, const double2 *resp, double2 *spec, double2 *in, cudaStream_t s) {
    k_fft_input<<<(J.fft + 255) / 256, 256, 0, s>>>(J, resp, in);
    k_dft_spec<<<(J.fft + 255) / 256, 256, 256 * sizeof(double2), s>>>(J, in, spec);
    return (int)cudaGetLastError();
}

int launch_fft1d(const FftJob &J, const double2 *resp, double2 *spec, cudaStream_t s) {
    double2 *in = nullptr;
    int e;
    if ((e = (int)cudaMallocAsync((void **)&in, sizeof(double2) * J.fft, s))) return e;
    k_fft_input<<<(J.fft + 255) / 256, 256, 0, s>>>(J, resp, in);
    k_dft_spec<<<(J.fft + 255) / 256, 256, 256 * sizeof(double2), s>>>(J, in, spec);
    e = (int)cudaGetLastError();
    cudaFreeAsync(in, s);
    return e;
}
