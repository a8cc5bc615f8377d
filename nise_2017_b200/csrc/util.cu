// Device measurement utilities.
#include <cuda_runtime.h>

#include "nise_b200.h"

extern "C" void nise_set_global_error(const char *msg);

namespace {
// Eight independent FMA chains per thread, long enough that issue, not
// latency, limits throughput.
__global__ void k_fma_probe(float *out, int iters, float a, float b) {
    float x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
          x7 = x0 + 7;
    for (int i = 0; i < iters; i++) {
        x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
        x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
    }
    float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 123.456f) out[0] = s;  // keeps the chains live
}
}  // namespace

extern "C" int nise_probe_fp32_peak(int device, double *tflops) {
    if (!tflops) return NISE_ERR_ARG;
    cudaDeviceProp prop;
    if (cudaSetDevice(device) != cudaSuccess || cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        nise_set_global_error("no CUDA device");
        return NISE_ERR_DEVICE;
    }
    float *out = nullptr;
    cudaMalloc(&out, sizeof(float));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int threads = 512, blocks = prop.multiProcessorCount * 4, iters = 1 << 16;
    k_fma_probe<<<blocks, threads>>>(out, 1024, 0.999f, 0.001f);  // warm-up
    cudaEventRecord(e0);
    k_fma_probe<<<blocks, threads>>>(out, iters, 0.999f, 0.001f);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess || ms <= 0) {
        nise_set_global_error(cudaGetErrorString(err));
        return NISE_ERR_DEVICE;
    }
    *tflops = 2.0 * 8.0 * iters * (double)threads * blocks / (ms * 1e-3) / 1e12;
    return NISE_OK;
}
