// FP32 FMA throughput of the device: the compute roofline of the superposition
// kernel (the superposition runs on the FP32 pipe, not on the tensor cores).
#include <cuda_runtime.h>

#include <string>

#include "../../include/subsecondpbs.h"
#include "context.h"

namespace pbs {

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) ffma_loop(float* out, float seed) {
    float a[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) a[c] = seed + float(threadIdx.x + c);
    const float m = 0.9999999f, k = 1e-7f;
    for (int i = 0; i < kIters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) a[c] = fmaf(a[c], m, k);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += a[c];
    if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the loop alive; never true in practice
}

}  // namespace

int measure_fp32_peak(int gpu, double* tflops) {
    cudaError_t e = cudaSetDevice(gpu);
    if (e != cudaSuccess) {
        set_error(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
        return PBS_ERR_CUDA;
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, gpu);
    const int blocks = sms * 8;
    float* out = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    float best = 1e30f;
    if ((e = cudaMalloc(&out, blocks * sizeof(float))) != cudaSuccess) goto done;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    for (int rep = 0; rep < 6; ++rep) {
        cudaEventRecord(a);
        ffma_loop<<<blocks, 256>>>(out, 1.0f + rep);
        cudaEventRecord(b);
        if ((e = cudaEventSynchronize(b)) != cudaSuccess) goto done;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (rep > 0 && ms < best) best = ms;  // first launch is a warm-up
    }
    e = cudaGetLastError();
done:
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (out) cudaFree(out);
    if (e != cudaSuccess) {
        set_error(std::string("fp32 peak probe: ") + cudaGetErrorString(e));
        return PBS_ERR_CUDA;
    }
    const double flops = 2.0 * double(blocks) * 256.0 * kChains * kIters;
    *tflops = flops / (double(best) * 1e-3) / 1e12;
    return PBS_OK;
}

}  // namespace pbs
