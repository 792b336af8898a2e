// bcc_diag.cu -- FP32 FMA-pipe peak probe: the roofline denominator of the
// checker, whose work is scalar FP32 (no tensor-core or HBM bound applies).
// Each thread runs 8 independent FMA chains; 2 FLOP per FMA.
#include <cuda_runtime.h>

#include "../../include/bcc.h"

namespace {

__global__ void __launch_bounds__(256) fma_peak_kernel(float* out, int iters, float a, float b) {
    float x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
    float x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
        }
    }
    const float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

extern "C" bcc_status bcc_measure_fp32_peak(int32_t device, double* tflops) {
    if (!tflops) return BCC_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return BCC_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 8, threads = 256, iters = 4096;
    float* out = nullptr;
    if (cudaMalloc(&out, sizeof(float) * blocks * threads) != cudaSuccess) return BCC_ERR_CUDA;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_peak_kernel<<<blocks, threads>>>(out, 64, 0.999f, 0.001f);
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(e0);
        fma_peak_kernel<<<blocks, threads>>>(out, iters, 0.999f, 0.001f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return BCC_ERR_CUDA;
    const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return BCC_OK;
}
