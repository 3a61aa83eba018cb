// probe.cu -- FP64 throughput of the device, the denominators of the
// rooflines (no FP64 figure is published for this pool):
//   ecg_probe_fp64_peak         FMA pipe: each thread runs 8 independent
//                               register-resident FMA chains (pair kernels)
//   ecg_probe_fp64_tensor_peak  FP64 tensor cores: each warp runs 8
//                               independent mma.sync.m8n8k4.f64 chains
//                               (the LDL^H and candidate GEMM tiles)
// Both grids cover every SM several times over.
#include <cuda_runtime.h>
#include "../../include/ecg_abi.h"

namespace {

__global__ void __launch_bounds__(256) k_fp64_fma(double* out, int iters, double a, double b)
{
    double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-10, x2 = x0 + 2e-10, x3 = x0 + 3e-10;
    double x4 = x0 + 4e-10, x5 = x0 + 5e-10, x6 = x0 + 6e-10, x7 = x0 + 7e-10;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    const double s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 12345.678) out[blockIdx.x] = s;  // keeps the chains live
}

__global__ void __launch_bounds__(256) k_fp64_mma(double* out, int iters, double a, double b)
{
    double c[8][2];
#pragma unroll
    for (int j = 0; j < 8; j++) c[j][0] = c[j][1] = threadIdx.x * 1e-9 + j;
    const double av = a + threadIdx.x * 1e-12;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int j = 0; j < 8; j++)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                         : "+d"(c[j][0]), "+d"(c[j][1])
                         : "d"(av), "d"(b));
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 8; j++) s += c[j][0] + c[j][1];
    if (s == 12345.678) out[blockIdx.x] = s;  // keeps the chains live
}

// Run `kern` once to warm up and once timed; flops per thread per iteration
// given by the caller.
template <typename F>
int time_probe(int device, F launch, double flops_per_iter_block, int blocks_per_sm, double* tflops)
{
    if (!tflops) return ECG_EARG;
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return ECG_ENODEV;
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * blocks_per_sm;
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * blocks) != cudaSuccess) {
        cudaGetLastError();
        return ECG_ENOMEM;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int iters = 4096;
    launch(blocks, out, 64);  // warm-up
    cudaEventRecord(e0);
    launch(blocks, out, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    *tflops = flops_per_iter_block * iters * blocks / (ms * 1e-3) / 1e12;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return cudaGetLastError() == cudaSuccess ? ECG_OK : ECG_ECUDA;
}

}  // namespace

extern "C" int ecg_probe_fp64_tensor_peak(int device, double* tflops)
{
    // per block and iteration: 8 warps x 8 mma x (2 x 8 x 8 x 4) flops
    return time_probe(
        device, [](int blocks, double* out, int it) { k_fp64_mma<<<blocks, 256>>>(out, it, 0.999999, 1e-7); },
        8.0 * 8 * 2 * 8 * 8 * 4, 4, tflops);
}

extern "C" int ecg_probe_fp64_peak(int device, double* tflops)
{
    if (!tflops) return ECG_EARG;
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return ECG_ENODEV;
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * sms * 16) != cudaSuccess) {
        cudaGetLastError();
        return ECG_ENOMEM;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8, iters = 4096;
    k_fp64_fma<<<blocks, 256>>>(out, 64, 0.999999, 1e-7);  // warm-up
    cudaEventRecord(e0);
    k_fp64_fma<<<blocks, 256>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    const double flops = 2.0 * 8 * 16 * (double)iters * blocks * 256;
    *tflops = flops / (ms * 1e-3) / 1e12;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return cudaGetLastError() == cudaSuccess ? ECG_OK : ECG_ECUDA;
}
