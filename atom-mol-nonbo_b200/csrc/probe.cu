// probe.cu -- FP64 FMA throughput of the device, the denominator of the
// pair kernels' roofline (no FP64 figure is published for this pool).
// Each thread runs 8 independent register-resident FMA chains; the grid
// covers every SM several times over.
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

}  // namespace

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
