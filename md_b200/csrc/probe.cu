// Diagnostic FMA throughput probe (mdf_probe_fma_tflops): the measured FP32 /
// FP64 CUDA-core peak that the pair kernel's roofline is quoted against.
// Independent dependency chains per thread keep every FMA pipe busy; the grid
// is a multiple of the SM count.
#include <cuda_runtime.h>

#include "mdf_internal.cuh"

namespace mdf {

template <typename R, int CHAINS, int ITERS>
__global__ void __launch_bounds__(256) k_fma_probe(R* out, R a, R b)
{
    R v[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) v[c] = (R)(threadIdx.x + c);
    for (int i = 0; i < ITERS; ++i) {
#pragma unroll
        for (int c = 0; c < CHAINS; ++c) v[c] = v[c] * a + b;
    }
    R s = 0;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += v[c];
    if (s == (R)-12345.678) out[0] = s;   // keeps the chains alive
}

template <typename R>
static double probe(int device)
{
    MDF_CUDA_TRY(cudaSetDevice(device));
    int sms = 0;
    MDF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    constexpr int CHAINS = 8, ITERS = 4096;
    const int threads = 256, blocks = sms * 16;
    R* out;
    MDF_CUDA_TRY(cudaMalloc(&out, sizeof(R)));
    cudaEvent_t e0, e1;
    MDF_CUDA_TRY(cudaEventCreate(&e0));
    MDF_CUDA_TRY(cudaEventCreate(&e1));
    k_fma_probe<R, CHAINS, ITERS><<<blocks, threads>>>(out, (R)0.999, (R)1e-3);   // warm-up
    MDF_CUDA_TRY(cudaGetLastError());
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        MDF_CUDA_TRY(cudaEventRecord(e0));
        k_fma_probe<R, CHAINS, ITERS><<<blocks, threads>>>(out, (R)0.999, (R)1e-3);
        MDF_CUDA_TRY(cudaEventRecord(e1));
        MDF_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0;
        MDF_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    double flops = 2.0 * CHAINS * (double)ITERS * threads * (double)blocks;
    return flops / (best * 1e-3) / 1e12;
}

}  // namespace mdf

extern "C" int mdf_probe_fma_tflops(int device, int precision, double* tflops)
{
    if (!tflops) return MDF_ERR_INVALID;
    try {
        *tflops = precision == MDF_PREC_FP64 ? mdf::probe<double>(device) : mdf::probe<float>(device);
        return MDF_OK;
    } catch (const mdf::CudaError&) {
        return MDF_ERR_CUDA;
    }
}
