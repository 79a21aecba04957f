// Diagnostic throughput probes: mdf_probe_fma_tflops, the measured FP32 /
// FP64 CUDA-core peak that the pair kernel's roofline is quoted against, and
// mdf_probe_l2_reductions, the measured L2 int64 reduction rate that the PME
// charge spread (an L2-resident fixed-point grid) is quoted against.
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

// L2 int64 reduction throughput on a buffer of `words` 64-bit words (sized
// to stay in L2, like the PME charge grid).  PATTERN 0 is the charge
// spread's: each thread adds 4 consecutive words (one 32-byte sector) at a
// pseudo-random 32-byte-aligned row; PATTERN 1 is the friendliest form: each
// warp adds 32 consecutive words (one 256-byte run) at a pseudo-random
// 256-byte-aligned base.  Indices come from a per-thread linear congruential
// sequence, reduced modulo the row count, so every access lies in the buffer.
template <int PATTERN>
__global__ void __launch_bounds__(256) k_red_probe(unsigned long long* __restrict__ buf, long long words, int iters)
{
    const unsigned tid = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned x = tid * 2654435761u + 12345u;
    if (PATTERN == 0) {
        const unsigned long long rows = (unsigned long long)(words / 4);
        for (int it = 0; it < iters; ++it) {
            x = x * 1664525u + 1013904223u;
            unsigned long long* p = buf + 4 * (unsigned long long)(x % rows);
#pragma unroll
            for (int k = 0; k < 4; ++k) atomicAdd(p + k, 1ull);
        }
    } else {
        const unsigned long long runs = (unsigned long long)(words / 32);
        unsigned w = (tid >> 5) * 2654435761u + 777u;
        for (int it = 0; it < iters; ++it) {
            w = w * 1664525u + 1013904223u;
            atomicAdd(buf + 32 * (unsigned long long)(w % runs) + (threadIdx.x & 31), 1ull);
        }
    }
}

static double probe_red(int device, long long words, int pattern)
{
    MDF_CUDA_TRY(cudaSetDevice(device));
    if (words < 1024) throw ApiError(MDF_ERR_INVALID, "probe buffer too small");
    int sms = 0;
    MDF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int threads = 256, blocks = sms * 8, iters = pattern == 0 ? 64 : 256;
    unsigned long long* buf;
    MDF_CUDA_TRY(cudaMalloc(&buf, sizeof(unsigned long long) * (size_t)words));
    MDF_CUDA_TRY(cudaMemset(buf, 0, sizeof(unsigned long long) * (size_t)words));
    cudaEvent_t e0, e1;
    MDF_CUDA_TRY(cudaEventCreate(&e0));
    MDF_CUDA_TRY(cudaEventCreate(&e1));
    auto launch = [&]() {
        if (pattern == 0) k_red_probe<0><<<blocks, threads>>>(buf, words, iters);
        else k_red_probe<1><<<blocks, threads>>>(buf, words, iters);
    };
    launch();   // warm-up (brings the buffer into L2)
    MDF_CUDA_TRY(cudaGetLastError());
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        MDF_CUDA_TRY(cudaEventRecord(e0));
        launch();
        MDF_CUDA_TRY(cudaEventRecord(e1));
        MDF_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0;
        MDF_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    const double reds = (double)threads * blocks * iters * (pattern == 0 ? 4.0 : 1.0);
    return reds / (best * 1e-3);
}

}  // namespace mdf

extern "C" int mdf_probe_l2_reductions(int device, int64_t words, int pattern, double* per_s)
{
    if (!per_s || (pattern != 0 && pattern != 1)) return MDF_ERR_INVALID;
    try {
        *per_s = mdf::probe_red(device, (long long)words, pattern);
        return MDF_OK;
    } catch (const mdf::ApiError& e) {
        return e.status;
    } catch (const mdf::CudaError&) {
        return MDF_ERR_CUDA;
    }
}

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
