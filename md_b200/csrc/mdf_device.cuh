// Device-side helpers shared by the libmdf kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mdf_internal.cuh"

namespace mdf {

template <typename R> struct V4;
template <> struct V4<float> { using type = float4; };
template <> struct V4<double> { using type = double4; };

__device__ __forceinline__ void status_set(unsigned* st, unsigned bit) { atomicOr(st, bit); }

// Fixed-point accumulation: order-independent, so results are bit-reproducible.
__device__ __forceinline__ void fx_add(unsigned long long* a, double v, double scale, unsigned* st)
{
    double s = v * scale;
    if (!(fabs(s) < 9.2e18)) {          // also catches NaN
        status_set(st, isfinite(v) ? ST_OVERFLOW : ST_NONFINITE);
        return;
    }
    atomicAdd(a, (unsigned long long)__double2ll_rn(s));
}

__device__ __forceinline__ void fx_add(unsigned long long* a, float v, double scale, unsigned* st)
{
    fx_add(a, (double)v, scale, st);
}

__device__ __forceinline__ long long to_fixed(double v, double scale) { return __double2ll_rn(v * scale); }

// FP32 force contribution straight to 2^-32 fixed point (the scaling is exact).
__device__ __forceinline__ void fx_add_force_f(unsigned long long* a, float v, unsigned* st)
{
    const float s = v * 4294967296.0f;
    if (!(fabsf(s) < 9.2e18f)) {
        status_set(st, isfinite(v) ? ST_OVERFLOW : ST_NONFINITE);
        return;
    }
    atomicAdd(a, (unsigned long long)__float2ll_rn(s));
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ long long warp_sum_ll(long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide deterministic sum of NV doubles per thread, converted to fixed
// point once per block and added to acc[idx[k]].  blockDim.x must be a
// multiple of 32 and <= 1024.  All threads of the block must call it.
template <int NV>
__device__ void block_acc_fixed(const double (&v)[NV], unsigned long long* acc, const int (&idx)[NV],
                                double scale, unsigned* st)
{
    __shared__ double red[32][NV > 0 ? NV : 1];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    double s[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) s[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) red[w][k] = s[k];
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = lane < nw ? red[lane][k] : 0.0;
            t = warp_sum(t);
            if (lane == 0 && t != 0.0) fx_add(acc + idx[k], t, scale, st);
        }
    }
    __syncthreads();
}

__host__ __device__ __forceinline__ double min_image(double d, double L) { return d - L * round(d / L); }

__host__ __device__ __forceinline__ double wrap_coord(double x, double L) { return x - L * floor(x / L); }

__device__ __forceinline__ void shift_decode(int code, int& sx, int& sy, int& sz)
{
    sx = code % 3 - 1;
    sy = (code / 3) % 3 - 1;
    sz = code / 9 - 1;
}

}  // namespace mdf
