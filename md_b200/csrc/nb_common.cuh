// Definitions shared by the pair kernel (nonbonded.cu) and its adjoint
// (adjoint.cu).
#pragma once

#include "mdf_internal.cuh"

namespace mdf {

constexpr int NB_WARPS = 8;
constexpr int NB_THREADS = NB_WARPS * 32;

template <typename R> struct V2;
template <> struct V2<float> { using type = float2; };
template <> struct V2<double> { using type = double2; };

struct NBParams {
    double box[3];
    double rc, rc2, rsw, inv_sw, kc, alpha, rlist2;
    int use_switch;
    int ntp;
    double ucut_pow6, ucut_pow12;   // rc^-6, rc^-12 (force-shift LJ)
};

// 2^x on the special-function unit (PTX ex2.approx.ftz: relative error ~2^-22).
__device__ __forceinline__ float ex2_approx(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// 1/sqrt(x) and 1/x on the special-function unit with denormal inputs flushed
// (PTX rsqrt.approx.ftz / rcp.approx.ftz): the library forms also handle
// denormal arguments, which a pair distance or 1 + p r never is, at the cost
// of extra instructions in the pair loop.
__device__ __forceinline__ float rsqrt_ftz(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float rcp_ftz(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Abramowitz & Stegun 7.1.26 (Hastings): erfc(x) ~ t (a1 + t (a2 + ...)) e^{-x^2},
// t = 1 / (1 + p x), |error| <= 1.5e-7.  Used by the FP32 pair kernel only.
__device__ __forceinline__ float erfc_as(float t, float ex)
{
    const float a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f, a4 = -1.453152027f,
                a5 = 1.061405429f;
    return t * (a1 + t * (a2 + t * (a3 + t * (a4 + t * a5)))) * ex;
}

// The table row at a byte offset (type indexes are kept pre-multiplied by the
// row size, so the address is one add).
template <typename T>
__device__ __forceinline__ const T& at_bytes(const T* __restrict__ base, int bytes)
{
    return *reinterpret_cast<const T*>(reinterpret_cast<const char*>(base) + bytes);
}

struct ShiftTable {
    float v[27][6];   // hi.x hi.y hi.z lo.x lo.y lo.z
};

NBParams make_params(const Ctx& c);
ShiftTable make_shift_table(const Ctx& c);

}  // namespace mdf
