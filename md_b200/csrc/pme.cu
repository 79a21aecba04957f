// Particle-mesh Ewald: charge spread, hand-written 3-D FFT, reciprocal
// convolution with the FP64 energy/virial reduction, and force gather.
//
// PHYSICAL semantics: smooth PME of order 4 (Essmann et al., J. Chem. Phys.
// 103, 8577 (1995)): E = 1/2 sum_m c(m) |S(m)|^2 with
// c(m) = k/(pi V) exp(-pi^2 m^2/alpha^2)/m^2 * B1 B2 B3, B_d = 1/|b_d(m_d)|^2.
// REFERENCE semantics: the reference's own chain, order 5 with its weights and
// grid offsets (src/System/PBC.cpp:183-250, :329-401), its moduli (:455-490),
// its solve with the extra 1/N and without the Coulomb constant (:501-564) and
// its gather (:576-653).  The reference discards those forces; they are
// returned separately for parity checks.
//
// FFT: mixed-radix Stockham autosort in shared memory (radix 4/2/3/5 and a
// generic small-prime butterfly).  Every butterfly's twiddle step and output
// index come from a table built on the host, so the passes do no integer
// division.  One kernel per dimension:
//   z: real -> half complex, two real lines packed per complex transform
//   y: complex, LP consecutive kz columns per block (coalesced along kz)
//   x: complex forward, convolution with the precomputed influence function
//      (+ FP64 energy and virial), complex inverse - one kernel
//   y: inverse
//   z: half complex -> real
// The charge grid is accumulated in int64 fixed point (2^-40), so the spread
// is deterministic regardless of atomic ordering.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "kargs.cuh"
#include "mdf_device.cuh"
#include "mdf_internal.cuh"

namespace mdf {

template <typename R> struct CT;
template <> struct CT<float> { using type = float2; };
template <> struct CT<double> { using type = double2; };

constexpr int FFT_THREADS = 128;


template <typename C>
__device__ __forceinline__ C cmul(C a, C b)
{
    C r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}

template <typename C>
__device__ __forceinline__ C cconj(C a)
{
    a.y = -a.y;
    return a;
}

// In-place DFT of v[0..R-1]; forward uses W = exp(-2 pi i / R).
template <typename C, typename R>
__device__ __forceinline__ void small_dft(C* v, int Rr, bool inverse, const C* tw, int n)
{
    const R s = inverse ? (R)1 : (R)-1;
    if (Rr == 2) {
        C a = v[0], b = v[1];
        v[0].x = a.x + b.x; v[0].y = a.y + b.y;
        v[1].x = a.x - b.x; v[1].y = a.y - b.y;
    } else if (Rr == 4) {
        C a = v[0], b = v[1], c = v[2], d = v[3];
        C t0 = {a.x + c.x, a.y + c.y}, t1 = {a.x - c.x, a.y - c.y};
        C t2 = {b.x + d.x, b.y + d.y}, t3 = {b.x - d.x, b.y - d.y};
        C t3r = {-s * t3.y, s * t3.x};   // t3 * (-i) forward, * (+i) inverse
        v[0].x = t0.x + t2.x; v[0].y = t0.y + t2.y;
        v[2].x = t0.x - t2.x; v[2].y = t0.y - t2.y;
        v[1].x = t1.x + t3r.x; v[1].y = t1.y + t3r.y;
        v[3].x = t1.x - t3r.x; v[3].y = t1.y - t3r.y;
    } else if (Rr == 3) {
        const R c1 = (R)-0.5, s1 = s * (R)0.86602540378443864676;
        C a = v[0], b = v[1], c = v[2];
        C t = {b.x + c.x, b.y + c.y}, u = {b.x - c.x, b.y - c.y};
        v[0].x = a.x + t.x; v[0].y = a.y + t.y;
        C m = {a.x + c1 * t.x, a.y + c1 * t.y};
        C w = {-s1 * u.y, s1 * u.x};
        v[1].x = m.x + w.x; v[1].y = m.y + w.y;
        v[2].x = m.x - w.x; v[2].y = m.y - w.y;
    } else if (Rr == 5) {
        const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;
        const R s1 = s * (R)0.95105651629515357212, s2 = s * (R)0.58778525229247312917;
        C a = v[0];
        C b1 = {v[1].x + v[4].x, v[1].y + v[4].y}, d1 = {v[1].x - v[4].x, v[1].y - v[4].y};
        C b2 = {v[2].x + v[3].x, v[2].y + v[3].y}, d2 = {v[2].x - v[3].x, v[2].y - v[3].y};
        v[0].x = a.x + b1.x + b2.x; v[0].y = a.y + b1.y + b2.y;
        C m1 = {a.x + c1 * b1.x + c2 * b2.x, a.y + c1 * b1.y + c2 * b2.y};
        C m2 = {a.x + c2 * b1.x + c1 * b2.x, a.y + c2 * b1.y + c1 * b2.y};
        C n1 = {s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y};
        C n2 = {s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y};
        v[1].x = m1.x - n1.y; v[1].y = m1.y + n1.x;
        v[4].x = m1.x + n1.y; v[4].y = m1.y - n1.x;
        v[2].x = m2.x - n2.y; v[2].y = m2.y + n2.x;
        v[3].x = m2.x + n2.y; v[3].y = m2.y - n2.x;
    } else {
        // generic prime radix through the line's twiddle table: W_R^q = W_n^{q n/R}
        C out[32];
        const int step = n / Rr;
        for (int t = 0; t < Rr; ++t) {
            C acc = {0, 0};
            for (int r = 0; r < Rr; ++r) {
                C w = tw[((r * t) % Rr) * step];
                if (inverse) w = cconj(w);
                C p = cmul(v[r], w);
                acc.x += p.x;
                acc.y += p.y;
            }
            out[t] = acc;
        }
        for (int t = 0; t < Rr; ++t) v[t] = out[t];
    }
}

// One Stockham stage (radix known at compile time) on this thread's line:
// butterflies j = lt, lt + tpl, ...; tab[j] = (twiddle step k*n/(Ns R), output index).
template <typename C, typename R, int RR>
__device__ __forceinline__ void stage_fixed(const C* in, C* out, int n, int Ns, const C* tw, const int2* tab, int lt,
                                            int tpl, bool inverse)
{
    const int nb = n / RR;
    for (int j = lt; j < nb; j += tpl) {
        const int2 t = tab[j];
        C v[RR];
#pragma unroll
        for (int r = 0; r < RR; ++r) {
            C x = in[j + r * nb];
            if (r && t.x) {
                C w = tw[r * t.x];
                if (inverse) w = cconj(w);
                x = cmul(x, w);
            }
            v[r] = x;
        }
        small_dft<C, R>(v, RR, inverse, tw, n);
#pragma unroll
        for (int r = 0; r < RR; ++r) out[t.y + r * Ns] = v[r];
    }
}

template <typename C, typename R>
__device__ void stage_generic(const C* in, C* out, int n, int Rr, int Ns, const C* tw, const int2* tab, int lt,
                              int tpl, bool inverse)
{
    const int nb = n / Rr;
    for (int j = lt; j < nb; j += tpl) {
        const int2 t = tab[j];
        C v[32];
        for (int r = 0; r < Rr; ++r) {
            C x = in[j + r * nb];
            if (r && t.x) {
                C w = tw[r * t.x];
                if (inverse) w = cconj(w);
                x = cmul(x, w);
            }
            v[r] = x;
        }
        small_dft<C, R>(v, Rr, inverse, tw, n);
        for (int r = 0; r < Rr; ++r) out[t.y + r * Ns] = v[r];
    }
}

// Stockham FFT of the block's lines stored [line][n] in shared memory; this
// thread works on line `line` with lane lt of tpl.  Returns the result buffer.
template <typename C, typename R>
__device__ C* fft_lines(C* a, C* b, const FFTDesc& d, const C* tw, const int2* tab, int line, int lt, int tpl,
                        bool inverse)
{
    const int n = d.n;
    for (int s = 0; s < d.nst; ++s) {
        const int Rr = d.radix[s];
        const C* in = a + line * n;
        C* out = b + line * n;
        const int2* ts = tab + d.toff[s];
        switch (Rr) {
            case 2: stage_fixed<C, R, 2>(in, out, n, d.ns[s], tw, ts, lt, tpl, inverse); break;
            case 3: stage_fixed<C, R, 3>(in, out, n, d.ns[s], tw, ts, lt, tpl, inverse); break;
            case 4: stage_fixed<C, R, 4>(in, out, n, d.ns[s], tw, ts, lt, tpl, inverse); break;
            case 5: stage_fixed<C, R, 5>(in, out, n, d.ns[s], tw, ts, lt, tpl, inverse); break;
            default: stage_generic<C, R>(in, out, n, Rr, d.ns[s], tw, ts, lt, tpl, inverse); break;
        }
        __syncthreads();
        C* t = a;
        a = b;
        b = t;
    }
    return a;
}

// shared memory: twiddles [n] | index table [ntab] | two line buffers [LP][n]
template <typename C>
__device__ __forceinline__ void fft_smem_setup(unsigned char* raw, const FFTDesc& d, const C* __restrict__ g_tw,
                                               const int2* __restrict__ g_tab, int LP, C*& tw, int2*& tab, C*& bufA,
                                               C*& bufB)
{
    tw = reinterpret_cast<C*>(raw);
    bufA = tw + d.n;
    bufB = bufA + LP * d.n;
    tab = reinterpret_cast<int2*>(bufB + LP * d.n);
    for (int i = threadIdx.x; i < d.n; i += blockDim.x) tw[i] = g_tw[i];
    for (int i = threadIdx.x; i < d.ntab; i += blockDim.x) tab[i] = g_tab[i];
}

// ------------------------------------------------------------- z passes
template <typename R>
__device__ __forceinline__ void fft_z_r2c_dev(const FFTZArgs<R>& A, int bx, int by)
{
    const unsigned long long* __restrict__ qgrid = A.qgrid;
    typename CT<R>::type* __restrict__ cgrid = A.cgrid;
    const int nlines = A.nlines;
    const FFTDesc& dz = A.d;
    const typename CT<R>::type* __restrict__ twz = A.tw;
    const int2* __restrict__ tabz = A.tab;
    const int LP = A.LP;
    using C = typename CT<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *tw, *bufA, *bufB;
    int2* tab;
    fft_smem_setup(smem_raw, dz, twz, tabz, LP, tw, tab, bufA, bufB);
    const int K2 = dz.n, Kc = K2 / 2 + 1;
    const int tpl = blockDim.x / LP, line = threadIdx.x / tpl, lt = threadIdx.x - line * tpl;
    const long long g0 = (long long)bx * 2 * LP + 2 * line;   // this thread's pair of real lines
    for (int z = lt; z < K2; z += tpl) {
        C v;
        v.x = g0 < nlines ? (R)((double)(long long)qgrid[g0 * K2 + z] * GRID_ISCALE) : (R)0;
        v.y = g0 + 1 < nlines ? (R)((double)(long long)qgrid[(g0 + 1) * K2 + z] * GRID_ISCALE) : (R)0;
        bufA[line * K2 + z] = v;
    }
    __syncthreads();
    const C* res = fft_lines<C, R>(bufA, bufB, dz, tw, tab, line, lt, tpl, false);
    for (int k = lt; k < Kc; k += tpl) {
        const C Z = res[line * K2 + k], Zc = cconj(res[line * K2 + (k == 0 ? 0 : K2 - k)]);
        const C A = {(R)0.5 * (Z.x + Zc.x), (R)0.5 * (Z.y + Zc.y)};
        const C B = {(R)0.5 * (Z.y - Zc.y), (R)-0.5 * (Z.x - Zc.x)};
        if (g0 < nlines) cgrid[g0 * Kc + k] = A;
        if (g0 + 1 < nlines) cgrid[(g0 + 1) * Kc + k] = B;
    }
}

template <typename R>
__device__ __forceinline__ void fft_z_c2r_dev(const FFTZArgs<R>& A, int bx, int by)
{
    const typename CT<R>::type* __restrict__ cgrid = A.cgrid;
    R* __restrict__ rgrid = A.rgrid;
    const int nlines = A.nlines;
    const FFTDesc& dz = A.d;
    const typename CT<R>::type* __restrict__ twz = A.tw;
    const int2* __restrict__ tabz = A.tab;
    const int LP = A.LP;
    using C = typename CT<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *tw, *bufA, *bufB;
    int2* tab;
    fft_smem_setup(smem_raw, dz, twz, tabz, LP, tw, tab, bufA, bufB);
    const int K2 = dz.n, Kc = K2 / 2 + 1;
    const int tpl = blockDim.x / LP, line = threadIdx.x / tpl, lt = threadIdx.x - line * tpl;
    const long long g0 = (long long)bx * 2 * LP + 2 * line;
    for (int k = lt; k < K2; k += tpl) {
        const int kk = k < Kc ? k : K2 - k;
        C A = {0, 0}, B = {0, 0};
        if (g0 < nlines) A = cgrid[g0 * Kc + kk];
        if (g0 + 1 < nlines) B = cgrid[(g0 + 1) * Kc + kk];
        if (k >= Kc) {
            A = cconj(A);
            B = cconj(B);
        }
        const C Z = {A.x - B.y, A.y + B.x};
        bufA[line * K2 + k] = Z;
    }
    __syncthreads();
    const C* res = fft_lines<C, R>(bufA, bufB, dz, tw, tab, line, lt, tpl, true);
    for (int k = lt; k < K2; k += tpl) {
        const C Z = res[line * K2 + k];
        if (g0 < nlines) rgrid[g0 * K2 + k] = Z.x;
        if (g0 + 1 < nlines) rgrid[(g0 + 1) * K2 + k] = Z.y;
    }
}

// ------------------------------------------------------------- y pass
template <typename R>
__device__ __forceinline__ void fft_y_dev(const FFTYArgs<R>& A, int bx, int by)
{
    typename CT<R>::type* __restrict__ cgrid = A.cgrid;
    const int Kc = A.Kc;
    const FFTDesc& dy = A.d;
    const typename CT<R>::type* __restrict__ twy = A.tw;
    const int2* __restrict__ taby = A.tab;
    const int LP = A.LP, lp_shift = A.lp_shift;
    const bool inverse = A.inverse != 0;
    using C = typename CT<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *tw, *bufA, *bufB;
    int2* tab;
    fft_smem_setup(smem_raw, dy, twy, taby, LP, tw, tab, bufA, bufB);
    const int K1 = dy.n;
    const int x = by, kz0 = bx * LP;
    const long long base = (long long)x * K1 * Kc;
    // loads: consecutive threads take consecutive kz (coalesced)
    for (int e = threadIdx.x; e < LP * K1; e += blockDim.x) {
        const int y = e >> lp_shift, l = e & (LP - 1), kz = kz0 + l;
        C v = {0, 0};
        if (kz < Kc) v = cgrid[base + (long long)y * Kc + kz];
        bufA[l * K1 + y] = v;
    }
    __syncthreads();
    const int tpl = blockDim.x / LP, line = threadIdx.x / tpl, lt = threadIdx.x - line * tpl;
    const C* res = fft_lines<C, R>(bufA, bufB, dy, tw, tab, line, lt, tpl, inverse);
    for (int e = threadIdx.x; e < LP * K1; e += blockDim.x) {
        const int y = e >> lp_shift, l = e & (LP - 1), kz = kz0 + l;
        if (kz < Kc) cgrid[base + (long long)y * Kc + kz] = res[l * K1 + y];
    }
}

// ------------------------------------------- x pass + convolution + inverse

template <typename R, bool ENERGY>
__device__ __forceinline__ void fft_x_conv_dev(const FFTXArgs<R>& A, int bx, int by)
{
    typename CT<R>::type* __restrict__ cgrid = A.cgrid;
    const int K1 = A.K1, Kc = A.Kc;
    const FFTDesc& dx = A.d;
    const typename CT<R>::type* __restrict__ twx = A.tw;
    const int2* __restrict__ tabx = A.tab;
    const int LP = A.LP, lp_shift = A.lp_shift;
    const ConvParams& cp = A.cp;
    const R* __restrict__ infl = A.infl;
    const double* __restrict__ mx = A.mx;
    const double* __restrict__ my = A.my;
    const double* __restrict__ mz = A.mz;
    unsigned long long* __restrict__ acc = A.acc;
    unsigned* st = A.st;
    using C = typename CT<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *tw, *bufA, *bufB;
    int2* tab;
    fft_smem_setup(smem_raw, dx, twx, tabx, LP, tw, tab, bufA, bufB);
    const int K0 = dx.n;
    const int y = by, kz0 = bx * LP;
    const long long stride = (long long)K1 * Kc;
    for (int e = threadIdx.x; e < LP * K0; e += blockDim.x) {
        const int x = e >> lp_shift, l = e & (LP - 1), kz = kz0 + l;
        C v = {0, 0};
        if (kz < Kc) v = cgrid[x * stride + (long long)y * Kc + kz];
        bufA[l * K0 + x] = v;
    }
    __syncthreads();
    const int tpl = blockDim.x / LP, line = threadIdx.x / tpl, lt = threadIdx.x - line * tpl;
    C* res = fft_lines<C, R>(bufA, bufB, dx, tw, tab, line, lt, tpl, false);
    C* other = (res == bufA) ? bufB : bufA;
    double e_sum = 0, w6[6] = {0, 0, 0, 0, 0, 0};
    const int kz = kz0 + line;
    if (kz < Kc) {
        // influence function laid out [ky][kz][kx]: this line is contiguous
        const R* fl = infl + ((long long)y * Kc + kz) * K0;
        const double wgt = (kz == 0 || ((cp.K[2] & 1) == 0 && kz == cp.K[2] / 2)) ? 1.0 : 2.0;
        for (int kx = lt; kx < K0; kx += tpl) {
            C S = res[line * K0 + kx];
            const R c = fl[kx];
            if (ENERGY && !cp.reference && c != (R)0) {
                const double s2 = (double)S.x * S.x + (double)S.y * S.y;
                const double em = 0.5 * (double)c * s2 * wgt;
                e_sum += em;
                const double m[3] = {mx[kx], my[y], mz[kz]};
                const double m2 = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
                const double vf = 2.0 * (1.0 + cp.pa2 * m2) / m2;
                int q = 0;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = a; b < 3; ++b) w6[q++] += em * ((a == b ? 1.0 : 0.0) - vf * m[a] * m[b]);
            }
            S.x *= c;
            S.y *= c;
            res[line * K0 + kx] = S;
        }
    }
    __syncthreads();
    const C* out = fft_lines<C, R>(res, other, dx, tw, tab, line, lt, tpl, true);
    for (int e = threadIdx.x; e < LP * K0; e += blockDim.x) {
        const int x = e >> lp_shift, l = e & (LP - 1), kzz = kz0 + l;
        if (kzz < Kc) cgrid[x * stride + (long long)y * Kc + kzz] = out[l * K0 + x];
    }
    if (ENERGY && !cp.reference) {
        const double v[7] = {e_sum, w6[0], w6[1], w6[2], w6[3], w6[4], w6[5]};
        const int idx[7] = {MDF_E_EE_RECIP, ACC_VIR + 0, ACC_VIR + 1, ACC_VIR + 2, ACC_VIR + 3, ACC_VIR + 4,
                            ACC_VIR + 5};
        block_acc_fixed<7>(v, acc, idx, ENERGY_SCALE, st);
    }
}

// One-system kernels (arguments by value) and their many-system forms: a
// one-dimensional grid of every system's blocks, block b running block
// bmap[b].y of system bmap[b].x (so systems of different sizes leave no idle
// blocks).
#define MDF_FFT_KERNELS(NAME, DEV, ARGS, ...)                                                                   \
    template <__VA_ARGS__>                                                                                    \
    __global__ void __launch_bounds__(FFT_THREADS) NAME(ARGS A)                                               \
    {                                                                                                         \
        DEV(A, blockIdx.x, blockIdx.y);                                                                       \
    }                                                                                                         \
    template <__VA_ARGS__>                                                                                    \
    __global__ void __launch_bounds__(FFT_THREADS) NAME##_multi(const ARGS* __restrict__ As,                  \
                                                                const int2* __restrict__ bmap)                \
    {                                                                                                         \
        const int2 m = bmap[blockIdx.x];                                                                      \
        const ARGS& A = As[m.x];                                                                              \
        DEV(A, m.y % A.gx, m.y / A.gx);                                                                       \
    }
MDF_FFT_KERNELS(k_fft_z_r2c, fft_z_r2c_dev<R>, FFTZArgs<R>, typename R)
MDF_FFT_KERNELS(k_fft_z_c2r, fft_z_c2r_dev<R>, FFTZArgs<R>, typename R)
MDF_FFT_KERNELS(k_fft_y, fft_y_dev<R>, FFTYArgs<R>, typename R)
#undef MDF_FFT_KERNELS

template <typename R, bool ENERGY>
__global__ void __launch_bounds__(FFT_THREADS) k_fft_x_conv(FFTXArgs<R> A)
{
    fft_x_conv_dev<R, ENERGY>(A, blockIdx.x, blockIdx.y);
}

// 64 registers (eight blocks per SM): the many-system grids are small and the
// pass is latency bound, so resident warps matter more than registers here
template <typename R, bool ENERGY>
__global__ void __launch_bounds__(FFT_THREADS, 8) k_fft_x_conv_multi(const FFTXArgs<R>* __restrict__ As,
                                                                     const int2* __restrict__ bmap)
{
    const int2 m = bmap[blockIdx.x];
    const FFTXArgs<R>& A = As[m.x];
    fft_x_conv_dev<R, ENERGY>(A, m.y % A.gx, m.y / A.gx);
}

// ------------------------------------------------------ spread / gather
// Cardinal B-spline of order 4: th[j] = M4(w + 3 - j), placed at base-1+j.
template <typename R>
__device__ __forceinline__ void bspline4(R w, R th[4], R dth[4])
{
    const R w2 = w * w, w3 = w2 * w, om = (R)1 - w;
    th[0] = om * om * om * (R)(1.0 / 6.0);
    th[1] = ((R)3 * w3 - (R)6 * w2 + (R)4) * (R)(1.0 / 6.0);
    th[2] = ((R)-3 * w3 + (R)3 * w2 + (R)3 * w + (R)1) * (R)(1.0 / 6.0);
    th[3] = w3 * (R)(1.0 / 6.0);
    if (dth) {
        dth[0] = (R)-0.5 * om * om;
        dth[1] = (R)1.5 * w2 - (R)2 * w;
        dth[2] = (R)-1.5 * w2 + w + (R)0.5;
        dth[3] = (R)0.5 * w2;
    }
}


template <typename R>
__global__ void k_spread4(int s0, int s1, const int* __restrict__ slot_atom, const double* __restrict__ xyz,
                          const double* __restrict__ q, GridGeom g, unsigned long long* __restrict__ qgrid,
                          unsigned* st)
{
    int s = s0 + blockIdx.x * blockDim.x + threadIdx.x;   // slots [s0, s1)
    if (s >= s1) return;
    int a = slot_atom[s];
    if (a < 0) return;
    double qa = q[a];
    if (qa == 0.0) return;
    int base[3];
    R th[3][4];
    for (int d = 0; d < 3; ++d) {
        double u = wrap_coord(xyz[3 * a + d], g.L[d]) * g.scale[d];
        if (!(u >= 0.0 && u <= (double)g.K[d])) {   // non-finite position
            status_set(st, ST_NONFINITE);
            return;
        }
        if (u >= g.K[d]) u -= g.K[d];
        int b = min((int)floor(u), g.K[d] - 1);
        base[d] = b;
        bspline4<R>((R)(u - b), th[d], nullptr);
    }
    const R qr = (R)qa;
    for (int i = 0; i < 4; ++i) {
        int kx = base[0] - 1 + i;
        kx += (kx < 0) ? g.K[0] : 0;
        kx -= (kx >= g.K[0]) ? g.K[0] : 0;
        for (int j = 0; j < 4; ++j) {
            int ky = base[1] - 1 + j;
            ky += (ky < 0) ? g.K[1] : 0;
            ky -= (ky >= g.K[1]) ? g.K[1] : 0;
            const R wxy = qr * th[0][i] * th[1][j];
            long long row = ((long long)kx * g.K[1] + ky) * g.K[2];
            for (int k = 0; k < 4; ++k) {
                int kz = base[2] - 1 + k;
                kz += (kz < 0) ? g.K[2] : 0;
                kz -= (kz >= g.K[2]) ? g.K[2] : 0;
                R v = wxy * th[2][k];
                atomicAdd(qgrid + row + kz, (unsigned long long)__double2ll_rn((double)v * GRID_SCALE));
            }
        }
    }
}

// One weight of the order-4 cardinal B-spline: th[j] of bspline4 for a single j.
template <typename R>
__device__ __forceinline__ R bspline4_one(R w, int j)
{
    const R w2 = w * w, w3 = w2 * w, om = (R)1 - w;
    R v;
    if (j == 0) v = om * om * om;
    else if (j == 1) v = (R)3 * w3 - (R)6 * w2 + (R)4;
    else if (j == 2) v = (R)-3 * w3 + (R)3 * w2 + (R)3 * w + (R)1;
    else v = w3;
    return v * (R)(1.0 / 6.0);
}

// Charge spread with 16 lanes per atom, four lanes per z run: lane (r, z)
// of an atom's group adds, in four steps t, the point (x = t, y = r, z) of the
// atom's 4 x 4 x 4 stencil.  At every step the 16 lanes of an atom hit four
// (x, y) rows with four consecutive z words each, so the L2 merges the
// reductions of a row (one or two 32-byte sectors per four words) instead of
// taking four separate requests from one lane.  Lane 0 of the group computes
// the atom's grid position and fractional offsets once and shares them.  The
// grid words are identical to the one-thread-per-atom form's (the same
// rounded fixed-point values, summed in any order).  Launched with a
// multiple of 16 threads per block.
template <typename R>
__device__ __forceinline__ void spread4_rows_dev(const SpreadArgs& A, int bx, int by)
{
    const int s0 = A.s0, s1 = A.s1;
    const int* __restrict__ slot_atom = A.slot_atom;
    const double* __restrict__ xyz = A.xyz;
    const double* __restrict__ q = A.q;
    const GridGeom& g = A.g;
    unsigned long long* __restrict__ qgrid = A.qgrid;
    unsigned* st = A.st;
    const long long t0 = (long long)bx * blockDim.x + threadIdx.x;
    const int s = s0 + (int)(t0 >> 4);
    const int l = (int)(t0 & 15), r = l >> 2, zz = l & 3;
    // the whole group of 16 lanes leaves together (same atom)
    if (s >= s1) return;
    const int a = slot_atom[s];
    if (a < 0) return;
    const double qa = q[a];
    if (qa == 0.0) return;
    const unsigned grp = 0xffffu << (threadIdx.x & 16);
    int base[3] = {0, 0, 0};
    double u[3] = {0, 0, 0};
    int bad = 0;
    if (l == 0) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double v = wrap_coord(xyz[3 * a + d], g.L[d]) * g.scale[d];
            if (!(v >= 0.0 && v <= (double)g.K[d])) bad = 1;   // non-finite position
            if (v >= g.K[d]) v -= g.K[d];
            const int b = bad ? 0 : min((int)floor(v), g.K[d] - 1);
            base[d] = b;
            u[d] = v - b;
        }
        if (!bad && A.win_n > 0) {
            // halo exchange: the stencil must start inside the rank's window
            int w = (base[0] - A.win_lo) % g.K[0];
            w += (w < 0) ? g.K[0] : 0;
            if (w >= A.win_n) bad = 2;
        }
    }
    bad = __shfl_sync(grp, bad, 0, 16);
    if (bad) {
        if (l == 0) status_set(st, bad == 1 ? ST_NONFINITE : ST_STALE);
        return;
    }
    R w[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        base[d] = __shfl_sync(grp, base[d], 0, 16);
        w[d] = (R)__shfl_sync(grp, u[d], 0, 16);
    }
    R thx[4];
    bspline4<R>(w[0], thx, nullptr);
    const R thy = bspline4_one<R>(w[1], r), thz = bspline4_one<R>(w[2], zz);
    int ky = base[1] - 1 + r;
    ky += (ky < 0) ? g.K[1] : 0;
    ky -= (ky >= g.K[1]) ? g.K[1] : 0;
    int kz = base[2] - 1 + zz;
    kz += (kz < 0) ? g.K[2] : 0;
    kz -= (kz >= g.K[2]) ? g.K[2] : 0;
    const R qr = (R)qa;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        int kx = base[0] - 1 + t;
        kx += (kx < 0) ? g.K[0] : 0;
        kx -= (kx >= g.K[0]) ? g.K[0] : 0;
        const R v = qr * thx[t] * thy * thz;
        long long fx;
        if (sizeof(R) == 4) fx = __float2ll_rn((float)v * 1099511627776.0f);   // exact 2^40 scaling
        else fx = __double2ll_rn((double)v * GRID_SCALE);
        atomicAdd(qgrid + ((long long)kx * g.K[1] + ky) * g.K[2] + kz, (unsigned long long)fx);
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_spread4_rows(SpreadArgs A)
{
    spread4_rows_dev<R>(A, blockIdx.x, 0);
}

template <typename R>
__global__ void __launch_bounds__(256) k_spread4_rows_multi(const SpreadArgs* __restrict__ As, const int2* __restrict__ bmap)
{
    const int2 m = bmap[blockIdx.x];
    spread4_rows_dev<R>(As[m.x], m.y, 0);
}

// Clear many systems' charge grids in one launch.
__global__ void k_zero_multi(const ZeroArgs* __restrict__ As, const int2* __restrict__ bmap)
{
    const int2 m = bmap[blockIdx.x];
    const ZeroArgs& A = As[m.x];
    for (long long i = (long long)m.y * blockDim.x + threadIdx.x; i < A.n; i += (long long)A.gx * blockDim.x)
        A.p[i] = 0ull;
}

template <typename R>
__device__ __forceinline__ void gather4_dev(const GatherArgs<R>& A, int bx, int by)
{
    const int s0 = A.s0, s1 = A.s1, nslots = A.nslots;
    const int* __restrict__ slot_atom = A.slot_atom;
    const double* __restrict__ xyz = A.xyz;
    const double* __restrict__ q = A.q;
    const GridGeom& g = A.g;
    const R* __restrict__ phi = A.phi;
    unsigned long long* __restrict__ fslot = A.fslot;
    unsigned* st = A.st;
    int s = s0 + bx * blockDim.x + threadIdx.x;   // slots [s0, s1) of nslots
    if (s >= s1) return;
    int a = slot_atom[s];
    if (a < 0) return;
    double qa = q[a];
    if (qa == 0.0) return;
    int base[3];
    R th[3][4], dth[3][4];
    for (int d = 0; d < 3; ++d) {
        double u = wrap_coord(xyz[3 * a + d], g.L[d]) * g.scale[d];
        if (!(u >= 0.0 && u <= (double)g.K[d])) {   // non-finite position
            status_set(st, ST_NONFINITE);
            return;
        }
        if (u >= g.K[d]) u -= g.K[d];
        int b = min((int)floor(u), g.K[d] - 1);
        base[d] = b;
        bspline4<R>((R)(u - b), th[d], dth[d]);
    }
    R gx = 0, gy = 0, gz = 0;
    for (int i = 0; i < 4; ++i) {
        int kx = base[0] - 1 + i;
        kx += (kx < 0) ? g.K[0] : 0;
        kx -= (kx >= g.K[0]) ? g.K[0] : 0;
        for (int j = 0; j < 4; ++j) {
            int ky = base[1] - 1 + j;
            ky += (ky < 0) ? g.K[1] : 0;
            ky -= (ky >= g.K[1]) ? g.K[1] : 0;
            long long row = ((long long)kx * g.K[1] + ky) * g.K[2];
            R sz = 0, dz = 0;
            for (int k = 0; k < 4; ++k) {
                int kz = base[2] - 1 + k;
                kz += (kz < 0) ? g.K[2] : 0;
                kz -= (kz >= g.K[2]) ? g.K[2] : 0;
                R p = phi[row + kz];
                sz += th[2][k] * p;
                dz += dth[2][k] * p;
            }
            gx += dth[0][i] * th[1][j] * sz;
            gy += th[0][i] * dth[1][j] * sz;
            gz += th[0][i] * th[1][j] * dz;
        }
    }
    const R qr = (R)qa;
    fx_add(fslot + s, -qr * gx * (R)g.scale[0], FORCE_SCALE, st);
    fx_add(fslot + nslots + s, -qr * gy * (R)g.scale[1], FORCE_SCALE, st);
    fx_add(fslot + 2 * nslots + s, -qr * gz * (R)g.scale[2], FORCE_SCALE, st);
}

template <typename R>
__global__ void k_gather4(GatherArgs<R> A)
{
    gather4_dev<R>(A, blockIdx.x, 0);
}

template <typename R>
__global__ void k_gather4_multi(const GatherArgs<R>* __restrict__ As, const int2* __restrict__ bmap)
{
    const int2 m = bmap[blockIdx.x];
    gather4_dev<R>(As[m.x], m.y, 0);
}

// The reference's order-5 weights (src/System/PBC.cpp:329-356 for the spread,
// :359-401 for the gather; the two differ in operation order).
__host__ __device__ __forceinline__ void ref_w5_spread(double u, double th[5])
{
    double c0 = 1.0 - u, c1 = u;
    double w0 = (1.0 / 2.0) * ((1.0 - u) * c0);
    double w1 = (1.0 / 2.0) * ((1.0 + u) * c0 + (2.0 - u) * c1);
    double w2 = (1.0 / 2.0) * ((1.0 + u) * c1);
    double x0 = (1.0 / 3.0) * ((1.0 - u) * w0);
    double x1 = (1.0 / 3.0) * ((2.0 + u) * w0 + (2.0 - u) * w1);
    double x2 = (1.0 / 3.0) * ((1.0 + u) * w1 + (3.0 - u) * w2);
    double x3 = (1.0 / 3.0) * ((2.0 + u) * w2);
    th[0] = (1.0 / 4.0) * ((1.0 - u) * x0);
    th[1] = (1.0 / 4.0) * ((3.0 + u) * x0 + (2.0 - u) * x1);
    th[2] = (1.0 / 4.0) * ((2.0 + u) * x1 + (3.0 - u) * x2);
    th[3] = (1.0 / 4.0) * ((1.0 + u) * x2 + (4.0 - u) * x3);
    th[4] = (1.0 / 4.0) * ((3.0 + u) * x3);
}

__device__ __forceinline__ void ref_w5_gather(double u, double th[5], double dth[5])
{
    double w20 = 1.0 - u, w21 = u;
    double w30 = 0.5 * (1.0 - u) * w20;
    double w31 = 0.5 * ((1.0 + u) * w20 + (2.0 - u) * w21);
    double w32 = 0.5 * (1.0 + u) * w21;
    const double d4 = 1.0 / 3.0;
    double w40 = d4 * (1.0 - u) * w30;
    double w41 = d4 * ((2.0 + u) * w30 + (2.0 - u) * w31);
    double w42 = d4 * ((1.0 + u) * w31 + (3.0 - u) * w32);
    double w43 = d4 * (2.0 + u) * w32;
    th[0] = 0.25 * (1.0 - u) * w40;
    th[1] = 0.25 * ((3.0 + u) * w40 + (2.0 - u) * w41);
    th[2] = 0.25 * ((2.0 + u) * w41 + (3.0 - u) * w42);
    th[3] = 0.25 * ((1.0 + u) * w42 + (4.0 - u) * w43);
    th[4] = 0.25 * (3.0 + u) * w43;
    dth[0] = -w40; dth[1] = w40 - w41; dth[2] = w41 - w42; dth[3] = w42 - w43; dth[4] = w43;
}

__global__ void k_spread_ref5(int N, const double* __restrict__ xyz, const double* __restrict__ q, GridGeom g,
                              unsigned long long* __restrict__ qgrid)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= N) return;
    double qa = q[a];
    if (qa == 0.0) return;
    int idx[3];
    double th[3][5];
    for (int d = 0; d < 3; ++d) {
        double u = wrap_coord(xyz[3 * a + d], g.L[d]) * g.scale[d];
        if (!(u >= 0.0 && u <= (double)g.K[d])) return;   // non-finite position
        idx[d] = (int)floor(u);
        ref_w5_spread(u - idx[d], th[d]);
    }
    for (int i = 0; i < 5; ++i) {
        int kx = ((idx[0] - 2 + i) % g.K[0] + g.K[0]) % g.K[0];
        for (int j = 0; j < 5; ++j) {
            int ky = ((idx[1] - 2 + j) % g.K[1] + g.K[1]) % g.K[1];
            double wxy = th[0][i] * th[1][j];
            for (int k = 0; k < 5; ++k) {
                int kz = ((idx[2] - 2 + k) % g.K[2] + g.K[2]) % g.K[2];
                double v = qa * wxy * th[2][k];
                atomicAdd(qgrid + ((long long)kx * g.K[1] + ky) * g.K[2] + kz,
                          (unsigned long long)__double2ll_rn(v * GRID_SCALE));
            }
        }
    }
}

__global__ void k_gather_ref5(int N, const double* __restrict__ xyz, const double* __restrict__ q, GridGeom g,
                              const double* __restrict__ phi, double* __restrict__ fout)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= N) return;
    double qa = q[a];
    double fx = 0, fy = 0, fz = 0;
    if (qa != 0.0) {
        int idx[3];
        double th[3][5], dth[3][5];
        for (int d = 0; d < 3; ++d) {
            double u = wrap_coord(xyz[3 * a + d], g.L[d]) * g.scale[d];
            if (!(u >= 0.0 && u <= (double)g.K[d])) u = 0.0;   // non-finite position
            idx[d] = (int)floor(u);
            ref_w5_gather(u - idx[d], th[d], dth[d]);
        }
        for (int i = 0; i < 5; ++i) {
            int kx = (idx[0] - 2 + i) % g.K[0];
            if (kx < 0) kx += g.K[0];
            for (int j = 0; j < 5; ++j) {
                int ky = (idx[1] - 2 + j) % g.K[1];
                if (ky < 0) ky += g.K[1];
                for (int k = 0; k < 5; ++k) {
                    int kz = (idx[2] - 2 + k) % g.K[2];
                    if (kz < 0) kz += g.K[2];
                    double pot = phi[((long long)kx * g.K[1] + ky) * g.K[2] + kz];
                    fx -= qa * pot * dth[0][i] * th[1][j] * th[2][k] * g.scale[0];
                    fy -= qa * pot * th[0][i] * dth[1][j] * th[2][k] * g.scale[1];
                    fz -= qa * pot * th[0][i] * th[1][j] * dth[2][k] * g.scale[2];
                }
            }
        }
    }
    fout[3 * a] = fx;
    fout[3 * a + 1] = fy;
    fout[3 * a + 2] = fz;
}

// ------------------------------------------------------------------ host
static FFTPlan1D make_plan(int n, std::vector<int2>& tab)
{
    FFTPlan1D p;
    p.n = n;
    p.nstages = 0;
    int m = n;
    auto push = [&](int f) {
        if (p.nstages >= 12) throw ApiError(MDF_ERR_UNSUPPORTED, "PME grid size has too many factors");
        p.radix[p.nstages++] = f;
        m /= f;
    };
    while (m % 4 == 0) push(4);
    while (m % 2 == 0) push(2);
    for (int f = 3; f <= 31 && m > 1; f += 2)
        while (m % f == 0) push(f);
    if (m != 1) throw ApiError(MDF_ERR_UNSUPPORTED, "PME grid size has a prime factor above 31");
    // per-butterfly table: Stockham stage s with radix R, Ns = product of the
    // earlier radices, butterfly j: twiddle step (j mod Ns) * n/(Ns R) and
    // output index (j div Ns) Ns R + (j mod Ns)
    tab.clear();
    int Ns = 1;
    for (int s = 0; s < p.nstages; ++s) {
        const int R = p.radix[s], nb = n / R, step = n / (Ns * R);
        p.ns[s] = Ns;
        p.toff[s] = (int)tab.size();
        for (int j = 0; j < nb; ++j) {
            const int k = j % Ns;
            tab.push_back(make_int2(k * step, (j / Ns) * Ns * R + k));
        }
        Ns *= R;
    }
    p.ntab = (int)tab.size();
    return p;
}

static FFTDesc to_desc(const FFTPlan1D& p)
{
    FFTDesc d;
    d.n = p.n;
    d.nst = p.nstages;
    for (int i = 0; i < 12; ++i) {
        d.radix[i] = i < p.nstages ? p.radix[i] : 1;
        d.ns[i] = i < p.nstages ? p.ns[i] : 1;
        d.toff[i] = i < p.nstages ? p.toff[i] : 0;
    }
    d.ntab = p.ntab;
    return d;
}

static void make_twiddles(int n, std::vector<double2>& tw)
{
    tw.resize(n);
    for (int q = 0; q < n; ++q) {
        double a = 2.0 * M_PI * (double)q / (double)n;
        tw[q] = make_double2(cos(a), -sin(a));
    }
}

// Cardinal B-spline M_n (Essmann et al. eq. 4.1 recursion).
static double cardinal_bspline(int n, double x)
{
    if (x <= 0.0 || x >= n) return 0.0;
    if (n == 2) return 1.0 - std::fabs(x - 1.0);
    return (x * cardinal_bspline(n - 1, x) + (n - x) * cardinal_bspline(n - 1, x - 1.0)) / (n - 1);
}

// Lines per block (a power of two dividing FFT_THREADS) within 46 KB of
// shared memory: mdf_params.fft_lines (1, 2, 4, 8, 16 or 32), or for 0 the
// most lines (at least 4) that leave every line as many threads as its
// radix-4 stages have butterflies (n/4): 4 at n = 100 or 216, 16 at n = 32.
static int lines_per_block(const FFTPlan1D& p, size_t csize, int cap = 0)
{
    int top = 4;
    if (cap == 1 || cap == 2 || cap == 4 || cap == 8 || cap == 16 || cap == 32) {
        top = cap;
    } else {
        const int need = (p.n + 3) / 4;
        while (top < 32 && FFT_THREADS / (2 * top) >= need) top *= 2;
    }
    for (int lp = top; lp >= 1; lp >>= 1) {
        size_t bytes = csize * ((size_t)p.n + 2 * (size_t)lp * p.n) + sizeof(int2) * (size_t)p.ntab;
        if (bytes <= 46 * 1024) return lp;
    }
    return 1;
}

static size_t fft_smem(const FFTPlan1D& p, size_t csize, int lp)
{
    return csize * ((size_t)p.n + 2 * (size_t)lp * p.n) + sizeof(int2) * (size_t)p.ntab;
}

static int ilog2(int v)
{
    int s = 0;
    while ((1 << s) < v) ++s;
    return s;
}

void setup_pme(Ctx& c)
{
    bool ref = c.p.semantics == MDF_SEM_REFERENCE;
    for (int d = 0; d < 3; ++d) {
        int K = c.p.grid[d];
        if (K <= 0) {
            // the reference's mesh formula (src/System/PBC.cpp:93-99)
            K = (int)((2 * c.alpha * c.box[d]) / (3 * std::pow(c.p.ewald_tol > 0 ? c.p.ewald_tol : 1e-6, 0.2)));
        }
        if (K < 5) throw ApiError(MDF_ERR_INVALID, "PME grid dimension below 5");
        c.K[d] = K;
        std::vector<int2> tab;
        c.plan[d] = make_plan(K, tab);
        c.fft_tab[d].upload(tab.data(), tab.size(), c.stream);
        std::vector<double> mv(K);
        for (int k = 0; k < K; ++k) mv[k] = ((k <= K / 2) ? k : k - K) / c.box[d];
        c.mvec[d].upload(mv.data(), K, c.stream);
    }
    c.order = ref ? 5 : (c.p.pme_order > 0 ? c.p.pme_order : 4);
    if (!ref && c.order != 4) throw ApiError(MDF_ERR_UNSUPPORTED, "PHYSICAL PME supports order 4");
    const int K0 = c.K[0], K1 = c.K[1], K2 = c.K[2], Kc = K2 / 2 + 1;
    long long ntot = (long long)K0 * K1 * K2;
    long long nc = (long long)K0 * K1 * Kc;
    c.qgrid.alloc(ntot);
    bool mixed = c.p.precision == MDF_PREC_MIXED && !ref;
    if (mixed) {
        c.cgrid_f.alloc(nc);
        c.rgrid_f.alloc(ntot);
    } else {
        c.cgrid_d.alloc(nc);
        c.rgrid_d.alloc(ntot);
    }
    // per-dimension factors: PHYSICAL 1/|b(m)|^2, REFERENCE the reference's moduli
    std::vector<double> bfac[3];
    for (int d = 0; d < 3; ++d) {
        int K = c.K[d];
        std::vector<double>& b = bfac[d];
        b.assign(K, 0.0);
        if (!ref) {
            // 1/|b(m)|^2 = |sum_{k=0}^{n-2} M_n(k+1) e^{2 pi i m k/K}|^2, zeros bridged
            for (int m = 0; m < K; ++m) {
                double sr = 0, si = 0;
                for (int k = 0; k <= c.order - 2; ++k) {
                    double v = cardinal_bspline(c.order, k + 1.0), a = 2.0 * M_PI * m * k / K;
                    sr += v * cos(a);
                    si += v * sin(a);
                }
                b[m] = sr * sr + si * si;
            }
            for (int m = 0; m < K; ++m)
                if (b[m] < 1e-7) b[m] = 0.5 * (b[(m - 1 + K) % K] + b[(m + 1) % K]);
            for (int m = 0; m < K; ++m) b[m] = 1.0 / b[m];
        } else {
            // |r2c of theta5(0) placed at 0,1,2,-1,-2|^2 (src/System/PBC.cpp:455-490)
            double th[5];
            ref_w5_spread(0.0, th);
            std::vector<double> rd(K, 0.0);
            rd[0] = th[2]; rd[1] = th[3]; rd[2] = th[4]; rd[K - 1] = th[1]; rd[K - 2] = th[0];
            for (int i = 0; i < K / 2 + 1; ++i) {
                double sr = 0, si = 0;
                for (int j = 0; j < K; ++j) {
                    double a = 2.0 * M_PI * (double)((long long)i * j % K) / K;
                    sr += rd[j] * cos(a);
                    si -= rd[j] * sin(a);
                }
                double m2 = sr * sr + si * si;
                b[i] = m2;
                if (i > 0 && i < (K + 1) / 2) b[K - i] = m2;
            }
        }
        std::vector<double2> tw;
        make_twiddles(K, tw);
        if (mixed) {
            std::vector<float2> twf(K);
            for (int i = 0; i < K; ++i) twf[i] = make_float2((float)tw[i].x, (float)tw[i].y);
            c.tw_f[d].upload(twf.data(), K, c.stream);
        } else {
            c.tw_d[d].upload(tw.data(), K, c.stream);
        }
    }
    // influence function, laid out [ky][kz][kx] (the x pass reads lines along kx)
    std::vector<double> infl((size_t)K1 * Kc * K0);
    const double V = c.box[0] * c.box[1] * c.box[2];
    for (int ky = 0; ky < K1; ++ky) {
        const int my_i = (ky <= K1 / 2) ? ky : ky - K1;
        for (int kz = 0; kz < Kc; ++kz)
            for (int kx = 0; kx < K0; ++kx) {
                const int mx_i = (kx <= K0 / 2) ? kx : kx - K0;
                double v;
                if (!ref) {
                    const double mx = mx_i / c.box[0], my = my_i / c.box[1], mz = kz / c.box[2];
                    const double m2 = mx * mx + my * my + mz * mz;
                    if (kx == 0 && ky == 0 && kz == 0) v = 0.0;
                    else
                        v = c.p.coulomb_const / (M_PI * V) * std::exp(-M_PI * M_PI * m2 / (c.alpha * c.alpha)) / m2 *
                            bfac[0][kx] * bfac[1][ky] * bfac[2][kz];
                } else {
                    // src/System/PBC.cpp:511-563: 4 pi / V exp(-k^2/(4 alpha^2)) / k^2 / moduli / N
                    const double kxv = 2.0 * M_PI * mx_i / c.box[0], kyv = 2.0 * M_PI * my_i / c.box[1],
                                 kzv = 2.0 * M_PI * kz / c.box[2];
                    const double ksq = kxv * kxv + kyv * kyv + kzv * kzv;
                    if (ksq < 1e-10) v = 0.0;
                    else {
                        const double influence = 4.0 * M_PI / V * std::exp(ksq * (-1.0 / (4.0 * c.alpha * c.alpha))) / ksq;
                        const double b_corr = 1.0 / (bfac[0][kx] * bfac[1][ky] * bfac[2][kz]);
                        v = influence * b_corr * (1.0 / (double)ntot);
                    }
                }
                infl[((size_t)ky * Kc + kz) * K0 + kx] = v;
            }
    }
    if (mixed) {
        std::vector<float> f(infl.begin(), infl.end());
        c.infl_f.upload(f.data(), f.size(), c.stream);
    } else {
        c.infl_d.upload(infl.data(), infl.size(), c.stream);
    }
    MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
}

// Device buffers of one precision.
template <typename R>
struct PmeBufs {
    using C = typename CT<R>::type;
    C* cg;
    R* rg;
    const C *twx, *twy, *twz;
    const R* infl;
    GridGeom g;
    explicit PmeBufs(Ctx& c)
    {
        if (sizeof(R) == 4) {
            cg = reinterpret_cast<C*>(c.cgrid_f.p); rg = reinterpret_cast<R*>(c.rgrid_f.p);
            twx = reinterpret_cast<const C*>(c.tw_f[0].p); twy = reinterpret_cast<const C*>(c.tw_f[1].p);
            twz = reinterpret_cast<const C*>(c.tw_f[2].p);
            infl = reinterpret_cast<const R*>(c.infl_f.p);
        } else {
            cg = reinterpret_cast<C*>(c.cgrid_d.p); rg = reinterpret_cast<R*>(c.rgrid_d.p);
            twx = reinterpret_cast<const C*>(c.tw_d[0].p); twy = reinterpret_cast<const C*>(c.tw_d[1].p);
            twz = reinterpret_cast<const C*>(c.tw_d[2].p);
            infl = reinterpret_cast<const R*>(c.infl_d.p);
        }
        for (int d = 0; d < 3; ++d) {
            g.K[d] = c.K[d];
            g.L[d] = c.box[d];
            g.scale[d] = (double)c.K[d] / c.box[d];
        }
    }
};

// The five FFT launches of one chain (fixed-point charge grid c.qgrid -> real
// potential grid): z, y, x + influence function (+ energy and virial), y^-1,
// z^-1, with their dynamic shared memory.
template <typename R>
FFTChain<R> make_fft_chain(const Ctx& c, bool energy)
{
    using C = typename CT<R>::type;
    const PmeBufs<R> B(const_cast<Ctx&>(c));
    FFTChain<R> F;
    const bool ref = c.p.semantics == MDF_SEM_REFERENCE;
    const int K0 = c.K[0], K1 = c.K[1], Kc = c.K[2] / 2 + 1;
    // z forward (real -> half complex) and z inverse share a geometry
    const int LPz = lines_per_block(c.plan[2], sizeof(C), c.p.fft_lines);
    F.smz = fft_smem(c.plan[2], sizeof(C), LPz);
    const int nlines = K0 * K1;
    F.zf.gx = (nlines + 2 * LPz - 1) / (2 * LPz);
    F.zf.gy = 1;
    F.zf.qgrid = c.qgrid.p;
    F.zf.cgrid = B.cg;
    F.zf.rgrid = B.rg;
    F.zf.nlines = nlines;
    F.zf.d = to_desc(c.plan[2]);
    F.zf.tw = B.twz;
    F.zf.tab = c.fft_tab[2].p;
    F.zf.LP = LPz;
    F.zi = F.zf;
    // y forward / inverse
    const int LPy = lines_per_block(c.plan[1], sizeof(C), c.p.fft_lines);
    F.smy = fft_smem(c.plan[1], sizeof(C), LPy);
    F.yf.gx = (Kc + LPy - 1) / LPy;
    F.yf.gy = K0;
    F.yf.cgrid = B.cg;
    F.yf.Kc = Kc;
    F.yf.d = to_desc(c.plan[1]);
    F.yf.tw = B.twy;
    F.yf.tab = c.fft_tab[1].p;
    F.yf.LP = LPy;
    F.yf.lp_shift = ilog2(LPy);
    F.yf.inverse = 0;
    F.yi = F.yf;
    F.yi.inverse = 1;
    // x forward + convolution + x inverse
    const int LP = lines_per_block(c.plan[0], sizeof(C), c.p.fft_lines);
    F.smx = fft_smem(c.plan[0], sizeof(C), LP);
    F.x.gx = (Kc + LP - 1) / LP;
    F.x.gy = K1;
    F.x.cgrid = B.cg;
    F.x.K1 = K1;
    F.x.Kc = Kc;
    F.x.d = to_desc(c.plan[0]);
    F.x.tw = B.twx;
    F.x.tab = c.fft_tab[0].p;
    F.x.LP = LP;
    F.x.lp_shift = ilog2(LP);
    for (int d = 0; d < 3; ++d) F.x.cp.K[d] = c.K[d];
    F.x.cp.pa2 = M_PI * M_PI / (c.alpha * c.alpha);
    F.x.cp.reference = ref ? 1 : 0;
    F.x.infl = B.infl;
    F.x.mx = c.mvec[0].p;
    F.x.my = c.mvec[1].p;
    F.x.mz = c.mvec[2].p;
    F.x.acc = c.acc.p;
    F.x.st = c.status.p;
    F.energy = energy;
    return F;
}
template FFTChain<float> make_fft_chain<float>(const Ctx&, bool);
template FFTChain<double> make_fft_chain<double>(const Ctx&, bool);

template <typename R>
static void conv_chain(Ctx& c, const PmeBufs<R>&, bool energy)
{
    const FFTChain<R> F = make_fft_chain<R>(c, energy);
    k_fft_z_r2c<R><<<grid_of(F.zf), FFT_THREADS, F.smz, c.stream>>>(F.zf);
    k_fft_y<R><<<grid_of(F.yf), FFT_THREADS, F.smy, c.stream>>>(F.yf);
    if (energy) k_fft_x_conv<R, true><<<grid_of(F.x), FFT_THREADS, F.smx, c.stream>>>(F.x);
    else k_fft_x_conv<R, false><<<grid_of(F.x), FFT_THREADS, F.smx, c.stream>>>(F.x);
    k_fft_y<R><<<grid_of(F.yi), FFT_THREADS, F.smy, c.stream>>>(F.yi);
    k_fft_z_c2r<R><<<grid_of(F.zi), FFT_THREADS, F.smz, c.stream>>>(F.zi);
}

// Many systems' FFT chains, one launch per pass (each struct array holds one
// entry per system; the block maps list every system's blocks; shared memory
// is the largest over systems).
template <typename R>
void launch_fft_chain_multi(const FFTChainDev<R>& D, const FFTChainMax& M, bool energy, cudaStream_t s)
{
    if (D.mz.n > 0) k_fft_z_r2c_multi<R><<<D.mz.n, FFT_THREADS, M.smz, s>>>(D.zf, D.mz.map);
    if (D.my.n > 0) k_fft_y_multi<R><<<D.my.n, FFT_THREADS, M.smy, s>>>(D.yf, D.my.map);
    if (D.mx.n > 0) {
        if (energy) k_fft_x_conv_multi<R, true><<<D.mx.n, FFT_THREADS, M.smx, s>>>(D.x, D.mx.map);
        else k_fft_x_conv_multi<R, false><<<D.mx.n, FFT_THREADS, M.smx, s>>>(D.x, D.mx.map);
    }
    if (D.my.n > 0) k_fft_y_multi<R><<<D.my.n, FFT_THREADS, M.smy, s>>>(D.yi, D.my.map);
    if (D.mz.n > 0) k_fft_z_c2r_multi<R><<<D.mz.n, FFT_THREADS, M.smz, s>>>(D.zi, D.mz.map);
    MDF_CUDA_TRY(cudaGetLastError());
}

// Spread and gather arguments of this rank's slots (PHYSICAL, order 4).
SpreadArgs make_spread_args(const Ctx& c)
{
    SpreadArgs A;
    long long s0, s1;
    slot_share(c, s0, s1);   // this rank's slots (all of them with one rank)
    A.s0 = (int)s0;
    A.s1 = (int)s1;
    A.gx = grid_blocks(16 * (s1 - s0), 256);
    A.gy = 1;
    A.slot_atom = c.slot_atom.p;
    A.xyz = c.xyz.p;
    A.q = c.q.p;
    for (int d = 0; d < 3; ++d) {
        A.g.K[d] = c.K[d];
        A.g.L[d] = c.box[d];
        A.g.scale[d] = (double)c.K[d] / c.box[d];
    }
    A.qgrid = c.qgrid.p;
    A.st = c.status.p;
    A.win_lo = 0;
    A.win_n = 0;
    if (halo_mode(c) && (int)c.win_n.size() == c.p.nranks) {
        A.win_lo = c.win_lo[c.p.rank];
        A.win_n = c.win_n[c.p.rank];
    }
    return A;
}

template <typename R>
GatherArgs<R> make_gather_args(const Ctx& c)
{
    GatherArgs<R> A;
    const PmeBufs<R> B(const_cast<Ctx&>(c));
    long long s0, s1;
    slot_share(c, s0, s1);
    A.s0 = (int)s0;
    A.s1 = (int)s1;
    A.nslots = c.n_slots;
    A.gx = grid_blocks(s1 - s0, 256);
    A.gy = 1;
    A.slot_atom = c.slot_atom.p;
    A.xyz = c.xyz.p;
    A.q = c.q.p;
    A.g = B.g;
    A.phi = B.rg;
    A.fslot = c.f_slot.p;
    A.st = c.status.p;
    return A;
}
template GatherArgs<float> make_gather_args<float>(const Ctx&);
template GatherArgs<double> make_gather_args<double>(const Ctx&);

template <typename R>
static void run_pme(Ctx& c, bool energy)
{
    const bool ref = c.p.semantics == MDF_SEM_REFERENCE;
    const PmeBufs<R> B(c);
    const long long ntot = (long long)c.K[0] * c.K[1] * c.K[2];
    MDF_CUDA_TRY(cudaMemsetAsync(c.qgrid.p, 0, sizeof(unsigned long long) * ntot, c.stream));
    const int th = 256;
    if (!ref) {
        const SpreadArgs S = make_spread_args(c);
        if (S.s1 > S.s0) k_spread4_rows<R><<<grid_of(S), th, 0, c.stream>>>(S);
        if (distributed(c)) allreduce_u64(c, c.qgrid.p, ntot);   // the whole charge grid on every rank
    } else {
        k_spread_ref5<<<grid_blocks(c.N, th), th, 0, c.stream>>>(c.N, c.xyz.p, c.q.p, B.g, c.qgrid.p);
    }
    mark(c, "pme_spread");
    conv_chain<R>(c, B, energy && rank0(c));   // reciprocal energy and virial counted once
    mark(c, "pme_fft_conv");
    if (!ref) {
        const GatherArgs<R> G = make_gather_args<R>(c);
        if (G.s1 > G.s0) k_gather4<R><<<grid_of(G), th, 0, c.stream>>>(G);
    } else {
        c.forces_pme_ref.alloc(3 * (size_t)c.N);
        k_gather_ref5<<<grid_blocks(c.N, th), th, 0, c.stream>>>(c.N, c.xyz.p, c.q.p, B.g,
                                                                 reinterpret_cast<const double*>(B.rg),
                                                                 c.forces_pme_ref.p);
    }
    mark(c, "pme_gather");
    MDF_CUDA_TRY(cudaGetLastError());
    c.launches += 7;   // spread, z, y, x+conv, y, z, gather
}

// ------------------------------------------- distributed reciprocal space
// x-slab decomposition over nranks (P): rank r owns planes [r K0p, (r+1) K0p)
// of the charge grid for the z and y passes and the y-range [r K1p, (r+1) K1p)
// for the x pass and the convolution; K0p = ceil(K0/P), K1p = ceil(K1/P).
// Transpose blocks are [P][K0p][K1p][Kc]: block t of a rank's send buffer
// holds its planes restricted to rank t's y-range.

// slab [K0p][K1][Kc] -> blocks [t][x][yl][kc] (y = t K1p + yl; zero past K1)
template <typename C>
__global__ void k_slab_to_blocks(const C* __restrict__ slab, C* __restrict__ blocks, int P, int K0p, int K1,
                                 int K1p, int Kc)
{
    const long long n = (long long)P * K0p * K1p * Kc;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int kc = (int)(e % Kc);
        long long rest = e / Kc;
        const int yl = (int)(rest % K1p);
        rest /= K1p;
        const int x = (int)(rest % K0p);
        const int t = (int)(rest / K0p);
        const int y = t * K1p + yl;
        C v;
        v.x = 0;
        v.y = 0;
        if (y < K1) v = slab[((long long)x * K1 + y) * Kc + kc];
        blocks[e] = v;
    }
}

// blocks [t][x][yl][kc] -> slab [K0p][K1][Kc]
template <typename C>
__global__ void k_blocks_to_slab(const C* __restrict__ blocks, C* __restrict__ slab, int K0p, int K1, int K1p, int Kc)
{
    const long long n = (long long)K0p * K1 * Kc;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int kc = (int)(e % Kc);
        const long long rest = e / Kc;
        const int y = (int)(rest % K1);
        const int x = (int)(rest / K1);
        const int t = y / K1p, yl = y - t * K1p;
        slab[e] = blocks[(((long long)t * K0p + x) * K1p + yl) * Kc + kc];
    }
}

static void coll_check(int rc, const char* what)
{
    if (rc != 0) throw ApiError(MDF_ERR_CUDA, std::string("the ") + what + " callback failed");
}

// Move n grid planes of `plane` words: plane k goes from src plane
// (src_pl ? src_pl[k] - src_off : k) to dst plane (dst_pl ? dst_pl[k] - dst_off
// : k), added (integer charge planes) or copied.  Packs and unpacks the halo
// exchange's buffers.
template <typename T, bool ADD>
__global__ void k_plane_move(const T* __restrict__ src, const int* __restrict__ src_pl, int src_off,
                             T* __restrict__ dst, const int* __restrict__ dst_pl, int dst_off, int n, long long plane)
{
    const long long total = (long long)n * plane;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(e / plane);
        const long long i = e - (long long)k * plane;
        const long long sp = src_pl ? src_pl[k] - src_off : k, dp = dst_pl ? dst_pl[k] - dst_off : k;
        if (ADD) dst[dp * plane + i] += src[sp * plane + i];
        else dst[dp * plane + i] = src[sp * plane + i];
    }
}

template <typename T, bool ADD>
static void plane_move(const T* src, const int* src_pl, int src_off, T* dst, const int* dst_pl, int dst_off, int n,
                       long long plane, cudaStream_t s)
{
    if (n <= 0) return;
    const int nb = (int)std::min<long long>(148 * 8, ((long long)n * plane + 255) / 256);
    k_plane_move<T, ADD><<<nb, 256, 0, s>>>(src, src_pl, src_off, dst, dst_pl, dst_off, n, plane);
    MDF_CUDA_TRY(cudaGetLastError());
}

// Per-rank byte counts of a halo exchange of planes: n[t] planes of `bytes` each.
static const int64_t* halo_counts(std::vector<int64_t>& out, const std::vector<int64_t>& n, size_t bytes)
{
    out.resize(n.size());
    for (size_t t = 0; t < n.size(); ++t) out[t] = n[t] * (int64_t)bytes;
    return out.data();
}

template <typename R>
static void run_pme_slab(Ctx& c, bool energy)
{
    using C = typename CT<R>::type;
    const int P = c.p.nranks, r = c.p.rank;
    const int K0 = c.K[0], K1 = c.K[1], K2 = c.K[2], Kc = K2 / 2 + 1;
    const int K0p = (K0 + P - 1) / P, K1p = (K1 + P - 1) / P;
    const long long plane = (long long)K1 * K2;
    const size_t blk = (size_t)K0p * K1p * Kc;
    // padded to P slabs: the planes past K0 stay zero
    c.qgrid.alloc((size_t)P * K0p * plane);
    if (sizeof(R) == 4) c.rgrid_f.alloc((size_t)P * K0p * plane);
    else c.rgrid_d.alloc((size_t)P * K0p * plane);
    c.q_slab.alloc((size_t)K0p * plane);
    c.pme_slab.alloc(sizeof(C) * (size_t)K0p * K1 * Kc);
    c.pme_send.alloc(sizeof(C) * P * blk);
    c.pme_recv.alloc(sizeof(C) * P * blk);
    c.pme_rslab.alloc(sizeof(R) * (size_t)K0p * plane);
    C* slab = reinterpret_cast<C*>(c.pme_slab.p);
    C* sendb = reinterpret_cast<C*>(c.pme_send.p);
    C* recvb = reinterpret_cast<C*>(c.pme_recv.p);
    R* rslab = reinterpret_cast<R*>(c.pme_rslab.p);
    const PmeBufs<R> B(c);
    const int th = 256;
    const bool halo = halo_mode(c);
    const int s_r = r * K0p;   // this rank's first plane
    const size_t hbytes = (size_t)plane * std::max(sizeof(unsigned long long), sizeof(R));
    if (halo) {
        c.halo_sendbuf.alloc(hbytes * (size_t)std::max(1, std::max(c.halo_n_send, c.halo_n_recv)));
        c.halo_recvbuf.alloc(hbytes * (size_t)std::max(1, std::max(c.halo_n_send, c.halo_n_recv)));
        // only the window's planes of the full-size grid are spread into
        for (int k = 0; k < 2; ++k)
            if (c.halo_rng[k][1] > 0)
                MDF_CUDA_TRY(cudaMemsetAsync(c.qgrid.p + (size_t)c.halo_rng[k][0] * plane, 0,
                                             sizeof(unsigned long long) * (size_t)c.halo_rng[k][1] * plane, c.stream));
    } else {
        MDF_CUDA_TRY(cudaMemsetAsync(c.qgrid.p, 0, sizeof(unsigned long long) * (size_t)P * K0p * plane, c.stream));
    }
    const SpreadArgs S = make_spread_args(c);
    if (S.s1 > S.s0) k_spread4_rows<R><<<grid_of(S), th, 0, c.stream>>>(S);
    MDF_CUDA_TRY(cudaGetLastError());
    if (halo) {
        // my slab = my own planes of my window + the planes other ranks spread into it
        using U = unsigned long long;
        U* hs = reinterpret_cast<U*>(c.halo_sendbuf.p);
        U* hr = reinterpret_cast<U*>(c.halo_recvbuf.p);
        MDF_CUDA_TRY(cudaMemsetAsync(c.q_slab.p, 0, sizeof(U) * (size_t)K0p * plane, c.stream));
        plane_move<U, true>(c.qgrid.p, c.halo_local_pl.p, 0, c.q_slab.p, c.halo_local_pl.p, s_r, c.halo_n_local, plane,
                            c.stream);
        plane_move<U, false>(c.qgrid.p, c.halo_send_pl.p, 0, hs, nullptr, 0, c.halo_n_send, plane, c.stream);
        coll_check(c.coll_a2av(hs, halo_counts(c.halo_bytes_a, c.halo_send_n, sizeof(U) * plane), hr,
                               halo_counts(c.halo_bytes_b, c.halo_recv_n, sizeof(U) * plane), (void*)c.stream,
                               c.coll_a2av_user),
                   "halo exchange");
        plane_move<U, true>(hr, nullptr, 0, c.q_slab.p, c.halo_recv_pl.p, s_r, c.halo_n_recv, plane, c.stream);
    } else {
        coll_check(c.coll_rs(reinterpret_cast<const uint64_t*>(c.qgrid.p), reinterpret_cast<uint64_t*>(c.q_slab.p),
                             (int64_t)K0p * plane, (void*)c.stream, c.coll_user),
                   "reduce-scatter");
    }
    mark(c, "pme_spread");
    FFTChain<R> F = make_fft_chain<R>(c, energy);
    const int nl = K0p * K1;
    F.zf.gx = (nl + 2 * F.zf.LP - 1) / (2 * F.zf.LP);
    F.zf.qgrid = c.q_slab.p;
    F.zf.cgrid = slab;
    F.zf.nlines = nl;
    F.zi = F.zf;
    F.zi.rgrid = rslab;
    F.yf.cgrid = slab;
    F.yf.gy = K0p;
    F.yi.cgrid = slab;
    F.yi.gy = K0p;
    const int ny = std::max(0, std::min(K1p, K1 - r * K1p));   // this rank's y planes
    F.x.cgrid = recvb;
    F.x.K1 = K1p;
    F.x.gy = ny;
    F.x.infl += (long long)r * K1p * Kc * K0;
    F.x.my += (long long)r * K1p;
    k_fft_z_r2c<R><<<grid_of(F.zf), FFT_THREADS, F.smz, c.stream>>>(F.zf);
    k_fft_y<R><<<grid_of(F.yf), FFT_THREADS, F.smy, c.stream>>>(F.yf);
    const int nb = (int)std::min<long long>(148 * 8, ((long long)P * blk + th - 1) / th);
    k_slab_to_blocks<C><<<nb, th, 0, c.stream>>>(slab, sendb, P, K0p, K1, K1p, Kc);
    MDF_CUDA_TRY(cudaGetLastError());
    coll_check(c.coll_a2a(sendb, recvb, (int64_t)(sizeof(C) * blk), (void*)c.stream, c.coll_user), "all-to-all");
    if (ny > 0) {
        if (energy) k_fft_x_conv<R, true><<<grid_of(F.x), FFT_THREADS, F.smx, c.stream>>>(F.x);
        else k_fft_x_conv<R, false><<<grid_of(F.x), FFT_THREADS, F.smx, c.stream>>>(F.x);
    }
    // back: the x-pass layout [s][x][yl][kc] is already one block per rank
    coll_check(c.coll_a2a(recvb, sendb, (int64_t)(sizeof(C) * blk), (void*)c.stream, c.coll_user), "all-to-all");
    k_blocks_to_slab<C><<<nb, th, 0, c.stream>>>(sendb, slab, K0p, K1, K1p, Kc);
    k_fft_y<R><<<grid_of(F.yi), FFT_THREADS, F.smy, c.stream>>>(F.yi);
    k_fft_z_c2r<R><<<grid_of(F.zi), FFT_THREADS, F.smz, c.stream>>>(F.zi);
    MDF_CUDA_TRY(cudaGetLastError());
    if (halo) {
        // the potential of my slab in place, and of my window's other planes from their owners
        R* ps = reinterpret_cast<R*>(c.halo_sendbuf.p);
        R* pr = reinterpret_cast<R*>(c.halo_recvbuf.p);
        const int nown = std::max(0, std::min(K0p, K0 - s_r));
        if (nown > 0)
            MDF_CUDA_TRY(cudaMemcpyAsync(B.rg + (size_t)s_r * plane, rslab, sizeof(R) * (size_t)nown * plane,
                                         cudaMemcpyDeviceToDevice, c.stream));
        plane_move<R, false>(rslab, c.halo_recv_pl.p, s_r, ps, nullptr, 0, c.halo_n_recv, plane, c.stream);
        coll_check(c.coll_a2av(ps, halo_counts(c.halo_bytes_a, c.halo_recv_n, sizeof(R) * plane), pr,
                               halo_counts(c.halo_bytes_b, c.halo_send_n, sizeof(R) * plane), (void*)c.stream,
                               c.coll_a2av_user),
                   "halo exchange");
        plane_move<R, false>(pr, nullptr, 0, B.rg, c.halo_send_pl.p, 0, c.halo_n_send, plane, c.stream);
    } else {
        coll_check(c.coll_ag(rslab, B.rg, (int64_t)(sizeof(R) * (size_t)K0p * plane), (void*)c.stream, c.coll_user),
                   "all-gather");
    }
    mark(c, "pme_fft_conv");
    const GatherArgs<R> G = make_gather_args<R>(c);
    if (G.s1 > G.s0) k_gather4<R><<<grid_of(G), th, 0, c.stream>>>(G);
    MDF_CUDA_TRY(cudaGetLastError());
    mark(c, "pme_gather");
    c.launches += 10;   // spread, z, y, pack, x+conv, unpack, y, z, gather (+ memset)
}

// Many systems: clear the charge grids, spread, the FFT chain, gather.
template <typename R>
void launch_pme_multi(const ZeroArgs* d_zero, BlockMap mzero, const SpreadArgs* d_spread, BlockMap mspread,
                      const FFTChainDev<R>& D, const FFTChainMax& M, const GatherArgs<R>* d_gather, BlockMap mgather,
                      bool energy, cudaStream_t s)
{
    if (mzero.n > 0) k_zero_multi<<<mzero.n, 256, 0, s>>>(d_zero, mzero.map);
    if (mspread.n > 0) k_spread4_rows_multi<R><<<mspread.n, 256, 0, s>>>(d_spread, mspread.map);
    MDF_CUDA_TRY(cudaGetLastError());
    launch_fft_chain_multi<R>(D, M, energy, s);
    if (mgather.n > 0) k_gather4_multi<R><<<mgather.n, 256, 0, s>>>(d_gather, mgather.map);
    MDF_CUDA_TRY(cudaGetLastError());
}
template void launch_pme_multi<float>(const ZeroArgs*, BlockMap, const SpreadArgs*, BlockMap, const FFTChainDev<float>&,
                                      const FFTChainMax&, const GatherArgs<float>*, BlockMap, bool, cudaStream_t);
template void launch_pme_multi<double>(const ZeroArgs*, BlockMap, const SpreadArgs*, BlockMap,
                                       const FFTChainDev<double>&, const FFTChainMax&, const GatherArgs<double>*,
                                       BlockMap, bool, cudaStream_t);

// ------------------------------------------------------------- adjoint
// Reciprocal-space part of mdf_backward.  With E = 1/2 Q^T C Q (Q the charge
// grid, C the convolution with the influence function), phi = C Q, F_a =
// -q_a grad phi(x_a), v = dL/dF and gE = dL/dE, the derivative of
// gE E + v.F with respect to q_a is
//   gE phi(x_a) - v_a . grad phi(x_a) - theta_a^T C P,
//   P = sum_b q_b (v_b . grad theta_b)   (a "dipole" grid).
// C is symmetric, so C P is the same convolution chain applied to P.

// Per slot: gE phi - v . grad phi at the atom, added to dq (fixed point).
template <typename R>
__global__ void k_adj_gather_phi(int nslots, const int* __restrict__ slot_atom, const double* __restrict__ xyz,
                                 GridGeom g, const R* __restrict__ phi, const typename V4<R>::type* __restrict__ vs,
                                 double gE, unsigned long long* __restrict__ dq, unsigned* st)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const int a = slot_atom[s];
    if (a < 0) return;
    int base[3];
    R th[3][4], dth[3][4];
    for (int d = 0; d < 3; ++d) {
        double u = wrap_coord(xyz[3 * a + d], g.L[d]) * g.scale[d];
        if (!(u >= 0.0 && u <= (double)g.K[d])) {
            status_set(st, ST_NONFINITE);
            return;
        }
        if (u >= g.K[d]) u -= g.K[d];
        const int b = min((int)floor(u), g.K[d] - 1);
        base[d] = b;
        bspline4<R>((R)(u - b), th[d], dth[d]);
    }
    R p = 0, gx = 0, gy = 0, gz = 0;
    for (int i = 0; i < 4; ++i) {
        int kx = base[0] - 1 + i;
        kx += (kx < 0) ? g.K[0] : 0;
        kx -= (kx >= g.K[0]) ? g.K[0] : 0;
        for (int j = 0; j < 4; ++j) {
            int ky = base[1] - 1 + j;
            ky += (ky < 0) ? g.K[1] : 0;
            ky -= (ky >= g.K[1]) ? g.K[1] : 0;
            const long long row = ((long long)kx * g.K[1] + ky) * g.K[2];
            R sz = 0, dz = 0;
            for (int k = 0; k < 4; ++k) {
                int kz = base[2] - 1 + k;
                kz += (kz < 0) ? g.K[2] : 0;
                kz -= (kz >= g.K[2]) ? g.K[2] : 0;
                const R v = phi[row + kz];
                sz += th[2][k] * v;
                dz += dth[2][k] * v;
            }
            p += th[0][i] * th[1][j] * sz;
            gx += dth[0][i] * th[1][j] * sz;
            gy += th[0][i] * dth[1][j] * sz;
            gz += th[0][i] * th[1][j] * dz;
        }
    }
    const typename V4<R>::type v = vs[s];
    const double val = gE * (double)p - ((double)v.x * (double)(gx * (R)g.scale[0]) +
                                         (double)v.y * (double)(gy * (R)g.scale[1]) +
                                         (double)v.z * (double)(gz * (R)g.scale[2]));
    fx_add(dq + s, val, FORCE_SCALE, st);
}

// Per slot: spread q_a (v_a . grad theta_a) onto the fixed-point grid.
template <typename R>
__global__ void k_adj_spread_dipole(int nslots, const int* __restrict__ slot_atom, const double* __restrict__ xyz,
                                    const double* __restrict__ q, GridGeom g,
                                    const typename V4<R>::type* __restrict__ vs, unsigned long long* __restrict__ qgrid,
                                    unsigned* st)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const int a = slot_atom[s];
    if (a < 0) return;
    const double qa = q[a];
    if (qa == 0.0) return;
    int base[3];
    R th[3][4], dth[3][4];
    for (int d = 0; d < 3; ++d) {
        double u = wrap_coord(xyz[3 * a + d], g.L[d]) * g.scale[d];
        if (!(u >= 0.0 && u <= (double)g.K[d])) {
            status_set(st, ST_NONFINITE);
            return;
        }
        if (u >= g.K[d]) u -= g.K[d];
        const int b = min((int)floor(u), g.K[d] - 1);
        base[d] = b;
        bspline4<R>((R)(u - b), th[d], dth[d]);
    }
    const typename V4<R>::type v = vs[s];
    const R cx = (R)qa * v.x * (R)g.scale[0], cy = (R)qa * v.y * (R)g.scale[1], cz = (R)qa * v.z * (R)g.scale[2];
    for (int i = 0; i < 4; ++i) {
        int kx = base[0] - 1 + i;
        kx += (kx < 0) ? g.K[0] : 0;
        kx -= (kx >= g.K[0]) ? g.K[0] : 0;
        for (int j = 0; j < 4; ++j) {
            int ky = base[1] - 1 + j;
            ky += (ky < 0) ? g.K[1] : 0;
            ky -= (ky >= g.K[1]) ? g.K[1] : 0;
            const long long row = ((long long)kx * g.K[1] + ky) * g.K[2];
            const R wx = cx * dth[0][i] * th[1][j], wy = cy * th[0][i] * dth[1][j], wz = cz * th[0][i] * th[1][j];
            for (int k = 0; k < 4; ++k) {
                int kz = base[2] - 1 + k;
                kz += (kz < 0) ? g.K[2] : 0;
                kz -= (kz >= g.K[2]) ? g.K[2] : 0;
                const R val = (wx + wy) * th[2][k] + wz * dth[2][k];
                atomicAdd(qgrid + row + kz, (unsigned long long)__double2ll_rn((double)val * GRID_SCALE));
            }
        }
    }
}

// Per slot: -theta_a^T (C P), added to dq.
template <typename R>
__global__ void k_adj_gather_dipole(int nslots, const int* __restrict__ slot_atom, const double* __restrict__ xyz,
                                    GridGeom g, const R* __restrict__ cp, unsigned long long* __restrict__ dq,
                                    unsigned* st)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const int a = slot_atom[s];
    if (a < 0) return;
    int base[3];
    R th[3][4];
    for (int d = 0; d < 3; ++d) {
        double u = wrap_coord(xyz[3 * a + d], g.L[d]) * g.scale[d];
        if (!(u >= 0.0 && u <= (double)g.K[d])) {
            status_set(st, ST_NONFINITE);
            return;
        }
        if (u >= g.K[d]) u -= g.K[d];
        const int b = min((int)floor(u), g.K[d] - 1);
        base[d] = b;
        bspline4<R>((R)(u - b), th[d], nullptr);
    }
    R p = 0;
    for (int i = 0; i < 4; ++i) {
        int kx = base[0] - 1 + i;
        kx += (kx < 0) ? g.K[0] : 0;
        kx -= (kx >= g.K[0]) ? g.K[0] : 0;
        for (int j = 0; j < 4; ++j) {
            int ky = base[1] - 1 + j;
            ky += (ky < 0) ? g.K[1] : 0;
            ky -= (ky >= g.K[1]) ? g.K[1] : 0;
            const long long row = ((long long)kx * g.K[1] + ky) * g.K[2];
            R sz = 0;
            for (int k = 0; k < 4; ++k) {
                int kz = base[2] - 1 + k;
                kz += (kz < 0) ? g.K[2] : 0;
                kz -= (kz >= g.K[2]) ? g.K[2] : 0;
                sz += th[2][k] * cp[row + kz];
            }
            p += th[0][i] * th[1][j] * sz;
        }
    }
    fx_add(dq + s, -(double)p, FORCE_SCALE, st);
}

template <typename R>
static void run_pme_adjoint(Ctx& c, double gE)
{
    const PmeBufs<R> B(c);
    const typename V4<R>::type* vs;
    if (sizeof(R) == 4) vs = reinterpret_cast<const typename V4<R>::type*>(c.adj_vs_f.p);
    else vs = reinterpret_cast<const typename V4<R>::type*>(c.adj_vs_d.p);
    const long long ntot = (long long)c.K[0] * c.K[1] * c.K[2];
    const int th = 256, nb = grid_blocks(c.n_slots, th);
    // phi = C Q
    MDF_CUDA_TRY(cudaMemsetAsync(c.qgrid.p, 0, sizeof(unsigned long long) * ntot, c.stream));
    k_spread4<R><<<nb, th, 0, c.stream>>>(0, c.n_slots, c.slot_atom.p, c.xyz.p, c.q.p, B.g, c.qgrid.p, c.status.p);
    conv_chain<R>(c, B, false);
    k_adj_gather_phi<R><<<nb, th, 0, c.stream>>>(c.n_slots, c.slot_atom.p, c.xyz.p, B.g, B.rg, vs, gE,
                                                 c.adj_dq_slot.p, c.status.p);
    // C P
    MDF_CUDA_TRY(cudaMemsetAsync(c.qgrid.p, 0, sizeof(unsigned long long) * ntot, c.stream));
    k_adj_spread_dipole<R><<<nb, th, 0, c.stream>>>(c.n_slots, c.slot_atom.p, c.xyz.p, c.q.p, B.g, vs, c.qgrid.p,
                                                    c.status.p);
    conv_chain<R>(c, B, false);
    k_adj_gather_dipole<R><<<nb, th, 0, c.stream>>>(c.n_slots, c.slot_atom.p, c.xyz.p, B.g, B.rg, c.adj_dq_slot.p,
                                                    c.status.p);
    MDF_CUDA_TRY(cudaGetLastError());
    c.launches += 14;
}

void pme_adjoint(Ctx& c, double gE, double)
{
    if (c.p.precision == MDF_PREC_MIXED) run_pme_adjoint<float>(c, gE);
    else run_pme_adjoint<double>(c, gE);
}

void launch_pme(Ctx& c, bool energy)
{
    const bool f32 = c.p.semantics == MDF_SEM_PHYSICAL && c.p.precision == MDF_PREC_MIXED;
    if (slab_mode(c)) {
        if (f32) run_pme_slab<float>(c, energy);
        else run_pme_slab<double>(c, energy);
    } else if (f32) {
        run_pme<float>(c, energy);
    } else {
        run_pme<double>(c, energy);
    }
}

}  // namespace mdf
