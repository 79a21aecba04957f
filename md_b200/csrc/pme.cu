// Particle-mesh Ewald: charge spread, hand-written 3-D FFT, reciprocal
// convolution with the FP64 energy/virial reduction, and force gather.
//
// PHYSICAL semantics: smooth PME of order n (Essmann et al., J. Chem. Phys.
// 103, 8577 (1995)): E = 1/2 sum_m c(m) |S(m)|^2 with
// c(m) = k/(pi V) exp(-pi^2 m^2/alpha^2)/m^2 * B1 B2 B3, B_d = 1/|b_d(m_d)|^2.
// REFERENCE semantics: the reference's own chain, order 5 with its weights and
// grid offsets (src/System/PBC.cpp:183-250, :329-401), its moduli (:455-490),
// its solve with the extra 1/N and without the Coulomb constant (:501-564) and
// its gather (:576-653).  The reference discards those forces; they are
// returned separately for parity checks.
//
// FFT: mixed-radix Stockham autosort in shared memory (radix 4/2/3/5 and a
// generic small-prime butterfly), one kernel per dimension:
//   z: real -> half complex, two real lines packed per complex transform
//   y: complex, LP consecutive kz columns per block (coalesced along kz)
//   x: complex forward, convolution, complex inverse in one kernel
//   y: inverse
//   z: half complex -> real
// The charge grid is accumulated in int64 fixed point (2^-40), so the spread
// is deterministic regardless of atomic ordering.
#include <algorithm>
#include <cmath>
#include <vector>

#include "mdf_device.cuh"
#include "mdf_internal.cuh"

namespace mdf {

template <typename R> struct CT;
template <> struct CT<float> { using type = float2; };
template <> struct CT<double> { using type = double2; };

struct FFTDesc {
    int n;
    int nst;
    int radix[16];
};

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
        // multiply t3 by -i (forward) or +i (inverse)
        C t3r = {-s * t3.y, s * t3.x};
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
        // i * (s1 d1 + s2 d2), i * (s2 d1 - s1 d2)
        C n1 = {s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y};
        C n2 = {s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y};
        v[1].x = m1.x - n1.y; v[1].y = m1.y + n1.x;
        v[4].x = m1.x + n1.y; v[4].y = m1.y - n1.x;
        v[2].x = m2.x - n2.y; v[2].y = m2.y + n2.x;
        v[3].x = m2.x + n2.y; v[3].y = m2.y - n2.x;
    } else {
        // generic prime radix via the line's twiddle table: W_R^q = W_n^{q n/R}
        C out[32];
        int step = n / Rr;
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

// One Stockham stage with a compile-time radix (registers only).
template <typename C, typename R, int RR>
__device__ __forceinline__ void stockham_stage(const C* a, C* b, int nl, int n, int Ns, const C* tw, bool inverse)
{
    const int nb = n / RR;
    const int step = n / (Ns * RR);
    for (int t = threadIdx.x; t < nl * nb; t += blockDim.x) {
        const int line = t / nb, j = t - line * nb;
        const C* in = a + line * n;
        C* out = b + line * n;
        const int k = j % Ns;
        C v[RR];
#pragma unroll
        for (int r = 0; r < RR; ++r) {
            C x = in[j + r * nb];
            if (r && k) {
                C w = tw[(r * k * step) % n];
                if (inverse) w = cconj(w);
                x = cmul(x, w);
            }
            v[r] = x;
        }
        small_dft<C, R>(v, RR, inverse, tw, n);
        const int idxD = (j / Ns) * Ns * RR + k;
#pragma unroll
        for (int r = 0; r < RR; ++r) out[idxD + r * Ns] = v[r];
    }
}

// Generic prime radix (7..31), runtime-sized.
template <typename C, typename R>
__device__ void stockham_stage_generic(const C* a, C* b, int nl, int n, int Ns, int Rr, const C* tw, bool inverse)
{
    const int nb = n / Rr;
    const int step = n / (Ns * Rr);
    for (int t = threadIdx.x; t < nl * nb; t += blockDim.x) {
        const int line = t / nb, j = t - line * nb;
        const C* in = a + line * n;
        C* out = b + line * n;
        const int k = j % Ns;
        C v[32];
        for (int r = 0; r < Rr; ++r) {
            C x = in[j + r * nb];
            if (r && k) {
                C w = tw[(r * k * step) % n];
                if (inverse) w = cconj(w);
                x = cmul(x, w);
            }
            v[r] = x;
        }
        small_dft<C, R>(v, Rr, inverse, tw, n);
        const int idxD = (j / Ns) * Ns * Rr + k;
        for (int r = 0; r < Rr; ++r) out[idxD + r * Ns] = v[r];
    }
}

// Stockham autosort FFT of nl lines stored [line][n] in shared memory.
// tw[q] = exp(-2 pi i q / n).  Returns the buffer holding the result.
template <typename C, typename R>
__device__ C* fft_lines(C* a, C* b, int nl, const FFTDesc& d, const C* tw, bool inverse)
{
    int Ns = 1;
    const int n = d.n;
    for (int s = 0; s < d.nst; ++s) {
        const int Rr = d.radix[s];
        switch (Rr) {
            case 2: stockham_stage<C, R, 2>(a, b, nl, n, Ns, tw, inverse); break;
            case 3: stockham_stage<C, R, 3>(a, b, nl, n, Ns, tw, inverse); break;
            case 4: stockham_stage<C, R, 4>(a, b, nl, n, Ns, tw, inverse); break;
            case 5: stockham_stage<C, R, 5>(a, b, nl, n, Ns, tw, inverse); break;
            default: stockham_stage_generic<C, R>(a, b, nl, n, Ns, Rr, tw, inverse); break;
        }
        __syncthreads();
        C* tmp = a;
        a = b;
        b = tmp;
        Ns *= Rr;
    }
    return a;
}

template <typename C>
__device__ void load_tw(C* s_tw, const C* __restrict__ g_tw, int n)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_tw[i] = g_tw[i];
}

// ------------------------------------------------------------- z passes
template <typename R>
__global__ void k_fft_z_r2c(const unsigned long long* __restrict__ qgrid, typename CT<R>::type* __restrict__ cgrid,
                            int nlines, int K2, FFTDesc dz, const typename CT<R>::type* __restrict__ twz, int LP)
{
    using C = typename CT<R>::type;
    extern __shared__ unsigned char smem_raw[];
    C* s_tw = reinterpret_cast<C*>(smem_raw);
    C* bufA = s_tw + K2;
    C* bufB = bufA + LP * K2;
    load_tw(s_tw, twz, K2);
    const long long line0 = (long long)blockIdx.x * 2 * LP;
    for (int e = threadIdx.x; e < 2 * LP * K2; e += blockDim.x) {
        int rl = e / K2, z = e - rl * K2;
        long long g = line0 + rl;
        R v = 0;
        if (g < nlines) v = (R)((double)(long long)qgrid[g * K2 + z] * GRID_ISCALE);
        R* comp = reinterpret_cast<R*>(&bufA[(rl >> 1) * K2 + z]);
        comp[rl & 1] = v;
    }
    __syncthreads();
    C* res = fft_lines<C, R>(bufA, bufB, LP, dz, s_tw, false);
    const int Kc = K2 / 2 + 1;
    for (int e = threadIdx.x; e < LP * Kc; e += blockDim.x) {
        int p = e / Kc, k = e - p * Kc;
        C Z = res[p * K2 + k], Zc = cconj(res[p * K2 + (K2 - k) % K2]);
        C A = {(R)0.5 * (Z.x + Zc.x), (R)0.5 * (Z.y + Zc.y)};
        C B = {(R)0.5 * (Z.y - Zc.y), (R)-0.5 * (Z.x - Zc.x)};
        long long g = line0 + 2 * p;
        if (g < nlines) cgrid[g * Kc + k] = A;
        if (g + 1 < nlines) cgrid[(g + 1) * Kc + k] = B;
    }
}

template <typename R>
__global__ void k_fft_z_c2r(const typename CT<R>::type* __restrict__ cgrid, R* __restrict__ rgrid, int nlines, int K2,
                            FFTDesc dz, const typename CT<R>::type* __restrict__ twz, int LP)
{
    using C = typename CT<R>::type;
    extern __shared__ unsigned char smem_raw[];
    C* s_tw = reinterpret_cast<C*>(smem_raw);
    C* bufA = s_tw + K2;
    C* bufB = bufA + LP * K2;
    load_tw(s_tw, twz, K2);
    const long long line0 = (long long)blockIdx.x * 2 * LP;
    const int Kc = K2 / 2 + 1;
    for (int e = threadIdx.x; e < LP * K2; e += blockDim.x) {
        int p = e / K2, k = e - p * K2;
        long long g = line0 + 2 * p;
        C A = {0, 0}, B = {0, 0};
        int kk = k < Kc ? k : K2 - k;
        if (g < nlines) A = cgrid[g * Kc + kk];
        if (g + 1 < nlines) B = cgrid[(g + 1) * Kc + kk];
        if (k >= Kc) {
            A = cconj(A);
            B = cconj(B);
        }
        C Z = {A.x - B.y, A.y + B.x};
        bufA[p * K2 + k] = Z;
    }
    __syncthreads();
    C* res = fft_lines<C, R>(bufA, bufB, LP, dz, s_tw, true);
    for (int e = threadIdx.x; e < LP * K2; e += blockDim.x) {
        int p = e / K2, k = e - p * K2;
        long long g = line0 + 2 * p;
        C Z = res[p * K2 + k];
        if (g < nlines) rgrid[g * K2 + k] = Z.x;
        if (g + 1 < nlines) rgrid[(g + 1) * K2 + k] = Z.y;
    }
}

// ------------------------------------------------------------- y pass
template <typename R>
__global__ void k_fft_y(typename CT<R>::type* __restrict__ cgrid, int K1, int Kc, FFTDesc dy,
                        const typename CT<R>::type* __restrict__ twy, int LP, bool inverse)
{
    using C = typename CT<R>::type;
    extern __shared__ unsigned char smem_raw[];
    C* s_tw = reinterpret_cast<C*>(smem_raw);
    C* bufA = s_tw + K1;
    C* bufB = bufA + LP * K1;
    load_tw(s_tw, twy, K1);
    const int x = blockIdx.y;
    const int kz0 = blockIdx.x * LP;
    const long long base = (long long)x * K1 * Kc;
    for (int e = threadIdx.x; e < LP * K1; e += blockDim.x) {
        int y = e / LP, l = e - y * LP;
        int kz = kz0 + l;
        C v = {0, 0};
        if (kz < Kc) v = cgrid[base + (long long)y * Kc + kz];
        bufA[l * K1 + y] = v;
    }
    __syncthreads();
    C* res = fft_lines<C, R>(bufA, bufB, LP, dy, s_tw, inverse);
    for (int e = threadIdx.x; e < LP * K1; e += blockDim.x) {
        int y = e / LP, l = e - y * LP;
        int kz = kz0 + l;
        if (kz < Kc) cgrid[base + (long long)y * Kc + kz] = res[l * K1 + y];
    }
}

// ------------------------------------------- x pass + convolution + inverse
struct ConvParams {
    int K[3];
    double L[3];
    double fac;       // PHYSICAL: k/(pi V); REFERENCE: 4 pi / V
    double pa2;       // PHYSICAL: pi^2/alpha^2; REFERENCE: 1/(4 alpha^2)
    double norm;      // REFERENCE: 1/(K0 K1 K2)
    int reference;
};

template <typename R, bool ENERGY>
__global__ void k_fft_x_conv(typename CT<R>::type* __restrict__ cgrid, int K1, int Kc, FFTDesc dx,
                             const typename CT<R>::type* __restrict__ twx, int LP, ConvParams cp,
                             const R* __restrict__ b0, const R* __restrict__ b1, const R* __restrict__ b2,
                             unsigned long long* __restrict__ acc, unsigned* st)
{
    using C = typename CT<R>::type;
    extern __shared__ unsigned char smem_raw[];
    const int K0 = cp.K[0];
    C* s_tw = reinterpret_cast<C*>(smem_raw);
    C* bufA = s_tw + K0;
    C* bufB = bufA + LP * K0;
    load_tw(s_tw, twx, K0);
    const int y = blockIdx.y;
    const int kz0 = blockIdx.x * LP;
    const long long stride = (long long)K1 * Kc;
    for (int e = threadIdx.x; e < LP * K0; e += blockDim.x) {
        int x = e / LP, l = e - x * LP;
        int kz = kz0 + l;
        C v = {0, 0};
        if (kz < Kc) v = cgrid[x * stride + (long long)y * Kc + kz];
        bufA[l * K0 + x] = v;
    }
    __syncthreads();
    C* res = fft_lines<C, R>(bufA, bufB, LP, dx, s_tw, false);
    C* other = (res == bufA) ? bufB : bufA;
    double e_sum = 0, w6[6] = {0, 0, 0, 0, 0, 0};
    const int my_i = (y <= cp.K[1] / 2) ? y : y - cp.K[1];
    for (int e = threadIdx.x; e < LP * K0; e += blockDim.x) {
        int l = e / K0, kx = e - l * K0;
        int kz = kz0 + l;
        C S = res[l * K0 + kx];
        if (kz >= Kc) continue;
        int mx_i = (kx <= K0 / 2) ? kx : kx - K0;
        if (!cp.reference) {
            double mx = mx_i / cp.L[0], my = my_i / cp.L[1], mz = kz / cp.L[2];
            double m2 = mx * mx + my * my + mz * mz;
            R c;
            if (kx == 0 && y == 0 && kz == 0) {
                c = 0;
            } else {
                c = (R)(cp.fac * exp(-cp.pa2 * m2) / m2) * b0[kx] * b1[y] * b2[kz];
                if (ENERGY) {
                    double wgt = (kz == 0 || ((cp.K[2] & 1) == 0 && kz == cp.K[2] / 2)) ? 1.0 : 2.0;
                    double s2 = (double)S.x * S.x + (double)S.y * S.y;
                    double em = 0.5 * (double)c * s2 * wgt;
                    e_sum += em;
                    double vf = 2.0 * (1.0 + cp.pa2 * m2) / m2;
                    double mv[3] = {mx, my, mz};
                    int q = 0;
                    for (int a = 0; a < 3; ++a)
                        for (int b = a; b < 3; ++b) w6[q++] += em * ((a == b ? 1.0 : 0.0) - vf * mv[a] * mv[b]);
                }
            }
            S.x *= c;
            S.y *= c;
        } else {
            // src/System/PBC.cpp:511-563
            const double PI = 3.14159265358979323846;
            double kxv = 2.0 * PI * mx_i / cp.L[0], kyv = 2.0 * PI * my_i / cp.L[1], kzv = 2.0 * PI * kz / cp.L[2];
            double ksq = kxv * kxv + kyv * kyv + kzv * kzv;
            if (ksq < 1e-10) {
                S.x = 0;
                S.y = 0;
            } else {
                double infl = cp.fac * exp(ksq * (-cp.pa2)) / ksq;
                double bc = 1.0 / ((double)b0[kx] * (double)b1[y] * (double)b2[kz]);
                double sc = infl * bc * cp.norm;
                S.x = (R)(S.x * sc);
                S.y = (R)(S.y * sc);
            }
        }
        res[l * K0 + kx] = S;
    }
    __syncthreads();
    C* out = fft_lines<C, R>(res, other, LP, dx, s_tw, true);
    for (int e = threadIdx.x; e < LP * K0; e += blockDim.x) {
        int x = e / LP, l = e - x * LP;
        int kz = kz0 + l;
        if (kz < Kc) cgrid[x * stride + (long long)y * Kc + kz] = out[l * K0 + x];
    }
    if (ENERGY && !cp.reference) {
        const double v[7] = {e_sum, w6[0], w6[1], w6[2], w6[3], w6[4], w6[5]};
        const int idx[7] = {MDF_E_EE_RECIP, ACC_VIR + 0, ACC_VIR + 1, ACC_VIR + 2, ACC_VIR + 3, ACC_VIR + 4,
                            ACC_VIR + 5};
        block_acc_fixed<7>(v, acc, idx, ENERGY_SCALE, st);
    }
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

struct GridGeom {
    int K[3];
    double L[3];
    double scale[3];   // K/L
};

template <typename R>
__global__ void k_spread4(int nslots, const int* __restrict__ slot_atom, const double* __restrict__ xyz,
                          const double* __restrict__ q, GridGeom g, unsigned long long* __restrict__ qgrid,
                          unsigned* st)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
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

template <typename R>
__global__ void k_gather4(int nslots, const int* __restrict__ slot_atom, const double* __restrict__ xyz,
                          const double* __restrict__ q, GridGeom g, const R* __restrict__ phi,
                          unsigned long long* __restrict__ fslot, unsigned* st)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
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

// The reference's order-5 weights (src/System/PBC.cpp:329-356 for the spread,
// :359-401 for the gather; the two differ in operation order).
__device__ __forceinline__ void ref_w5_spread(double u, double th[5])
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
static FFTPlan1D make_plan(int n)
{
    FFTPlan1D p;
    p.n = n;
    p.nstages = 0;
    int m = n;
    while (m % 4 == 0) { p.radix[p.nstages++] = 4; m /= 4; }
    while (m % 2 == 0) { p.radix[p.nstages++] = 2; m /= 2; }
    for (int f = 3; f <= 31 && m > 1; f += 2)
        while (m % f == 0) {
            if (p.nstages >= 16) throw ApiError(MDF_ERR_UNSUPPORTED, "FFT size has too many factors");
            p.radix[p.nstages++] = f;
            m /= f;
        }
    if (m != 1) throw ApiError(MDF_ERR_UNSUPPORTED, "PME grid size has a prime factor above 31");
    return p;
}

static FFTDesc to_desc(const FFTPlan1D& p)
{
    FFTDesc d;
    d.n = p.n;
    d.nst = p.nstages;
    for (int i = 0; i < 16; ++i) d.radix[i] = i < p.nstages ? p.radix[i] : 1;
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

// Cardinal B-spline M_n at integer points 1..n-1 (Essmann eq. 4.1 recursion).
static double cardinal_bspline(int n, double x)
{
    if (x <= 0.0 || x >= n) return 0.0;
    if (n == 2) return 1.0 - std::fabs(x - 1.0);
    return (x * cardinal_bspline(n - 1, x) + (n - x) * cardinal_bspline(n - 1, x - 1.0)) / (n - 1);
}

static void ref_w5_spread_host(double u, double th[5])
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

static int lines_per_block(int n, size_t csize)
{
    // two ping-pong buffers + twiddles within 48 KB
    // few lines per block: many small blocks keep every SM busy on these
    // latency-bound, L2-resident passes
    size_t budget = 46 * 1024;
    int lp = (int)((budget / csize - n) / (2 * (size_t)n));
    return std::max(1, std::min(4, lp));
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
        c.plan[d] = make_plan(K);
    }
    c.order = ref ? 5 : (c.p.pme_order > 0 ? c.p.pme_order : 4);
    if (!ref && c.order != 4) throw ApiError(MDF_ERR_UNSUPPORTED, "PHYSICAL PME supports order 4");
    long long ntot = (long long)c.K[0] * c.K[1] * c.K[2];
    long long nc = (long long)c.K[0] * c.K[1] * (c.K[2] / 2 + 1);
    c.qgrid.alloc(ntot);
    bool mixed = c.p.precision == MDF_PREC_MIXED && !ref;
    if (mixed) {
        c.cgrid_f.alloc(nc);
        c.rgrid_f.alloc(ntot);
    } else {
        c.cgrid_d.alloc(nc);
        c.rgrid_d.alloc(ntot);
    }
    for (int d = 0; d < 3; ++d) {
        int K = c.K[d];
        std::vector<double> b(K);
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
            // the reference's moduli: |r2c of theta5(0) at 0,1,2,-1,-2|^2 (src/System/PBC.cpp:455-490)
            double th[5];
            ref_w5_spread_host(0.0, th);
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
            std::vector<float> bf(K);
            std::vector<float2> twf(K);
            for (int i = 0; i < K; ++i) {
                bf[i] = (float)b[i];
                twf[i] = make_float2((float)tw[i].x, (float)tw[i].y);
            }
            c.bmod_f[d].upload(bf.data(), K, c.stream);
            c.tw_f[d].upload(twf.data(), K, c.stream);
        } else {
            c.bmod[d].upload(b.data(), K, c.stream);
            c.tw_d[d].upload(tw.data(), K, c.stream);
        }
    }
    MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
}

template <typename R>
static void run_pme(Ctx& c, bool energy)
{
    using C = typename CT<R>::type;
    const bool ref = c.p.semantics == MDF_SEM_REFERENCE;
    const int K0 = c.K[0], K1 = c.K[1], K2 = c.K[2], Kc = K2 / 2 + 1;
    C* cg;
    R* rg;
    const C *twx, *twy, *twz;
    const R *b0, *b1, *b2;
    if (sizeof(R) == 4) {
        cg = reinterpret_cast<C*>(c.cgrid_f.p); rg = reinterpret_cast<R*>(c.rgrid_f.p);
        twx = reinterpret_cast<const C*>(c.tw_f[0].p); twy = reinterpret_cast<const C*>(c.tw_f[1].p);
        twz = reinterpret_cast<const C*>(c.tw_f[2].p);
        b0 = reinterpret_cast<const R*>(c.bmod_f[0].p); b1 = reinterpret_cast<const R*>(c.bmod_f[1].p);
        b2 = reinterpret_cast<const R*>(c.bmod_f[2].p);
    } else {
        cg = reinterpret_cast<C*>(c.cgrid_d.p); rg = reinterpret_cast<R*>(c.rgrid_d.p);
        twx = reinterpret_cast<const C*>(c.tw_d[0].p); twy = reinterpret_cast<const C*>(c.tw_d[1].p);
        twz = reinterpret_cast<const C*>(c.tw_d[2].p);
        b0 = reinterpret_cast<const R*>(c.bmod[0].p); b1 = reinterpret_cast<const R*>(c.bmod[1].p);
        b2 = reinterpret_cast<const R*>(c.bmod[2].p);
    }
    GridGeom g;
    for (int d = 0; d < 3; ++d) {
        g.K[d] = c.K[d];
        g.L[d] = c.box[d];
        g.scale[d] = (double)c.K[d] / c.box[d];
    }
    long long ntot = (long long)K0 * K1 * K2;
    MDF_CUDA_TRY(cudaMemsetAsync(c.qgrid.p, 0, sizeof(unsigned long long) * ntot, c.stream));
    const int th = 256;
    if (!ref) {
        k_spread4<R><<<grid_blocks(c.n_slots, th), th, 0, c.stream>>>(c.n_slots, c.slot_atom.p, c.xyz.p, c.q.p, g,
                                                                      c.qgrid.p, c.status.p);
    } else {
        k_spread_ref5<<<grid_blocks(c.N, th), th, 0, c.stream>>>(c.N, c.xyz.p, c.q.p, g, c.qgrid.p);
    }
    mark(c, "pme_spread");
    const int fth = 128;
    // z forward (real -> half complex)
    {
        int LP = lines_per_block(K2, sizeof(C));
        size_t sm = sizeof(C) * ((size_t)K2 + 2 * (size_t)LP * K2);
        int nlines = K0 * K1;
        int nb = (nlines + 2 * LP - 1) / (2 * LP);
        k_fft_z_r2c<R><<<nb, fth, sm, c.stream>>>(c.qgrid.p, cg, nlines, K2, to_desc(c.plan[2]), twz, LP);
    }
    // y forward
    int LPy = lines_per_block(K1, sizeof(C));
    size_t smy = sizeof(C) * ((size_t)K1 + 2 * (size_t)LPy * K1);
    dim3 gy((Kc + LPy - 1) / LPy, K0);
    k_fft_y<R><<<gy, fth, smy, c.stream>>>(cg, K1, Kc, to_desc(c.plan[1]), twy, LPy, false);
    // x forward + convolution + x inverse
    {
        int LP = lines_per_block(K0, sizeof(C));
        size_t sm = sizeof(C) * ((size_t)K0 + 2 * (size_t)LP * K0);
        dim3 gx((Kc + LP - 1) / LP, K1);
        ConvParams cp;
        for (int d = 0; d < 3; ++d) {
            cp.K[d] = c.K[d];
            cp.L[d] = c.box[d];
        }
        double V = c.box[0] * c.box[1] * c.box[2];
        cp.reference = ref ? 1 : 0;
        if (!ref) {
            cp.fac = c.p.coulomb_const / (M_PI * V);
            cp.pa2 = M_PI * M_PI / (c.alpha * c.alpha);
            cp.norm = 1.0;
        } else {
            cp.fac = 4.0 * M_PI / V;
            cp.pa2 = 1.0 / (4.0 * c.alpha * c.alpha);
            cp.norm = 1.0 / (double)ntot;
        }
        if (energy)
            k_fft_x_conv<R, true><<<gx, fth, sm, c.stream>>>(cg, K1, Kc, to_desc(c.plan[0]), twx, LP, cp, b0, b1, b2,
                                                            c.acc.p, c.status.p);
        else
            k_fft_x_conv<R, false><<<gx, fth, sm, c.stream>>>(cg, K1, Kc, to_desc(c.plan[0]), twx, LP, cp, b0, b1,
                                                             b2, c.acc.p, c.status.p);
    }
    // y inverse
    k_fft_y<R><<<gy, fth, smy, c.stream>>>(cg, K1, Kc, to_desc(c.plan[1]), twy, LPy, true);
    // z inverse (half complex -> real)
    {
        int LP = lines_per_block(K2, sizeof(C));
        size_t sm = sizeof(C) * ((size_t)K2 + 2 * (size_t)LP * K2);
        int nlines = K0 * K1;
        int nb = (nlines + 2 * LP - 1) / (2 * LP);
        k_fft_z_c2r<R><<<nb, fth, sm, c.stream>>>(cg, rg, nlines, K2, to_desc(c.plan[2]), twz, LP);
    }
    mark(c, "pme_fft_conv");
    if (!ref) {
        k_gather4<R><<<grid_blocks(c.n_slots, th), th, 0, c.stream>>>(c.n_slots, c.slot_atom.p, c.xyz.p, c.q.p, g, rg,
                                                                      c.f_slot.p, c.status.p);
    } else {
        c.forces_pme_ref.alloc(3 * (size_t)c.N);
        k_gather_ref5<<<grid_blocks(c.N, th), th, 0, c.stream>>>(c.N, c.xyz.p, c.q.p, g,
                                                                 reinterpret_cast<const double*>(rg),
                                                                 c.forces_pme_ref.p);
    }
    mark(c, "pme_gather");
    MDF_CUDA_TRY(cudaGetLastError());
    c.launches += 7;   // spread, z, y, x+conv, y, z, gather
}

void launch_pme(Ctx& c, bool energy)
{
    if (c.p.semantics == MDF_SEM_PHYSICAL && c.p.precision == MDF_PREC_MIXED) run_pme<float>(c, energy);
    else run_pme<double>(c, energy);
}

}  // namespace mdf
