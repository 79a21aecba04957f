// Nonbonded pair kernel and the FP64 excluded-pair / 1-4 kernels.
//
// Replaces, in REFERENCE semantics:
//   calculate_LJ_energy_pairlist     src/System/NonBondedEnergy.cpp:79-131
//   calculate_EE_energy (all pairs)  src/System/NonBondedEnergy.cpp:133-174
//   calculate_EE_energy_pairlist     :176-204, ..._with_cutoff :206-234
//   calculate_EE_ewald_direct_term   :236-305
//   calculate_forces_LJ_pairlist     src/System/NonBondedForces.cpp:92-155
//   calculate_forces_EE_pairlist     src/System/NonBondedForces.cpp:207-241
// and in PHYSICAL semantics the erfc real-space Ewald sum with switched LJ,
// the excluded-pair erf corrections and the scaled 1-4 pairs.
//
// Pair kernel layout: one warp per i cluster (8 atoms).  The warp walks the
// cluster's half list four j clusters at a time; lane = (jslot, ii) with
// jslot = lane/8 selecting the j cluster and ii = lane%8 the i atom.  The four
// j clusters are staged in shared memory; in step t lane (jslot, ii) computes
// the pair (ii, (ii+t)&7), so the eight lanes of a j slot touch eight different
// j atoms at every step and the j-force accumulators simply rotate one lane
// per step (3 shuffles per pair instead of a 3-level reduction).  i forces
// stay in registers for the whole list; j forces go to int64 fixed-point
// accumulators once per cluster pair.
#include <cmath>
#include <map>
#include <tuple>

#include "kargs.cuh"
#include "mdf_device.cuh"
#include "mdf_internal.cuh"
#include "nb_common.cuh"

namespace mdf {

template <typename R, int SEM, bool ENERGY>
__device__ __forceinline__ void pairs_dev(const PairArgs<R>& A)
{
    const int nlist = A.nlist;
    const ILRange* __restrict__ ilist = A.ilist;
    const PairEntry* __restrict__ plist = A.plist;
    const typename V4<R>::type* __restrict__ xq = A.xq;
    const int* __restrict__ stype = A.stype;
    const double4* __restrict__ center = A.center;
    const typename V2<R>::type* __restrict__ ljAB = A.ljAB;
    const int* __restrict__ ljvalid = A.ljvalid;
    const NBParams& P = A.P;
    unsigned long long* __restrict__ fslot = A.fslot;
    const int nslots = A.nslots;
    unsigned long long* __restrict__ acc = A.acc;
    unsigned long long* __restrict__ npairs = A.npairs;
    const int count = A.count;
    unsigned* st = A.st;
    using V4t = typename V4<R>::type;
    using V2t = typename V2<R>::type;
    __shared__ V4t sx[NB_WARPS][4][CLUSTER + 1];
    __shared__ int stj[NB_WARPS][4][CLUSTER];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = blockIdx.x * (blockDim.x >> 5) + wib;
    const int jslot = lane >> 3, ii = lane & 7;
    const unsigned FULL = 0xffffffffu;

    double e_lj = 0, e_dir = 0, e_all = 0, e_pl = 0, e_cut = 0;
    int npc = 0;
    R fix = 0, fiy = 0, fiz = 0;
    const R rc2 = (R)P.rc2, rsw = (R)P.rsw, inv_sw = (R)P.inv_sw, alpha = (R)P.alpha;
    const R two_a_spi = (R)(2.0 * P.alpha / 1.7724538509055160273);

    if (w < nlist) {
        const ILRange L = ilist[w];
        const int I = L.i;
        const V4t xi = xq[I * CLUSTER + ii];
        const int ti = stype[I * CLUSTER + ii];
        const double4 cI = center[I];
        const R qik = (R)P.kc * xi.w;
        for (int b = 0; b < L.count; b += 4) {
            const int e = b + jslot;
            const bool valid = e < L.count;
            PairEntry pe;
            if (valid) {
                pe = plist[L.start + e];
            } else {
                pe.j = I; pe.shift = 13; pe.mask = 0ull;
            }
            const int J = pe.j;
            sx[wib][jslot][ii] = xq[J * CLUSTER + ii];
            stj[wib][jslot][ii] = stype[J * CLUSTER + ii];
            const double4 cJ = center[J];
            int ssx, ssy, ssz;
            shift_decode(pe.shift, ssx, ssy, ssz);
            const R xix = xi.x + (R)(cI.x - cJ.x - ssx * P.box[0]);
            const R xiy = xi.y + (R)(cI.y - cJ.y - ssy * P.box[1]);
            const R xiz = xi.z + (R)(cI.z - cJ.z - ssz * P.box[2]);
            const unsigned long long mask = pe.mask;
            __syncwarp();
            R fjx = 0, fjy = 0, fjz = 0;
            R el_e = 0, ed_e = 0;   // this entry's energies in working precision; summed in FP64 below
            const int rot_src = (lane & ~7) | ((ii + 1) & 7);
#pragma unroll
            for (int t = 0; t < CLUSTER; ++t) {
                const int jj = (ii + t) & 7;
                const V4t xj = sx[wib][jslot][jj];
                const R dx = xix - xj.x, dy = xiy - xj.y, dz = xiz - xj.z;
                const R r2 = dx * dx + dy * dy + dz * dz;
                bool on = ((mask >> (ii * 8 + jj)) & 1ull) && r2 <= rc2;
                if (SEM == MDF_SEM_REFERENCE) on = on && r2 >= (R)1e-12;
                if (on) {
                    const int tj = stj[wib][jslot][jj];
                    const int tp = ti * P.ntp + tj;
                    R g = 0;
                    if (SEM == MDF_SEM_PHYSICAL) {
                        R rinv, r, rinv2;
                        if (sizeof(R) == 4) {
                            rinv = rsqrtf((float)r2);
                        } else {
                            rinv = (R)1 / sqrt((double)r2);
                        }
                        r = r2 * rinv;
                        rinv2 = rinv * rinv;
                        // Lennard-Jones 12-6, switched (or force-shifted)
                        const V2t ab = ljAB[tp];
                        const R rinv6 = rinv2 * rinv2 * rinv2;
                        R U = (ab.x * rinv6 - ab.y) * rinv6;
                        R G = ((R)12 * ab.x * rinv6 - (R)6 * ab.y) * rinv6 * rinv2;
                        if (P.use_switch) {
                            if (r > rsw) {
                                const R x = (r - rsw) * inv_sw, x2 = x * x, x3 = x2 * x;
                                const R S = (R)1 + x3 * ((R)-10 + x * ((R)15 - (R)6 * x));
                                const R dS = x2 * ((R)-30 + x * ((R)60 - (R)30 * x)) * inv_sw;
                                G = S * G - U * dS * rinv;
                                U = U * S;
                            }
                        } else {
                            const R uc = ab.x * (R)P.ucut_pow12 - ab.y * (R)P.ucut_pow6;
                            const R gc = ((R)12 * ab.x * (R)P.ucut_pow12 - (R)6 * ab.y * (R)P.ucut_pow6) / (R)P.rc2;
                            U = U - uc + (r - (R)P.rc) * (gc * (R)P.rc);
                            G = G - gc * (R)P.rc * rinv;
                        }
                        // erfc real-space Ewald
                        const R qq = qik * xj.w;
                        const R ar = alpha * r;
                        R erfcv, ex;
                        if (sizeof(R) == 4) {
                            ex = __expf(-(float)(ar * ar));
                            const float tt = __fdividef(1.0f, 1.0f + 0.3275911f * (float)ar);
                            erfcv = erfc_as(tt, (float)ex);
                        } else {
                            ex = exp(-(double)(ar * ar));
                            erfcv = erfc((double)ar);
                        }
                        const R ec = qq * erfcv * rinv;
                        g = G + (ec + qq * two_a_spi * ex) * rinv2;
                        if (ENERGY) {
                            el_e += U;
                            ed_e += ec;
                        }
                        ++npc;
                    } else {
                        // REFERENCE formulas, operation for operation
                        const double r2d = (double)r2, r = sqrt(r2d);
                        const double qq = (double)xi.w * (double)xj.w;
                        const double ecoul = (qq / r) * P.kc;
                        if (ENERGY) e_all += ecoul;
                        if (ljvalid[tp]) {
                            const V2t ab = ljAB[tp];
                            const double A = (double)ab.x, B = (double)ab.y;
                            const double i2 = 1.0 / r2d, i4 = i2 * i2, i6 = i4 * i2, i8 = i4 * i4, i12 = i6 * i6,
                                         i14 = i12 * i2;
                            double U = A * i12 - B * i6;
                            double G = 12.0 * A * i14 - 6.0 * B * i8;
                            if (P.use_switch) {
                                double S = 1.0, dS = 0.0;
                                if (r > P.rsw) {
                                    if (r >= P.rc) {
                                        S = 0.0;
                                    } else {
                                        const double x = (r - P.rsw) * P.inv_sw, x2 = x * x, x3 = x2 * x,
                                                     x4 = x2 * x2, x5 = x4 * x;
                                        S = 1.0 - 10.0 * x3 + 15.0 * x4 - 6.0 * x5;
                                        dS = (-30.0 * x2 + 60.0 * x3 - 30.0 * x4) * P.inv_sw;
                                    }
                                }
                                G = S * G - (U / r) * dS;
                                U = U * S;
                            } else {
                                const double rc2d = P.rc2, c2 = 1.0 / rc2d, c4 = c2 * c2, c6 = c4 * c2, c8 = c4 * c4,
                                             c12 = c6 * c6, c14 = c12 * c2;
                                const double ucut = A * c12 - B * c6, gcut = 12.0 * A * c14 - 6.0 * B * c8;
                                U = U - ucut + (r - P.rc) * (gcut * P.rc);
                                G = G - gcut * (P.rc / r);
                            }
                            g = (R)(G + ((qq / (r2d * r)) * P.kc));
                            if (ENERGY) {
                                e_lj += U;
                                e_pl += ecoul;
                                e_cut += (qq * P.kc) * (1.0 / r - 1.0 / P.rc);
                                e_dir += (qq / r) * erfc(P.alpha * r) * P.kc;
                            }
                            ++npc;
                        }
                    }
                    fix += g * dx; fiy += g * dy; fiz += g * dz;
                    fjx -= g * dx; fjy -= g * dy; fjz -= g * dz;
                }
                fjx = __shfl_sync(FULL, fjx, rot_src);
                fjy = __shfl_sync(FULL, fjy, rot_src);
                fjz = __shfl_sync(FULL, fjz, rot_src);
            }
            if (ENERGY && SEM == MDF_SEM_PHYSICAL) {
                e_lj += (double)el_e;
                e_dir += (double)ed_e;
            }
            if (valid && (fjx != (R)0 || fjy != (R)0 || fjz != (R)0)) {
                const int sl = J * CLUSTER + ii;
                fx_add(fslot + sl, fjx, FORCE_SCALE, st);
                fx_add(fslot + nslots + sl, fjy, FORCE_SCALE, st);
                fx_add(fslot + 2 * nslots + sl, fjz, FORCE_SCALE, st);
            }
            __syncwarp();
        }
        fix += __shfl_xor_sync(FULL, fix, 8); fix += __shfl_xor_sync(FULL, fix, 16);
        fiy += __shfl_xor_sync(FULL, fiy, 8); fiy += __shfl_xor_sync(FULL, fiy, 16);
        fiz += __shfl_xor_sync(FULL, fiz, 8); fiz += __shfl_xor_sync(FULL, fiz, 16);
        if (jslot == 0) {
            const int sl = I * CLUSTER + ii;
            fx_add(fslot + sl, fix, FORCE_SCALE, st);
            fx_add(fslot + nslots + sl, fiy, FORCE_SCALE, st);
            fx_add(fslot + 2 * nslots + sl, fiz, FORCE_SCALE, st);
        }
    }
    if (ENERGY) {
        if (SEM == MDF_SEM_PHYSICAL) {
            const double v[2] = {e_lj, e_dir};
            const int idx[2] = {MDF_E_VDW, MDF_E_EE_DIRECT};
            block_acc_fixed<2>(v, acc, idx, ENERGY_SCALE, st);
        } else {
            const double v[5] = {e_lj, e_all, e_pl, e_cut, e_dir};
            const int idx[5] = {MDF_E_VDW, MDF_E_EE, MDF_E_EE_PAIRLIST, MDF_E_EE_CUTOFF, MDF_E_EE_DIRECT};
            block_acc_fixed<5>(v, acc, idx, ENERGY_SCALE, st);
        }
    }
    if (count) {
        long long np = warp_sum_ll((long long)npc);
        if (lane == 0 && np) atomicAdd(npairs, (unsigned long long)np);
    }
}

template <typename R, int SEM, bool ENERGY>
__global__ void __launch_bounds__(NB_THREADS) k_pairs(PairArgs<R> A)
{
    pairs_dev<R, SEM, ENERGY>(A);
}

template <typename R, int SEM, bool ENERGY>
__global__ void __launch_bounds__(NB_THREADS) k_pairs_multi(const PairArgs<R>* __restrict__ As)
{
    const PairArgs<R>& A = As[blockIdx.z];
    if ((int)blockIdx.x >= A.gx) return;
    pairs_dev<R, SEM, ENERGY>(A);
}

// ------------------------------------------------- FP32 PHYSICAL pair kernel
// Periodic image offsets s*L of the 27 shift codes as an FP32 hi + lo pair.

// The mixed-precision production kernel (PHYSICAL semantics).  Same warp
// layout as k_pairs; differences that matter for speed and accuracy:
//  * cluster centres lie on a 2^-k grid and are exact in FP32, so the centre
//    difference is exact and the image offset enters as hi + lo: the pair
//    vector carries ~1e-6 A rounding, not the 1e-5 A of raw FP32 coordinates;
//  * the lane's row of the 8x8 mask is rotated once per entry so step t tests
//    bit t;
//  * the pair arithmetic is branch-free (inactive pairs are selected out);
//  * energies are summed in FP32 per entry and in FP64 across entries.

// The mixed-precision production kernel (PHYSICAL semantics).  Same warp
// layout as k_pairs; differences that matter for speed and accuracy:
//  * cluster centres lie on a 2^-k grid and are exact in FP32, so the centre
//    difference is exact and the image offset enters as hi + lo: the pair
//    vector carries ~1e-6 A rounding, not the 1e-5 A of raw FP32 coordinates;
//  * the lane's row of the 8x8 mask is rotated once per entry so step t tests
//    bit t;
//  * the pair arithmetic is branch-free: with the LJ switch an inactive pair
//    (masked, or beyond the cutoff) is evaluated at r^2 = 1e30, where every
//    term is exactly zero; with the force-shifted LJ its results are selected
//    out at the end (a masked pair at r = 0 only produces values that are
//    dropped);
//  * the LJ table holds (A, B, 12A, 6B) per type pair, in shared memory when it
//    fits (lj_smem), and the Gaussian uses 2^(kex r^2) on the SFU;
//  * each lane loads its entry of the next batch of four one batch ahead;
//  * energies are summed in FP32 per entry and in FP64 across entries.

// Static shared arrays of the pair bodies, declared once per kernel (each
// kernel inlines two forms of its body, see pairs_f32_body).
struct SmemF32W {
    float4 sx[NB_WARPS][4][2 * CLUSTER];
    int stj[NB_WARPS][4][2 * CLUSTER];
    float sh[27][6];
};
struct SmemF32H {
    float4 sxi[NB_WARPS][8];    // the item's four i atoms (I frame, charge x kc), twice
    int sti[NB_WARPS][8];       // their LJ table rows
    float sh[27][6];
};
struct SmemF64W {
    double4 sx[NB_WARPS][4][2 * CLUSTER];
    int stj[NB_WARPS][4][2 * CLUSTER];
    double sh[27][3];
};
struct SmemF64H {
    double4 sxi[NB_WARPS][8];
    int sti[NB_WARPS][8];
    double sh[27][3];
};

template <bool ENERGY, bool SWITCH, bool COUNT, bool LJS>
__device__ __forceinline__ void pairs_f32_body_t(SmemF32W& S,
    int nlist, const ILRange* __restrict__ ilist, const PairEntry* __restrict__ plist, const float4* __restrict__ xq,
    const int* __restrict__ stype, const float4* __restrict__ centerf, const float4* __restrict__ lj4, int ntp,
    int lj_smem, float kc, const PairConstF& Kin, const ShiftTable& shifts, unsigned long long* __restrict__ fslot,
    int nslots, unsigned long long* __restrict__ acc, unsigned long long* __restrict__ npairs,
    unsigned long long* __restrict__ next, int persist, unsigned* st)
{
    const PairConstF K = Kin;   // registers (the multi-system launch reads it from device memory)
    extern __shared__ float4 s_lj[];
    // each staged j cluster is stored twice in a row, so the atom a lane meets
    // at step t, (ii + t) mod 8, sits at the compile-time offset t from the
    // lane's own slot: no index arithmetic in the pair loop
    auto& sx = S.sx;
    auto& stj = S.stj;
    auto& sh = S.sh;
    for (int k = threadIdx.x; k < 27 * 6; k += blockDim.x) sh[k / 6][k % 6] = shifts.v[k / 6][k % 6];
    if (LJS)
        for (int k = threadIdx.x; k < ntp * ntp; k += blockDim.x) s_lj[k] = lj4[k];
    __syncthreads();
    const float4* __restrict__ ljt = LJS ? s_lj : lj4;
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int jslot = lane >> 3, ii = lane & 7;
    const unsigned FULL = 0xffffffffu;
    int npc = 0;
    // persist: persistent warps, each taking the next i cluster from the work
    // counter until the list is done (no SM idles behind a slow block or a
    // partial last wave); otherwise warp w takes i cluster w.  Energies go to
    // fixed point once per i cluster (a fixed-order FP64 sum), so they do not
    // depend on which warp took which cluster.
    for (int round = 0;; ++round) {
        int w = 0;
        if (persist) {
            if (lane == 0) w = (int)atomicAdd(next, 1ull);
            w = __shfl_sync(FULL, w, 0);
        } else {
            if (round) break;
            w = blockIdx.x * (blockDim.x >> 5) + wib;
        }
        if (w >= nlist) break;
        double e_lj = 0, e_dir = 0;
        float fix = 0.f, fiy = 0.f, fiz = 0.f;
        const ILRange L = ilist[w];
        const int I = L.i;
        const float4 xi = xq[I * CLUSTER + ii];
        const int trow = stype[I * CLUSTER + ii] * ntp * (int)sizeof(float4);   // byte offsets
        const float4 cI = centerf[I];
        const float qik = kc * xi.w;
        const float qik2 = qik * K.two_a_spi;
        const int rot_src = (lane & ~7) | ((ii + 1) & 7);
        // the lane's entry of the next batch is loaded one batch ahead
        PairEntry pn;
        if (jslot < L.count) {
            pn = plist[L.start + jslot];
        } else {
            pn.j = I; pn.shift = 13; pn.mask = 0ull;
        }
        for (int b = 0; b < L.count; b += 4) {
            const int e = b + jslot;
            const PairEntry pe = pn;
            if (e + 4 < L.count) {
                pn = plist[L.start + e + 4];
            } else {
                pn.j = I; pn.shift = 13; pn.mask = 0ull;
            }
            const int J = pe.j;
            const float4 xjj = xq[J * CLUSTER + ii];
            const int tjj = stype[J * CLUSTER + ii] * (int)sizeof(float4);
            sx[wib][jslot][ii] = xjj;
            sx[wib][jslot][ii + CLUSTER] = xjj;
            stj[wib][jslot][ii] = tjj;
            stj[wib][jslot][ii + CLUSTER] = tjj;
            const float4 cJ = centerf[J];
            const float* s6 = sh[pe.shift];
            const float xix = xi.x + (((cI.x - cJ.x) - s6[0]) - s6[3]);
            const float xiy = xi.y + (((cI.y - cJ.y) - s6[1]) - s6[4]);
            const float xiz = xi.z + (((cI.z - cJ.z) - s6[2]) - s6[5]);
            const unsigned rowm = (unsigned)(pe.mask >> (ii * 8)) & 0xffu;
            const unsigned rot = ((rowm >> ii) | (rowm << (8 - ii))) & 0xffu;
            __syncwarp();
            float fjx = 0.f, fjy = 0.f, fjz = 0.f, el = 0.f, ed = 0.f;
            const float4* __restrict__ sxl = &sx[wib][jslot][ii];
            const int* __restrict__ stl = &stj[wib][jslot][ii];
#pragma unroll
            for (int t = 0; t < CLUSTER; ++t) {
                const float4 xj = sxl[t];
                const float dx = xix - xj.x, dy = xiy - xj.y, dz = xiz - xj.z;
                const float r2r = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                const bool on = ((rot >> t) & 1u) && r2r <= K.rc2;
                // switched LJ: a slot outside the list or the cutoff takes r^2 = 1e30,
                // at which every term below is exactly zero (r^-6 underflows, the
                // Gaussian is 0 and the switch is 0 at x = 1), so no result needs a select
                const float r2 = SWITCH ? (on ? r2r : 1e30f) : r2r;
                const float rinv = rsqrt_ftz(r2);
                const float r = r2 * rinv, rinv2 = rinv * rinv, rinv6 = rinv2 * rinv2 * rinv2;
                const float4 ab = at_bytes(ljt, trow + stl[t]);      // A, B, 12A, 6B
                float U = rinv6 * fmaf(ab.x, rinv6, -ab.y);
                float G = (rinv6 * rinv2) * fmaf(ab.z, rinv6, -ab.w);
                if (SWITCH) {
                    const float x = __saturatef(fmaf(r, K.inv_sw, -K.rsw_inv)), x2 = x * x;
                    const float S = fmaf(x2 * x, fmaf(x, fmaf(x, -6.f, 15.f), -10.f), 1.f);
                    const float dSr = x2 * fmaf(x, fmaf(x, K.d30, K.d60), K.d30) * rinv;   // dS/dr / r
                    G = fmaf(S, G, -U * dSr);
                    U = U * S;
                } else {
                    const float uc = ab.x * K.uc12 - ab.y * K.uc6;
                    const float gc = (ab.z * K.uc12 - ab.w * K.uc6) / K.rc2f;
                    U = U - uc + (r - K.rcf) * (gc * K.rcf);
                    G = G - gc * K.rcf * rinv;
                }
                const float ex = ex2_approx(K.kex * r2);
                const float erfcv = erfc_as(rcp_ftz(fmaf(K.pa, r, 1.0f)), ex);
                const float ec = (qik * xj.w) * erfcv * rinv;
                float g = fmaf(fmaf(qik2 * xj.w, ex, ec), rinv2, G);
                if (!SWITCH) g = on ? g : 0.f;
                if (ENERGY) {
                    el += SWITCH ? U : (on ? U : 0.f);
                    ed += SWITCH ? ec : (on ? ec : 0.f);
                }
                if (COUNT) npc += on ? 1 : 0;
                fix = fmaf(g, dx, fix); fiy = fmaf(g, dy, fiy); fiz = fmaf(g, dz, fiz);
                fjx = fmaf(-g, dx, fjx); fjy = fmaf(-g, dy, fjy); fjz = fmaf(-g, dz, fjz);
                fjx = __shfl_sync(FULL, fjx, rot_src);
                fjy = __shfl_sync(FULL, fjy, rot_src);
                fjz = __shfl_sync(FULL, fjz, rot_src);
            }
            if (ENERGY) {
                e_lj += (double)el;
                e_dir += (double)ed;
            }
            if (e < L.count && (fjx != 0.f || fjy != 0.f || fjz != 0.f)) {
                const int sl = J * CLUSTER + ii;
                fx_add_force_f(fslot + sl, fjx, st);
                fx_add_force_f(fslot + nslots + sl, fjy, st);
                fx_add_force_f(fslot + 2 * nslots + sl, fjz, st);
            }
            __syncwarp();
        }
        fix += __shfl_xor_sync(FULL, fix, 8); fix += __shfl_xor_sync(FULL, fix, 16);
        fiy += __shfl_xor_sync(FULL, fiy, 8); fiy += __shfl_xor_sync(FULL, fiy, 16);
        fiz += __shfl_xor_sync(FULL, fiz, 8); fiz += __shfl_xor_sync(FULL, fiz, 16);
        if (jslot == 0) {
            const int sl = I * CLUSTER + ii;
            fx_add_force_f(fslot + sl, fix, st);
            fx_add_force_f(fslot + nslots + sl, fiy, st);
            fx_add_force_f(fslot + 2 * nslots + sl, fiz, st);
        }
        if (ENERGY) {
            const double s_lj = warp_sum(e_lj), s_dir = warp_sum(e_dir);
            if (lane == 0) {
                if (s_lj != 0.0) fx_add(acc + MDF_E_VDW, s_lj, ENERGY_SCALE, st);
                if (s_dir != 0.0) fx_add(acc + MDF_E_EE_DIRECT, s_dir, ENERGY_SCALE, st);
            }
        }
    }
    if (COUNT) {
        long long np = warp_sum_ll((long long)npc);
        if (lane == 0 && np) atomicAdd(npairs, (unsigned long long)np);
    }
}

// ---------------------------------------- half-cluster (4 x 8) FP32 kernel
// The same pair arithmetic over half entries: an item is (i cluster, half h)
// with the list of j clusters that have an atom pair within the cutoff of
// i atoms 4h..4h+3 (the half prune builds it, ILRange.pad = h).  At c1 half
// entries keep 45% of their atom pairs inside the cutoff against 39% for
// whole 8 x 8 entries.  Lane (e, jj) owns j atom jj of entry e of a batch of
// four; in step t it meets i atom 4h + ((jj + t) & 3), read from shared
// memory (stored twice so the step's atom sits at a compile-time offset), so
// the j force stays in the lane's registers and the i-force accumulators
// rotate one lane per step (the lane's i atom repeats every four lanes, so
// the same shuffle as the whole-entry kernel works).  After the item the
// eight partial sums of each i atom are reduced by three butterfly steps.
template <bool ENERGY, bool SWITCH, bool COUNT, bool LJS>
__device__ __forceinline__ void pairs_f32_half_body_t(SmemF32H& S, const PairF32Args& A)
{
    extern __shared__ float4 s_lj[];
    auto& sxi = S.sxi;
    auto& sti = S.sti;
    auto& sh = S.sh;
    const int nlist = A.nlist, ntp = A.ntp, nslots = A.nslots;
    const ILRange* __restrict__ ilist = A.ilist;
    const PairEntry* __restrict__ plist = A.plist;
    const float4* __restrict__ xq = A.xq;
    const int* __restrict__ stype = A.stype;
    const float4* __restrict__ centerf = A.centerf;
    unsigned long long* __restrict__ fslot = A.fslot;
    unsigned* st = A.st;
    const PairConstF K = A.K;
    for (int k = threadIdx.x; k < 27 * 6; k += blockDim.x) sh[k / 6][k % 6] = A.shifts.v[k / 6][k % 6];
    if (LJS)
        for (int k = threadIdx.x; k < ntp * ntp; k += blockDim.x) s_lj[k] = A.lj4[k];
    __syncthreads();
    const float4* __restrict__ ljt = LJS ? s_lj : A.lj4;
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int eslot = lane >> 3, jj = lane & 7, i4 = jj & 3;
    const unsigned FULL = 0xffffffffu;
    const int rot_src = (lane & ~7) | ((jj + 1) & 7);
    int npc = 0;
    for (int round = 0;; ++round) {
        int w = 0;
        if (A.persist) {
            if (lane == 0) w = (int)atomicAdd(A.next, 1ull);
            w = __shfl_sync(FULL, w, 0);
        } else {
            if (round) break;
            w = blockIdx.x * (blockDim.x >> 5) + wib;
        }
        if (w >= nlist) break;
        const ILRange L = ilist[w];
        const int I = L.i, h = L.pad;
        if (lane < 8) {
            float4 v = xq[I * CLUSTER + 4 * h + (lane & 3)];
            v.w *= A.kc;
            sxi[wib][lane] = v;
            sti[wib][lane] = stype[I * CLUSTER + 4 * h + (lane & 3)] * ntp * (int)sizeof(float4);   // bytes
        }
        __syncwarp();
        const float4 cI = centerf[I];
        const float4* __restrict__ sxl = &sxi[wib][i4];
        const int* __restrict__ stl = &sti[wib][i4];
        double e_lj = 0, e_dir = 0;
        float fix = 0.f, fiy = 0.f, fiz = 0.f;   // the i atom (jj + t) & 3 at step t
        // the lane's entry of the next batch is loaded one batch ahead
        PairEntry pn;
        if (eslot < L.count) {
            pn = plist[L.start + eslot];
        } else {
            pn.j = I; pn.shift = 13; pn.mask = 0ull;
        }
        for (int b = 0; b < L.count; b += 4) {
            const int e = b + eslot;
            const PairEntry pe = pn;
            if (e + 4 < L.count) {
                pn = plist[L.start + e + 4];
            } else {
                pn.j = I; pn.shift = 13; pn.mask = 0ull;
            }
            const int J = pe.j;
            const float4 xj = xq[J * CLUSTER + jj];
            const int tj = stype[J * CLUSTER + jj] * (int)sizeof(float4);
            const float4 cJ = centerf[J];
            const float* s6 = sh[pe.shift];
            // the j atom in I's frame: x_j - D, D = (c_I - c_J) - image offset
            const float pjx = xj.x - (((cI.x - cJ.x) - s6[0]) - s6[3]);
            const float pjy = xj.y - (((cI.y - cJ.y) - s6[1]) - s6[4]);
            const float pjz = xj.z - (((cI.z - cJ.z) - s6[2]) - s6[5]);
            // mask bits (4h + i) * 8 + jj, i = 0..3, rotated so step t tests bit t
            const unsigned long long mc = pe.mask >> (32 * h + jj);
            const unsigned nib = (unsigned)((mc & 1ull) | ((mc >> 7) & 2ull) | ((mc >> 14) & 4ull) | ((mc >> 21) & 8ull));
            const unsigned rot = ((nib >> i4) | (nib << (4 - i4))) & 0xfu;
            float fjx = 0.f, fjy = 0.f, fjz = 0.f, el = 0.f, ed = 0.f;
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const float4 xi = sxl[t];
                const float dx = xi.x - pjx, dy = xi.y - pjy, dz = xi.z - pjz;
                const float r2r = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                const bool on = ((rot >> t) & 1u) && r2r <= K.rc2;
                const float r2 = SWITCH ? (on ? r2r : 1e30f) : r2r;   // as in the whole-entry kernel
                const float rinv = rsqrt_ftz(r2);
                const float r = r2 * rinv, rinv2 = rinv * rinv, rinv6 = rinv2 * rinv2 * rinv2;
                const float4 ab = at_bytes(ljt, stl[t] + tj);      // A, B, 12A, 6B
                float U = rinv6 * fmaf(ab.x, rinv6, -ab.y);
                float G = (rinv6 * rinv2) * fmaf(ab.z, rinv6, -ab.w);
                if (SWITCH) {
                    const float x = __saturatef(fmaf(r, K.inv_sw, -K.rsw_inv)), x2 = x * x;
                    const float S = fmaf(x2 * x, fmaf(x, fmaf(x, -6.f, 15.f), -10.f), 1.f);
                    const float dSr = x2 * fmaf(x, fmaf(x, K.d30, K.d60), K.d30) * rinv;   // dS/dr / r
                    G = fmaf(S, G, -U * dSr);
                    U = U * S;
                } else {
                    const float uc = ab.x * K.uc12 - ab.y * K.uc6;
                    const float gc = (ab.z * K.uc12 - ab.w * K.uc6) / K.rc2f;
                    U = U - uc + (r - K.rcf) * (gc * K.rcf);
                    G = G - gc * K.rcf * rinv;
                }
                const float ex = ex2_approx(K.kex * r2);
                const float erfcv = erfc_as(rcp_ftz(fmaf(K.pa, r, 1.0f)), ex);
                const float qq = xi.w * xj.w;
                const float ec = qq * erfcv * rinv;
                float g = fmaf(fmaf(qq * K.two_a_spi, ex, ec), rinv2, G);
                if (!SWITCH) g = on ? g : 0.f;
                if (ENERGY) {
                    el += SWITCH ? U : (on ? U : 0.f);
                    ed += SWITCH ? ec : (on ? ec : 0.f);
                }
                if (COUNT) npc += on ? 1 : 0;
                fix = fmaf(g, dx, fix); fiy = fmaf(g, dy, fiy); fiz = fmaf(g, dz, fiz);
                fjx = fmaf(-g, dx, fjx); fjy = fmaf(-g, dy, fjy); fjz = fmaf(-g, dz, fjz);
                fix = __shfl_sync(FULL, fix, rot_src);
                fiy = __shfl_sync(FULL, fiy, rot_src);
                fiz = __shfl_sync(FULL, fiz, rot_src);
            }
            if (ENERGY) {
                e_lj += (double)el;
                e_dir += (double)ed;
            }
            if (e < L.count && (fjx != 0.f || fjy != 0.f || fjz != 0.f)) {
                const int sl = J * CLUSTER + jj;
                fx_add_force_f(fslot + sl, fjx, st);
                fx_add_force_f(fslot + nslots + sl, fjy, st);
                fx_add_force_f(fslot + 2 * nslots + sl, fjz, st);
            }
        }
        // lane jj holds a partial sum for i atom jj & 3: eight per atom
        fix += __shfl_xor_sync(FULL, fix, 4); fix += __shfl_xor_sync(FULL, fix, 8); fix += __shfl_xor_sync(FULL, fix, 16);
        fiy += __shfl_xor_sync(FULL, fiy, 4); fiy += __shfl_xor_sync(FULL, fiy, 8); fiy += __shfl_xor_sync(FULL, fiy, 16);
        fiz += __shfl_xor_sync(FULL, fiz, 4); fiz += __shfl_xor_sync(FULL, fiz, 8); fiz += __shfl_xor_sync(FULL, fiz, 16);
        if (lane < 4) {
            const int sl = I * CLUSTER + 4 * h + lane;
            fx_add_force_f(fslot + sl, fix, st);
            fx_add_force_f(fslot + nslots + sl, fiy, st);
            fx_add_force_f(fslot + 2 * nslots + sl, fiz, st);
        }
        if (ENERGY) {
            const double s_lj = warp_sum(e_lj), s_dir = warp_sum(e_dir);
            if (lane == 0) {
                if (s_lj != 0.0) fx_add(A.acc + MDF_E_VDW, s_lj, ENERGY_SCALE, st);
                if (s_dir != 0.0) fx_add(A.acc + MDF_E_EE_DIRECT, s_dir, ENERGY_SCALE, st);
            }
        }
        __syncwarp();   // the next item overwrites this warp's i atoms
    }
    if (COUNT) {
        long long np = warp_sum_ll((long long)npc);
        if (lane == 0 && np) atomicAdd(A.npairs, (unsigned long long)np);
    }
}

#define MDF_PF32_UNPACK(A)                                                                                       \
    A.nlist, A.ilist, A.plist, A.xq, A.stype, A.centerf, A.lj4, A.ntp, A.lj_smem, A.kc, A.K, A.shifts, A.fslot,      \
        A.nslots, A.acc, A.npairs, A.next, A.persist, A.st

// Every pair kernel holds two forms of its body: with the LJ table copied to
// shared memory (lj_smem, when it fits) and read from global memory.  Either
// way the table loads in the pair loop have a known address space (a generic
// pointer chosen at run time measured 5% slower at 100k atoms).
template <bool ENERGY, bool SWITCH, bool COUNT>
__device__ __forceinline__ void pairs_f32_body(const PairF32Args& A)
{
    __shared__ SmemF32W S;
    if (A.lj_smem) pairs_f32_body_t<ENERGY, SWITCH, COUNT, true>(S, MDF_PF32_UNPACK(A));
    else pairs_f32_body_t<ENERGY, SWITCH, COUNT, false>(S, MDF_PF32_UNPACK(A));
}

template <bool ENERGY, bool SWITCH, bool COUNT>
__device__ __forceinline__ void pairs_f32_half_body(const PairF32Args& A)
{
    __shared__ SmemF32H S;
    if (A.lj_smem) pairs_f32_half_body_t<ENERGY, SWITCH, COUNT, true>(S, A);
    else pairs_f32_half_body_t<ENERGY, SWITCH, COUNT, false>(S, A);
}

// With energies: up to 80 registers, three blocks per SM (left to itself the
// compiler picks 64 and spills, which measured 1-2% slower).
template <bool SWITCH, bool COUNT>
__global__ void __launch_bounds__(NB_THREADS, 3) k_pairs_f32(PairF32Args A)
{
    pairs_f32_body<true, SWITCH, COUNT>(A);
}

// Forces only (every dynamics step but the last of a chunk): 64 registers
// with no spills, four blocks per SM (+4% dynamics steps/s).
template <bool SWITCH, bool COUNT>
__global__ void __launch_bounds__(NB_THREADS, 4) k_pairs_f32_force(PairF32Args A)
{
    pairs_f32_body<false, SWITCH, COUNT>(A);
}

// The half-entry (4 x 8) forms, same register budgets.
template <bool SWITCH, bool COUNT>
__global__ void __launch_bounds__(NB_THREADS) k_pairs_f32_half(PairF32Args A)
{
    pairs_f32_half_body<true, SWITCH, COUNT>(A);
}

template <bool SWITCH, bool COUNT>
__global__ void __launch_bounds__(NB_THREADS, 4) k_pairs_f32_half_force(PairF32Args A)
{
    pairs_f32_half_body<false, SWITCH, COUNT>(A);
}

// The many-system kernels hold one form of the body: LJS is the batch's
// choice for all its systems (shared memory when every system's table fits).
template <bool SWITCH, bool LJS>
__global__ void __launch_bounds__(NB_THREADS) k_pairs_f32_half_multi(const PairF32Args* __restrict__ As)
{
    __shared__ SmemF32H S;
    const PairF32Args& A = As[blockIdx.z];
    if ((int)blockIdx.x >= A.gx) return;
    pairs_f32_half_body_t<true, SWITCH, false, LJS>(S, A);
}

template <bool SWITCH, bool LJS>
__global__ void __launch_bounds__(NB_THREADS, 4) k_pairs_f32_half_force_multi(const PairF32Args* __restrict__ As)
{
    __shared__ SmemF32H S;
    const PairF32Args& A = As[blockIdx.z];
    if ((int)blockIdx.x >= A.gx) return;
    pairs_f32_half_body_t<false, SWITCH, false, LJS>(S, A);
}

// Many systems in one launch (blockIdx.z = system), with the same register
// budgets as the one-system kernels above.
template <bool SWITCH, bool LJS>
__global__ void __launch_bounds__(NB_THREADS, 3) k_pairs_f32_multi(const PairF32Args* __restrict__ As)
{
    __shared__ SmemF32W S;
    const PairF32Args& A = As[blockIdx.z];
    if ((int)blockIdx.x >= A.gx) return;
    pairs_f32_body_t<true, SWITCH, false, LJS>(S, MDF_PF32_UNPACK(A));
}

template <bool SWITCH, bool LJS>
__global__ void __launch_bounds__(NB_THREADS, 4) k_pairs_f32_force_multi(const PairF32Args* __restrict__ As)
{
    __shared__ SmemF32W S;
    const PairF32Args& A = As[blockIdx.z];
    if ((int)blockIdx.x >= A.gx) return;
    pairs_f32_body_t<false, SWITCH, false, LJS>(S, MDF_PF32_UNPACK(A));
}
#undef MDF_PF32_UNPACK

// ------------------------------------------------ FP64 PHYSICAL pair kernel
// The FP32 kernel's structure in double precision: the same warp layout and
// lane rotation, j clusters staged twice in shared memory (compile-time
// offsets), the lane's mask row rotated once per entry, branch-free
// selection of the inactive pairs, an (A, B, 12A, 6B) table in shared memory
// and constants folded on the host.  The arithmetic differs only where
// precision does: FP64 rsqrt, exp and erfc (the CUDA math library) instead of
// the SFU forms and the A&S erfc, and FP64 image offsets from FP64 centres.
template <bool ENERGY, bool SWITCH, bool COUNT, bool LJS>
__device__ __forceinline__ void pairs_f64_body_t(SmemF64W& S, const PairF64Args& A)
{
    extern __shared__ double4 s_lj_d[];
    auto& sx = S.sx;
    auto& stj = S.stj;
    auto& sh = S.sh;
    const int nlist = A.nlist;
    const ILRange* __restrict__ ilist = A.ilist;
    const PairEntry* __restrict__ plist = A.plist;
    const double4* __restrict__ xq = A.xq;
    const int* __restrict__ stype = A.stype;
    const double4* __restrict__ center = A.center;
    const int ntp = A.ntp;
    unsigned long long* __restrict__ fslot = A.fslot;
    const int nslots = A.nslots;
    unsigned* st = A.st;
    const PairConstD K = A.K;
    for (int k = threadIdx.x; k < 27 * 3; k += blockDim.x) sh[k / 3][k % 3] = A.shifts.v[k / 3][k % 3];
    if (LJS)
        for (int k = threadIdx.x; k < ntp * ntp; k += blockDim.x) s_lj_d[k] = A.lj4[k];
    __syncthreads();
    const double4* __restrict__ ljt = LJS ? s_lj_d : A.lj4;
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int jslot = lane >> 3, ii = lane & 7;
    const unsigned FULL = 0xffffffffu;
    int npc = 0;
    // warp schedule and per-cluster energies as in the FP32 kernel
    for (int round = 0;; ++round) {
        int w = 0;
        if (A.persist) {
            if (lane == 0) w = (int)atomicAdd(A.next, 1ull);
            w = __shfl_sync(FULL, w, 0);
        } else {
            if (round) break;
            w = blockIdx.x * (blockDim.x >> 5) + wib;
        }
        if (w >= nlist) break;
        double e_lj = 0, e_dir = 0;
        double fix = 0, fiy = 0, fiz = 0;
        const ILRange L = ilist[w];
        const int I = L.i;
        const double4 xi = xq[I * CLUSTER + ii];
        const int trow = stype[I * CLUSTER + ii] * ntp * (int)sizeof(double4);   // byte offsets
        const double4 cI = center[I];
        const double qik = A.kc * xi.w;
        const double qik2 = qik * K.two_a_spi;
        const int rot_src = (lane & ~7) | ((ii + 1) & 7);
        // the lane's entry of the next batch is loaded one batch ahead
        PairEntry pn;
        if (jslot < L.count) {
            pn = plist[L.start + jslot];
        } else {
            pn.j = I; pn.shift = 13; pn.mask = 0ull;
        }
        for (int b = 0; b < L.count; b += 4) {
            const int e = b + jslot;
            const PairEntry pe = pn;
            if (e + 4 < L.count) {
                pn = plist[L.start + e + 4];
            } else {
                pn.j = I; pn.shift = 13; pn.mask = 0ull;
            }
            const int J = pe.j;
            const double4 xjj = xq[J * CLUSTER + ii];
            const int tjj = stype[J * CLUSTER + ii] * (int)sizeof(double4);
            sx[wib][jslot][ii] = xjj;
            sx[wib][jslot][ii + CLUSTER] = xjj;
            stj[wib][jslot][ii] = tjj;
            stj[wib][jslot][ii + CLUSTER] = tjj;
            const double4 cJ = center[J];
            const double* s3 = sh[pe.shift];
            const double xix = xi.x + ((cI.x - cJ.x) - s3[0]);
            const double xiy = xi.y + ((cI.y - cJ.y) - s3[1]);
            const double xiz = xi.z + ((cI.z - cJ.z) - s3[2]);
            const unsigned rowm = (unsigned)(pe.mask >> (ii * 8)) & 0xffu;
            const unsigned rot = ((rowm >> ii) | (rowm << (8 - ii))) & 0xffu;
            __syncwarp();
            double fjx = 0, fjy = 0, fjz = 0, el = 0, ed = 0;
            const double4* __restrict__ sxl = &sx[wib][jslot][ii];
            const int* __restrict__ stl = &stj[wib][jslot][ii];
#pragma unroll
            for (int t = 0; t < CLUSTER; ++t) {
                const double4 xj = sxl[t];
                const double dx = xix - xj.x, dy = xiy - xj.y, dz = xiz - xj.z;
                const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
                const bool on = ((rot >> t) & 1u) && r2 <= K.rc2;
                const double rinv = rsqrt(r2);
                const double r = r2 * rinv, rinv2 = rinv * rinv, rinv6 = rinv2 * rinv2 * rinv2;
                const double4 ab = at_bytes(ljt, trow + stl[t]);      // A, B, 12A, 6B
                double U = rinv6 * fma(ab.x, rinv6, -ab.y);
                double G = (rinv6 * rinv2) * fma(ab.z, rinv6, -ab.w);
                if (SWITCH) {
                    const double x = fmax(0.0, fma(r, K.inv_sw, -K.rsw_inv)), x2 = x * x;
                    const double S = fma(x2 * x, fma(x, fma(x, -6.0, 15.0), -10.0), 1.0);
                    const double dSr = x2 * fma(x, fma(x, K.d30, K.d60), K.d30) * rinv;   // dS/dr / r
                    G = fma(S, G, -U * dSr);
                    U = U * S;
                } else {
                    const double uc = ab.x * K.uc12 - ab.y * K.uc6;
                    const double gc = (ab.z * K.uc12 - ab.w * K.uc6) / K.rc2;
                    U = U - uc + (r - K.rc) * (gc * K.rc);
                    G = G - gc * K.rc * rinv;
                }
                const double ar = K.alpha * r;
                const double ex = exp(-ar * ar);
                const double ec = (qik * xj.w) * erfc(ar) * rinv;
                double g = fma(fma(qik2 * xj.w, ex, ec), rinv2, G);
                g = on ? g : 0.0;
                if (ENERGY) {
                    el += on ? U : 0.0;
                    ed += on ? ec : 0.0;
                }
                if (COUNT) npc += on ? 1 : 0;
                fix = fma(g, dx, fix); fiy = fma(g, dy, fiy); fiz = fma(g, dz, fiz);
                fjx = fma(-g, dx, fjx); fjy = fma(-g, dy, fjy); fjz = fma(-g, dz, fjz);
                fjx = __shfl_sync(FULL, fjx, rot_src);
                fjy = __shfl_sync(FULL, fjy, rot_src);
                fjz = __shfl_sync(FULL, fjz, rot_src);
            }
            if (ENERGY) {
                e_lj += el;
                e_dir += ed;
            }
            if (e < L.count && (fjx != 0.0 || fjy != 0.0 || fjz != 0.0)) {
                const int sl = J * CLUSTER + ii;
                fx_add(fslot + sl, fjx, FORCE_SCALE, st);
                fx_add(fslot + nslots + sl, fjy, FORCE_SCALE, st);
                fx_add(fslot + 2 * nslots + sl, fjz, FORCE_SCALE, st);
            }
            __syncwarp();
        }
        fix += __shfl_xor_sync(FULL, fix, 8); fix += __shfl_xor_sync(FULL, fix, 16);
        fiy += __shfl_xor_sync(FULL, fiy, 8); fiy += __shfl_xor_sync(FULL, fiy, 16);
        fiz += __shfl_xor_sync(FULL, fiz, 8); fiz += __shfl_xor_sync(FULL, fiz, 16);
        if (jslot == 0) {
            const int sl = I * CLUSTER + ii;
            fx_add(fslot + sl, fix, FORCE_SCALE, st);
            fx_add(fslot + nslots + sl, fiy, FORCE_SCALE, st);
            fx_add(fslot + 2 * nslots + sl, fiz, FORCE_SCALE, st);
        }
        if (ENERGY) {
            const double s_lj = warp_sum(e_lj), s_dir = warp_sum(e_dir);
            if (lane == 0) {
                if (s_lj != 0.0) fx_add(A.acc + MDF_E_VDW, s_lj, ENERGY_SCALE, st);
                if (s_dir != 0.0) fx_add(A.acc + MDF_E_EE_DIRECT, s_dir, ENERGY_SCALE, st);
            }
        }
    }
    if (COUNT) {
        long long np = warp_sum_ll((long long)npc);
        if (lane == 0 && np) atomicAdd(A.npairs, (unsigned long long)np);
    }
}

// The half-entry (4 x 8) layout in FP64: the FP32 half kernel's structure
// with the FP64 kernel's arithmetic.
template <bool ENERGY, bool SWITCH, bool COUNT, bool LJS>
__device__ __forceinline__ void pairs_f64_half_body_t(SmemF64H& S, const PairF64Args& A)
{
    extern __shared__ double4 s_lj_d[];
    auto& sxi = S.sxi;
    auto& sti = S.sti;
    auto& sh = S.sh;
    const int nlist = A.nlist, ntp = A.ntp, nslots = A.nslots;
    const ILRange* __restrict__ ilist = A.ilist;
    const PairEntry* __restrict__ plist = A.plist;
    const double4* __restrict__ xq = A.xq;
    const int* __restrict__ stype = A.stype;
    const double4* __restrict__ center = A.center;
    unsigned long long* __restrict__ fslot = A.fslot;
    unsigned* st = A.st;
    const PairConstD K = A.K;
    for (int k = threadIdx.x; k < 27 * 3; k += blockDim.x) sh[k / 3][k % 3] = A.shifts.v[k / 3][k % 3];
    if (LJS)
        for (int k = threadIdx.x; k < ntp * ntp; k += blockDim.x) s_lj_d[k] = A.lj4[k];
    __syncthreads();
    const double4* __restrict__ ljt = LJS ? s_lj_d : A.lj4;
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int eslot = lane >> 3, jj = lane & 7, i4 = jj & 3;
    const unsigned FULL = 0xffffffffu;
    const int rot_src = (lane & ~7) | ((jj + 1) & 7);
    int npc = 0;
    for (int round = 0;; ++round) {
        int w = 0;
        if (A.persist) {
            if (lane == 0) w = (int)atomicAdd(A.next, 1ull);
            w = __shfl_sync(FULL, w, 0);
        } else {
            if (round) break;
            w = blockIdx.x * (blockDim.x >> 5) + wib;
        }
        if (w >= nlist) break;
        const ILRange L = ilist[w];
        const int I = L.i, h = L.pad;
        if (lane < 8) {
            double4 v = xq[I * CLUSTER + 4 * h + (lane & 3)];
            v.w *= A.kc;
            sxi[wib][lane] = v;
            sti[wib][lane] = stype[I * CLUSTER + 4 * h + (lane & 3)] * ntp * (int)sizeof(double4);   // bytes
        }
        __syncwarp();
        const double4 cI = center[I];
        const double4* __restrict__ sxl = &sxi[wib][i4];
        const int* __restrict__ stl = &sti[wib][i4];
        double e_lj = 0, e_dir = 0;
        double fix = 0, fiy = 0, fiz = 0;
        // the lane's entry of the next batch is loaded one batch ahead
        PairEntry pn;
        if (eslot < L.count) {
            pn = plist[L.start + eslot];
        } else {
            pn.j = I; pn.shift = 13; pn.mask = 0ull;
        }
        for (int b = 0; b < L.count; b += 4) {
            const int e = b + eslot;
            const PairEntry pe = pn;
            if (e + 4 < L.count) {
                pn = plist[L.start + e + 4];
            } else {
                pn.j = I; pn.shift = 13; pn.mask = 0ull;
            }
            const int J = pe.j;
            const double4 xj = xq[J * CLUSTER + jj];
            const int tj = stype[J * CLUSTER + jj] * (int)sizeof(double4);
            const double4 cJ = center[J];
            const double* s3 = sh[pe.shift];
            const double pjx = xj.x - ((cI.x - cJ.x) - s3[0]);
            const double pjy = xj.y - ((cI.y - cJ.y) - s3[1]);
            const double pjz = xj.z - ((cI.z - cJ.z) - s3[2]);
            const unsigned long long mc = pe.mask >> (32 * h + jj);
            const unsigned nib = (unsigned)((mc & 1ull) | ((mc >> 7) & 2ull) | ((mc >> 14) & 4ull) | ((mc >> 21) & 8ull));
            const unsigned rot = ((nib >> i4) | (nib << (4 - i4))) & 0xfu;
            double fjx = 0, fjy = 0, fjz = 0, el = 0, ed = 0;
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const double4 xi = sxl[t];
                const double dx = xi.x - pjx, dy = xi.y - pjy, dz = xi.z - pjz;
                const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
                const bool on = ((rot >> t) & 1u) && r2 <= K.rc2;
                const double rinv = rsqrt(r2);
                const double r = r2 * rinv, rinv2 = rinv * rinv, rinv6 = rinv2 * rinv2 * rinv2;
                const double4 ab = at_bytes(ljt, stl[t] + tj);      // A, B, 12A, 6B
                double U = rinv6 * fma(ab.x, rinv6, -ab.y);
                double G = (rinv6 * rinv2) * fma(ab.z, rinv6, -ab.w);
                if (SWITCH) {
                    const double x = fmax(0.0, fma(r, K.inv_sw, -K.rsw_inv)), x2 = x * x;
                    const double S = fma(x2 * x, fma(x, fma(x, -6.0, 15.0), -10.0), 1.0);
                    const double dSr = x2 * fma(x, fma(x, K.d30, K.d60), K.d30) * rinv;   // dS/dr / r
                    G = fma(S, G, -U * dSr);
                    U = U * S;
                } else {
                    const double uc = ab.x * K.uc12 - ab.y * K.uc6;
                    const double gc = (ab.z * K.uc12 - ab.w * K.uc6) / K.rc2;
                    U = U - uc + (r - K.rc) * (gc * K.rc);
                    G = G - gc * K.rc * rinv;
                }
                const double ar = K.alpha * r;
                const double ex = exp(-ar * ar);
                const double qq = xi.w * xj.w;
                const double ec = qq * erfc(ar) * rinv;
                double g = fma(fma(qq * K.two_a_spi, ex, ec), rinv2, G);
                g = on ? g : 0.0;
                if (ENERGY) {
                    el += on ? U : 0.0;
                    ed += on ? ec : 0.0;
                }
                if (COUNT) npc += on ? 1 : 0;
                fix = fma(g, dx, fix); fiy = fma(g, dy, fiy); fiz = fma(g, dz, fiz);
                fjx = fma(-g, dx, fjx); fjy = fma(-g, dy, fjy); fjz = fma(-g, dz, fjz);
                fix = __shfl_sync(FULL, fix, rot_src);
                fiy = __shfl_sync(FULL, fiy, rot_src);
                fiz = __shfl_sync(FULL, fiz, rot_src);
            }
            if (ENERGY) {
                e_lj += el;
                e_dir += ed;
            }
            if (e < L.count && (fjx != 0.0 || fjy != 0.0 || fjz != 0.0)) {
                const int sl = J * CLUSTER + jj;
                fx_add(fslot + sl, fjx, FORCE_SCALE, st);
                fx_add(fslot + nslots + sl, fjy, FORCE_SCALE, st);
                fx_add(fslot + 2 * nslots + sl, fjz, FORCE_SCALE, st);
            }
        }
        fix += __shfl_xor_sync(FULL, fix, 4); fix += __shfl_xor_sync(FULL, fix, 8); fix += __shfl_xor_sync(FULL, fix, 16);
        fiy += __shfl_xor_sync(FULL, fiy, 4); fiy += __shfl_xor_sync(FULL, fiy, 8); fiy += __shfl_xor_sync(FULL, fiy, 16);
        fiz += __shfl_xor_sync(FULL, fiz, 4); fiz += __shfl_xor_sync(FULL, fiz, 8); fiz += __shfl_xor_sync(FULL, fiz, 16);
        if (lane < 4) {
            const int sl = I * CLUSTER + 4 * h + lane;
            fx_add(fslot + sl, fix, FORCE_SCALE, st);
            fx_add(fslot + nslots + sl, fiy, FORCE_SCALE, st);
            fx_add(fslot + 2 * nslots + sl, fiz, FORCE_SCALE, st);
        }
        if (ENERGY) {
            const double s_lj = warp_sum(e_lj), s_dir = warp_sum(e_dir);
            if (lane == 0) {
                if (s_lj != 0.0) fx_add(A.acc + MDF_E_VDW, s_lj, ENERGY_SCALE, st);
                if (s_dir != 0.0) fx_add(A.acc + MDF_E_EE_DIRECT, s_dir, ENERGY_SCALE, st);
            }
        }
        __syncwarp();
    }
    if (COUNT) {
        long long np = warp_sum_ll((long long)npc);
        if (lane == 0 && np) atomicAdd(A.npairs, (unsigned long long)np);
    }
}

template <bool ENERGY, bool SWITCH, bool COUNT>
__device__ __forceinline__ void pairs_f64_body(const PairF64Args& A)
{
    __shared__ SmemF64W S;
    if (A.lj_smem) pairs_f64_body_t<ENERGY, SWITCH, COUNT, true>(S, A);
    else pairs_f64_body_t<ENERGY, SWITCH, COUNT, false>(S, A);
}

template <bool ENERGY, bool SWITCH, bool COUNT>
__device__ __forceinline__ void pairs_f64_half_body(const PairF64Args& A)
{
    __shared__ SmemF64H S;
    if (A.lj_smem) pairs_f64_half_body_t<ENERGY, SWITCH, COUNT, true>(S, A);
    else pairs_f64_half_body_t<ENERGY, SWITCH, COUNT, false>(S, A);
}

template <bool ENERGY, bool SWITCH, bool COUNT>
__global__ void __launch_bounds__(NB_THREADS, 2) k_pairs_f64_half(PairF64Args A)
{
    pairs_f64_half_body<ENERGY, SWITCH, COUNT>(A);
}

template <bool ENERGY, bool SWITCH, bool LJS>
__global__ void __launch_bounds__(NB_THREADS) k_pairs_f64_half_multi(const PairF64Args* __restrict__ As)
{
    __shared__ SmemF64H S;
    const PairF64Args& A = As[blockIdx.z];
    if ((int)blockIdx.x >= A.gx) return;
    pairs_f64_half_body_t<ENERGY, SWITCH, false, LJS>(S, A);
}

template <bool ENERGY, bool SWITCH, bool COUNT>
__global__ void __launch_bounds__(NB_THREADS) k_pairs_f64(PairF64Args A)
{
    pairs_f64_body<ENERGY, SWITCH, COUNT>(A);
}

template <bool ENERGY, bool SWITCH, bool LJS>
__global__ void __launch_bounds__(NB_THREADS) k_pairs_f64_multi(const PairF64Args* __restrict__ As)
{
    __shared__ SmemF64W S;
    const PairF64Args& A = As[blockIdx.z];
    if ((int)blockIdx.x >= A.gx) return;
    pairs_f64_body_t<ENERGY, SWITCH, false, LJS>(S, A);
}

// --------------------------------------------------------------- FP64 pairs
__device__ __forceinline__ void pair_vec(const double* __restrict__ xyz, int a, int b, const NBParams& P,
                                         double d[3])
{
    d[0] = min_image(xyz[3 * a] - xyz[3 * b], P.box[0]);
    d[1] = min_image(xyz[3 * a + 1] - xyz[3 * b + 1], P.box[1]);
    d[2] = min_image(xyz[3 * a + 2] - xyz[3 * b + 2], P.box[2]);
}

__device__ __forceinline__ void add_pair_force(unsigned long long* f, int N, int a, int b, double g, const double d[3],
                                               unsigned* st)
{
    for (int k = 0; k < 3; ++k) {
        fx_add(f + k * N + a, g * d[k], FORCE_SCALE, st);
        fx_add(f + k * N + b, -g * d[k], FORCE_SCALE, st);
    }
}

// Excluded pairs.  PHYSICAL: -k q q erf(alpha r)/r with its force (every
// excluded pair, min image, no cutoff).  REFERENCE: the same energy for
// excluded pairs that are not 1-4 (src/System/NonBondedEnergy.cpp:271-304),
// no force.
template <int SEM, bool ENERGY>
__device__ __forceinline__ void exclusions_dev(const ExclArgs& A)
{
    const int n = A.n;
    const int* __restrict__ pairs = A.pairs;
    const int* __restrict__ is14 = A.is14;
    const double* __restrict__ xyz = A.xyz;
    const double* __restrict__ q = A.q;
    const NBParams& P = A.P;
    const int N = A.N;
    unsigned long long* __restrict__ fatom = A.fatom;
    unsigned long long* __restrict__ acc = A.acc;
    unsigned* st = A.st;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (k < n && !(SEM == MDF_SEM_REFERENCE && is14[k])) {
        int a = pairs[2 * k], b = pairs[2 * k + 1];
        double d[3];
        pair_vec(xyz, a, b, P, d);
        double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2], r = sqrt(r2);
        if (SEM == MDF_SEM_PHYSICAL) {
            double qq = q[a] * q[b] * P.kc, ar = P.alpha * r;
            e = -qq * erf(ar) / r;
            double g = (e + qq * (2.0 * P.alpha / 1.7724538509055160273) * exp(-ar * ar)) / r2;
            add_pair_force(fatom, N, a, b, g, d, st);
        } else {
            e = -P.kc * (q[a] * q[b] / r) * erf(P.alpha * r);
        }
    }
    if (ENERGY) {
        const double v[1] = {e};
        const int idx[1] = {SEM == MDF_SEM_PHYSICAL ? MDF_E_EE_EXCL : MDF_E_EE_DIRECT};
        block_acc_fixed<1>(v, acc, idx, ENERGY_SCALE, st);
    }
}

// 1-4 pairs.  PHYSICAL: k q q / (scee r) + (A14/r^12 - B14/r^6) / scnb.
// REFERENCE: the reference's is14 branches of the list loops (A14/B14 with the
// switch, Coulomb / scee, and CalculateEnergyEwaldDirectTerm_14's erf(r)).
template <int SEM, bool ENERGY>
__global__ void k_exclusions(ExclArgs A)
{
    exclusions_dev<SEM, ENERGY>(A);
}

template <int SEM, bool ENERGY>
__global__ void k_exclusions_multi(const ExclArgs* __restrict__ As)
{
    const ExclArgs& A = As[blockIdx.z];
    if ((int)blockIdx.x >= A.gx) return;
    exclusions_dev<SEM, ENERGY>(A);
}

template <int SEM, bool ENERGY>
__device__ __forceinline__ void pairs14_dev(const Pair14Args& A)
{
    const int n = A.n;
    const int* __restrict__ pairs = A.pairs;
    const double2* __restrict__ scale = A.scale;
    const double* __restrict__ xyz = A.xyz;
    const double* __restrict__ q = A.q;
    const int* __restrict__ type = A.type;
    const double2* __restrict__ lj14 = A.lj14;
    const int* __restrict__ ljvalid = A.ljvalid;
    const NBParams& P = A.P;
    const int N = A.N;
    unsigned long long* __restrict__ fatom = A.fatom;
    unsigned long long* __restrict__ acc = A.acc;
    unsigned* st = A.st;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    double ev = 0, ec = 0, eall = 0, epl = 0, ecut = 0, edir = 0;
    if (k < n) {
        int a = pairs[2 * k], b = pairs[2 * k + 1];
        double d[3];
        pair_vec(xyz, a, b, P, d);
        double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2], r = sqrt(r2);
        double2 sc = scale[k];
        int tp = type[a] * P.ntp + type[b];
        double2 ab = lj14[tp];
        double i2 = 1.0 / r2, i4 = i2 * i2, i6 = i4 * i2, i8 = i4 * i4, i12 = i6 * i6, i14 = i12 * i2;
        if (SEM == MDF_SEM_PHYSICAL) {
            double qq = q[a] * q[b] * P.kc / sc.x;
            ec = qq / r;
            double g = ec / r2;
            if (ljvalid[tp]) {
                ev = (ab.x * i12 - ab.y * i6) / sc.y;
                g += (12.0 * ab.x * i14 - 6.0 * ab.y * i8) / sc.y;
            }
            add_pair_force(fatom, N, a, b, g, d, st);
        } else {
            double qq = q[a] * q[b];
            double scee = sc.x;
            if (r2 <= P.rc2 && r2 >= 1e-12) eall = (1.0 / scee) * ((qq / r) * P.kc);
            bool in_list = r2 <= P.rlist2 && r2 > 1e-12 && ljvalid[tp];
            if (in_list && r2 <= P.rc2 && r2 >= 1e-12) {
                double U = ab.x * i12 - ab.y * i6, G = 12.0 * ab.x * i14 - 6.0 * ab.y * i8;
                if (P.use_switch) {
                    double S = 1.0, dS = 0.0;
                    if (r > P.rsw) {
                        if (r >= P.rc) S = 0.0;
                        else {
                            double x = (r - P.rsw) * P.inv_sw, x2 = x * x, x3 = x2 * x, x4 = x2 * x2, x5 = x4 * x;
                            S = 1.0 - 10.0 * x3 + 15.0 * x4 - 6.0 * x5;
                            dS = (-30.0 * x2 + 60.0 * x3 - 30.0 * x4) * P.inv_sw;
                        }
                    }
                    G = S * G - (U / r) * dS;
                    U = U * S;
                } else {
                    double c2 = 1.0 / P.rc2, c4 = c2 * c2, c6 = c4 * c2, c8 = c4 * c4, c12 = c6 * c6, c14 = c12 * c2;
                    double ucut = ab.x * c12 - ab.y * c6, gcut = 12.0 * ab.x * c14 - 6.0 * ab.y * c8;
                    U = U - ucut + (r - P.rc) * (gcut * P.rc);
                    G = G - gcut * (P.rc / r);
                }
                ev = U;
                epl = (1.0 / scee) * ((qq / r) * P.kc);
                ecut = (1.0 / scee) * (qq * P.kc) * (1.0 / r - 1.0 / P.rc);
                edir = ((1.0 / (scee * r)) - (erf(r) / r)) * (qq * P.kc);
                double g = G + (1.0 / scee) * ((qq / (r2 * r)) * P.kc);
                add_pair_force(fatom, N, a, b, g, d, st);
            }
        }
    }
    if (ENERGY) {
        if (SEM == MDF_SEM_PHYSICAL) {
            const double v[2] = {ev, ec};
            const int idx[2] = {MDF_E_VDW14, MDF_E_EE14};
            block_acc_fixed<2>(v, acc, idx, ENERGY_SCALE, st);
        } else {
            const double v[5] = {ev, eall, epl, ecut, edir};
            const int idx[5] = {MDF_E_VDW, MDF_E_EE, MDF_E_EE_PAIRLIST, MDF_E_EE_CUTOFF, MDF_E_EE_DIRECT};
            block_acc_fixed<5>(v, acc, idx, ENERGY_SCALE, st);
        }
    }
}

template <int SEM, bool ENERGY>
__global__ void k_pairs14(Pair14Args A)
{
    pairs14_dev<SEM, ENERGY>(A);
}

template <int SEM, bool ENERGY>
__global__ void k_pairs14_multi(const Pair14Args* __restrict__ As)
{
    const Pair14Args& A = As[blockIdx.z];
    if ((int)blockIdx.x >= A.gx) return;
    pairs14_dev<SEM, ENERGY>(A);
}

// ------------------------------------------------------------------ host
NBParams make_params(const Ctx& c)
{
    NBParams P;
    for (int d = 0; d < 3; ++d) P.box[d] = c.box[d];
    P.rc = c.p.cutoff;
    P.rc2 = c.p.cutoff * c.p.cutoff;
    P.use_switch = c.p.switch_radius > 0.0;
    P.rsw = P.use_switch ? c.p.switch_radius : c.p.cutoff;
    P.inv_sw = P.use_switch ? 1.0 / (c.p.cutoff - c.p.switch_radius) : 0.0;
    P.kc = c.p.coulomb_const;
    P.alpha = c.alpha;
    double rl = c.p.cutoff + c.p.skin;
    P.rlist2 = rl * rl;
    P.ntp = c.ntp;
    double i2 = 1.0 / P.rc2, i6 = i2 * i2 * i2;
    P.ucut_pow6 = i6;
    P.ucut_pow12 = i6 * i6;
    return P;
}

// Warps per block of the pair kernels: mdf_params.pair_warps (2, 4 or 8; 0 = 8).
static int pair_warps(const Ctx& c)
{
    const int w = c.p.pair_warps;
    return (w == 2 || w == 4 || w == 8) ? w : NB_WARPS;
}

// Blocks of a persistent pair kernel: as many as stay resident on the device
// at once (SMs x resident blocks per SM for this kernel, block size and
// shared memory), cached per kernel and launch shape.
int persistent_blocks(const void* fn, int threads, size_t dyn)
{
    struct Key {
        const void* fn;
        int threads;
        size_t dyn;
        int dev;
        bool operator<(const Key& o) const
        {
            return std::tie(fn, threads, dyn, dev) < std::tie(o.fn, o.threads, o.dyn, o.dev);
        }
    };
    static thread_local std::map<Key, int> cache;
    int dev = 0;
    MDF_CUDA_TRY(cudaGetDevice(&dev));
    const Key k{fn, threads, dyn, dev};
    auto it = cache.find(k);
    if (it != cache.end()) return it->second;
    int sms = 0, per = 0;
    MDF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MDF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, dyn));
    const int n = std::max(1, sms * std::max(1, per));
    cache[k] = n;
    return n;
}

int pair_threads(const Ctx& c)
{
    return 32 * pair_warps(c);
}

// Atom pairs within the cutoff are counted by the first evaluation after a
// pairlist build only (the count costs instructions in the pair loop).
static bool begin_pair_count(Ctx& c)
{
    if (!c.count_next) return false;
    MDF_CUDA_TRY(cudaMemsetAsync(c.npairs_dev.p, 0, sizeof(unsigned long long), c.stream));
    c.count_next = false;
    c.counted = true;
    c.counting = true;
    return true;
}

// Pair-kernel arguments of this rank's i clusters.  With count set the kernel
// counts the atom pairs inside the cutoff (first evaluation after a build).
template <typename R>
PairArgs<R> make_pair_args(const Ctx& c, bool count)
{
    PairArgs<R> A;
    A.P = make_params(c);
    const int wpb = pair_warps(c);
    long long lo, hi;
    cluster_share(c, lo, hi);   // this rank's i clusters
    A.nlist = (int)(hi - lo);
    A.gx = grid_blocks(A.nlist, wpb);
    A.gy = 1;
    const bool pruned = c.p.prune_every != 0 && c.pruned_valid;
    A.ilist = (pruned ? c.ilist_in.p : c.ilist.p) + lo;
    A.plist = pruned ? c.plist_in.p : c.plist.p;
    if (sizeof(R) == 4) {
        A.xq = reinterpret_cast<const typename V4<R>::type*>(c.xq_f.p);
        A.ljAB = reinterpret_cast<const typename V2<R>::type*>(c.ljAB_f.p);
    } else {
        A.xq = reinterpret_cast<const typename V4<R>::type*>(c.xq_d.p);
        A.ljAB = reinterpret_cast<const typename V2<R>::type*>(c.ljAB.p);
    }
    A.stype = c.slot_type.p;
    A.center = c.center.p;
    A.ljvalid = c.ljvalid.p;
    A.fslot = c.f_slot.p;
    A.nslots = c.n_slots;
    A.acc = c.acc.p;
    A.npairs = c.npairs_dev.p;
    A.count = count ? 1 : 0;
    A.st = c.status.p;
    return A;
}
template PairArgs<float> make_pair_args<float>(const Ctx&, bool);
template PairArgs<double> make_pair_args<double>(const Ctx&, bool);

template <typename R, int SEM>
static void launch_pairs_t(Ctx& c, bool energy)
{
    const bool count = begin_pair_count(c);
    const PairArgs<R> A = make_pair_args<R>(c, count);
    if (A.nlist == 0) return;
    const int th = 32 * pair_warps(c);
    if (energy) k_pairs<R, SEM, true><<<grid_of(A), th, 0, c.stream>>>(A);
    else k_pairs<R, SEM, false><<<grid_of(A), th, 0, c.stream>>>(A);
    MDF_CUDA_TRY(cudaGetLastError());
    c.launches += 1;
}


ShiftTable make_shift_table(const Ctx& c)
{
    ShiftTable t;
    for (int code = 0; code < 27; ++code) {
        int s[3] = {code % 3 - 1, (code / 3) % 3 - 1, code / 9 - 1};
        for (int d = 0; d < 3; ++d) {
            double v = s[d] * c.box[d];
            float hi = (float)v;
            t.v[code][d] = hi;
            t.v[code][3 + d] = (float)(v - (double)hi);
        }
    }
    return t;
}

// FP32 pair-kernel arguments (PHYSICAL) of this rank's i clusters; *dyn gets
// the dynamic shared memory the LJ table needs (0 when it stays in global
// memory).
PairF32Args make_pair_f32_args(const Ctx& c, size_t* dyn)
{
    PairF32Args A;
    const NBParams P = make_params(c);
    A.shifts = make_shift_table(c);
    PairConstF& K = A.K;
    K.rc2 = (float)P.rc2;
    K.kex = (float)(-P.alpha * P.alpha * 1.4426950408889634074);
    K.pa = (float)(0.3275911 * P.alpha);
    K.two_a_spi = (float)(2.0 * P.alpha / 1.7724538509055160273);
    K.inv_sw = (float)P.inv_sw;
    K.rsw_inv = (float)(P.rsw * P.inv_sw);
    K.d30 = (float)(-30.0 * P.inv_sw);
    K.d60 = (float)(60.0 * P.inv_sw);
    K.uc6 = (float)P.ucut_pow6;
    K.uc12 = (float)P.ucut_pow12;
    K.rcf = (float)P.rc;
    K.rc2f = (float)P.rc2;
    const int ntp2 = c.ntp * c.ntp;
    const size_t lj_bytes = sizeof(float4) * (size_t)ntp2;
    A.lj_smem = lj_bytes <= 40 * 1024 ? 1 : 0;
    if (dyn) *dyn = A.lj_smem ? lj_bytes : 0;
    const int wpb = pair_warps(c);
    long long lo, hi;
    cluster_share(c, lo, hi);   // this rank's i clusters
    A.nlist = (int)(hi - lo);
    A.gx = grid_blocks(A.nlist, wpb);
    A.gy = 1;
    const bool pruned = c.p.prune_every != 0 && c.pruned_valid;
    A.half = pruned && c.pruned_half ? 1 : 0;
    A.ilist = A.half ? c.ilist_h.p + 2 * lo : (pruned ? c.ilist_in.p : c.ilist.p) + lo;
    A.plist = pruned ? (A.half ? c.plist_h.p : c.plist_in.p) : c.plist.p;
    if (A.half) {
        A.nlist *= 2;   // two half items per i cluster
        A.gx = grid_blocks(A.nlist, wpb);
    }
    A.xq = c.xq_f.p;
    A.stype = c.slot_type.p;
    A.centerf = c.centerf.p;
    A.lj4 = c.ljAB4_f.p;
    A.ntp = c.ntp;
    A.kc = (float)P.kc;
    A.fslot = c.f_slot.p;
    A.nslots = c.n_slots;
    A.acc = c.acc.p;
    A.npairs = c.npairs_dev.p;
    A.next = c.scal.p + SCAL_WORK;
    A.persist = c.p.pair_schedule == 1 ? 1 : 0;
    A.st = c.status.p;
    return A;
}

static void launch_pairs_f32(Ctx& c, bool energy)
{
    const bool count = begin_pair_count(c);
    size_t dyn = 0;
    const PairF32Args A = make_pair_f32_args(c, &dyn);
    if (A.nlist == 0) return;
    const int th = 32 * pair_warps(c);
    const bool sw = c.p.switch_radius > 0.0;
#define MDF_PF32(E, S, K_)                                                                                     \
    do {                                                                                                       \
        const void* fn = A.half ? ((E) ? (const void*)k_pairs_f32_half<S, K_>                                  \
                                       : (const void*)k_pairs_f32_half_force<S, K_>)                           \
                                : ((E) ? (const void*)k_pairs_f32<S, K_> : (const void*)k_pairs_f32_force<S, K_>); \
        const int nb = A.persist ? std::min(A.gx, persistent_blocks(fn, th, dyn)) : A.gx;                       \
        if (A.half) {                                                                                          \
            if (E) k_pairs_f32_half<S, K_><<<nb, th, dyn, c.stream>>>(A);                                        \
            else k_pairs_f32_half_force<S, K_><<<nb, th, dyn, c.stream>>>(A);                                    \
        } else {                                                                                               \
            if (E) k_pairs_f32<S, K_><<<nb, th, dyn, c.stream>>>(A);                                             \
            else k_pairs_f32_force<S, K_><<<nb, th, dyn, c.stream>>>(A);                                         \
        }                                                                                                      \
    } while (0)
#define MDF_PF32_K(E, S) \
    do { if (count) MDF_PF32(E, S, true); else MDF_PF32(E, S, false); } while (0)
    if (energy) {
        if (sw) MDF_PF32_K(true, true); else MDF_PF32_K(true, false);
    } else {
        if (sw) MDF_PF32_K(false, true); else MDF_PF32_K(false, false);
    }
#undef MDF_PF32_K
#undef MDF_PF32
    MDF_CUDA_TRY(cudaGetLastError());
    c.launches += 1;
}

void launch_pairs_f32_multi(const PairF32Args* d_args, int nsys, int gx, int threads, size_t dyn, bool energy,
                            bool use_switch, bool persist, bool half, bool lj_smem, cudaStream_t s)
{
#define MDF_PF32M(KERN)                                                                                        \
    do {                                                                                                       \
        const dim3 g(persist ? std::min(gx, persistent_blocks((const void*)KERN, threads, dyn)) : gx, 1, nsys); \
        KERN<<<g, threads, dyn, s>>>(d_args);                                                                  \
    } while (0)
#define MDF_PF32S(S, L)                                                                                        \
    do {                                                                                                       \
        if (half) {                                                                                            \
            if (energy) MDF_PF32M((k_pairs_f32_half_multi<S, L>));                                             \
            else MDF_PF32M((k_pairs_f32_half_force_multi<S, L>));                                              \
        } else {                                                                                               \
            if (energy) MDF_PF32M((k_pairs_f32_multi<S, L>));                                                  \
            else MDF_PF32M((k_pairs_f32_force_multi<S, L>));                                                   \
        }                                                                                                      \
    } while (0)
    if (use_switch) {
        if (lj_smem) MDF_PF32S(true, true); else MDF_PF32S(true, false);
    } else {
        if (lj_smem) MDF_PF32S(false, true); else MDF_PF32S(false, false);
    }
#undef MDF_PF32S
#undef MDF_PF32M
    MDF_CUDA_TRY(cudaGetLastError());
}

// FP64 pair-kernel arguments (PHYSICAL) of this rank's i clusters; *dyn gets
// the dynamic shared memory of the LJ table (0 when it stays in global memory).
PairF64Args make_pair_f64_args(const Ctx& c, size_t* dyn)
{
    PairF64Args A;
    const NBParams P = make_params(c);
    for (int code = 0; code < 27; ++code) {
        const int sv[3] = {code % 3 - 1, (code / 3) % 3 - 1, code / 9 - 1};
        for (int d = 0; d < 3; ++d) A.shifts.v[code][d] = sv[d] * c.box[d];
    }
    PairConstD& K = A.K;
    K.rc2 = P.rc2;
    K.alpha = P.alpha;
    K.two_a_spi = 2.0 * P.alpha / 1.7724538509055160273;
    K.inv_sw = P.inv_sw;
    K.rsw_inv = P.rsw * P.inv_sw;
    K.d30 = -30.0 * P.inv_sw;
    K.d60 = 60.0 * P.inv_sw;
    K.uc6 = P.ucut_pow6;
    K.uc12 = P.ucut_pow12;
    K.rc = P.rc;
    const size_t lj_bytes = sizeof(double4) * (size_t)c.ntp * c.ntp;
    A.lj_smem = lj_bytes <= 96 * 1024 ? 1 : 0;
    if (dyn) *dyn = A.lj_smem ? lj_bytes : 0;
    const int wpb = pair_warps(c);
    long long lo, hi;
    cluster_share(c, lo, hi);   // this rank's i clusters
    A.nlist = (int)(hi - lo);
    A.gx = grid_blocks(A.nlist, wpb);
    A.gy = 1;
    const bool pruned = c.p.prune_every != 0 && c.pruned_valid;
    A.half = pruned && c.pruned_half ? 1 : 0;
    A.ilist = A.half ? c.ilist_h.p + 2 * lo : (pruned ? c.ilist_in.p : c.ilist.p) + lo;
    A.plist = pruned ? (A.half ? c.plist_h.p : c.plist_in.p) : c.plist.p;
    if (A.half) {
        A.nlist *= 2;   // two half items per i cluster
        A.gx = grid_blocks(A.nlist, wpb);
    }
    A.xq = c.xq_d.p;
    A.stype = c.slot_type.p;
    A.center = c.center.p;
    A.lj4 = c.ljAB4_d.p;
    A.ntp = c.ntp;
    A.kc = P.kc;
    A.fslot = c.f_slot.p;
    A.nslots = c.n_slots;
    A.acc = c.acc.p;
    A.npairs = c.npairs_dev.p;
    A.next = c.scal.p + SCAL_WORK;
    A.persist = c.p.pair_schedule == 1 ? 1 : 0;
    A.st = c.status.p;
    return A;
}

// The table above 48 KB needs the opt-in dynamic shared memory size.
template <typename KernelT>
static void allow_smem(KernelT* k, size_t dyn)
{
    if (dyn > 48 * 1024)
        MDF_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
}

static void launch_pairs_f64(Ctx& c, bool energy)
{
    const bool count = begin_pair_count(c);
    size_t dyn = 0;
    const PairF64Args A = make_pair_f64_args(c, &dyn);
    if (A.nlist == 0) return;
    const int th = 32 * pair_warps(c);
    const bool sw = c.p.switch_radius > 0.0;
#define MDF_PF64(E, S, K_)                                                                                     \
    do {                                                                                                       \
        if (A.half) {                                                                                          \
            allow_smem(k_pairs_f64_half<E, S, K_>, dyn);                                                       \
            const int nb = A.persist                                                                           \
                               ? std::min(A.gx, persistent_blocks((const void*)k_pairs_f64_half<E, S, K_>, th, dyn)) \
                               : A.gx;                                                                         \
            k_pairs_f64_half<E, S, K_><<<nb, th, dyn, c.stream>>>(A);                                          \
        } else {                                                                                               \
            allow_smem(k_pairs_f64<E, S, K_>, dyn);                                                            \
            const int nb = A.persist                                                                           \
                               ? std::min(A.gx, persistent_blocks((const void*)k_pairs_f64<E, S, K_>, th, dyn))  \
                               : A.gx;                                                                         \
            k_pairs_f64<E, S, K_><<<nb, th, dyn, c.stream>>>(A);                                               \
        }                                                                                                      \
    } while (0)
#define MDF_PF64_K(E, S) \
    do { if (count) MDF_PF64(E, S, true); else MDF_PF64(E, S, false); } while (0)
    if (energy) {
        if (sw) MDF_PF64_K(true, true); else MDF_PF64_K(true, false);
    } else {
        if (sw) MDF_PF64_K(false, true); else MDF_PF64_K(false, false);
    }
#undef MDF_PF64_K
#undef MDF_PF64
    MDF_CUDA_TRY(cudaGetLastError());
    c.launches += 1;
}

void launch_pairs_f64_multi(const PairF64Args* d_args, int nsys, int gx, int threads, size_t dyn, bool energy,
                            bool use_switch, bool persist, bool half, bool lj_smem, cudaStream_t s)
{
#define MDF_PF64K(KERN)                                                                                        \
    do {                                                                                                       \
        allow_smem(KERN, dyn);                                                                                 \
        const dim3 gp(persist ? std::min(gx, persistent_blocks((const void*)KERN, threads, dyn)) : gx, 1, nsys); \
        KERN<<<gp, threads, dyn, s>>>(d_args);                                                                 \
    } while (0)
#define MDF_PF64M(E, S)                                                                                        \
    do {                                                                                                       \
        if (half) {                                                                                            \
            if (lj_smem) MDF_PF64K((k_pairs_f64_half_multi<E, S, true>));                                      \
            else MDF_PF64K((k_pairs_f64_half_multi<E, S, false>));                                             \
        } else {                                                                                               \
            if (lj_smem) MDF_PF64K((k_pairs_f64_multi<E, S, true>));                                           \
            else MDF_PF64K((k_pairs_f64_multi<E, S, false>));                                                  \
        }                                                                                                      \
    } while (0)
    if (energy) {
        if (use_switch) MDF_PF64M(true, true); else MDF_PF64M(true, false);
    } else {
        if (use_switch) MDF_PF64M(false, true); else MDF_PF64M(false, false);
    }
#undef MDF_PF64M
#undef MDF_PF64K
    MDF_CUDA_TRY(cudaGetLastError());
}

void launch_nonbonded(Ctx& c, bool energy)
{
    if (c.n_clusters == 0) return;
    bool phys = c.p.semantics == MDF_SEM_PHYSICAL;
    if (c.p.precision == MDF_PREC_MIXED) {
        if (phys) launch_pairs_f32(c, energy);
        else launch_pairs_t<float, MDF_SEM_REFERENCE>(c, energy);
    } else {
        if (phys) launch_pairs_f64(c, energy);
        else launch_pairs_t<double, MDF_SEM_REFERENCE>(c, energy);
    }
}

// This rank's excluded pairs and 1-4 pairs.
ExclArgs make_excl_args(const Ctx& c)
{
    ExclArgs A;
    long long e0, e1;
    rank_slice(c, c.n_excl, e0, e1);
    A.n = (int)(e1 - e0);
    A.gx = grid_blocks(A.n, 256);
    A.gy = 1;
    A.pairs = c.excl_pairs.p + 2 * e0;
    A.is14 = c.excl_is14.p + e0;
    A.xyz = c.xyz.p;
    A.q = c.q.p;
    A.P = make_params(c);
    A.N = c.N;
    A.fatom = c.f_atom.p;
    A.acc = c.acc.p;
    A.st = c.status.p;
    return A;
}

Pair14Args make_pair14_args(const Ctx& c)
{
    Pair14Args A;
    long long p0, p1;
    rank_slice(c, c.n_14, p0, p1);
    A.n = (int)(p1 - p0);
    A.gx = grid_blocks(A.n, 256);
    A.gy = 1;
    A.pairs = c.pairs14.p + 2 * p0;
    A.scale = c.p14_scale.p + p0;
    A.xyz = c.xyz.p;
    A.q = c.q.p;
    A.type = c.type.p;
    A.lj14 = c.lj14AB.p;
    A.ljvalid = c.ljvalid.p;
    A.P = make_params(c);
    A.N = c.N;
    A.fatom = c.f_atom.p;
    A.acc = c.acc.p;
    A.st = c.status.p;
    return A;
}

void launch_exclusions(Ctx& c, bool energy)
{
    const int th = 256;
    const bool phys = c.p.semantics == MDF_SEM_PHYSICAL;
    const ExclArgs E = make_excl_args(c);
    if (E.n > 0) {
#define MDF_EXCL(S, EN) k_exclusions<S, EN><<<grid_of(E), th, 0, c.stream>>>(E)
        if (phys) { if (energy) MDF_EXCL(MDF_SEM_PHYSICAL, true); else MDF_EXCL(MDF_SEM_PHYSICAL, false); }
        else if (energy) MDF_EXCL(MDF_SEM_REFERENCE, true);
#undef MDF_EXCL
        if (phys || energy) c.launches += 1;
    }
    const Pair14Args P14 = make_pair14_args(c);
    if (P14.n > 0) {
#define MDF_P14(S, EN) k_pairs14<S, EN><<<grid_of(P14), th, 0, c.stream>>>(P14)
        if (phys) { if (energy) MDF_P14(MDF_SEM_PHYSICAL, true); else MDF_P14(MDF_SEM_PHYSICAL, false); }
        else { if (energy) MDF_P14(MDF_SEM_REFERENCE, true); else MDF_P14(MDF_SEM_REFERENCE, false); }
#undef MDF_P14
        c.launches += 1;
    }
    MDF_CUDA_TRY(cudaGetLastError());
}

void launch_exclusions_multi(const ExclArgs* d_excl, int gx_excl, const Pair14Args* d_14, int gx_14, int nsys,
                             bool energy, cudaStream_t s)
{
    if (gx_excl > 0) {
        if (energy) k_exclusions_multi<MDF_SEM_PHYSICAL, true><<<dim3(gx_excl, 1, nsys), 256, 0, s>>>(d_excl);
        else k_exclusions_multi<MDF_SEM_PHYSICAL, false><<<dim3(gx_excl, 1, nsys), 256, 0, s>>>(d_excl);
    }
    if (gx_14 > 0) {
        if (energy) k_pairs14_multi<MDF_SEM_PHYSICAL, true><<<dim3(gx_14, 1, nsys), 256, 0, s>>>(d_14);
        else k_pairs14_multi<MDF_SEM_PHYSICAL, false><<<dim3(gx_14, 1, nsys), 256, 0, s>>>(d_14);
    }
    MDF_CUDA_TRY(cudaGetLastError());
}

}  // namespace mdf
