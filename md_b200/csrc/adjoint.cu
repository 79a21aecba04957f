// Adjoint (vector-Jacobian product) of the PHYSICAL energy and forces with
// respect to the per-atom charges and the Lennard-Jones A/B coefficients.
//
// Given v = dL/dF (3N, forces as returned by mdf_compute) and gE = dL/dE
// (total energy), the gradient of the loss is the gradient, at fixed
// positions, of
//     Phi(q, A, B) = gE E + sum_a v_a . F_a .
// Every nonbonded pair contributes E_ab = A e_A(r) + B e_B(r) + q_a q_b e_0(r)
// and F_a = -F_b = g(r) d with g linear in the same coefficients, so per pair
//     dPhi/dA_ab = gE e_A + g_A w,   dPhi/dB_ab = gE e_B + g_B w,
//     dPhi/dq_a += q_b (gE e_0 + g_0 w),   w = (v_a - v_b) . d .
// The pair kernel is recomputed (nothing is stored by the forward pass).  The
// exclusion corrections, the 1-4 Coulomb pairs, the self energy and the net
// charge term follow the same pattern; the reciprocal space is in pme.cu.
//
// dL/dq is accumulated in int64 fixed point (deterministic); dL/dA and dL/dB
// per NONBONDED_PARM_INDEX entry in FP64 through per-block shared-memory
// partials (atomics in FP64: reproducible to rounding, not bitwise).
#include <algorithm>
#include <cmath>
#include <vector>

#include "mdf_device.cuh"
#include "mdf_internal.cuh"
#include "nb_common.cuh"

namespace mdf {

// dL/dq and the normalised v are scaled by 1/scale so that the fixed-point
// accumulators keep their resolution whatever the loss' magnitude.
template <typename R>
__global__ void k_adj_pack(int nslots, const int* __restrict__ slot_atom, const double* __restrict__ v,
                           typename V4<R>::type* __restrict__ vs)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const int a = slot_atom[s];
    typename V4<R>::type o;
    o.x = 0; o.y = 0; o.z = 0; o.w = 0;
    if (a >= 0) {
        o.x = (R)v[3 * a];
        o.y = (R)v[3 * a + 1];
        o.z = (R)v[3 * a + 2];
    }
    vs[s] = o;
}

// Frame offset of J's cluster frame seen from I's frame, as in the forward kernels.
template <typename R> struct Frame;
template <> struct Frame<float> {
    __device__ static void offset(const float4* cf, const double4*, const float (*sh)[6], const NBParams&, int I,
                                  int J, int shift, float o[3])
    {
        const float4 cI = cf[I], cJ = cf[J];
        const float* s6 = sh[shift];
        o[0] = ((cI.x - cJ.x) - s6[0]) - s6[3];
        o[1] = ((cI.y - cJ.y) - s6[1]) - s6[4];
        o[2] = ((cI.z - cJ.z) - s6[2]) - s6[5];
    }
};
template <> struct Frame<double> {
    __device__ static void offset(const float4*, const double4* c, const float (*)[6], const NBParams& P, int I,
                                  int J, int shift, double o[3])
    {
        const double4 cI = c[I], cJ = c[J];
        int sx, sy, sz;
        shift_decode(shift, sx, sy, sz);
        o[0] = cI.x - cJ.x - sx * P.box[0];
        o[1] = cI.y - cJ.y - sy * P.box[1];
        o[2] = cI.z - cJ.z - sz * P.box[2];
    }
};

template <typename R> __device__ __forceinline__ R rsqrt_r(R x);
template <> __device__ __forceinline__ float rsqrt_r<float>(float x) { return rsqrt_ftz(x); }
template <> __device__ __forceinline__ double rsqrt_r<double>(double x) { return 1.0 / sqrt(x); }

template <typename R> __device__ __forceinline__ void erfc_exp(R ar, R& erfcv, R& ex);
template <> __device__ __forceinline__ void erfc_exp<float>(float ar, float& erfcv, float& ex)
{
    ex = ex2_approx(-1.4426950408889634f * ar * ar);
    erfcv = erfc_as(rcp_ftz(1.0f + 0.3275911f * ar), ex);
}
template <> __device__ __forceinline__ void erfc_exp<double>(double ar, double& erfcv, double& ex)
{
    ex = exp(-ar * ar);
    erfcv = erfc(ar);
}

// Adjoint pair kernel: the forward kernel's warp layout (warp per i cluster,
// lane = (j slot, i atom), the j accumulator rotating one lane per step).
// Shared memory: the 8 warps' staged j atoms, then 2 * nlj partial sums
// (dA | dB) when nlj > 0; nlj == 0 sends every LJ term straight to global
// memory.
template <typename R, bool SWITCH>
__global__ void __launch_bounds__(NB_THREADS) k_adj_pairs(
    int nlist, const ILRange* __restrict__ ilist, const PairEntry* __restrict__ plist,
    const typename V4<R>::type* __restrict__ xq, const typename V4<R>::type* __restrict__ vs,
    const int* __restrict__ stype, const float4* __restrict__ centerf, const double4* __restrict__ center,
    ShiftTable shifts, const int* __restrict__ nbidx, NBParams P, double gE, int nlj,
    unsigned long long* __restrict__ dq_slot, double* __restrict__ dab, int n_ljpair, unsigned* st)
{
    using V4t = typename V4<R>::type;
    extern __shared__ __align__(16) unsigned char adj_smem[];
    V4t* sx = reinterpret_cast<V4t*>(adj_smem);                      // [NB_WARPS][4][8]
    V4t* sv = sx + NB_WARPS * 4 * CLUSTER;                           // [NB_WARPS][4][8]
    int* stj = reinterpret_cast<int*>(sv + NB_WARPS * 4 * CLUSTER);  // [NB_WARPS][4][8]
    R* part = reinterpret_cast<R*>(stj + NB_WARPS * 4 * CLUSTER);    // [2 * nlj]
    __shared__ float sh[27][6];
    for (int k = threadIdx.x; k < 27 * 6; k += blockDim.x) sh[k / 6][k % 6] = shifts.v[k / 6][k % 6];
    for (int k = threadIdx.x; k < 2 * nlj; k += blockDim.x) part[k] = (R)0;
    __syncthreads();
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = blockIdx.x * NB_WARPS + wib;
    const int jslot = lane >> 3, ii = lane & 7;
    const unsigned FULL = 0xffffffffu;
    const R rc2 = (R)P.rc2, rsw = (R)P.rsw, inv_sw = (R)P.inv_sw, alpha = (R)P.alpha, kc = (R)P.kc;
    const R two_a_spi = (R)(2.0 * P.alpha / 1.7724538509055160273);
    const R gEr = (R)gE;
    const R c6 = (R)P.ucut_pow6, c12 = (R)P.ucut_pow12, rcr = (R)P.rc;
    V4t* wsx = sx + wib * 4 * CLUSTER;
    V4t* wsv = sv + wib * 4 * CLUSTER;
    int* wst = stj + wib * 4 * CLUSTER;
    R dqi = 0;
    // LJ parameter derivatives: a one-entry cache per lane (most pairs of a
    // solvent share one type pair), flushed to the block sums when the type
    // pair changes and at the end
    int kcache = -1;
    R ca = 0, cb = 0;
    auto flush_lj = [&]() {
        if (kcache < 0) return;
        if (nlj > 0) {
            atomicAdd(part + kcache, ca);
            atomicAdd(part + nlj + kcache, cb);
        } else {
            atomicAdd(dab + kcache, (double)ca);
            atomicAdd(dab + n_ljpair + kcache, (double)cb);
        }
    };
    if (w < nlist) {
        const ILRange L = ilist[w];
        const int I = L.i;
        const V4t xi = xq[I * CLUSTER + ii];
        const V4t vi = vs[I * CLUSTER + ii];
        const int trow = stype[I * CLUSTER + ii] * P.ntp;
        const int rot_src = (lane & ~7) | ((ii + 1) & 7);
        for (int b = 0; b < L.count; b += 4) {
            const int e = b + jslot;
            PairEntry pe;
            if (e < L.count) {
                pe = plist[L.start + e];
            } else {
                pe.j = I; pe.shift = 13; pe.mask = 0ull;
            }
            const int J = pe.j;
            wsx[jslot * CLUSTER + ii] = xq[J * CLUSTER + ii];
            wsv[jslot * CLUSTER + ii] = vs[J * CLUSTER + ii];
            wst[jslot * CLUSTER + ii] = stype[J * CLUSTER + ii];
            R o[3];
            Frame<R>::offset(centerf, center, sh, P, I, J, pe.shift, o);
            const R xix = xi.x + o[0], xiy = xi.y + o[1], xiz = xi.z + o[2];
            const unsigned long long mask = pe.mask;
            __syncwarp();
            R dqj = 0;
#pragma unroll
            for (int t = 0; t < CLUSTER; ++t) {
                const int jj = (ii + t) & 7;
                const V4t xj = wsx[jslot * CLUSTER + jj];
                const R dx = xix - xj.x, dy = xiy - xj.y, dz = xiz - xj.z;
                const R r2 = dx * dx + dy * dy + dz * dz;
                const bool on = ((mask >> (ii * 8 + jj)) & 1ull) && r2 <= rc2;
                if (on) {
                    const V4t vj = wsv[jslot * CLUSTER + jj];
                    const R wv = (vi.x - vj.x) * dx + (vi.y - vj.y) * dy + (vi.z - vj.z) * dz;
                    const R rinv = rsqrt_r<R>(r2), r = r2 * rinv, rinv2 = rinv * rinv;
                    // Coulomb (erfc real space)
                    const R ar = alpha * r;
                    R erfcv, ex;
                    erfc_exp<R>(ar, erfcv, ex);
                    const R e0 = kc * erfcv * rinv;
                    const R g0 = (e0 + kc * two_a_spi * ex) * rinv2;
                    const R psi = gEr * e0 + g0 * wv;
                    dqi += xj.w * psi;
                    dqj += xi.w * psi;
                    // Lennard-Jones: E = A eA + B eB, g = A gA + B gB
                    const int k = nbidx[trow + wst[jslot * CLUSTER + jj]];
                    if (k >= 0) {
                        const R rinv6 = rinv2 * rinv2 * rinv2;
                        R eA = rinv6 * rinv6, eB = -rinv6;
                        R gA = (R)12 * eA * rinv2, gB = (R)-6 * rinv6 * rinv2;
                        if (SWITCH) {
                            if (r > rsw) {
                                const R x = (r - rsw) * inv_sw, x2 = x * x, x3 = x2 * x;
                                const R S = (R)1 + x3 * ((R)-10 + x * ((R)15 - (R)6 * x));
                                const R dS = x2 * ((R)-30 + x * ((R)60 - (R)30 * x)) * inv_sw;
                                gA = S * gA - eA * dS * rinv;
                                gB = S * gB - eB * dS * rinv;
                                eA *= S;
                                eB *= S;
                            }
                        } else {
                            // force-shifted: U - U(rc) + (r - rc) g(rc) rc, linear in A and B
                            const R gcA = (R)12 * c12 / rc2, gcB = (R)-6 * c6 / rc2;
                            eA = eA - c12 + (r - rcr) * (gcA * rcr);
                            eB = eB + c6 + (r - rcr) * (gcB * rcr);
                            gA = gA - gcA * rcr * rinv;
                            gB = gB - gcB * rcr * rinv;
                        }
                        const R da = gEr * eA + gA * wv, db = gEr * eB + gB * wv;
                        if (k == kcache) {
                            ca += da;
                            cb += db;
                        } else {
                            flush_lj();
                            kcache = k;
                            ca = da;
                            cb = db;
                        }
                    }
                }
                dqj = __shfl_sync(FULL, dqj, rot_src);
            }
            if (e < L.count && dqj != (R)0) fx_add(dq_slot + J * CLUSTER + ii, (double)dqj, FORCE_SCALE, st);
            __syncwarp();
        }
        dqi += __shfl_xor_sync(FULL, dqi, 8);
        dqi += __shfl_xor_sync(FULL, dqi, 16);
        if (jslot == 0 && dqi != (R)0) fx_add(dq_slot + I * CLUSTER + ii, (double)dqi, FORCE_SCALE, st);
    }
    flush_lj();
    if (nlj > 0) {
        __syncthreads();
        for (int k = threadIdx.x; k < 2 * nlj; k += blockDim.x) {
            const R v = part[k];
            if (v != (R)0) atomicAdd(dab + (k < nlj ? k : n_ljpair + k - nlj), (double)v);
        }
    }
}

// Excluded pairs (-k q q erf(alpha r)/r) and 1-4 Coulomb pairs (k q q/(scee r)),
// FP64, minimum image, atom order.
__global__ void k_adj_pairs_fp64(int nex, const int* __restrict__ excl, int n14, const int* __restrict__ p14,
                                 const double2* __restrict__ scale14, const double* __restrict__ xyz,
                                 const double* __restrict__ q, const double* __restrict__ v, NBParams P, double gE,
                                 unsigned long long* __restrict__ dq, unsigned* st)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nex + n14) return;
    const bool ex = k < nex;
    const int a = ex ? excl[2 * k] : p14[2 * (k - nex)], b = ex ? excl[2 * k + 1] : p14[2 * (k - nex) + 1];
    double d[3];
    for (int c = 0; c < 3; ++c) d[c] = min_image(xyz[3 * a + c] - xyz[3 * b + c], P.box[c]);
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2], r = sqrt(r2);
    double e0, g0;
    if (ex) {
        const double ar = P.alpha * r;
        e0 = -P.kc * erf(ar) / r;
        g0 = (e0 + P.kc * (2.0 * P.alpha / 1.7724538509055160273) * exp(-ar * ar)) / r2;
    } else {
        e0 = P.kc / (scale14[k - nex].x * r);
        g0 = e0 / r2;
    }
    const double w = (v[3 * a] - v[3 * b]) * d[0] + (v[3 * a + 1] - v[3 * b + 1]) * d[1] +
                     (v[3 * a + 2] - v[3 * b + 2]) * d[2];
    const double psi = gE * e0 + g0 * w;
    fx_add(dq + a, q[b] * psi, FORCE_SCALE, st);
    fx_add(dq + b, q[a] * psi, FORCE_SCALE, st);
}

// Self energy and net-charge term, and the final sum (atom order, unscaled).
__global__ void k_adj_finish(int N, const double* __restrict__ q, const int* __restrict__ atom_slot,
                             const unsigned long long* __restrict__ dq_atom,
                             const unsigned long long* __restrict__ dq_slot, double self_coef, double net_coef,
                             double scale, double* __restrict__ out)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= N) return;
    const long long f = (long long)dq_atom[a] + (long long)dq_slot[atom_slot[a]];
    out[a] = ((double)f * FORCE_ISCALE + self_coef * q[a] + net_coef) * scale;
}

__global__ void k_scale(int n, double* __restrict__ x, double s)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] *= s;
}

template <typename R>
static void launch_adj_pairs(Ctx& c, const NBParams& P, double gE)
{
    using V4t = typename V4<R>::type;
    const bool pruned = c.p.prune_every != 0 && c.pruned_valid && !c.pruned_half;
    const ILRange* il = pruned ? c.ilist_in.p : c.ilist.p;
    const PairEntry* pl = pruned ? c.plist_in.p : c.plist.p;
    const V4t* xq = sizeof(R) == 4 ? reinterpret_cast<const V4t*>(c.xq_f.p) : reinterpret_cast<const V4t*>(c.xq_d.p);
    const V4t* vs =
        sizeof(R) == 4 ? reinterpret_cast<const V4t*>(c.adj_vs_f.p) : reinterpret_cast<const V4t*>(c.adj_vs_d.p);
    const size_t stage = (size_t)NB_WARPS * 4 * CLUSTER * (2 * sizeof(V4t) + sizeof(int));
    int nlj = c.n_ljpair;
    size_t smem = stage + 2 * (size_t)nlj * sizeof(R);
    if (smem > 96 * 1024) {   // too many LJ entries for per-block partials: global atomics
        nlj = 0;
        smem = stage;
    }
    const ShiftTable sh = make_shift_table(c);
    const int nb = grid_blocks(c.n_clusters, NB_WARPS);
    if (P.use_switch) {
        MDF_CUDA_TRY(cudaFuncSetAttribute(k_adj_pairs<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        k_adj_pairs<R, true><<<nb, NB_THREADS, smem, c.stream>>>(c.n_clusters, il, pl, xq, vs, c.slot_type.p,
                                                                 c.centerf.p, c.center.p, sh, c.nbidx.p, P, gE, nlj,
                                                                 c.adj_dq_slot.p, c.adj_dab.p, c.n_ljpair,
                                                                 c.status.p);
    } else {
        MDF_CUDA_TRY(cudaFuncSetAttribute(k_adj_pairs<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        k_adj_pairs<R, false><<<nb, NB_THREADS, smem, c.stream>>>(c.n_clusters, il, pl, xq, vs, c.slot_type.p,
                                                                  c.centerf.p, c.center.p, sh, c.nbidx.p, P, gE, nlj,
                                                                  c.adj_dq_slot.p, c.adj_dab.p, c.n_ljpair,
                                                                  c.status.p);
    }
    MDF_CUDA_TRY(cudaGetLastError());
}

void backward(Ctx& c, const double* dL_dF, double dL_dE, double* dL_dq, double* dL_dA, double* dL_dB)
{
    if (c.p.semantics != MDF_SEM_PHYSICAL)
        throw ApiError(MDF_ERR_UNSUPPORTED, "mdf_backward needs PHYSICAL semantics (REFERENCE forces are not "
                                            "the gradient of its energy)");
    if (!c.have_positions) throw ApiError(MDF_ERR_STATE, "positions not set");
    if (!c.have_list) build_pairlist(c);
    cudaStream_t s = c.stream;
    const bool mixed = c.p.precision == MDF_PREC_MIXED;
    // normalise: scale = max(|gE|, max |v|)
    double scale = std::fabs(dL_dE);
    if (dL_dF)
        for (long long i = 0; i < 3LL * c.N; ++i) scale = std::max(scale, std::fabs(dL_dF[i]));
    const int nlj = c.n_ljpair;
    c.adj_dq.alloc(c.N);
    c.adj_dab.alloc(2 * (size_t)std::max(nlj, 1));
    if (scale == 0.0 || !std::isfinite(scale)) {
        if (!std::isfinite(scale)) throw ApiError(MDF_ERR_NONFINITE, "non-finite dL/dF or dL/dE");
        if (dL_dq) std::fill(dL_dq, dL_dq + c.N, 0.0);
        if (dL_dA) std::fill(dL_dA, dL_dA + nlj, 0.0);
        if (dL_dB) std::fill(dL_dB, dL_dB + nlj, 0.0);
        return;
    }
    std::vector<double> vn(3 * (size_t)c.N, 0.0);
    if (dL_dF)
        for (long long i = 0; i < 3LL * c.N; ++i) vn[i] = dL_dF[i] / scale;
    const double gE = dL_dE / scale;
    c.adj_v.upload(vn.data(), vn.size(), s);
    c.adj_dq_slot.alloc(c.n_slots);
    c.adj_dq_atom.alloc(c.N);
    MDF_CUDA_TRY(cudaMemsetAsync(c.adj_dq_slot.p, 0, sizeof(unsigned long long) * c.n_slots, s));
    MDF_CUDA_TRY(cudaMemsetAsync(c.adj_dq_atom.p, 0, sizeof(unsigned long long) * c.N, s));
    MDF_CUDA_TRY(cudaMemsetAsync(c.adj_dab.p, 0, sizeof(double) * 2 * std::max(nlj, 1), s));
    MDF_CUDA_TRY(cudaMemsetAsync(c.status.p, 0, sizeof(unsigned), s));
    const int th = 256;
    // current cluster frame and pruned list, as a forward evaluation builds them
    pack_positions(c);
    if (c.p.prune_every != 0) {
        prune_pairlist(c, true);   // whole entries: the adjoint kernel walks 8 x 8 cluster pairs
        c.since_prune = 1;
        if (half_layout(c)) c.pruned_valid = false;   // the next forward prunes its half lists again
    }
    if (mixed) {
        c.adj_vs_f.alloc(c.n_slots);
        k_adj_pack<float><<<grid_blocks(c.n_slots, th), th, 0, s>>>(c.n_slots, c.slot_atom.p, c.adj_v.p,
                                                                     c.adj_vs_f.p);
    } else {
        c.adj_vs_d.alloc(c.n_slots);
        k_adj_pack<double><<<grid_blocks(c.n_slots, th), th, 0, s>>>(c.n_slots, c.slot_atom.p, c.adj_v.p,
                                                                      c.adj_vs_d.p);
    }
    const NBParams P = make_params(c);
    // the reciprocal-space part runs on the side stream, concurrently with
    // the pair adjoint (both only add into the fixed-point dq accumulators)
    MDF_CUDA_TRY(cudaEventRecord(c.ev_fork, s));
    MDF_CUDA_TRY(cudaStreamWaitEvent(c.side, c.ev_fork, 0));
    c.stream = c.side;
    try {
        pme_adjoint(c, gE, 1.0);
    } catch (...) {
        c.stream = s;
        throw;
    }
    c.stream = s;
    MDF_CUDA_TRY(cudaEventRecord(c.ev_join, c.side));
    if (mixed) launch_adj_pairs<float>(c, P, gE);
    else launch_adj_pairs<double>(c, P, gE);
    if (c.n_excl + c.n_14 > 0)
        k_adj_pairs_fp64<<<grid_blocks(c.n_excl + c.n_14, th), th, 0, s>>>(
            c.n_excl, c.excl_pairs.p, c.n_14, c.pairs14.p, c.p14_scale.p, c.xyz.p, c.q.p, c.adj_v.p, P, gE,
            c.adj_dq_atom.p, c.status.p);
    MDF_CUDA_TRY(cudaStreamWaitEvent(s, c.ev_join, 0));
    // d/dq_a of gE (E_self + E_net): -2 k alpha/sqrt(pi) q_a and -k pi Q / (V alpha^2)
    const double V = c.box[0] * c.box[1] * c.box[2];
    const double self_coef = gE * (-2.0 * c.p.coulomb_const * c.alpha / std::sqrt(M_PI));
    const double net_coef = gE * (-c.p.coulomb_const * M_PI * c.q_total / (V * c.alpha * c.alpha));
    k_adj_finish<<<grid_blocks(c.N, th), th, 0, s>>>(c.N, c.q.p, c.atom_slot.p, c.adj_dq_atom.p, c.adj_dq_slot.p,
                                                     self_coef, net_coef, scale, c.adj_dq.p);
    if (nlj > 0) k_scale<<<grid_blocks(2 * nlj, th), th, 0, s>>>(2 * nlj, c.adj_dab.p, scale);
    MDF_CUDA_TRY(cudaGetLastError());
    c.launches += 6;
    unsigned st = 0;
    MDF_CUDA_TRY(cudaMemcpyAsync(&st, c.status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    if (dL_dq) MDF_CUDA_TRY(cudaMemcpyAsync(dL_dq, c.adj_dq.p, sizeof(double) * c.N, cudaMemcpyDeviceToHost, s));
    if (dL_dA && nlj > 0)
        MDF_CUDA_TRY(cudaMemcpyAsync(dL_dA, c.adj_dab.p, sizeof(double) * nlj, cudaMemcpyDeviceToHost, s));
    if (dL_dB && nlj > 0)
        MDF_CUDA_TRY(cudaMemcpyAsync(dL_dB, c.adj_dab.p + nlj, sizeof(double) * nlj, cudaMemcpyDeviceToHost, s));
    // the status word belongs to the forward's scalar block: leave it clear
    MDF_CUDA_TRY(cudaMemsetAsync(c.status.p, 0, sizeof(unsigned), s));
    MDF_CUDA_TRY(cudaStreamSynchronize(s));
    if (st & ST_NONFINITE) throw ApiError(MDF_ERR_NONFINITE, "non-finite value in the adjoint");
    if (st & ST_OVERFLOW) throw ApiError(MDF_ERR_OVERFLOW, "fixed-point accumulator range exceeded in the adjoint");
}

}  // namespace mdf
