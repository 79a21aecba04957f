// C ABI of libmdf (include/mdf.h): context lifetime, uploads, evaluation
// sequencing and result readback.  The evaluation replaces the reference's
// System::calculate_forces() + calculate_energies() + PME chain
// (src/System/System.cpp:9-39, src/System/init.cpp:59-64).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "kargs.cuh"
#include "mdf_device.cuh"
#include "mdf_internal.cuh"

namespace mdf {

CudaError::CudaError(cudaError_t e, const char* what, const char* file, int line) : err(e)
{
    char buf[512];
    snprintf(buf, sizeof(buf), "CUDA error %s (%s) at %s:%d: %s", cudaGetErrorName(e), cudaGetErrorString(e), file,
             line, what);
    msg = buf;
}

void mark(Ctx& c, const char* name)
{
    if (!c.timing) return;
    if (c.nev >= (int)c.evpool.size()) {
        cudaEvent_t ev;
        MDF_CUDA_TRY(cudaEventCreate(&ev));
        c.evpool.push_back(ev);
        c.evname.push_back(name);
    }
    c.evname[c.nev] = name;
    MDF_CUDA_TRY(cudaEventRecord(c.evpool[c.nev], c.stream));
    ++c.nev;
}

// Forces out in atom order, and every accumulator cleared for the next
// evaluation (read-and-clear: an evaluation needs no memsets).  The scalar
// block was copied to the host before this kernel runs.
__device__ __forceinline__ void finalize_dev(const FinalizeArgs& A, int bx, int by)
{
    const int N = A.N, nslots = A.nslots;
    unsigned long long* __restrict__ fatom = A.fatom;
    unsigned long long* __restrict__ fslot = A.fslot;
    const int* __restrict__ atom_slot = A.atom_slot;
    double* __restrict__ out = A.out;
    unsigned long long* __restrict__ scal = A.scal;
    unsigned long long* __restrict__ host_scal = A.host_scal;
    int a = bx * blockDim.x + threadIdx.x;
    if (a < NUM_SCAL) {
        host_scal[a] = scal[a];   // mapped pinned memory: no copy-engine round trip
        scal[a] = 0ull;
    }
    if (a >= N) return;
    const int s = atom_slot[a];
    // all loads before any store, so the six loads are in flight together
    long long v[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
        v[k] = (long long)fatom[(long long)k * N + a] + (long long)fslot[(long long)k * nslots + s];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        fatom[(long long)k * N + a] = 0ull;
        fslot[(long long)k * nslots + s] = 0ull;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) out[3 * a + k] = (double)v[k] * FORCE_ISCALE;
}

__global__ void k_finalize(FinalizeArgs A)
{
    finalize_dev(A, blockIdx.x, 0);
}

__global__ void k_finalize_multi(const FinalizeArgs* __restrict__ As, const int2* __restrict__ bmap)
{
    const int2 m = bmap[blockIdx.x];
    finalize_dev(As[m.x], m.y, 0);
}

// Distributed force return.  Fold the per-atom accumulators into slot order
// and lay the slots out as nranks blocks of Sb slots, [P][3][Sb], reading
// and clearing both accumulators (padding slots past nslots are zero).
__global__ void k_stage_forces(int N, int nslots, int Sb, int P, unsigned long long* __restrict__ fatom,
                               unsigned long long* __restrict__ fslot, const int* __restrict__ slot_atom,
                               unsigned long long* __restrict__ stage)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P * Sb) return;
    const int blk = s / Sb, sl = s - blk * Sb;
    const int a = s < nslots ? slot_atom[s] : -1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        unsigned long long v = 0ull;
        if (s < nslots) {
            v = fslot[(long long)k * nslots + s];
            fslot[(long long)k * nslots + s] = 0ull;
            if (a >= 0) {
                v += fatom[(long long)k * N + a];
                fatom[(long long)k * N + a] = 0ull;
            }
        }
        stage[((long long)blk * 3 + k) * Sb + sl] = v;
    }
}

// This rank's block of summed slots -> FP64 forces [Sb][3]; also the scalar
// block to the mapped host copy and cleared (as k_finalize does).
__global__ void k_finish_block(int nslots, int Sb, int rank, const unsigned long long* __restrict__ mine,
                               double* __restrict__ out, unsigned long long* __restrict__ scal,
                               unsigned long long* __restrict__ host_scal)
{
    const int sl = blockIdx.x * blockDim.x + threadIdx.x;
    if (sl < NUM_SCAL) {
        host_scal[sl] = scal[sl];
        scal[sl] = 0ull;
    }
    if (sl >= Sb) return;
    const bool real = (long long)rank * Sb + sl < nslots;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        out[3 * sl + k] = real ? (double)(long long)mine[(long long)k * Sb + sl] * FORCE_ISCALE : 0.0;
}

// All ranks' finished slots [P Sb][3] -> forces in atom order.
__global__ void k_slots_to_atoms(int N, const int* __restrict__ atom_slot, const double* __restrict__ all,
                                 double* __restrict__ out)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= N) return;
    const int s = atom_slot[a];
#pragma unroll
    for (int k = 0; k < 3; ++k) out[3 * a + k] = all[3 * (long long)s + k];
}

static void finish_slab_forces(Ctx& c, double* d_forces)
{
    const int P = c.p.nranks, S = c.n_slots, Sb = (S + P - 1) / P;
    c.f_stage.alloc((size_t)P * 3 * Sb);
    c.f_mine.alloc((size_t)3 * Sb);
    c.f_out_blk.alloc((size_t)3 * Sb);
    c.f_out_all.alloc((size_t)3 * Sb * P);
    k_stage_forces<<<grid_blocks((long long)P * Sb, 256), 256, 0, c.stream>>>(c.N, S, Sb, P, c.f_atom.p, c.f_slot.p,
                                                                            c.slot_atom.p, c.f_stage.p);
    MDF_CUDA_TRY(cudaGetLastError());
    if (c.coll_rs(reinterpret_cast<const uint64_t*>(c.f_stage.p), reinterpret_cast<uint64_t*>(c.f_mine.p),
                  (int64_t)3 * Sb, (void*)c.stream, c.coll_user) != 0)
        throw ApiError(MDF_ERR_CUDA, "the reduce-scatter callback failed");
    k_finish_block<<<grid_blocks(std::max(Sb, NUM_SCAL), 256), 256, 0, c.stream>>>(S, Sb, c.p.rank, c.f_mine.p,
                                                                                  c.f_out_blk.p, c.scal.p,
                                                                                  c.d_hscal);
    MDF_CUDA_TRY(cudaGetLastError());
    if (c.coll_ag(c.f_out_blk.p, c.f_out_all.p, (int64_t)(sizeof(double) * 3 * Sb), (void*)c.stream,
                  c.coll_user) != 0)
        throw ApiError(MDF_ERR_CUDA, "the all-gather callback failed");
    k_slots_to_atoms<<<grid_blocks(c.N, 256), 256, 0, c.stream>>>(c.N, c.atom_slot.p, c.f_out_all.p, d_forces);
    MDF_CUDA_TRY(cudaGetLastError());
    c.launches += 3;
}

FinalizeArgs make_finalize_args(const Ctx& c, double* d_forces)
{
    FinalizeArgs A;
    A.gx = grid_blocks(std::max(c.N, NUM_SCAL), 256);
    A.gy = 1;
    A.N = c.N;
    A.nslots = c.n_slots;
    A.fatom = c.f_atom.p;
    A.fslot = c.f_slot.p;
    A.atom_slot = c.atom_slot.p;
    A.out = d_forces;
    A.scal = c.scal.p;
    A.host_scal = c.d_hscal;
    return A;
}

void launch_finalize(Ctx& c, double* d_forces, bool)
{
    if (c.fin_wait) MDF_CUDA_TRY(cudaStreamWaitEvent(c.stream, c.fin_wait, 0));
    FinalizeArgs A = make_finalize_args(c, c.fin_forces ? c.fin_forces : d_forces);
    if (c.fin_hscal) A.host_scal = c.fin_hscal;
    k_finalize<<<grid_of(A), 256, 0, c.stream>>>(A);
    MDF_CUDA_TRY(cudaGetLastError());
    c.launches += 1;
}

void launch_finalize_multi(const FinalizeArgs* d_args, BlockMap bm, cudaStream_t s)
{
    if (bm.n <= 0) return;
    k_finalize_multi<<<bm.n, 256, 0, s>>>(d_args, bm.map);
    MDF_CUDA_TRY(cudaGetLastError());
}

static void check_index(const int32_t* a, long long n, int N, const char* what)
{
    for (long long i = 0; i < n; ++i)
        if (a[i] < 0 || a[i] >= N) throw ApiError(MDF_ERR_INVALID, std::string("atom index out of range in ") + what);
}

// Pair tables over (ntypes + 1)^2, the extra type being cluster padding, from
// the LJ coefficients per NONBONDED_PARM_INDEX entry; also the table mapping a
// type pair to its 0-based entry (-1: no LJ).
void set_lj_tables(Ctx& c, const double* lj_a, const double* lj_b)
{
    cudaStream_t s = c.stream;
    const int ntp = c.ntp;
    std::vector<double2> ab(ntp * ntp, make_double2(0, 0)), ab14(ntp * ntp, make_double2(0, 0));
    std::vector<float2> abf(ntp * ntp, make_float2(0, 0));
    std::vector<float4> ab4(ntp * ntp, make_float4(0, 0, 0, 0));
    std::vector<double4> ab4d(ntp * ntp, make_double4(0, 0, 0, 0));
    std::vector<int> valid(ntp * ntp, 0), idx(ntp * ntp, -1);
    for (int i = 0; i < c.ntypes; ++i)
        for (int j = 0; j < c.ntypes; ++j) {
            const int nb = c.h_nb_index[i * c.ntypes + j];
            if (nb == 0) continue;
            const int tp = i * ntp + j;
            ab[tp] = make_double2(lj_a[nb - 1], lj_b[nb - 1]);
            abf[tp] = make_float2((float)lj_a[nb - 1], (float)lj_b[nb - 1]);
            ab4[tp] = make_float4((float)lj_a[nb - 1], (float)lj_b[nb - 1], (float)(12.0 * lj_a[nb - 1]),
                                  (float)(6.0 * lj_b[nb - 1]));
            ab4d[tp] = make_double4(lj_a[nb - 1], lj_b[nb - 1], 12.0 * lj_a[nb - 1], 6.0 * lj_b[nb - 1]);
            ab14[tp] = make_double2(c.h_lj14a[nb - 1], c.h_lj14b[nb - 1]);
            valid[tp] = 1;
            idx[tp] = nb - 1;
        }
    c.ljAB.upload(ab.data(), ab.size(), s);
    c.ljAB_f.upload(abf.data(), abf.size(), s);
    c.ljAB4_f.upload(ab4.data(), ab4.size(), s);
    c.ljAB4_d.upload(ab4d.data(), ab4d.size(), s);
    c.lj14AB.upload(ab14.data(), ab14.size(), s);
    c.ljvalid.upload(valid.data(), valid.size(), s);
    c.nbidx.upload(idx.data(), idx.size(), s);
    MDF_CUDA_TRY(cudaStreamSynchronize(s));
}

// Charge-dependent constants: self energy -k alpha / sqrt(pi) sum q^2
// (src/System/NonBondedEnergy.cpp:307-316) and the net charge.
void set_charge_constants(Ctx& c, const double* charge)
{
    long double q2 = 0, qt = 0;
    for (int i = 0; i < c.N; ++i) {
        q2 += (long double)charge[i] * charge[i];
        qt += charge[i];
    }
    c.e_self = (double)(-(long double)c.p.coulomb_const * (c.alpha / std::sqrt(M_PI)) * q2);
    c.q_total = (double)qt;
}

void upload_topology(Ctx& c, const mdf_topology* t)
{
    cudaStream_t s = c.stream;
    if (!t || t->natoms <= 0) throw ApiError(MDF_ERR_INVALID, "topology has no atoms");
    if (!t->charge || !t->type || !t->nb_index || t->ntypes <= 0)
        throw ApiError(MDF_ERR_INVALID, "topology misses charges, types or the nonbonded index");
    // the pair kernels address the (ntypes + 1)^2 table of 32-byte rows with int byte offsets
    if (t->ntypes > 8000) throw ApiError(MDF_ERR_CAPACITY, "more than 8000 atom types");
    c.N = t->natoms;
    c.ntypes = t->ntypes;
    c.ntp = t->ntypes + 1;
    for (int i = 0; i < c.N; ++i)
        if (t->type[i] < 0 || t->type[i] >= t->ntypes) throw ApiError(MDF_ERR_INVALID, "atom type out of range");
    c.n_ljpair = t->n_ljpair;
    c.h_nb_index.assign(t->nb_index, t->nb_index + (size_t)c.ntypes * c.ntypes);
    for (int i = 0; i < c.ntypes; ++i)
        for (int j = 0; j < c.ntypes; ++j) {
            int nb = t->nb_index[i * c.ntypes + j];
            if (nb != t->nb_index[j * c.ntypes + i])
                throw ApiError(MDF_ERR_UNSUPPORTED, "NONBONDED_PARM_INDEX is not symmetric");
            if (nb < 0 || nb > t->n_ljpair) throw ApiError(MDF_ERR_INVALID, "NONBONDED_PARM_INDEX out of range");
        }
    if (t->lj14_a && t->lj14_b) {
        c.h_lj14a.assign(t->lj14_a, t->lj14_a + c.n_ljpair);
        c.h_lj14b.assign(t->lj14_b, t->lj14_b + c.n_ljpair);
    } else {
        c.h_lj14a.assign(t->lj_a, t->lj_a + c.n_ljpair);
        c.h_lj14b.assign(t->lj_b, t->lj_b + c.n_ljpair);
    }
    set_lj_tables(c, t->lj_a, t->lj_b);
    c.q.upload(t->charge, c.N, s);
    c.type.upload(t->type, c.N, s);

    // bonded terms
    auto pack2 = [](int n, const double* a, const double* b) {
        std::vector<double2> v(n);
        for (int i = 0; i < n; ++i) v[i] = make_double2(a[i], b[i]);
        return v;
    };
    c.n_bonds = t->n_bonds; c.n_ub = t->n_ub; c.n_angles = t->n_angles;
    c.n_dih = t->n_dihedrals; c.n_imp = t->n_impropers; c.n_cmap = t->n_cmaps;
    check_index(t->bond_atoms, 2LL * c.n_bonds, c.N, "bonds");
    check_index(t->ub_atoms, 2LL * c.n_ub, c.N, "Urey-Bradley");
    check_index(t->angle_atoms, 3LL * c.n_angles, c.N, "angles");
    check_index(t->dihedral_atoms, 4LL * c.n_dih, c.N, "dihedrals");
    check_index(t->improper_atoms, 4LL * c.n_imp, c.N, "impropers");
    check_index(t->cmap_atoms, 5LL * c.n_cmap, c.N, "CMAP");
    c.bond_atoms.upload(t->bond_atoms, 2 * (size_t)c.n_bonds, s);
    { auto v = pack2(c.n_bonds, t->bond_k, t->bond_r0); c.bond_par.upload(v.data(), v.size(), s); }
    c.ub_atoms.upload(t->ub_atoms, 2 * (size_t)c.n_ub, s);
    { auto v = pack2(c.n_ub, t->ub_k, t->ub_r0); c.ub_par.upload(v.data(), v.size(), s); }
    c.angle_atoms.upload(t->angle_atoms, 3 * (size_t)c.n_angles, s);
    { auto v = pack2(c.n_angles, t->angle_k, t->angle_theta0); c.angle_par.upload(v.data(), v.size(), s); }
    c.dih_atoms.upload(t->dihedral_atoms, 4 * (size_t)c.n_dih, s);
    {
        std::vector<double> v(3 * (size_t)c.n_dih);
        for (int i = 0; i < c.n_dih; ++i) {
            v[3 * i] = t->dihedral_k[i]; v[3 * i + 1] = t->dihedral_n[i]; v[3 * i + 2] = t->dihedral_phase[i];
        }
        c.dih_par.upload(v.data(), v.size(), s);
    }
    c.imp_atoms.upload(t->improper_atoms, 4 * (size_t)c.n_imp, s);
    { auto v = pack2(c.n_imp, t->improper_k, t->improper_phase); c.imp_par.upload(v.data(), v.size(), s); }
    c.cmap_atoms.upload(t->cmap_atoms, 5 * (size_t)c.n_cmap, s);
    c.cmap_set.upload(t->cmap_set, c.n_cmap, s);
    c.cmap_res = t->cmap_res > 0 ? t->cmap_res : 24;
    c.cmap_nsets = t->cmap_nsets;
    for (int i = 0; i < c.n_cmap; ++i)
        if (t->cmap_set[i] < 0 || t->cmap_set[i] >= c.cmap_nsets) throw ApiError(MDF_ERR_INVALID, "CMAP set out of range");
    if (c.n_cmap > 0) {
        if (!t->cmap_coeff) throw ApiError(MDF_ERR_INVALID, "CMAP coefficients missing");
        c.cmap_coeff.upload(t->cmap_coeff, (size_t)c.cmap_nsets * c.cmap_res * c.cmap_res * 16, s);
    }

    // exclusions and 1-4 pairs
    c.n_excl = t->n_excl;
    c.n_14 = t->n_pairs14;
    check_index(t->excl_pairs, 2LL * c.n_excl, c.N, "exclusions");
    check_index(t->pairs14, 2LL * c.n_14, c.N, "1-4 pairs");
    std::vector<int> ex(2 * (size_t)c.n_excl), is14(c.n_excl, 0);
    std::set<std::pair<int, int>> s14;
    for (int i = 0; i < c.n_14; ++i) {
        int a = t->pairs14[2 * i], b = t->pairs14[2 * i + 1];
        s14.insert({std::min(a, b), std::max(a, b)});
    }
    std::set<std::pair<int, int>> sex;
    for (int i = 0; i < c.n_excl; ++i) {
        int a = t->excl_pairs[2 * i], b = t->excl_pairs[2 * i + 1];
        if (a == b) throw ApiError(MDF_ERR_INVALID, "excluded pair of an atom with itself");
        ex[2 * i] = std::min(a, b);
        ex[2 * i + 1] = std::max(a, b);
        is14[i] = s14.count({ex[2 * i], ex[2 * i + 1]}) ? 1 : 0;
        sex.insert({ex[2 * i], ex[2 * i + 1]});
    }
    for (auto& pr : s14)
        if (!sex.count(pr)) throw ApiError(MDF_ERR_INVALID, "1-4 pair missing from the exclusion list");
    c.excl_pairs.upload(ex.data(), ex.size(), s);
    c.excl_is14.upload(is14.data(), is14.size(), s);
    {
        std::vector<int> p(2 * (size_t)c.n_14);
        std::vector<double2> sc(c.n_14);
        for (int i = 0; i < c.n_14; ++i) {
            p[2 * i] = t->pairs14[2 * i];
            p[2 * i + 1] = t->pairs14[2 * i + 1];
            sc[i] = make_double2(t->scee14 ? t->scee14[i] : 1.0, t->scnb14 ? t->scnb14[i] : 1.0);
        }
        c.pairs14.upload(p.data(), p.size(), s);
        c.p14_scale.upload(sc.data(), sc.size(), s);
    }

    set_charge_constants(c, t->charge);

    c.xyz.alloc(3 * (size_t)c.N);
    c.f_atom.alloc(3 * (size_t)c.N);
    c.forces_out.alloc(3 * (size_t)c.N);
    c.scal.alloc(NUM_SCAL);
    c.acc.p = c.scal.p;
    c.npairs_cut.p = c.scal.p + NUM_ACC;
    c.status.p = reinterpret_cast<unsigned*>(c.scal.p + NUM_ACC + 1);
    c.need_clear = true;
    MDF_CUDA_TRY(cudaStreamSynchronize(s));
}

void allreduce_u64(Ctx& c, unsigned long long* d, long long n)
{
    if (!c.allreduce) throw ApiError(MDF_ERR_STATE, "nranks > 1 needs mdf_set_allreduce");
    if (n <= 0) return;
    if (c.allreduce(reinterpret_cast<uint64_t*>(d), (int64_t)n, (void*)c.stream, c.allreduce_user) != 0)
        throw ApiError(MDF_ERR_CUDA, "the allreduce callback failed");
}

void eval_async_impl(Ctx& c, uint32_t flags)
{
    if (!c.have_positions) throw ApiError(MDF_ERR_STATE, "positions not set");
    if (distributed(c) && !c.allreduce) throw ApiError(MDF_ERR_STATE, "nranks > 1 needs mdf_set_allreduce");
    if (!c.have_list) build_pairlist(c);
    cudaStream_t s = c.stream;
    bool energy = (flags & MDF_COMPUTE_ENERGY) != 0;
    bool phys = c.p.semantics == MDF_SEM_PHYSICAL;
    c.nev = 0;
    mark(c, "start");
    if (c.need_clear) {
        // first evaluation on these buffers (later ones are cleared by k_finalize)
        MDF_CUDA_TRY(cudaMemsetAsync(c.f_slot.p, 0, sizeof(unsigned long long) * 3 * (size_t)c.n_slots, s));
        MDF_CUDA_TRY(cudaMemsetAsync(c.f_atom.p, 0, sizeof(unsigned long long) * 3 * (size_t)c.N, s));
        MDF_CUDA_TRY(cudaMemsetAsync(c.scal.p, 0, sizeof(unsigned long long) * NUM_SCAL, s));
        c.need_clear = false;
    }
    // The exclusion, 1-4, bonded and PME kernels only read positions and
    // charges and add into the fixed-point accumulators, so they run on the
    // side stream while the main stream packs, prunes and runs the pair
    // kernel; the main stream waits for them before k_finalize.  With timing enabled every
    // kernel runs on the main stream so the per-phase times are separable.
    const bool want_pme = phys || (flags & MDF_COMPUTE_PME_REFERENCE);
    const bool overlap = want_pme && !c.timing;
    if (overlap) {
        MDF_CUDA_TRY(cudaEventRecord(c.ev_fork, s));
        MDF_CUDA_TRY(cudaStreamWaitEvent(c.side, c.ev_fork, 0));
        c.stream = c.side;
        try {
            launch_exclusions(c, energy);
            launch_bonded(c, energy);
            launch_pme(c, energy);
        } catch (...) {
            c.stream = s;
            throw;
        }
        c.stream = s;
        c.have_pme_ref = !phys;
        MDF_CUDA_TRY(cudaEventRecord(c.ev_join, c.side));
    }
    pack_positions(c);
    mark(c, "pack");
    if (c.p.prune_every > 0) {
        if (!c.pruned_valid || c.since_prune >= c.p.prune_every) {
            prune_pairlist(c);
            c.since_prune = 0;
        }
        ++c.since_prune;
        mark(c, "prune");
    } else if (c.p.prune_every < 0) {
        prune_pairlist(c);   // self-pruning: the kernel returns at once while the last lists hold
        mark(c, "prune");
    }
    launch_nonbonded(c, energy);
    mark(c, "pairs");
    if (!overlap) {
        launch_exclusions(c, energy);
        mark(c, "excl_14");
        launch_bonded(c, energy);
        mark(c, "bonded");
    }
    if (want_pme && !overlap) {
        launch_pme(c, energy);
        c.have_pme_ref = !phys;
    }
    if (overlap) MDF_CUDA_TRY(cudaStreamWaitEvent(s, c.ev_join, 0));
    if (slab_mode(c)) {
        // energies, virial and pair count summed; the forces by reduce-scatter
        // of the accumulators and all-gather of the finished forces
        allreduce_u64(c, c.scal.p, NUM_ACC + 1);
        if (c.counting) allreduce_u64(c, c.npairs_dev.p, 1);
        c.counting = false;
        finish_slab_forces(c, c.forces_out.p);
        mark(c, "finalize");
        c.pending = true;
        c.pending_flags = flags;
        return;
    }
    if (distributed(c)) {
        // every rank's partial forces, energies, virial and pair count, summed
        // (the status word stays per rank)
        allreduce_u64(c, c.f_slot.p, 3LL * c.n_slots);
        allreduce_u64(c, c.f_atom.p, 3LL * c.N);
        allreduce_u64(c, c.scal.p, NUM_ACC + 1);
        if (c.counting) allreduce_u64(c, c.npairs_dev.p, 1);
    }
    c.counting = false;
    launch_finalize(c, c.forces_out.p, false);
    mark(c, "finalize");
    c.pending = true;
    c.pending_flags = flags;
}

static void eval_async(Ctx& c, uint32_t flags)
{
    try {
        eval_async_impl(c, flags);
    } catch (...) {
        c.need_clear = true;
        throw;
    }
}

// Energies of the last finished evaluation from the host copy of its scalar
// block (written by k_finalize into mapped host memory).
void host_energies(const Ctx& c, uint32_t flags, mdf_energies* e_out)
{
    host_energies_from(c, c.h_scal, flags, e_out);
}

void host_energies_from(const Ctx& c, const unsigned long long* hs, uint32_t flags, mdf_energies* e_out)
{
    memset(e_out, 0, sizeof(*e_out));
    if (!(flags & MDF_COMPUTE_ENERGY)) return;
    for (int k = 0; k < MDF_E_COUNT; ++k) e_out->e[k] = (double)(long long)hs[k] * ENERGY_ISCALE;
    e_out->e[MDF_E_EE_SELF] += c.e_self;
    const bool phys = c.p.semantics == MDF_SEM_PHYSICAL;
    if (phys) {
        const double V = c.box[0] * c.box[1] * c.box[2];
        e_out->e[MDF_E_EE_RECIP] += -c.p.coulomb_const * M_PI * c.q_total * c.q_total / (2.0 * V * c.alpha * c.alpha);
        const int vmap[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        for (int k = 0; k < 9; ++k) e_out->virial[k] = (double)(long long)hs[ACC_VIR + vmap[k]] * ENERGY_ISCALE;
        double tot = 0;
        const int terms[] = {MDF_E_BOND, MDF_E_ANGLE, MDF_E_DIHEDRAL, MDF_E_UB, MDF_E_IMPROPER, MDF_E_CMAP,
                             MDF_E_VDW, MDF_E_VDW14, MDF_E_EE_DIRECT, MDF_E_EE14, MDF_E_EE_EXCL,
                             MDF_E_EE_SELF, MDF_E_EE_RECIP};
        for (int k : terms) tot += e_out->e[k];
        e_out->total = tot;
    } else {
        double tot = 0;
        const int terms[] = {MDF_E_BOND, MDF_E_ANGLE, MDF_E_DIHEDRAL, MDF_E_UB, MDF_E_IMPROPER, MDF_E_CMAP,
                             MDF_E_VDW, MDF_E_EE};
        for (int k : terms) tot += e_out->e[k];
        e_out->total = tot;
    }
}

// Status bits of the last finished evaluation, as an exception.
void check_host_status(const Ctx& c)
{
    check_status_word(c.h_scal);
}

void check_status_word(const unsigned long long* hs)
{
    const unsigned st = (unsigned)hs[NUM_ACC + 1];
    if (st & ST_NONFINITE) throw ApiError(MDF_ERR_NONFINITE, "non-finite force or energy contribution");
    if (st & ST_OVERFLOW) throw ApiError(MDF_ERR_OVERFLOW, "fixed-point accumulator range exceeded");
    if (st & ST_STALE)
        throw ApiError(MDF_ERR_STATE, "an atom drifted more than half the skin out of this rank's band since the list "
                                      "build: rebuild the pair list");
}

static void fetch(Ctx& c, double* forces_out, mdf_energies* e_out)
{
    if (!c.pending) throw ApiError(MDF_ERR_STATE, "no evaluation to fetch");
    MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
    check_host_status(c);
    if (c.timing) {
        c.tlast.clear();
        for (int i = 1; i < c.nev; ++i) {
            float ms = 0;
            cudaEventElapsedTime(&ms, c.evpool[i - 1], c.evpool[i]);
            c.tlast.emplace_back(c.evname[i], ms);
        }
    }
    if (e_out) host_energies(c, c.pending_flags, e_out);
    if (forces_out)
        MDF_CUDA_TRY(cudaMemcpy(forces_out, c.forces_out.p, sizeof(double) * 3 * (size_t)c.N, cudaMemcpyDeviceToHost));
}

// Pipelined evaluation: the positions go in on one copy stream (into the
// stage's buffer, then one device copy on the evaluation stream), the
// evaluation runs on the context's stream and writes the stage's forces and
// scalar block, and the forces go out on a second copy stream (so the next
// evaluation's positions never queue behind this one's forces).  With two stages the
// copies of one evaluation overlap the computation of the other.
static void submit(Ctx& c, uint32_t flags, const double* xyz, double* forces_out)
{
    if (c.inflight >= 2) throw ApiError(MDF_ERR_STATE, "two evaluations in flight: collect one first");
    if (distributed(c)) throw ApiError(MDF_ERR_UNSUPPORTED, "not available with nranks > 1");
    const size_t n3 = 3 * (size_t)c.N;
    if (!c.copy) MDF_CUDA_TRY(cudaStreamCreateWithFlags(&c.copy, cudaStreamNonBlocking));
    if (!c.copy_out) MDF_CUDA_TRY(cudaStreamCreateWithFlags(&c.copy_out, cudaStreamNonBlocking));
    Ctx::Stage& S = c.stage[c.stage_next];
    if (!S.h_scal) {
        MDF_CUDA_TRY(cudaHostAlloc((void**)&S.h_scal, sizeof(unsigned long long) * NUM_SCAL, cudaHostAllocMapped));
        memset(S.h_scal, 0, sizeof(unsigned long long) * NUM_SCAL);
        MDF_CUDA_TRY(cudaHostGetDevicePointer((void**)&S.d_hscal, S.h_scal, 0));
        for (cudaEvent_t* e : {&S.h2d, &S.consumed, &S.done, &S.d2h})
            MDF_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    S.xyz.alloc(n3);
    S.forces.alloc(n3);
    // positions in: the stage buffer is free once the stage's last evaluation copied it
    MDF_CUDA_TRY(cudaStreamWaitEvent(c.copy, S.consumed, 0));
    MDF_CUDA_TRY(cudaMemcpyAsync(S.xyz.p, xyz, sizeof(double) * n3, cudaMemcpyHostToDevice, c.copy));
    MDF_CUDA_TRY(cudaEventRecord(S.h2d, c.copy));
    MDF_CUDA_TRY(cudaStreamWaitEvent(c.stream, S.h2d, 0));
    MDF_CUDA_TRY(cudaMemcpyAsync(c.xyz.p, S.xyz.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c.stream));
    MDF_CUDA_TRY(cudaEventRecord(S.consumed, c.stream));
    c.have_positions = true;
    // the evaluation, finalising into the stage (after its last forces left)
    c.fin_forces = S.forces.p;
    c.fin_hscal = S.d_hscal;
    c.fin_wait = S.d2h;
    try {
        eval_async_impl(c, flags);
    } catch (...) {
        c.fin_forces = nullptr; c.fin_hscal = nullptr; c.fin_wait = nullptr;
        c.need_clear = true;
        throw;
    }
    c.fin_forces = nullptr; c.fin_hscal = nullptr; c.fin_wait = nullptr;
    c.pending = false;   // results belong to the stage, not to mdf_fetch
    MDF_CUDA_TRY(cudaEventRecord(S.done, c.stream));
    // forces out
    MDF_CUDA_TRY(cudaStreamWaitEvent(c.copy_out, S.done, 0));
    if (forces_out)
        MDF_CUDA_TRY(cudaMemcpyAsync(forces_out, S.forces.p, sizeof(double) * n3, cudaMemcpyDeviceToHost,
                                     c.copy_out));
    MDF_CUDA_TRY(cudaEventRecord(S.d2h, c.copy_out));
    S.flags = flags;
    c.stage_next ^= 1;
    ++c.inflight;
}

static void collect(Ctx& c, mdf_energies* e_out)
{
    if (c.inflight == 0) throw ApiError(MDF_ERR_STATE, "no submitted evaluation to collect");
    Ctx::Stage& S = c.stage[c.stage_old];
    c.stage_old ^= 1;
    --c.inflight;
    MDF_CUDA_TRY(cudaEventSynchronize(S.d2h));
    check_status_word(S.h_scal);
    if (e_out) host_energies_from(c, S.h_scal, S.flags, e_out);
}

}  // namespace mdf

using namespace mdf;

template <typename F>
static int guarded(mdf_ctx* ctx, F&& f)
{
    try {
        f();
        if (ctx) ctx->c.last_error.clear();
        return MDF_OK;
    } catch (const ApiError& e) {
        if (ctx) ctx->c.last_error = e.msg;
        return e.status;
    } catch (const CudaError& e) {
        if (ctx) ctx->c.last_error = e.msg;
        return MDF_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        if (ctx) ctx->c.last_error = "host allocation failed";
        return MDF_ERR_NOMEM;
    } catch (const std::exception& e) {
        if (ctx) ctx->c.last_error = e.what();
        return MDF_ERR_INVALID;
    }
}

static thread_local std::string g_create_error;

// Live contexts per device; when the last one on a device is destroyed the
// no-allocation entry point forgets that device's scratch address.
static std::mutex g_live_mutex;
static std::map<int, int> g_live;

extern "C" {

void mdf_params_default(mdf_params* p)
{
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->semantics = MDF_SEM_REFERENCE;
    p->precision = MDF_PREC_FP64;
    p->cutoff = 10.0;
    p->skin = 2.0;
    p->switch_radius = 9.0;
    p->ewald_tol = 1e-6;
    p->ewald_alpha = 0.0;
    p->pme_order = 4;
    long double r = 18.2206899283247L;
    p->coulomb_const = (double)(r * r);
    p->device = 0;
    p->prune_every = 1;
    p->prune_margin = 0.0;
}

const char* mdf_status_string(int status)
{
    switch (status) {
        case MDF_OK: return "MDF_OK";
        case MDF_ERR_INVALID: return "MDF_ERR_INVALID";
        case MDF_ERR_CUDA: return "MDF_ERR_CUDA";
        case MDF_ERR_CAPACITY: return "MDF_ERR_CAPACITY";
        case MDF_ERR_NONFINITE: return "MDF_ERR_NONFINITE";
        case MDF_ERR_OVERFLOW: return "MDF_ERR_OVERFLOW";
        case MDF_ERR_TIMEOUT: return "MDF_ERR_TIMEOUT";
        case MDF_ERR_STATE: return "MDF_ERR_STATE";
        case MDF_ERR_NOMEM: return "MDF_ERR_NOMEM";
        case MDF_ERR_UNSUPPORTED: return "MDF_ERR_UNSUPPORTED";
        default: return "MDF_ERR_UNKNOWN";
    }
}

const char* mdf_last_error(const mdf_ctx* ctx)
{
    if (!ctx) return g_create_error.c_str();
    return ctx->c.last_error.c_str();
}

int mdf_create(const mdf_topology* top, const mdf_params* p, mdf_ctx** out)
{
    if (!out || !top || !p) {
        g_create_error = "null argument";
        return MDF_ERR_INVALID;
    }
    *out = nullptr;
    mdf_ctx* ctx = new mdf_ctx();
    int rc = guarded(ctx, [&] {
        Ctx& c = ctx->c;
        c.p = *p;
        if (c.p.semantics != MDF_SEM_REFERENCE && c.p.semantics != MDF_SEM_PHYSICAL)
            throw ApiError(MDF_ERR_INVALID, "unknown semantics");
        if (c.p.precision != MDF_PREC_FP64 && c.p.precision != MDF_PREC_MIXED)
            throw ApiError(MDF_ERR_INVALID, "unknown precision");
        if (!(c.p.cutoff > 0) || c.p.skin < 0) throw ApiError(MDF_ERR_INVALID, "bad cutoff or skin");
        if (c.p.nranks < 0 || (c.p.nranks > 1 && (c.p.rank < 0 || c.p.rank >= c.p.nranks)) ||
            (c.p.nranks <= 1 && c.p.rank != 0))
            throw ApiError(MDF_ERR_INVALID, "rank must lie in [0, nranks)");
        if (c.p.nranks > 1 && c.p.semantics != MDF_SEM_PHYSICAL)
            throw ApiError(MDF_ERR_UNSUPPORTED, "the work split needs PHYSICAL semantics");
        if (c.p.switch_radius > 0 && !(c.p.switch_radius < c.p.cutoff))
            throw ApiError(MDF_ERR_INVALID, "lj_switch must be < lj_cutoff");
        int ndev = 0;
        cudaError_t e = cudaGetDeviceCount(&ndev);
        if (e != cudaSuccess || ndev == 0) throw ApiError(MDF_ERR_CUDA, "no CUDA device available");
        if (c.p.device < 0 || c.p.device >= ndev) throw ApiError(MDF_ERR_INVALID, "device ordinal out of range");
        c.device = c.p.device;
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        MDF_CUDA_TRY(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
        c.own_stream = true;
        {
            // The side stream (exclusions, 1-4, bonded, PME) gets the highest
            // priority: its kernels are short and few-block, and scheduled
            // first they finish inside the pair kernel instead of stretching
            // its tail (c1 mixed: 0.364 vs 0.386 ms per evaluation).
            int lo = 0, hi = 0;
            MDF_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            MDF_CUDA_TRY(cudaStreamCreateWithPriority(&c.side, cudaStreamNonBlocking, hi));
        }
        MDF_CUDA_TRY(cudaEventCreateWithFlags(&c.ev_fork, cudaEventDisableTiming));
        MDF_CUDA_TRY(cudaEventCreateWithFlags(&c.ev_join, cudaEventDisableTiming));
        MDF_CUDA_TRY(cudaHostAlloc((void**)&c.h_scal, sizeof(unsigned long long) * NUM_SCAL, cudaHostAllocMapped));
        memset(c.h_scal, 0, sizeof(unsigned long long) * NUM_SCAL);
        MDF_CUDA_TRY(cudaHostGetDevicePointer((void**)&c.d_hscal, c.h_scal, 0));
        for (int d = 0; d < 3; ++d) c.box[d] = c.p.box[d];
        double tol = c.p.ewald_tol > 0 ? c.p.ewald_tol : 1e-6;
        c.alpha = c.p.ewald_alpha > 0 ? c.p.ewald_alpha : std::sqrt(std::log(2 * tol) * -1) / c.p.cutoff;
        // ewald_tol >= 0.5 gives no splitting parameter; the FP32 pair kernel
        // also relies on exp(-alpha^2 r^2) vanishing at r^2 = 1e30
        if (!(std::isfinite(c.alpha) && c.alpha >= 1e-12))
            throw ApiError(MDF_ERR_INVALID, "Ewald alpha must be finite and >= 1e-12 (ewald_tol in (0, 0.5))");
        upload_topology(c, top);
        if (!(c.box[0] > 0 && c.box[1] > 0 && c.box[2] > 0))
            throw ApiError(MDF_ERR_INVALID, "periodic box required");
        setup_pme(c);
    });
    if (rc != MDF_OK) {
        g_create_error = ctx->c.last_error;
        mdf_destroy(ctx);
        return rc;
    }
    {
        std::lock_guard<std::mutex> lock(g_live_mutex);
        ++g_live[ctx->c.device];
        ctx->c.counted_live = true;
    }
    *out = ctx;
    return MDF_OK;
}

void mdf_destroy(mdf_ctx* ctx)
{
    if (!ctx) return;
    Ctx& c = ctx->c;
    if (c.counted_live) {
        std::lock_guard<std::mutex> lock(g_live_mutex);
        if (--g_live[c.device] == 0) noalloc_forget_device(c.device);
    }
    cudaSetDevice(c.device);
    if (c.stream) cudaStreamSynchronize(c.stream);
    for (auto& e : c.evpool) cudaEventDestroy(e);
    c.q.release(); c.type.release(); c.ljAB.release(); c.ljAB4_f.release(); c.ljAB4_d.release(); c.ljAB_f.release(); c.lj14AB.release(); c.ljvalid.release();
    c.bond_atoms.release(); c.ub_atoms.release(); c.angle_atoms.release(); c.dih_atoms.release();
    c.imp_atoms.release(); c.cmap_atoms.release(); c.cmap_set.release(); c.bond_par.release(); c.ub_par.release();
    c.angle_par.release(); c.imp_par.release(); c.dih_par.release(); c.cmap_coeff.release();
    c.excl_pairs.release(); c.pairs14.release(); c.p14_scale.release(); c.excl_is14.release();
    c.xyz.release(); c.atom_col.release(); c.col_count.release(); c.col_start.release(); c.col_cstart.release();
    c.col_atoms.release(); c.slot_atom.release(); c.atom_slot.release(); c.slot_type.release(); c.center.release(); c.centerf.release();
    c.bb_lo.release(); c.bb_hi.release(); c.xq_f.release(); c.xq_d.release(); c.cluster_col.release();
    c.ilist.release(); c.plist.release(); c.scan_tmp.release(); c.f_slot.release();
    c.plist_in.release(); c.ilist_in.release(); c.cur_lo.release(); c.cur_hi.release(); c.xq_snap.release();
    c.q_slab.release(); c.pme_slab.release(); c.pme_send.release(); c.pme_recv.release(); c.pme_rslab.release();
    c.f_stage.release(); c.f_mine.release(); c.f_out_blk.release(); c.f_out_all.release();
    c.f_atom.release(); c.scal.release(); c.npairs_dev.release(); c.forces_out.release(); c.forces_pme_ref.release();
    c.qgrid.release(); c.cgrid_f.release(); c.cgrid_d.release(); c.rgrid_f.release();
    c.rgrid_d.release(); c.infl_f.release(); c.infl_d.release();
    for (int d = 0; d < 3; ++d) {
        c.tw_d[d].release(); c.tw_f[d].release(); c.fft_tab[d].release(); c.mvec[d].release();
    }
    if (c.h_scal) cudaFreeHost(c.h_scal);
    if (c.h_build) cudaFreeHost(c.h_build);
    for (auto& S : c.stage) {
        if (S.h_scal) cudaFreeHost(S.h_scal);
        for (cudaEvent_t e : {S.h2d, S.consumed, S.done, S.d2h})
            if (e) cudaEventDestroy(e);
        S.xyz.release();
        S.forces.release();
    }
    for (cudaStream_t cs : {c.copy, c.copy_out})
        if (cs) {
            cudaStreamSynchronize(cs);
            cudaStreamDestroy(cs);
        }
    c.d_build.release();
    if (c.md_exec) cudaGraphExecDestroy(c.md_exec);
    if (c.md_graph) cudaGraphDestroy(c.md_graph);
    if (c.md_host) cudaFreeHost(c.md_host);
    c.md_v.release(); c.md_invm.release(); c.md_xref.release(); c.min_x.release(); c.min_f.release(); c.md_words.release();
    if (c.stream && c.own_stream) cudaStreamDestroy(c.stream);
    if (c.side) cudaStreamDestroy(c.side);
    if (c.ev_fork) cudaEventDestroy(c.ev_fork);
    if (c.ev_join) cudaEventDestroy(c.ev_join);
    delete ctx;
}

int mdf_set_positions(mdf_ctx* ctx, const double* xyz)
{
    if (!ctx || !xyz) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        MDF_CUDA_TRY(cudaMemcpyAsync(c.xyz.p, xyz, sizeof(double) * 3 * (size_t)c.N, cudaMemcpyHostToDevice, c.stream));
        c.have_positions = true;
    });
}

int mdf_set_positions_device(mdf_ctx* ctx, const double* d_xyz)
{
    if (!ctx || !d_xyz) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        MDF_CUDA_TRY(cudaMemcpyAsync(c.xyz.p, d_xyz, sizeof(double) * 3 * (size_t)c.N, cudaMemcpyDeviceToDevice,
                                     c.stream));
        c.have_positions = true;
    });
}

int mdf_set_box(mdf_ctx* ctx, const double box[3])
{
    if (!ctx || !box) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        for (int d = 0; d < 3; ++d) {
            if (!(box[d] > 0)) throw ApiError(MDF_ERR_INVALID, "box lengths must be positive");
            c.box[d] = box[d];
            c.p.box[d] = box[d];
        }
        c.have_list = false;
        setup_pme(c);
    });
}

int mdf_build_pairlist(mdf_ctx* ctx)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        if (!c.have_positions) throw ApiError(MDF_ERR_STATE, "positions not set");
        build_pairlist(c);
    });
}

int mdf_compute_async(mdf_ctx* ctx, uint32_t flags)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        MDF_CUDA_TRY(cudaSetDevice(ctx->c.device));
        eval_async(ctx->c, flags);
    });
}

int mdf_fetch(mdf_ctx* ctx, double* forces_out, mdf_energies* e_out)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        MDF_CUDA_TRY(cudaSetDevice(ctx->c.device));
        fetch(ctx->c, forces_out, e_out);
    });
}

int mdf_submit(mdf_ctx* ctx, uint32_t flags, const double* xyz, double* forces_out)
{
    if (!ctx || !xyz) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        MDF_CUDA_TRY(cudaSetDevice(ctx->c.device));
        submit(ctx->c, flags, xyz, forces_out);
    });
}

int mdf_collect(mdf_ctx* ctx, mdf_energies* e_out)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        MDF_CUDA_TRY(cudaSetDevice(ctx->c.device));
        collect(ctx->c, e_out);
    });
}

int mdf_compute(mdf_ctx* ctx, uint32_t flags, double* forces_out, mdf_energies* e_out)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        eval_async(c, flags);
        // the force copy joins the evaluation's stream: one synchronisation for both
        if (forces_out)
            MDF_CUDA_TRY(cudaMemcpyAsync(forces_out, c.forces_out.p, sizeof(double) * 3 * (size_t)c.N,
                                         cudaMemcpyDeviceToHost, c.stream));
        fetch(c, nullptr, e_out);
    });
}

int mdf_forces_device(mdf_ctx* ctx, double* d_forces_out)
{
    if (!ctx || !d_forces_out) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        MDF_CUDA_TRY(cudaMemcpyAsync(d_forces_out, c.forces_out.p, sizeof(double) * 3 * (size_t)c.N,
                                     cudaMemcpyDeviceToDevice, c.stream));
    });
}

int mdf_pme_grids(mdf_ctx* ctx, int32_t grid_out[3], double* charge_grid, double* potential_grid)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        if (grid_out)
            for (int d = 0; d < 3; ++d) grid_out[d] = c.K[d];
        if (!charge_grid && !potential_grid) return;
        if (!c.pending) throw ApiError(MDF_ERR_STATE, "no evaluation yet");
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
        const size_t n = (size_t)c.K[0] * c.K[1] * c.K[2];
        if (charge_grid) {
            std::vector<long long> q(n);
            MDF_CUDA_TRY(cudaMemcpy(q.data(), c.qgrid.p, sizeof(long long) * n, cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n; ++i) charge_grid[i] = (double)q[i] * GRID_ISCALE;
        }
        if (potential_grid) {
            if (c.rgrid_f.p) {
                std::vector<float> r(n);
                MDF_CUDA_TRY(cudaMemcpy(r.data(), c.rgrid_f.p, sizeof(float) * n, cudaMemcpyDeviceToHost));
                for (size_t i = 0; i < n; ++i) potential_grid[i] = r[i];
            } else {
                MDF_CUDA_TRY(cudaMemcpy(potential_grid, c.rgrid_d.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
            }
        }
    });
}

int mdf_get_pme_forces(mdf_ctx* ctx, double* forces_out)
{
    if (!ctx || !forces_out) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        if (!c.have_pme_ref) throw ApiError(MDF_ERR_STATE, "no reference PME evaluation available");
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
        MDF_CUDA_TRY(cudaMemcpy(forces_out, c.forces_pme_ref.p, sizeof(double) * 3 * (size_t)c.N,
                                cudaMemcpyDeviceToHost));
    });
}

int mdf_set_stream(mdf_ctx* ctx, void* stream)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
        if (c.own_stream && c.stream) cudaStreamDestroy(c.stream);
        if (stream) {
            c.stream = (cudaStream_t)stream;
            c.own_stream = false;
        } else {
            MDF_CUDA_TRY(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
            c.own_stream = true;
        }
    });
}

int mdf_pairlist_info(mdf_ctx* ctx, int64_t* n_clusters, int64_t* n_cluster_pairs, int64_t* n_cluster_pairs_pruned,
                      int64_t* n_pairs_in_cutoff)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        if (n_clusters) *n_clusters = c.have_list ? c.n_clusters : -1;
        if (n_cluster_pairs) *n_cluster_pairs = c.have_list ? c.n_entries : -1;
        if (n_cluster_pairs_pruned) {
            // entries the pair kernel walks: the counts of the last prune's item ranges
            long long v = 0;
            const bool ok = c.have_list && c.pruned_valid && c.p.prune_every != 0;
            if (ok) {
                long long lo, hi;
                cluster_share(c, lo, hi);
                const bool half = c.pruned_half;
                const size_t n = (size_t)(hi - lo) * (half ? 2 : 1);
                std::vector<ILRange> r(n);
                MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
                if (n)
                    MDF_CUDA_TRY(cudaMemcpy(r.data(), half ? c.ilist_h.p + 2 * lo : c.ilist_in.p + lo,
                                            sizeof(ILRange) * n, cudaMemcpyDeviceToHost));
                for (const ILRange& x : r) v += x.count;
            }
            *n_cluster_pairs_pruned = ok ? (int64_t)v : -1;
        }
        if (n_pairs_in_cutoff) {
            unsigned long long v = 0;
            const bool ok = c.have_list && c.counted;
            if (ok) {
                MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
                MDF_CUDA_TRY(cudaMemcpy(&v, c.npairs_dev.p, sizeof(v), cudaMemcpyDeviceToHost));
            }
            *n_pairs_in_cutoff = ok ? (int64_t)v : -1;
        }
    });
}

int mdf_set_parameters(mdf_ctx* ctx, const double* charge, const double* lj_a, const double* lj_b)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
        if ((lj_a == nullptr) != (lj_b == nullptr)) throw ApiError(MDF_ERR_INVALID, "give both lj_a and lj_b or neither");
        if (charge) {
            for (int i = 0; i < c.N; ++i)
                if (!std::isfinite(charge[i])) throw ApiError(MDF_ERR_INVALID, "non-finite charge");
            c.q.upload(charge, c.N, c.stream);
            set_charge_constants(c, charge);
        }
        if (lj_a) {
            for (int k = 0; k < c.n_ljpair; ++k)
                if (!std::isfinite(lj_a[k]) || !std::isfinite(lj_b[k]))
                    throw ApiError(MDF_ERR_INVALID, "non-finite LJ coefficient");
            set_lj_tables(c, lj_a, lj_b);
        }
        MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
    });
}

int mdf_backward(mdf_ctx* ctx, const double* dL_dF, double dL_dE, double* dL_dq, double* dL_dA, double* dL_dB)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        if (distributed(ctx->c)) throw ApiError(MDF_ERR_UNSUPPORTED, "not available with nranks > 1");
        Ctx& c = ctx->c;
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        backward(c, dL_dF, dL_dE, dL_dq, dL_dA, dL_dB);
    });
}

int mdf_autotune(mdf_ctx* ctx, int reps, mdf_tune_report* rep)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        if (distributed(c)) throw ApiError(MDF_ERR_UNSUPPORTED, "not available with nranks > 1");
        if (!c.have_positions) throw ApiError(MDF_ERR_STATE, "positions not set");
        if (!c.have_list) build_pairlist(c);
        const int R = reps > 0 ? reps : 5;
        const uint32_t flags = MDF_COMPUTE_ENERGY | MDF_COMPUTE_FORCES;
        const int warps[3] = {2, 4, 8}, lines[4] = {2, 4, 8, 16}, prune[2] = {0, 1}, sched[2] = {0, 1};
        const bool timing = c.timing;
        c.timing = false;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        try {
            MDF_CUDA_TRY(cudaEventCreate(&e0));
            MDF_CUDA_TRY(cudaEventCreate(&e1));
            auto apply = [&](int w, int l, int p, int sc, int ly) {
                c.p.pair_warps = w;
                c.p.fft_lines = l;
                c.p.pair_schedule = sc;
                if (c.p.prune_every != p || c.p.pair_layout != ly) {
                    c.p.prune_every = p;
                    c.p.pair_layout = ly;
                    c.pruned_valid = false;
                    c.since_prune = 0;
                }
            };
            auto time_it = [&]() {
                eval_async(c, flags);   // untimed: first use of this shape
                MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
                check_host_status(c);
                MDF_CUDA_TRY(cudaEventRecord(e0, c.stream));
                for (int r = 0; r < R; ++r) eval_async(c, flags);
                MDF_CUDA_TRY(cudaEventRecord(e1, c.stream));
                MDF_CUDA_TRY(cudaEventSynchronize(e1));
                check_host_status(c);
                float ms = 0;
                MDF_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
                return (double)ms / R;
            };
            const int w0 = c.p.pair_warps, l0 = c.p.fft_lines, p0 = c.p.prune_every, s0 = c.p.pair_schedule,
                      y0 = c.p.pair_layout;
            const double t_default = time_it();
            double best = t_default;
            int bw = w0, bl = l0, bp = p0, bs = s0, by = y0, tried = 0;
            // a self-pruning context (prune_every < 0) keeps that mode
            const int prune_self[1] = {c.p.prune_every};
            const int* popts = c.p.prune_every < 0 ? prune_self : prune;
            const int np = c.p.prune_every < 0 ? 1 : 2;
            for (int sc : sched)
                for (int pi = 0; pi < np; ++pi)
                    for (int ly = 0, p = popts[pi]; ly <= (p != 0 ? 1 : 0); ++ly)   // half layout: pruned lists only
                        for (int w : warps)
                            for (int l : lines) {
                                apply(w, l, p, sc, ly);
                                const double t = time_it();
                                ++tried;
                                if (t < best) {
                                    best = t;
                                    bw = w; bl = l; bp = p; bs = sc; by = ly;
                                }
                            }
            apply(bw, bl, bp, bs, by);
            if (rep) {
                rep->pair_warps = bw;
                rep->fft_lines = bl;
                rep->prune_every = bp;
                rep->pair_schedule = bs;
                rep->pair_layout = by;
                rep->n_tried = tried;
                rep->best_ms = best;
                rep->default_ms = t_default;
            }
        } catch (...) {
            c.timing = timing;
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            throw;
        }
        c.timing = timing;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        c.pending = false;
        c.md_stale = true;   // a recorded dynamics graph holds the old shapes
    });
}

int mdf_set_collectives(mdf_ctx* ctx, mdf_reduce_scatter_u64 reduce_scatter, mdf_allgather_bytes allgather,
                        mdf_alltoall_bytes alltoall, void* user)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        const bool all = reduce_scatter && allgather && alltoall, none = !reduce_scatter && !allgather && !alltoall;
        if (!all && !none) throw ApiError(MDF_ERR_INVALID, "give all three collectives or none");
        ctx->c.coll_rs = reduce_scatter;
        ctx->c.coll_ag = allgather;
        ctx->c.coll_a2a = alltoall;
        ctx->c.coll_user = user;
    });
}

int mdf_set_halo_exchange(mdf_ctx* ctx, mdf_alltoallv_bytes alltoallv, void* user)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        ctx->c.coll_a2av = alltoallv;
        ctx->c.coll_a2av_user = user;
    });
}

int mdf_set_allreduce(mdf_ctx* ctx, mdf_allreduce_u64 fn, void* user)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        ctx->c.allreduce = fn;
        ctx->c.allreduce_user = user;
    });
}

int mdf_minimize(mdf_ctx* ctx, int32_t max_iter, double fmax_tol, double max_step, mdf_min_report* report)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        if (distributed(ctx->c)) throw ApiError(MDF_ERR_UNSUPPORTED, "not available with nranks > 1");
        MDF_CUDA_TRY(cudaSetDevice(ctx->c.device));
        minimize(ctx->c, max_iter, fmax_tol, max_step, report);
    });
}

int mdf_minimize_lbfgs(mdf_ctx* ctx, int32_t max_iter, double fmax_tol, double max_step, int32_t history,
                       mdf_min_report* report)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        if (distributed(ctx->c)) throw ApiError(MDF_ERR_UNSUPPORTED, "not available with nranks > 1");
        MDF_CUDA_TRY(cudaSetDevice(ctx->c.device));
        minimize_lbfgs(ctx->c, max_iter, fmax_tol, max_step, history, report);
    });
}

int mdf_md_init(mdf_ctx* ctx, const double* masses, const double* velocities, double temperature, uint64_t seed)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        if (distributed(ctx->c)) throw ApiError(MDF_ERR_UNSUPPORTED, "not available with nranks > 1");
        MDF_CUDA_TRY(cudaSetDevice(ctx->c.device));
        md_init(ctx->c, masses, velocities, temperature, seed);
    });
}

int mdf_md_run(mdf_ctx* ctx, int64_t nsteps, double dt_ps, int32_t chunk, int32_t rebuild_every, double* samples,
               int64_t cap, mdf_md_report* report)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        if (distributed(ctx->c)) throw ApiError(MDF_ERR_UNSUPPORTED, "not available with nranks > 1");
        MDF_CUDA_TRY(cudaSetDevice(ctx->c.device));
        md_run(ctx->c, nsteps, dt_ps, chunk, rebuild_every, samples, cap, report);
    });
}

int mdf_md_state(mdf_ctx* ctx, double* xyz, double* velocities)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        MDF_CUDA_TRY(cudaSetDevice(ctx->c.device));
        md_state(ctx->c, xyz, velocities);
    });
}

int mdf_md_write_rst7(mdf_ctx* ctx, const char* path, const char* title, double time_ps)
{
    if (!ctx) return MDF_ERR_INVALID;
    return guarded(ctx, [&] {
        MDF_CUDA_TRY(cudaSetDevice(ctx->c.device));
        md_write_rst7(ctx->c, path, title, time_ps);
    });
}

int64_t mdf_kernel_launches(const mdf_ctx* ctx)
{
    return ctx ? (int64_t)ctx->c.launches : -1;
}

int mdf_enable_timing(mdf_ctx* ctx, int enable)
{
    if (!ctx) return MDF_ERR_INVALID;
    ctx->c.timing = enable != 0;
    return MDF_OK;
}

int mdf_kernel_times(mdf_ctx* ctx, const char** names, float* ms, int max_entries)
{
    if (!ctx) return 0;
    int n = 0;
    for (auto& t : ctx->c.tlast) {
        if (n >= max_entries) break;
        if (names) names[n] = t.first;
        if (ms) ms[n] = t.second;
        ++n;
    }
    return n;
}

}  // extern "C"
