// Internal declarations shared by the libmdf translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/mdf.h"

namespace mdf {

// ---------------------------------------------------------------- constants
constexpr int CLUSTER = 8;                 // atoms per cluster
constexpr double FORCE_SCALE = 4294967296.0;          // 2^32 fixed point for forces
constexpr double FORCE_ISCALE = 1.0 / 4294967296.0;
constexpr double ENERGY_SCALE = 4294967296.0;         // 2^32 fixed point for energies
constexpr double ENERGY_ISCALE = 1.0 / 4294967296.0;
constexpr double GRID_SCALE = 1099511627776.0;        // 2^40 fixed point for PME charge grid
constexpr double GRID_ISCALE = 1.0 / 1099511627776.0;
constexpr int NUM_ACC = MDF_E_COUNT + 6;   // energies + 6 virial components
constexpr int ACC_VIR = MDF_E_COUNT;
constexpr int NUM_SCAL = NUM_ACC + 4;      // + pairs in cutoff + status word + pair-kernel work counter + displacement
constexpr int SCAL_WORK = NUM_ACC + 2;     // work counter of the persistent pair kernels (cleared with the block)
constexpr int SCAL_DISP = NUM_ACC + 3;     // largest squared displacement since the last prune (FP32 bits; self-pruning mode)

// device status bits
enum : unsigned {
    ST_NONFINITE = 1u,
    ST_OVERFLOW = 2u,
    ST_CAPACITY_PAIRS = 4u,
    ST_CAPACITY_COLUMN = 8u,
    ST_BAD_INDEX = 16u,
    ST_STALE = 32u,   // an atom left its rank's band (halo exchange): the list needs a rebuild
};

struct PairEntry {          // one cluster pair of the half list (16 B)
    int j;                  // j cluster
    int shift;              // periodic image code (sx+1) + 3 (sy+1) + 9 (sz+1)
    unsigned long long mask;  // bit (ii*8 + jj): atom pair interacts
};

struct ILRange {            // one i cluster's span of entries
    int i;
    int start;
    int count;
    int pad;
};

// --------------------------------------------------------------- utilities
#define MDF_CUDA_TRY(expr)                                                          \
    do {                                                                            \
        cudaError_t _e = (expr);                                                    \
        if (_e != cudaSuccess) {                                                    \
            throw mdf::CudaError(_e, #expr, __FILE__, __LINE__);                    \
        }                                                                           \
    } while (0)

struct CudaError {
    cudaError_t err;
    std::string msg;
    CudaError(cudaError_t e, const char* what, const char* file, int line);
};

struct ApiError {
    int status;
    std::string msg;
    ApiError(int s, std::string m) : status(s), msg(std::move(m)) {}
};

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        if (count <= n && p) return;
        // a buffer that has to grow (pair lists, slots after a rebuild) gets
        // 1/8 headroom, so lists that creep up between rebuilds do not pay a
        // cudaFree + cudaMalloc at every build
        if (p) count += count / 8;
        release();
        size_t bytes = count * sizeof(T);
        if (bytes == 0) bytes = sizeof(T);
        MDF_CUDA_TRY(cudaMalloc((void**)&p, bytes));
        n = count;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    template <typename U>
    void upload(const U* host, size_t count, cudaStream_t s) {
        alloc(count);
        if (count) MDF_CUDA_TRY(cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
};

// Non-owning view into a DevBuf.
template <typename T>
struct DevView {
    T* p = nullptr;
};

// ----------------------------------------------------------- PME plan bits
struct FFTPlan1D {
    int n = 0;
    int nstages = 0;
    int radix[12];
    int ns[12];     // product of the radices before stage s
    int toff[12];   // offset of stage s in the per-butterfly index table
    int ntab = 0;   // entries of the index table
};

// --------------------------------------------------------------- context
struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t side = nullptr;         // the PME chain runs here, concurrently with the pair kernel
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    mdf_params p{};
    int N = 0;
    int ntypes = 0;
    std::string last_error;

    // topology on device
    DevBuf<double> q;          // [N]
    DevBuf<int> type;          // [N]
    DevBuf<double2> ljAB;      // [(ntypes+1)^2] pair table (A,B); last row/col = padding type
    DevBuf<float2> ljAB_f;
    DevBuf<float4> ljAB4_f;        // (A, B, 12A, 6B) per type pair, FP32 pair kernel
    DevBuf<double4> ljAB4_d;       // the same in FP64 (FP64 PHYSICAL pair kernel)
    DevBuf<double2> lj14AB;    // same indexing, 1-4 tables
    DevBuf<int> ljvalid;       // [(ntypes+1)^2] nb != 0
    int ntp = 0;               // ntypes + 1 (padding type appended)
    int n_ljpair = 0;
    std::vector<int> h_nb_index;         // [ntypes^2] NONBONDED_PARM_INDEX (host copy)
    std::vector<double> h_lj14a, h_lj14b;  // [n_ljpair] 1-4 coefficients (host copy)
    DevBuf<int> nbidx;                   // [(ntypes+1)^2] 0-based LJ entry of a type pair, -1 = none

    int n_bonds = 0, n_ub = 0, n_angles = 0, n_dih = 0, n_imp = 0, n_cmap = 0;
    DevBuf<int> bond_atoms, ub_atoms, angle_atoms, dih_atoms, imp_atoms, cmap_atoms, cmap_set;
    DevBuf<double2> bond_par, ub_par, angle_par, imp_par;
    DevBuf<double> dih_par;    // 3 per term
    DevBuf<double> cmap_coeff;
    int cmap_res = 24, cmap_nsets = 0;

    int n_excl = 0, n_14 = 0;
    DevBuf<int> excl_pairs, pairs14;
    DevBuf<double2> p14_scale;     // (scee, scnb)
    DevBuf<int> excl_is14;         // per excluded pair: 1 if it is a 1-4 pair

    double e_self = 0.0;           // constant for fixed charges
    double q_total = 0.0;

    // positions
    DevBuf<double> xyz;            // [3N] raw as given
    bool have_positions = false;
    double box[3] = {0, 0, 0};

    // clusters / pairlist
    int ncol_x = 0, ncol_y = 0, ncols = 0;
    int n_clusters = 0, n_slots = 0;
    bool have_list = false;
    DevBuf<int> atom_col;          // [N]
    DevBuf<int> col_count, col_start, col_cstart;   // [ncols + 1]
    DevBuf<int> col_atoms;         // [N] atoms bucketed by column
    DevBuf<int> slot_atom;         // [n_slots]
    DevBuf<int> atom_slot;         // [N]
    DevBuf<int> slot_type;         // [n_slots]
    DevBuf<double4> center;        // [n_clusters] (x,y,z,n_real_atoms) cluster centre
    DevBuf<float4> centerf;        // the same centres, exact in FP32 (they lie on a 2^-k grid)
    double center_quantum = 0.0;
    DevBuf<float4> bb_lo, bb_hi;   // [n_clusters] bounding boxes (wrapped coordinates)
    DevBuf<float4> cur_lo, cur_hi; // [n_clusters] current boxes in the cluster frame (per evaluation)
    DevBuf<float4> xq_f;           // [n_slots] offset from center + q (mixed)
    DevBuf<double4> xq_d;          // [n_slots] (FP64)
    DevBuf<int> cluster_col;       // [n_clusters]
    DevBuf<ILRange> ilist;         // [n_clusters]
    DevBuf<PairEntry> plist;       // [cap] outer list (cutoff + skin)
    long long n_entries = 0;
    DevBuf<PairEntry> plist_in;    // pruned list the pair kernel walks (same offsets as plist)
    DevBuf<ILRange> ilist_in;
    DevBuf<ILRange> ilist_h;       // half layout: [2 n_clusters] items (ILRange.pad = half)
    DevBuf<PairEntry> plist_h;     // half layout: [2 x outer capacity]
    bool pruned_half = false;      // the last prune wrote the half lists
    DevBuf<unsigned char> xq_snap; // self-pruning mode: the cluster-frame positions of the last prune, per slot
    int since_prune = 0;
    bool pruned_valid = false;
    DevBuf<int> scan_tmp;
    DevBuf<int> d_build;           // [4] list entries claimed by the search
    int* h_build = nullptr;        // pinned: cluster count, entry count, status of the last build

    // accumulators.  The force accumulators are cleared by the kernel that
    // reads them (k_finalize); the scalar block is copied to the host and then
    // cleared by k_finalize too, so an evaluation needs no memsets.
    DevBuf<unsigned long long> f_slot;   // [3 * n_slots] fixed point, SoA x|y|z
    DevBuf<unsigned long long> f_atom;   // [3 * N]
    DevBuf<unsigned long long> scal;     // [NUM_SCAL]: energies + virial | pairs in cutoff | status
    DevView<unsigned long long> acc;     // = scal[0 .. NUM_ACC)
    DevView<unsigned long long> npairs_cut;  // = scal[NUM_ACC] (unused word)
    DevBuf<unsigned long long> npairs_dev;   // [1] atom pairs within the cutoff (first evaluation after a build)
    bool count_next = false;             // the next evaluation counts them
    bool counted = false;                // npairs_dev holds a count for the current list
    bool counting = false;               // this evaluation counts (its count is summed over ranks)
    DevView<unsigned> status;            // = (unsigned*)&scal[NUM_ACC + 1]
    DevBuf<double> forces_out;           // [3N]
    DevBuf<double> forces_pme_ref;       // [3N]
    unsigned long long* h_scal = nullptr;  // mapped pinned copy of scal, written by k_finalize
    unsigned long long* d_hscal = nullptr; // its device address
    bool need_clear = true;              // accumulators not known to be zero

    // PME
    int K[3] = {0, 0, 0};
    int order = 4;
    double alpha = 0.0;
    DevBuf<unsigned long long> qgrid;    // [K0*K1*K2] fixed point
    DevBuf<float2> cgrid_f;              // [K0*K1*(K2/2+1)]
    DevBuf<double2> cgrid_d;
    DevBuf<float> rgrid_f;               // [K0*K1*K2] potential
    DevBuf<double> rgrid_d;
    DevBuf<double2> tw_d[3];             // twiddles per dimension
    DevBuf<float2> tw_f[3];
    FFTPlan1D plan[3];
    DevBuf<int2> fft_tab[3];             // per-butterfly (twiddle step, output index) per dimension
    DevBuf<float> infl_f;                // influence function [ky][kz][kx] (mixed)
    DevBuf<double> infl_d;               // influence function [ky][kz][kx] (FP64 / reference solve)
    DevBuf<double> mvec[3];              // m_d = signed frequency / L_d per grid index
    bool have_pme_ref = false;           // forces_pme_ref holds the reference chain's forces

    // adjoint (mdf_backward)
    DevBuf<double> adj_v;                // [3N] dL/dF, atom order, normalised
    DevBuf<float4> adj_vs_f;             // [n_slots] the same per slot (mixed)
    DevBuf<double4> adj_vs_d;            // [n_slots] (FP64)
    DevBuf<unsigned long long> adj_dq_slot, adj_dq_atom;   // fixed-point dL/dq
    DevBuf<double> adj_dab;              // [2 n_ljpair] dL/dA | dL/dB
    DevBuf<double> adj_dq;               // [N] dL/dq out

    // dynamics and minimiser (md.cu)
    DevBuf<double> md_v;                 // [3N] velocities, A/ps
    DevBuf<double> md_invm;              // [N] 418.4 / mass (0 = frozen)
    DevBuf<double> md_xref;              // [3N] positions at the last list build
    DevBuf<double> min_x, min_f;         // minimiser: positions and forces before the trial move
    DevBuf<double> lb_s, lb_y;           // L-BFGS history [m][3N] (position and gradient differences)
    DevBuf<double> lb_q, lb_part, lb_scal;   // two-loop vector, dot partials, recursion scalars
    unsigned long long* md_host = nullptr;   // mapped host copy of the reduction words (see md.cu)
    unsigned long long* md_hmap = nullptr;   // its device address
    DevBuf<unsigned long long> md_words; // the reduction words in device memory
    unsigned long long* md_dev = nullptr;    // = md_words.p
    unsigned* md_dev_st = nullptr;
    bool md_ready = false;
    mdf_allreduce_u64 allreduce = nullptr;   // sum over ranks (nranks > 1)
    void* allreduce_user = nullptr;
    // distributed reciprocal space and force return (mdf_set_collectives)
    mdf_reduce_scatter_u64 coll_rs = nullptr;
    mdf_allgather_bytes coll_ag = nullptr;
    mdf_alltoall_bytes coll_a2a = nullptr;
    void* coll_user = nullptr;
    DevBuf<unsigned long long> q_slab;       // this rank's planes of the charge grid [K0p][K1][K2]
    DevBuf<unsigned char> pme_slab;          // complex slab [K0p][K1][Kc] (float2 / double2)
    DevBuf<unsigned char> pme_send, pme_recv;   // transpose blocks [nranks][K0p][K1p][Kc]
    DevBuf<unsigned char> pme_rslab;         // real potential slab [K0p][K1][K2]
    // Bands of a split evaluation (set by the list build, nranks > 1): rank r
    // owns the i clusters [band_cl[r], band_cl[r+1]), the x-columns whose
    // centres lie in its x-slab of the PME grid.  Its atoms' spread stencils
    // start at grid planes (base) within win_lo[r] .. win_lo[r] + win_n[r] - 1
    // (mod K0) while no atom drifted more than half the skin.
    std::vector<long long> band_cl;
    std::vector<int> win_lo, win_n;
    // halo exchange of grid planes (mdf_set_halo_exchange): this rank's
    // planes sent to / received from each rank (absolute plane indexes,
    // concatenated in rank order), the planes of its own window inside its
    // slab, and the window's plane ranges (at most two after wrapping)
    mdf_alltoallv_bytes coll_a2av = nullptr;
    void* coll_a2av_user = nullptr;
    DevBuf<int> halo_send_pl, halo_recv_pl, halo_local_pl;
    std::vector<int64_t> halo_send_n, halo_recv_n;   // planes per rank
    int halo_n_send = 0, halo_n_recv = 0, halo_n_local = 0;
    int halo_rng[2][2] = {{0, 0}, {0, 0}};           // (first plane, count) of the window
    std::vector<int64_t> halo_bytes_a, halo_bytes_b;  // per-rank byte counts of the current exchange
    DevBuf<unsigned char> halo_sendbuf, halo_recvbuf;
    DevBuf<unsigned long long> f_stage;      // force blocks for the reduce-scatter [nranks][3][Sb]
    DevBuf<unsigned long long> f_mine;       // this rank's block [3][Sb]
    DevBuf<double> f_out_blk, f_out_all;     // finished forces: this rank's slots [Sb][3], all slots [nranks*Sb][3]
    cudaGraph_t md_graph = nullptr;
    cudaGraphExec_t md_exec = nullptr;
    int md_graph_steps = 0;
    double md_graph_dt = 0.0;
    bool md_stale = false;               // list rebuilt since the graph was recorded

    // timing
    bool timing = false;
    std::vector<cudaEvent_t> evpool;          // reused timing events
    std::vector<const char*> evname;
    int nev = 0;
    std::vector<std::pair<const char*, float>> tlast;
    long long launches = 0;                   // kernels launched by evaluations

    bool counted_live = false;           // counted in the per-device live-context table

    // pipelined evaluations (mdf_submit / mdf_collect): two stages, each with
    // its staged positions, its forces, its mapped scalar block and events
    struct Stage {
        DevBuf<double> xyz;                      // positions copied in on the copy stream
        DevBuf<double> forces;                   // this stage's evaluation writes its forces here
        unsigned long long* h_scal = nullptr;    // mapped pinned scalar block of this stage
        unsigned long long* d_hscal = nullptr;
        cudaEvent_t h2d = nullptr, consumed = nullptr, done = nullptr, d2h = nullptr;
        uint32_t flags = 0;
    };
    cudaStream_t copy = nullptr;         // host -> device copies of the pipelined path
    cudaStream_t copy_out = nullptr;     // device -> host copies (its own stream, so the next
                                         // evaluation's positions need not wait behind them)
    Stage stage[2];
    int stage_next = 0, stage_old = 0, inflight = 0;
    double* fin_forces = nullptr;              // k_finalize targets for this evaluation (nullptr: the defaults)
    unsigned long long* fin_hscal = nullptr;
    cudaEvent_t fin_wait = nullptr;            // event the stream waits for before k_finalize

    // last evaluation bookkeeping
    bool pending = false;
    uint32_t pending_flags = 0;
};

// ------------------------------------------------------ launch helpers (.cu)
void upload_topology(Ctx& c, const mdf_topology* t);
void set_lj_tables(Ctx& c, const double* lj_a, const double* lj_b);
void set_charge_constants(Ctx& c, const double* charge);
void md_init(Ctx& c, const double* masses, const double* vel, double temperature, uint64_t seed);
void md_run(Ctx& c, long long nsteps, double dt, int chunk, int rebuild_every, double* samples, long long cap,
            mdf_md_report* rep);
void md_state(Ctx& c, double* xyz, double* vel);
void md_write_rst7(Ctx& c, const char* path, const char* title, double time_ps);
void minimize(Ctx& c, int max_iter, double fmax_tol, double max_step, mdf_min_report* rep);
void minimize_lbfgs(Ctx& c, int max_iter, double fmax_tol, double max_step, int history, mdf_min_report* rep);
void backward(Ctx& c, const double* dL_dF, double dL_dE, double* dL_dq, double* dL_dA, double* dL_dB);
void pme_adjoint(Ctx& c, double gE, double vscale);
void build_pairlist(Ctx& c);
void build_bands(Ctx& c);   // rank bands and halo plane lists of a split evaluation
void pack_positions(Ctx& c);
void prune_pairlist(Ctx& c, bool whole_entries = false);
// half-entry lists in use by the pair kernel (layout 1, pruned)
inline bool half_layout(const Ctx& c) { return c.p.pair_layout == 1 && c.p.prune_every != 0; }
// prune_every < 0: the device prunes when an atom moved more than prune_margin / 2
// since the last prune (one context per system; with several ranks it prunes every evaluation)
inline bool self_pruning(const Ctx& c) { return c.p.prune_every < 0 && c.p.nranks <= 1 && c.xq_snap.p != nullptr; }
void launch_nonbonded(Ctx& c, bool energy);
void launch_exclusions(Ctx& c, bool energy);
void launch_bonded(Ctx& c, bool energy);
void launch_bonded_into(Ctx& c, bool energy, unsigned long long* f, unsigned long long* acc, unsigned* st);
void setup_pme(Ctx& c);
void launch_pme(Ctx& c, bool energy);
void launch_finalize(Ctx& c, double* d_forces, bool pme_ref);
void mark(Ctx& c, const char* name);
void eval_async_impl(Ctx& c, uint32_t flags);
void host_energies(const Ctx& c, uint32_t flags, mdf_energies* e_out);
void host_energies_from(const Ctx& c, const unsigned long long* hs, uint32_t flags, mdf_energies* e_out);
void check_host_status(const Ctx& c);
void check_status_word(const unsigned long long* hs);
void noalloc_forget_device(int device);

int grid_blocks(long long n, int threads);

// This rank's share [lo, hi) of n items (the whole range with one rank).
inline void rank_slice(const Ctx& c, long long n, long long& lo, long long& hi)
{
    const long long P = c.p.nranks > 1 ? c.p.nranks : 1, r = P > 1 ? c.p.rank : 0;
    lo = n * r / P;
    hi = n * (r + 1) / P;
}
inline bool distributed(const Ctx& c) { return c.p.nranks > 1; }
// This rank's i clusters: its band (all of them with one rank).
inline void cluster_share(const Ctx& c, long long& lo, long long& hi)
{
    if (distributed(c) && (int)c.band_cl.size() == c.p.nranks + 1) {
        lo = c.band_cl[c.p.rank];
        hi = c.band_cl[c.p.rank + 1];
    } else {
        rank_slice(c, c.n_clusters, lo, hi);
    }
}
// This rank's atom slots (PME spread and gather): its band's clusters.
inline void slot_share(const Ctx& c, long long& lo, long long& hi)
{
    cluster_share(c, lo, hi);
    lo *= CLUSTER;
    hi *= CLUSTER;
}
// nranks > 1 with the reduce-scatter / all-gather / all-to-all collectives
inline bool slab_mode(const Ctx& c) { return distributed(c) && c.coll_rs && c.coll_ag && c.coll_a2a; }
// slab mode with the grid planes exchanged as halos (mdf_set_halo_exchange)
inline bool halo_mode(const Ctx& c) { return slab_mode(c) && c.coll_a2av != nullptr; }
inline bool rank0(const Ctx& c) { return !distributed(c) || c.p.rank == 0; }
// In-place sum over the ranks through the registered collective, on c.stream.
void allreduce_u64(Ctx& c, unsigned long long* d, long long n);

}  // namespace mdf

// The opaque handle of the C ABI.
struct mdf_ctx {
    mdf::Ctx c;
};
