// Batched evaluation of many independent systems (uneven atom counts, boxes
// and PME grids) as one CUDA graph launch.
//
// Each system keeps its own context (device buffers, pairlist, PME plan); a
// batch evaluation is captured once into a graph:
//   host->device copy of every system's positions (one pinned buffer)
//   -> one scatter kernel into the systems' position arrays
//   -> every system's evaluation on its own stream (a fork/join of streams,
//      so the systems' kernels run concurrently; each system's PME chain is
//      a further branch)
//   -> one gather kernel of all forces -> device->host copy (one buffer).
// Replaying the graph evaluates the whole batch with one launch from the
// host.  The graph is recaptured when the flags change, after a pairlist
// rebuild or a change of launch shapes.
//
// mdf_batch_autotune times the candidate launch shapes (pair-kernel warps per
// block, FFT lines per block, per-evaluation pruning on or off, pair-kernel
// schedule and layout) on the batch itself and keeps the fastest; the choice
// changes results only through the order of the floating-point sums of each
// i cluster's forces (pruning, layout), never through the atomics (fixed
// point).  mdf_batch_submit / mdf_batch_collect pipeline consecutive batches.
#include <algorithm>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "kargs.cuh"
#include "mdf_device.cuh"
#include "mdf_internal.cuh"

using namespace mdf;

struct mdf_batch {
    int nsys = 0;
    int device = 0;
    std::vector<mdf_ctx*> sys;
    std::vector<long long> off;          // [nsys + 1] offsets into the concatenated xyz (doubles)
    long long total = 0;                 // 3 * total atoms
    int max_len = 0;                     // longest system in doubles
    cudaStream_t main = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool have_graph = false;
    uint32_t graph_flags = 0;
    long long graph_kernels = 0;
    bool have_positions = false;
    bool have_lists = false;
    double* h_pos = nullptr;             // pinned [total]
    double* h_forces = nullptr;          // pinned [total]
    DevBuf<double> d_pos, d_forces;
    DevBuf<double*> d_xyz_ptr, d_f_ptr;
    DevBuf<long long> d_off;
    std::string last_error;
    // one launch per kernel for all systems (uniform launch parameters), or
    // every system's own kernel chain in the graph
    bool multi = false;
    cudaStream_t side = nullptr;         // PME, bonded, exclusions: concurrent with pack/prune/pairs
    cudaEvent_t ev_fork2 = nullptr, ev_join2 = nullptr;
    // per-kernel argument arrays of the multi form (rebuilt before each capture)
    DevBuf<unsigned char> args;          // one allocation, the arrays below point into it
    size_t args_cap = 0;
    // pipelined evaluation (mdf_batch_submit / mdf_batch_collect): two stages,
    // each with its own graph (no copies inside), device position and force
    // buffers and host scalar blocks; the copies run on two copy streams
    struct Stage {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        uint32_t graph_flags = 0;
        DevBuf<double> d_pos, d_forces;
        DevBuf<unsigned char> args;
        unsigned long long* h_scal = nullptr;    // mapped pinned [nsys][NUM_SCAL]
        unsigned long long* d_hscal = nullptr;
        cudaEvent_t h2d = nullptr, consumed = nullptr, done = nullptr, d2h = nullptr;
        uint32_t flags = 0;
    };
    Stage stage[2];
    int stage_next = 0, stage_old = 0, inflight = 0;
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
};

namespace {

__global__ void k_batch_scatter(const long long* __restrict__ off, const double* __restrict__ src,
                                double* const* __restrict__ dst)
{
    const int s = blockIdx.y;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = off[s + 1] - off[s];
    if (i < n) dst[s][i] = src[off[s] + i];
}

__global__ void k_batch_gather(const long long* __restrict__ off, const double* const* __restrict__ src,
                               double* __restrict__ dst)
{
    const int s = blockIdx.y;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = off[s + 1] - off[s];
    if (i < n) dst[off[s] + i] = src[s][i];
}

template <typename F>
int batch_guard(mdf_batch* b, F&& f)
{
    try {
        f();
        if (b) b->last_error.clear();
        return MDF_OK;
    } catch (const ApiError& e) {
        if (b) b->last_error = e.msg;
        return e.status;
    } catch (const CudaError& e) {
        if (b) b->last_error = e.msg;
        return MDF_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        if (b) b->last_error = "host allocation failed";
        return MDF_ERR_NOMEM;
    } catch (const std::exception& e) {
        if (b) b->last_error = e.what();
        return MDF_ERR_INVALID;
    }
}

void drop_graph(mdf_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->have_graph = false;
    if (b->inflight) cudaStreamSynchronize(b->main);   // stage graphs still queued finish first
    for (auto& S : b->stage) {
        if (S.exec) cudaGraphExecDestroy(S.exec);
        if (S.graph) cudaGraphDestroy(S.graph);
        S.exec = nullptr;
        S.graph = nullptr;
    }
}

// Enqueue one batch evaluation on b->main (used both plainly and under capture).
void enqueue(mdf_batch* b, uint32_t flags)
{
    const int th = 256;
    const dim3 grid((unsigned)((b->max_len + th - 1) / th), (unsigned)b->nsys);
    MDF_CUDA_TRY(cudaMemcpyAsync(b->d_pos.p, b->h_pos, sizeof(double) * b->total, cudaMemcpyHostToDevice, b->main));
    k_batch_scatter<<<grid, th, 0, b->main>>>(b->d_off.p, b->d_pos.p, b->d_xyz_ptr.p);
    MDF_CUDA_TRY(cudaGetLastError());
    MDF_CUDA_TRY(cudaEventRecord(b->fork, b->main));
    long long k0 = 0;
    for (int s = 0; s < b->nsys; ++s) {
        Ctx& c = b->sys[s]->c;
        MDF_CUDA_TRY(cudaStreamWaitEvent(c.stream, b->fork, 0));
        const long long l0 = c.launches;
        eval_async_impl(c, flags);
        k0 += c.launches - l0;
        MDF_CUDA_TRY(cudaEventRecord(b->join[s], c.stream));
        MDF_CUDA_TRY(cudaStreamWaitEvent(b->main, b->join[s], 0));
    }
    k_batch_gather<<<grid, th, 0, b->main>>>(b->d_off.p, b->d_f_ptr.p, b->d_forces.p);
    MDF_CUDA_TRY(cudaGetLastError());
    MDF_CUDA_TRY(cudaMemcpyAsync(b->h_forces, b->d_forces.p, sizeof(double) * b->total, cudaMemcpyDeviceToHost,
                                 b->main));
    b->graph_kernels = k0 + 2;
}

// ----------------------------------------------------------- multi form
// Every kernel of an evaluation is launched once for all systems (grid z =
// system, each block reads its system's arguments from device memory), so a
// batch evaluation is ~17 graph nodes whatever the number of systems.  It
// needs the launch-selecting parameters to agree across systems: precision,
// LJ switch on or off, pruning on or off, pair-kernel warps and FFT lines.
bool uniform_launches(const mdf_batch* b)
{
    const mdf_params& p0 = b->sys[0]->c.p;
    for (const mdf_ctx* x : b->sys) {
        const mdf_params& p = x->c.p;
        if (p.precision != p0.precision || (p.switch_radius > 0) != (p0.switch_radius > 0) ||
            (p.prune_every != 0) != (p0.prune_every != 0) || p.pair_warps != p0.pair_warps ||
            p.fft_lines != p0.fft_lines || p.pair_schedule != p0.pair_schedule ||
            half_layout(x->c) != half_layout(b->sys[0]->c) || p.nranks > 1)
            return false;
    }
    return true;
}

// Host-built argument arrays of one batch evaluation, copied to the device
// before capture; the captured launches read them at every replay.
template <typename R>
struct MultiArgs {
    std::vector<PackArgs<R>> pack;
    std::vector<PruneArgs<R>> prune;
    std::vector<PairF32Args> pf32;
    std::vector<PairF64Args> p64;
    std::vector<ExclArgs> excl;
    std::vector<Pair14Args> p14;
    std::vector<BondedArgs> bonded;
    std::vector<ZeroArgs> zero;
    std::vector<SpreadArgs> spread;
    std::vector<FFTZArgs<R>> zf, zi;
    std::vector<FFTYArgs<R>> yf, yi;
    std::vector<FFTXArgs<R>> x;
    std::vector<GatherArgs<R>> gather;
    std::vector<FinalizeArgs> fin;
    // block maps of the kernels whose per-system grids differ most between
    // systems (one entry per block actually needed: no idle blocks)
    std::vector<int2> map_pack, map_zero, map_spread, map_z, map_y, map_x, map_gather, map_fin;
    FFTChainMax fm{};
    int gx_prune = 0, gx_pairs = 0, gx_excl = 0, gx_14 = 0, gx_bonded = 0;
    size_t dyn_pairs = 0;
    int threads = 256;
    bool prune_on = false, use_switch = false, energy = false, persist = false, half = false;
    bool lj_smem = true;   // every system's LJ table in shared memory (one kernel form for the batch)
};

template <typename R>
struct MultiDev {
    const PackArgs<R>* pack;
    const PruneArgs<R>* prune;
    const PairF32Args* pf32;
    const PairF64Args* p64;
    const ExclArgs* excl;
    const Pair14Args* p14;
    const BondedArgs* bonded;
    const ZeroArgs* zero;
    const SpreadArgs* spread;
    FFTChainDev<R> fft;
    const GatherArgs<R>* gather;
    const FinalizeArgs* fin;
    BlockMap pack_m, zero_m, spread_m, gather_m, fin_m;
};

// Append system s's blocks (a gx x gy grid, linear index) to a block map.
inline void add_blocks(std::vector<int2>& map, int s, int gx, int gy)
{
    for (int b = 0; b < gx * gy; ++b) map.push_back(make_int2(s, b));
}

template <typename T>
size_t arr_bytes(const std::vector<T>& v)
{
    return (v.size() * sizeof(T) + 255) & ~(size_t)255;
}

// Build every system's arguments into M and copy them into b->args
// (synchronously, outside any capture); returns the device arrays.  (The
// prune kernel's kept-entry counter is not cleared per evaluation here: a
// batch does not report it.)
// d_forces: the concatenated force buffer the finalize kernels write;
// hscal: per-system host scalar blocks ([nsys][NUM_SCAL], device view of
// mapped memory; nullptr = each context's own); args: the device allocation
// of the argument arrays.
template <typename R>
MultiDev<R> prepare_multi(mdf_batch* b, uint32_t flags, MultiArgs<R>& M, double* d_forces,
                          unsigned long long* hscal, DevBuf<unsigned char>& args)
{
    const int n = b->nsys;
    const bool energy = (flags & MDF_COMPUTE_ENERGY) != 0;
    M.energy = energy;
    const Ctx& c0 = b->sys[0]->c;
    M.prune_on = c0.p.prune_every != 0;
    M.use_switch = c0.p.switch_radius > 0;
    M.threads = pair_threads(c0);
    M.persist = c0.p.pair_schedule == 1;
    M.half = half_layout(c0);
    for (int s = 0; s < n; ++s) {
        Ctx& c = b->sys[s]->c;
        if (M.half) ensure_half_lists(c);
        if (M.prune_on) {
            // the captured chain prunes before the pair kernel.  A self-pruning
            // system whose lists are not valid (new list, new layout) prunes once
            // here, so the captured prunes can leave the decision to the device.
            if (self_pruning(c) && (!c.pruned_valid || c.pruned_half != M.half)) {
                prune_pairlist(c);
                MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
            }
            c.pruned_valid = true;
            c.pruned_half = M.half;
        }
        M.pack.push_back(make_pack_args<R>(c));
        M.prune.push_back(M.half ? make_prune_half_args<R>(c) : make_prune_args<R>(c));
        if (sizeof(R) == 4) {
            size_t dyn = 0;
            M.pf32.push_back(make_pair_f32_args(c, &dyn));
            M.dyn_pairs = std::max(M.dyn_pairs, dyn);
        } else {
            size_t dyn = 0;
            M.p64.push_back(make_pair_f64_args(c, &dyn));
            M.dyn_pairs = std::max(M.dyn_pairs, dyn);
        }
        M.excl.push_back(make_excl_args(c));
        M.p14.push_back(make_pair14_args(c));
        M.bonded.push_back(make_bonded_args(c, false, c.f_atom.p, c.acc.p, c.status.p));
        const long long ntot = (long long)c.K[0] * c.K[1] * c.K[2];
        ZeroArgs z;
        z.gx = grid_blocks(ntot, 256 * 8);
        z.gy = 1;
        z.p = c.qgrid.p;
        z.n = ntot;
        M.zero.push_back(z);
        M.spread.push_back(make_spread_args(c));
        const FFTChain<R> F = make_fft_chain<R>(c, energy);
        M.zf.push_back(F.zf);
        M.yf.push_back(F.yf);
        M.x.push_back(F.x);
        M.yi.push_back(F.yi);
        M.zi.push_back(F.zi);
        add_blocks(M.map_z, s, F.zf.gx, F.zf.gy);
        add_blocks(M.map_y, s, F.yf.gx, F.yf.gy);
        add_blocks(M.map_x, s, F.x.gx, F.x.gy);
        M.fm.smz = std::max(M.fm.smz, F.smz);
        M.fm.smy = std::max(M.fm.smy, F.smy);
        M.fm.smx = std::max(M.fm.smx, F.smx);
        M.gather.push_back(make_gather_args<R>(c));
        // forces straight into the batch's concatenated device buffer
        M.fin.push_back(make_finalize_args(c, d_forces + b->off[s]));
        if (hscal) M.fin.back().host_scal = hscal + (size_t)s * NUM_SCAL;
    }
    auto gmax = [](const auto& v) {
        int g = 0;
        for (const auto& a : v) g = std::max(g, a.gx);
        return g;
    };
    // the pair kernel reads the LJ tables from shared memory only when all fit
    for (const auto& a : M.pf32) M.lj_smem = M.lj_smem && a.lj_smem;
    for (const auto& a : M.p64) M.lj_smem = M.lj_smem && a.lj_smem;
    if (!M.lj_smem) {
        for (auto& a : M.pf32) a.lj_smem = 0;
        for (auto& a : M.p64) a.lj_smem = 0;
        M.dyn_pairs = 0;
    }
    M.gx_prune = gmax(M.prune);
    M.gx_pairs = sizeof(R) == 4 ? gmax(M.pf32) : gmax(M.p64);
    M.gx_excl = gmax(M.excl);
    M.gx_14 = gmax(M.p14);
    M.gx_bonded = gmax(M.bonded);
    for (int s = 0; s < n; ++s) {
        add_blocks(M.map_pack, s, M.pack[s].gx, 1);
        add_blocks(M.map_zero, s, M.zero[s].gx, 1);
        add_blocks(M.map_spread, s, M.spread[s].gx, 1);
        add_blocks(M.map_gather, s, M.gather[s].gx, 1);
        add_blocks(M.map_fin, s, M.fin[s].gx, 1);
    }
    // one device allocation for every array
    const size_t total = arr_bytes(M.pack) + arr_bytes(M.prune) + arr_bytes(M.pf32) + arr_bytes(M.p64) +
                         arr_bytes(M.excl) + arr_bytes(M.p14) + arr_bytes(M.bonded) + arr_bytes(M.zero) +
                         arr_bytes(M.spread) + arr_bytes(M.zf) + arr_bytes(M.yf) + arr_bytes(M.x) +
                         arr_bytes(M.yi) + arr_bytes(M.zi) + arr_bytes(M.gather) + arr_bytes(M.fin) +
                         arr_bytes(M.map_pack) + arr_bytes(M.map_zero) + arr_bytes(M.map_spread) +
                         arr_bytes(M.map_z) + arr_bytes(M.map_y) + arr_bytes(M.map_x) + arr_bytes(M.map_gather) +
                         arr_bytes(M.map_fin);
    std::vector<unsigned char> host(total);
    args.alloc(total);
    size_t off = 0;
    MultiDev<R> D;
    auto put = [&](const auto& v, auto*& dptr) {
        using T = typename std::decay_t<decltype(v)>::value_type;
        if (!v.empty()) memcpy(host.data() + off, v.data(), v.size() * sizeof(T));
        dptr = reinterpret_cast<T*>(args.p + off);
        off += arr_bytes(v);
    };
    put(M.pack, D.pack);
    put(M.prune, D.prune);
    put(M.pf32, D.pf32);
    put(M.p64, D.p64);
    put(M.excl, D.excl);
    put(M.p14, D.p14);
    put(M.bonded, D.bonded);
    put(M.zero, D.zero);
    put(M.spread, D.spread);
    put(M.zf, D.fft.zf);
    put(M.yf, D.fft.yf);
    put(M.x, D.fft.x);
    put(M.yi, D.fft.yi);
    put(M.zi, D.fft.zi);
    put(M.gather, D.gather);
    put(M.fin, D.fin);
    auto putmap = [&](const std::vector<int2>& v, BlockMap& bm) {
        const int2* p = nullptr;
        put(v, p);
        bm.map = p;
        bm.n = (int)v.size();
    };
    putmap(M.map_pack, D.pack_m);
    putmap(M.map_zero, D.zero_m);
    putmap(M.map_spread, D.spread_m);
    putmap(M.map_gather, D.gather_m);
    putmap(M.map_fin, D.fin_m);
    putmap(M.map_z, D.fft.mz);
    putmap(M.map_y, D.fft.my);
    putmap(M.map_x, D.fft.mx);
    MDF_CUDA_TRY(cudaMemcpyAsync(args.p, host.data(), total, cudaMemcpyHostToDevice, b->main));
    MDF_CUDA_TRY(cudaStreamSynchronize(b->main));
    return D;
}

// One batch evaluation in the multi form.  copies: the host<->device copies
// of the batch's own pinned buffers at both ends (the plain graph); without
// them the evaluation reads positions from d_pos and leaves forces where the
// finalize arguments point (the pipelined stages).
template <typename R>
void enqueue_multi(mdf_batch* b, const MultiArgs<R>& M, const MultiDev<R>& D, const double* d_pos, bool copies)
{
    const int n = b->nsys, th = 256;
    const dim3 grid((unsigned)((b->max_len + th - 1) / th), (unsigned)n);
    if (copies)
        MDF_CUDA_TRY(cudaMemcpyAsync(b->d_pos.p, b->h_pos, sizeof(double) * b->total, cudaMemcpyHostToDevice,
                                     b->main));
    k_batch_scatter<<<grid, th, 0, b->main>>>(b->d_off.p, d_pos, b->d_xyz_ptr.p);
    MDF_CUDA_TRY(cudaGetLastError());
    long long k = 2;   // scatter + finalize
    // side stream: exclusions, 1-4, bonded terms, PME (they only read positions
    // and charges and add into the fixed-point accumulators)
    MDF_CUDA_TRY(cudaEventRecord(b->ev_fork2, b->main));
    MDF_CUDA_TRY(cudaStreamWaitEvent(b->side, b->ev_fork2, 0));
    launch_exclusions_multi(D.excl, M.gx_excl, D.p14, M.gx_14, n, M.energy, b->side);
    k += (M.gx_excl > 0) + (M.gx_14 > 0);
    launch_bonded_multi(D.bonded, n, M.gx_bonded, M.energy, b->side);
    k += M.gx_bonded > 0;
    launch_pme_multi<R>(D.zero, D.zero_m, D.spread, D.spread_m, D.fft, M.fm, D.gather, D.gather_m, M.energy,
                        b->side);
    k += 8;   // grid clear, spread, five FFT passes, gather
    MDF_CUDA_TRY(cudaEventRecord(b->ev_join2, b->side));
    // main stream: pack, prune, pair kernel
    launch_pack_multi<R>(D.pack, D.pack_m, b->main);
    ++k;
    if (M.prune_on) {
        launch_prune_multi<R>(D.prune, n, M.gx_prune, M.half, b->main);
        ++k;
    }
    if (M.gx_pairs > 0) {
        if (sizeof(R) == 4)
            launch_pairs_f32_multi(D.pf32, n, M.gx_pairs, M.threads, M.dyn_pairs, M.energy, M.use_switch, M.persist,
                                   M.half, M.lj_smem, b->main);
        else
            launch_pairs_f64_multi(D.p64, n, M.gx_pairs, M.threads, M.dyn_pairs, M.energy, M.use_switch, M.persist,
                                   M.half, M.lj_smem, b->main);
        ++k;
    }
    MDF_CUDA_TRY(cudaStreamWaitEvent(b->main, b->ev_join2, 0));
    launch_finalize_multi(D.fin, D.fin_m, b->main);
    if (copies)
        MDF_CUDA_TRY(cudaMemcpyAsync(b->h_forces, b->d_forces.p, sizeof(double) * b->total, cudaMemcpyDeviceToHost,
                                     b->main));
    b->graph_kernels = k;
}

void capture(mdf_batch* b, uint32_t flags)
{
    drop_graph(b);
    b->multi = uniform_launches(b);
    const bool fp32 = b->sys[0]->c.p.precision == MDF_PREC_MIXED;
    MultiArgs<float> Mf;
    MultiArgs<double> Md;
    MultiDev<float> Df{};
    MultiDev<double> Dd{};
    if (b->multi) {
        if (fp32) Df = prepare_multi<float>(b, flags, Mf, b->d_forces.p, nullptr, b->args);
        else Dd = prepare_multi<double>(b, flags, Md, b->d_forces.p, nullptr, b->args);
    }
    MDF_CUDA_TRY(cudaStreamBeginCapture(b->main, cudaStreamCaptureModeThreadLocal));
    try {
        if (!b->multi) enqueue(b, flags);
        else if (fp32) enqueue_multi<float>(b, Mf, Df, b->d_pos.p, true);
        else enqueue_multi<double>(b, Md, Dd, b->d_pos.p, true);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(b->main, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    MDF_CUDA_TRY(cudaStreamEndCapture(b->main, &b->graph));
    MDF_CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->have_graph = true;
    b->graph_flags = flags;
}

void build_lists(mdf_batch* b)
{
    if (!b->have_positions) throw ApiError(MDF_ERR_STATE, "positions not set");
    drop_graph(b);
    for (int s = 0; s < b->nsys; ++s) {
        Ctx& c = b->sys[s]->c;
        MDF_CUDA_TRY(cudaMemcpyAsync(c.xyz.p, b->h_pos + b->off[s], sizeof(double) * 3 * (size_t)c.N,
                                     cudaMemcpyHostToDevice, c.stream));
        c.have_positions = true;
        build_pairlist(c);
        // one plain evaluation: clears the accumulators and counts pairs, so
        // the captured evaluations need no first-use work
        eval_async_impl(c, MDF_COMPUTE_ENERGY | MDF_COMPUTE_FORCES);
    }
    for (int s = 0; s < b->nsys; ++s) MDF_CUDA_TRY(cudaStreamSynchronize(b->sys[s]->c.stream));
    b->have_lists = true;
}

void run(mdf_batch* b, uint32_t flags)
{
    if (!b->have_lists) build_lists(b);
    if (!b->have_graph || b->graph_flags != flags) capture(b, flags);
    MDF_CUDA_TRY(cudaGraphLaunch(b->exec, b->main));
}

void collect(mdf_batch* b, uint32_t flags, double* forces, mdf_energies* e)
{
    MDF_CUDA_TRY(cudaStreamSynchronize(b->main));
    for (int s = 0; s < b->nsys; ++s) {
        const Ctx& c = b->sys[s]->c;
        try {
            check_host_status(c);
        } catch (const ApiError& err) {
            throw ApiError(err.status, "system " + std::to_string(s) + ": " + err.msg);
        }
        if (e) host_energies(c, flags, e + s);
    }
    if (forces) memcpy(forces, b->h_forces, sizeof(double) * b->total);
}

// The graph of pipeline stage st: the multi-form evaluation reading the
// stage's device positions and writing its device forces and host scalar blocks.
void capture_stage(mdf_batch* b, uint32_t flags, int st)
{
    mdf_batch::Stage& S = b->stage[st];
    if (S.exec) cudaGraphExecDestroy(S.exec);
    if (S.graph) cudaGraphDestroy(S.graph);
    S.exec = nullptr;
    S.graph = nullptr;
    if (!uniform_launches(b))
        throw ApiError(MDF_ERR_UNSUPPORTED, "pipelined batches need the same launch parameters in every system");
    const bool fp32 = b->sys[0]->c.p.precision == MDF_PREC_MIXED;
    MultiArgs<float> Mf;
    MultiArgs<double> Md;
    MultiDev<float> Df{};
    MultiDev<double> Dd{};
    if (fp32) Df = prepare_multi<float>(b, flags, Mf, S.d_forces.p, S.d_hscal, S.args);
    else Dd = prepare_multi<double>(b, flags, Md, S.d_forces.p, S.d_hscal, S.args);
    MDF_CUDA_TRY(cudaStreamBeginCapture(b->main, cudaStreamCaptureModeThreadLocal));
    try {
        if (fp32) enqueue_multi<float>(b, Mf, Df, S.d_pos.p, false);
        else enqueue_multi<double>(b, Md, Dd, S.d_pos.p, false);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(b->main, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    MDF_CUDA_TRY(cudaStreamEndCapture(b->main, &S.graph));
    MDF_CUDA_TRY(cudaGraphInstantiate(&S.exec, S.graph, 0));
    S.graph_flags = flags;
}

void submit(mdf_batch* b, uint32_t flags, const double* xyz, double* forces)
{
    if (b->inflight >= 2) throw ApiError(MDF_ERR_STATE, "two batch evaluations in flight: collect one first");
    if (!b->have_lists) {
        // the first evaluation: lists from these positions (through the batch's own buffer)
        if (xyz != b->h_pos) memcpy(b->h_pos, xyz, sizeof(double) * b->total);
        b->have_positions = true;
        build_lists(b);
    }
    if (!b->copy_in) MDF_CUDA_TRY(cudaStreamCreateWithFlags(&b->copy_in, cudaStreamNonBlocking));
    if (!b->copy_out) MDF_CUDA_TRY(cudaStreamCreateWithFlags(&b->copy_out, cudaStreamNonBlocking));
    mdf_batch::Stage& S = b->stage[b->stage_next];
    if (!S.h_scal) {
        MDF_CUDA_TRY(cudaHostAlloc((void**)&S.h_scal, sizeof(unsigned long long) * NUM_SCAL * (size_t)b->nsys,
                                   cudaHostAllocMapped));
        memset(S.h_scal, 0, sizeof(unsigned long long) * NUM_SCAL * (size_t)b->nsys);
        MDF_CUDA_TRY(cudaHostGetDevicePointer((void**)&S.d_hscal, S.h_scal, 0));
        for (cudaEvent_t* e : {&S.h2d, &S.consumed, &S.done, &S.d2h})
            MDF_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        S.d_pos.alloc(b->total);
        S.d_forces.alloc(b->total);
    }
    if (!S.exec || S.graph_flags != flags) capture_stage(b, flags, b->stage_next);
    // positions in (the stage buffer is free once its last evaluation ran)
    MDF_CUDA_TRY(cudaStreamWaitEvent(b->copy_in, S.consumed, 0));
    MDF_CUDA_TRY(cudaMemcpyAsync(S.d_pos.p, xyz, sizeof(double) * b->total, cudaMemcpyHostToDevice, b->copy_in));
    MDF_CUDA_TRY(cudaEventRecord(S.h2d, b->copy_in));
    // the evaluation, after its positions and after the stage's last forces left
    MDF_CUDA_TRY(cudaStreamWaitEvent(b->main, S.h2d, 0));
    MDF_CUDA_TRY(cudaStreamWaitEvent(b->main, S.d2h, 0));
    MDF_CUDA_TRY(cudaGraphLaunch(S.exec, b->main));
    MDF_CUDA_TRY(cudaEventRecord(S.consumed, b->main));
    MDF_CUDA_TRY(cudaEventRecord(S.done, b->main));
    // forces out
    MDF_CUDA_TRY(cudaStreamWaitEvent(b->copy_out, S.done, 0));
    if (forces)
        MDF_CUDA_TRY(cudaMemcpyAsync(forces, S.d_forces.p, sizeof(double) * b->total, cudaMemcpyDeviceToHost,
                                     b->copy_out));
    MDF_CUDA_TRY(cudaEventRecord(S.d2h, b->copy_out));
    S.flags = flags;
    b->stage_next ^= 1;
    ++b->inflight;
}

void collect_stage(mdf_batch* b, mdf_energies* e)
{
    if (b->inflight == 0) throw ApiError(MDF_ERR_STATE, "no submitted batch evaluation to collect");
    mdf_batch::Stage& S = b->stage[b->stage_old];
    b->stage_old ^= 1;
    --b->inflight;
    MDF_CUDA_TRY(cudaEventSynchronize(S.d2h));
    for (int s = 0; s < b->nsys; ++s) {
        const unsigned long long* hs = S.h_scal + (size_t)s * NUM_SCAL;
        try {
            check_status_word(hs);
        } catch (const ApiError& err) {
            throw ApiError(err.status, "system " + std::to_string(s) + ": " + err.msg);
        }
        if (e) host_energies_from(b->sys[s]->c, hs, S.flags, e + s);
    }
}

}  // namespace

extern "C" {

int mdf_batch_create(int nsys, const mdf_topology* const* topos, const mdf_params* params, mdf_batch** out)
{
    if (!out || nsys <= 0 || !topos || !params) return MDF_ERR_INVALID;
    *out = nullptr;
    mdf_batch* b = new mdf_batch();
    int rc = batch_guard(b, [&] {
        b->nsys = nsys;
        b->device = params[0].device;
        b->sys.assign(nsys, nullptr);
        b->off.assign(nsys + 1, 0);
        for (int s = 0; s < nsys; ++s) {
            if (params[s].device != b->device) throw ApiError(MDF_ERR_INVALID, "all systems must use one device");
            if (params[s].semantics != MDF_SEM_PHYSICAL)
                throw ApiError(MDF_ERR_UNSUPPORTED, "batches run PHYSICAL semantics");
            int r = mdf_create(topos[s], &params[s], &b->sys[s]);
            if (r != MDF_OK)
                throw ApiError(r, "system " + std::to_string(s) + ": " + mdf_last_error(nullptr));
            const int len = 3 * b->sys[s]->c.N;
            b->off[s + 1] = b->off[s] + len;
            b->max_len = std::max(b->max_len, len);
        }
        b->total = b->off[nsys];
        MDF_CUDA_TRY(cudaSetDevice(b->device));
        MDF_CUDA_TRY(cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking));
        MDF_CUDA_TRY(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
        {
            int lo = 0, hi = 0;   // the short PME / bonded kernels first (as in one context)
            MDF_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            MDF_CUDA_TRY(cudaStreamCreateWithPriority(&b->side, cudaStreamNonBlocking, hi));
        }
        MDF_CUDA_TRY(cudaEventCreateWithFlags(&b->ev_fork2, cudaEventDisableTiming));
        MDF_CUDA_TRY(cudaEventCreateWithFlags(&b->ev_join2, cudaEventDisableTiming));
        b->join.assign(nsys, nullptr);
        for (int s = 0; s < nsys; ++s) MDF_CUDA_TRY(cudaEventCreateWithFlags(&b->join[s], cudaEventDisableTiming));
        MDF_CUDA_TRY(cudaHostAlloc((void**)&b->h_pos, sizeof(double) * b->total, cudaHostAllocDefault));
        MDF_CUDA_TRY(cudaHostAlloc((void**)&b->h_forces, sizeof(double) * b->total, cudaHostAllocDefault));
        b->d_pos.alloc(b->total);
        b->d_forces.alloc(b->total);
        std::vector<double*> xp(nsys), fp(nsys);
        for (int s = 0; s < nsys; ++s) {
            xp[s] = b->sys[s]->c.xyz.p;
            fp[s] = b->sys[s]->c.forces_out.p;
        }
        b->d_xyz_ptr.upload(xp.data(), nsys, b->main);
        b->d_f_ptr.upload(fp.data(), nsys, b->main);
        b->d_off.upload(b->off.data(), nsys + 1, b->main);
        MDF_CUDA_TRY(cudaStreamSynchronize(b->main));
    });
    if (rc != MDF_OK) {
        std::string msg = b->last_error;
        mdf_batch_destroy(b);
        (void)msg;
        return rc;
    }
    *out = b;
    return MDF_OK;
}

void mdf_batch_destroy(mdf_batch* b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    // submitted evaluations (and their copies) finish before anything is freed
    for (cudaStream_t cs : {b->main, b->copy_in, b->copy_out})
        if (cs) cudaStreamSynchronize(cs);
    b->inflight = 0;
    drop_graph(b);
    for (mdf_ctx* c : b->sys)
        if (c) mdf_destroy(c);
    b->d_pos.release();
    b->d_forces.release();
    b->d_xyz_ptr.release();
    b->d_f_ptr.release();
    b->d_off.release();
    if (b->h_pos) cudaFreeHost(b->h_pos);
    if (b->h_forces) cudaFreeHost(b->h_forces);
    for (cudaEvent_t e : b->join)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->ev_fork2) cudaEventDestroy(b->ev_fork2);
    if (b->ev_join2) cudaEventDestroy(b->ev_join2);
    if (b->side) cudaStreamDestroy(b->side);
    b->args.release();
    for (auto& S : b->stage) {
        if (S.h_scal) cudaFreeHost(S.h_scal);
        for (cudaEvent_t e : {S.h2d, S.consumed, S.done, S.d2h})
            if (e) cudaEventDestroy(e);
        S.d_pos.release();
        S.d_forces.release();
        S.args.release();
    }
    for (cudaStream_t cs : {b->copy_in, b->copy_out})
        if (cs) {
            cudaStreamSynchronize(cs);
            cudaStreamDestroy(cs);
        }
    if (b->main) cudaStreamDestroy(b->main);
    delete b;
}

const char* mdf_batch_last_error(const mdf_batch* b)
{
    return b ? b->last_error.c_str() : "null batch";
}

int mdf_batch_info(const mdf_batch* b, int64_t* n_systems, int64_t* total_atoms, int64_t* graph_kernels)
{
    if (!b) return MDF_ERR_INVALID;
    if (n_systems) *n_systems = b->nsys;
    if (total_atoms) *total_atoms = b->total / 3;
    if (graph_kernels) *graph_kernels = b->have_graph ? b->graph_kernels : -1;
    return MDF_OK;
}

int mdf_batch_set_positions(mdf_batch* b, const double* xyz)
{
    if (!b || !xyz) return MDF_ERR_INVALID;
    return batch_guard(b, [&] {
        if (xyz != b->h_pos) memcpy(b->h_pos, xyz, sizeof(double) * b->total);   // own buffer: written in place
        b->have_positions = true;
    });
}

int mdf_batch_host_buffers(mdf_batch* b, double** positions, double** forces)
{
    if (!b) return MDF_ERR_INVALID;
    if (positions) *positions = b->h_pos;
    if (forces) *forces = b->h_forces;
    return MDF_OK;
}

int mdf_batch_build_pairlists(mdf_batch* b)
{
    if (!b) return MDF_ERR_INVALID;
    return batch_guard(b, [&] {
        MDF_CUDA_TRY(cudaSetDevice(b->device));
        build_lists(b);
    });
}

int mdf_batch_compute(mdf_batch* b, uint32_t flags, double* forces, mdf_energies* energies)
{
    if (!b) return MDF_ERR_INVALID;
    return batch_guard(b, [&] {
        MDF_CUDA_TRY(cudaSetDevice(b->device));
        if (!b->have_positions) throw ApiError(MDF_ERR_STATE, "positions not set");
        run(b, flags);
        collect(b, flags, forces, energies);
    });
}

int mdf_batch_launch(mdf_batch* b, uint32_t flags, void* stream)
{
    if (!b) return MDF_ERR_INVALID;
    return batch_guard(b, [&] {
        MDF_CUDA_TRY(cudaSetDevice(b->device));
        if (!b->have_positions) throw ApiError(MDF_ERR_STATE, "positions not set");
        if (stream) {
            // order the launch after the caller's stream and the caller's stream after it
            MDF_CUDA_TRY(cudaEventRecord(b->fork, (cudaStream_t)stream));
            MDF_CUDA_TRY(cudaStreamWaitEvent(b->main, b->fork, 0));
        }
        run(b, flags);
        if (stream) {
            MDF_CUDA_TRY(cudaEventRecord(b->join[0], b->main));
            MDF_CUDA_TRY(cudaStreamWaitEvent((cudaStream_t)stream, b->join[0], 0));
        }
    });
}

int mdf_batch_submit(mdf_batch* b, uint32_t flags, const double* xyz, double* forces)
{
    if (!b || !xyz) return MDF_ERR_INVALID;
    return batch_guard(b, [&] {
        MDF_CUDA_TRY(cudaSetDevice(b->device));
        submit(b, flags, xyz, forces);
    });
}

int mdf_batch_collect(mdf_batch* b, mdf_energies* energies)
{
    if (!b) return MDF_ERR_INVALID;
    return batch_guard(b, [&] {
        MDF_CUDA_TRY(cudaSetDevice(b->device));
        collect_stage(b, energies);
    });
}

int mdf_batch_fetch(mdf_batch* b, uint32_t flags, double* forces, mdf_energies* energies)
{
    if (!b) return MDF_ERR_INVALID;
    return batch_guard(b, [&] {
        MDF_CUDA_TRY(cudaSetDevice(b->device));
        collect(b, flags, forces, energies);
    });
}

int mdf_batch_autotune(mdf_batch* b, int reps, mdf_tune_report* rep)
{
    if (!b) return MDF_ERR_INVALID;
    return batch_guard(b, [&] {
        MDF_CUDA_TRY(cudaSetDevice(b->device));
        if (!b->have_positions) throw ApiError(MDF_ERR_STATE, "positions not set");
        if (!b->have_lists) build_lists(b);
        const int R = reps > 0 ? reps : 5;
        const uint32_t flags = MDF_COMPUTE_ENERGY | MDF_COMPUTE_FORCES;
        const int warps[3] = {2, 4, 8}, lines[4] = {2, 4, 8, 16}, prune[2] = {0, 1}, sched[2] = {0, 1};
        cudaEvent_t e0, e1;
        MDF_CUDA_TRY(cudaEventCreate(&e0));
        MDF_CUDA_TRY(cudaEventCreate(&e1));
        auto apply = [&](int w, int l, int p, int sc, int ly) {
            for (mdf_ctx* x : b->sys) {
                Ctx& c = x->c;
                c.p.pair_warps = w;
                c.p.fft_lines = l;
                c.p.pair_schedule = sc;
                if (c.p.prune_every != p || c.p.pair_layout != ly) {
                    c.p.prune_every = p;
                    c.p.pair_layout = ly;
                    c.pruned_valid = false;
                    c.since_prune = 0;
                }
            }
            drop_graph(b);
        };
        auto time_it = [&]() {
            run(b, flags);   // capture + first replay (untimed)
            MDF_CUDA_TRY(cudaStreamSynchronize(b->main));
            MDF_CUDA_TRY(cudaEventRecord(e0, b->main));
            for (int r = 0; r < R; ++r) MDF_CUDA_TRY(cudaGraphLaunch(b->exec, b->main));
            MDF_CUDA_TRY(cudaEventRecord(e1, b->main));
            MDF_CUDA_TRY(cudaEventSynchronize(e1));
            float ms = 0;
            MDF_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
            return (double)ms / R;
        };
        const Ctx& c0 = b->sys[0]->c;
        const int w0 = c0.p.pair_warps, l0 = c0.p.fft_lines, p0 = c0.p.prune_every, s0 = c0.p.pair_schedule,
                  y0 = c0.p.pair_layout;
        double t_default = time_it();
        double best = 1e300;
        int bw = w0, bl = l0, bp = p0, bs = s0, by = y0, tried = 0;
        // self-pruning systems (prune_every < 0) keep that mode
        const int prune_self[1] = {p0};
        const int* popts = p0 < 0 ? prune_self : prune;
        const int np = p0 < 0 ? 1 : 2;
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
        run(b, flags);
        MDF_CUDA_TRY(cudaStreamSynchronize(b->main));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
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
    });
}

}  // extern "C"
