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
// block, FFT lines per block, per-evaluation pruning on or off) on the batch
// itself and keeps the fastest; results do not depend on the choice (all
// sums are fixed point).
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

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

void capture(mdf_batch* b, uint32_t flags)
{
    drop_graph(b);
    MDF_CUDA_TRY(cudaStreamBeginCapture(b->main, cudaStreamCaptureModeThreadLocal));
    try {
        enqueue(b, flags);
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
    if (b->main) cudaStreamSynchronize(b->main);
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
        const int warps[3] = {2, 4, 8}, lines[3] = {1, 2, 4}, prune[2] = {0, 1};
        cudaEvent_t e0, e1;
        MDF_CUDA_TRY(cudaEventCreate(&e0));
        MDF_CUDA_TRY(cudaEventCreate(&e1));
        auto apply = [&](int w, int l, int p) {
            for (mdf_ctx* x : b->sys) {
                Ctx& c = x->c;
                c.p.pair_warps = w;
                c.p.fft_lines = l;
                if (c.p.prune_every != p) {
                    c.p.prune_every = p;
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
        const int w0 = c0.p.pair_warps, l0 = c0.p.fft_lines, p0 = c0.p.prune_every;
        double t_default = time_it();
        double best = 1e300;
        int bw = w0, bl = l0, bp = p0, tried = 0;
        for (int p : prune)
            for (int w : warps)
                for (int l : lines) {
                    apply(w, l, p);
                    const double t = time_it();
                    ++tried;
                    if (t < best) {
                        best = t;
                        bw = w; bl = l; bp = p;
                    }
                }
        apply(bw, bl, bp);
        run(b, flags);
        MDF_CUDA_TRY(cudaStreamSynchronize(b->main));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (rep) {
            rep->pair_warps = bw;
            rep->fft_lines = bl;
            rep->prune_every = bp;
            rep->n_tried = tried;
            rep->best_ms = best;
            rep->default_ms = t_default;
        }
    });
}

}  // extern "C"
