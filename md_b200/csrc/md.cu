// Velocity-Verlet NVE dynamics and a steepest-descent minimiser on the
// device, with the pairlist rebuild trigger of the reference
// (src/System/NonBondedUtils.cpp:87-100: rebuild when the largest
// displacement since the last build exceeds half the skin) and an Amber rst7
// writer for positions and velocities.
//
// Units: positions A, velocities A/ps, masses amu, forces kcal/mol/A;
// a = F/m * 418.4 (1 kcal/mol = 418.4 amu A^2 ps^-2).
//
// Steps run in chunks of `chunk` steps, each chunk one CUDA graph:
//   per step: v += dt/2 a; x += dt v | forces (the full evaluation) |
//             v += dt/2 a (+ kinetic energy on the chunk's last step) |
//             largest displacement since the last build (running max)
// The host looks at the chunk's end: energies for the record, and the
// displacement and the largest speed for the rebuild decision (rebuild when
// the displacement plus twice what the fastest atom can cover in one chunk
// would pass half the skin; passing half the skin inside a chunk is reported
// as an error).  A rebuild (host-synchronous list build) is followed by a new
// capture.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "mdf_device.cuh"
#include "mdf_internal.cuh"

namespace mdf {

constexpr double MD_ACCEL = 418.4;          // (kcal/mol/A)/amu -> A/ps^2
constexpr double KB_KCAL = 0.0019872041;    // kcal/mol/K
constexpr double AMBER_VEL = 20.455;        // A/ps per Amber velocity unit

// Reduction words: kinetic energy (fixed point) | max displacement^2 bits |
// status | max |F| bits (minimiser) | max speed^2 bits.  Kernels reduce into
// device memory (every warp adds or takes a maximum); one small kernel then
// publishes the words to mapped host memory for the host to read after the
// stream is synchronised.  (Atomics straight into mapped host memory would
// cross the host link once per warp.)
constexpr int MD_WORDS = 5;

__global__ void k_md_publish(const unsigned long long* __restrict__ src, unsigned long long* __restrict__ dst)
{
    const int i = threadIdx.x;
    if (i < MD_WORDS) dst[i] = src[i];
}

// Zero the words whose bit is set in mask.
__global__ void k_md_reset(unsigned long long* __restrict__ w, unsigned mask)
{
    const int i = threadIdx.x;
    if (i < MD_WORDS && ((mask >> i) & 1u)) w[i] = 0ull;
}

static double bits_to_double(unsigned long long u)
{
    double d;
    memcpy(&d, &u, sizeof(d));
    return d;
}

__global__ void k_md_kick_drift(int N, double* __restrict__ x, double* __restrict__ v,
                                const double* __restrict__ f, const double* __restrict__ invm, double dt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * N) return;
    const double a = f[i] * invm[i / 3];
    const double vh = v[i] + 0.5 * dt * a;
    v[i] = vh;
    x[i] += dt * vh;
}

// Second half kick; with ke != nullptr also the kinetic energy 1/2 m v^2 in
// kcal/mol (fixed point, deterministic) and the largest speed^2.
__global__ void k_md_kick(int N, double* __restrict__ v, const double* __restrict__ f,
                          const double* __restrict__ invm, double dt, unsigned long long* __restrict__ ke,
                          unsigned long long* __restrict__ vmax2, unsigned* st)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0, s = 0.0;
    if (a < N) {
        const double im = invm[a];
        for (int k = 0; k < 3; ++k) {
            const double vv = v[3 * a + k] + 0.5 * dt * f[3 * a + k] * im;
            v[3 * a + k] = vv;
            s += vv * vv;
        }
        if (im > 0.0) e = 0.5 * s / im;   // 1/2 m v^2 / 418.4 = 1/2 v^2 / invm
    }
    if (ke) {
        double m = s;
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(vmax2, (unsigned long long)__double_as_longlong(m));
        const double vals[1] = {e};
        const int idx[1] = {0};
        block_acc_fixed<1>(vals, ke, idx, ENERGY_SCALE, st);
    }
}

// Running maximum of the squared displacement since the last list build (raw
// coordinates: the integrator never wraps them).  Non-negative doubles order
// like their bit patterns, so atomicMax on the bits works.
__global__ void k_md_displacement(int N, const double* __restrict__ x, const double* __restrict__ xref,
                                  unsigned long long* __restrict__ dmax2)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    double d2 = 0.0;
    if (a < N) {
        for (int k = 0; k < 3; ++k) {
            const double d = x[3 * a + k] - xref[3 * a + k];
            d2 += d * d;
        }
    }
    for (int o = 16; o > 0; o >>= 1) d2 = fmax(d2, __shfl_xor_sync(0xffffffffu, d2, o));
    if ((threadIdx.x & 31) == 0 && d2 > 0.0) atomicMax(dmax2, (unsigned long long)__double_as_longlong(d2));
}

static void md_words(Ctx& c)
{
    if (!c.md_host) {
        MDF_CUDA_TRY(cudaHostAlloc((void**)&c.md_host, sizeof(unsigned long long) * MD_WORDS, cudaHostAllocMapped));
        MDF_CUDA_TRY(cudaHostGetDevicePointer((void**)&c.md_hmap, c.md_host, 0));
        memset(c.md_host, 0, sizeof(unsigned long long) * MD_WORDS);
        c.md_words.alloc(MD_WORDS);
        MDF_CUDA_TRY(cudaMemsetAsync(c.md_words.p, 0, sizeof(unsigned long long) * MD_WORDS, c.stream));
        c.md_dev = c.md_words.p;
        c.md_dev_st = reinterpret_cast<unsigned*>(c.md_dev + 2);
    }
}

static void md_drop_graph(Ctx& c)
{
    if (c.md_exec) cudaGraphExecDestroy(c.md_exec);
    if (c.md_graph) cudaGraphDestroy(c.md_graph);
    c.md_exec = nullptr;
    c.md_graph = nullptr;
}

// Record one chunk of `steps` steps into a new graph (not instantiated).
static cudaGraph_t md_record(Ctx& c, int steps, double dt)
{
    cudaStream_t s = c.stream;
    const int th = 256;
    const bool timing = c.timing;
    c.timing = false;   // no per-phase events inside a captured chunk
    cudaGraph_t g = nullptr;
    MDF_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
        k_md_reset<<<1, 32, 0, s>>>(c.md_dev, (1u << 0) | (1u << 2) | (1u << 4));
        for (int k = 0; k < steps; ++k) {
            const bool last = k == steps - 1;
            k_md_kick_drift<<<grid_blocks(3LL * c.N, th), th, 0, s>>>(c.N, c.xyz.p, c.md_v.p, c.forces_out.p,
                                                                    c.md_invm.p, dt);
            eval_async_impl(c, MDF_COMPUTE_FORCES | (last ? MDF_COMPUTE_ENERGY : 0u));
            k_md_kick<<<grid_blocks(c.N, th), th, 0, s>>>(c.N, c.md_v.p, c.forces_out.p, c.md_invm.p, dt,
                                                          last ? c.md_dev : nullptr, c.md_dev + 4, c.md_dev_st);
            k_md_displacement<<<grid_blocks(c.N, th), th, 0, s>>>(c.N, c.xyz.p, c.md_xref.p, c.md_dev + 1);
        }
        k_md_publish<<<1, 32, 0, s>>>(c.md_dev, c.md_hmap);
        MDF_CUDA_TRY(cudaGetLastError());
    } catch (...) {
        c.timing = timing;
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    c.timing = timing;
    MDF_CUDA_TRY(cudaStreamEndCapture(s, &g));
    return g;
}

// A ready graph for `steps` steps: instantiate on first use; after a list
// rebuild re-record and update the instantiated graph in place (same shape,
// new sizes and pointers), instantiating afresh only if the update is refused.
static void md_prepare(Ctx& c, int steps, double dt)
{
    if (c.md_exec && c.md_graph_steps == steps && c.md_graph_dt == dt && !c.md_stale) return;
    cudaGraph_t g = md_record(c, steps, dt);
    if (c.md_exec && c.md_graph_steps == steps && c.md_graph_dt == dt) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(c.md_exec, g, &info) == cudaSuccess) {
            if (c.md_graph) cudaGraphDestroy(c.md_graph);
            c.md_graph = g;
            c.md_stale = false;
            return;
        }
        (void)cudaGetLastError();   // the refusal is not an error here
    }
    md_drop_graph(c);
    c.md_graph = g;
    MDF_CUDA_TRY(cudaGraphInstantiate(&c.md_exec, c.md_graph, 0));
    c.md_graph_steps = steps;
    c.md_graph_dt = dt;
    c.md_stale = false;
}

// New pairlist at the current positions.  With need_forces the forces are
// evaluated too (start of a run); otherwise the last chunk's forces, at these
// same positions, stay in place for the next half kick.
static void md_rebuild(Ctx& c, bool need_forces)
{
    build_pairlist(c);
    MDF_CUDA_TRY(cudaMemcpyAsync(c.md_xref.p, c.xyz.p, sizeof(double) * 3 * (size_t)c.N, cudaMemcpyDeviceToDevice,
                                 c.stream));
    if (need_forces) {
        eval_async_impl(c, MDF_COMPUTE_FORCES);   // also clears the accumulators and counts pairs
    } else {
        // the slot layout changed: clear the accumulators here rather than in
        // every replay of the next graph; pairs are not counted inside graphs
        MDF_CUDA_TRY(cudaMemsetAsync(c.f_slot.p, 0, sizeof(unsigned long long) * 3 * (size_t)c.n_slots, c.stream));
        MDF_CUDA_TRY(cudaMemsetAsync(c.f_atom.p, 0, sizeof(unsigned long long) * 3 * (size_t)c.N, c.stream));
        c.need_clear = false;
        c.count_next = false;
    }
    k_md_reset<<<1, 32, 0, c.stream>>>(c.md_dev, 1u << 1);   // displacement since this build
    MDF_CUDA_TRY(cudaGetLastError());
    MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
    if (need_forces) check_host_status(c);
    c.md_host[1] = 0;
    c.md_stale = true;
}

void md_init(Ctx& c, const double* masses, const double* vel, double temperature, uint64_t seed)
{
    if (c.p.semantics != MDF_SEM_PHYSICAL) throw ApiError(MDF_ERR_UNSUPPORTED, "dynamics needs PHYSICAL semantics");
    if (!masses) throw ApiError(MDF_ERR_INVALID, "masses are required");
    if (!c.have_positions) throw ApiError(MDF_ERR_STATE, "positions not set");
    std::vector<double> invm(c.N), v(3 * (size_t)c.N, 0.0);
    double mtot = 0;
    for (int i = 0; i < c.N; ++i) {
        if (!(masses[i] >= 0.0) || !std::isfinite(masses[i])) throw ApiError(MDF_ERR_INVALID, "bad mass");
        invm[i] = masses[i] > 0.0 ? MD_ACCEL / masses[i] : 0.0;
        mtot += masses[i];
    }
    if (vel) {
        for (size_t k = 0; k < v.size(); ++k) v[k] = vel[k];
    } else if (temperature > 0.0) {
        // Maxwell-Boltzmann at T, then the centre-of-mass motion removed
        std::mt19937_64 rng(seed);
        std::normal_distribution<double> nd(0.0, 1.0);
        double p[3] = {0, 0, 0};
        for (int i = 0; i < c.N; ++i) {
            if (masses[i] <= 0.0) continue;
            const double sd = std::sqrt(KB_KCAL * temperature * MD_ACCEL / masses[i]);
            for (int k = 0; k < 3; ++k) {
                v[3 * i + k] = sd * nd(rng);
                p[k] += masses[i] * v[3 * i + k];
            }
        }
        if (mtot > 0)
            for (int i = 0; i < c.N; ++i)
                if (masses[i] > 0.0)
                    for (int k = 0; k < 3; ++k) v[3 * i + k] -= p[k] / mtot;
    }
    double v2 = 0;
    for (double x : v) v2 = std::max(v2, x * x);
    c.md_invm.upload(invm.data(), invm.size(), c.stream);
    c.md_v.upload(v.data(), v.size(), c.stream);
    c.md_xref.alloc(3 * (size_t)c.N);
    md_words(c);
    MDF_CUDA_TRY(cudaMemsetAsync(c.md_words.p, 0, sizeof(unsigned long long) * MD_WORDS, c.stream));
    memset(c.md_host, 0, sizeof(unsigned long long) * MD_WORDS);
    double vmax2 = 3.0 * v2;   // bound until the first chunk has measured it
    memcpy(&c.md_host[4], &vmax2, sizeof(double));
    c.md_ready = true;
    md_drop_graph(c);
    md_rebuild(c, true);
}

void md_run(Ctx& c, long long nsteps, double dt, int chunk, int rebuild_every, double* samples, long long cap,
            mdf_md_report* rep)
{
    if (!c.md_ready) throw ApiError(MDF_ERR_STATE, "mdf_md_init first");
    if (nsteps < 0 || !(dt > 0.0)) throw ApiError(MDF_ERR_INVALID, "bad step count or time step");
    if (chunk <= 0) chunk = 10;
    const double half_skin = 0.5 * c.p.skin;
    mdf_md_report r;
    memset(&r, 0, sizeof(r));
    const auto t0 = std::chrono::steady_clock::now();
    long long done = 0, since_build = 0, nsamp = 0;
    while (done < nsteps) {
        const int steps = (int)std::min<long long>(chunk, nsteps - done);
        const bool due = rebuild_every > 0 && since_build >= rebuild_every;
        // the next chunk can move an atom by about steps * dt * vmax; keep
        // twice that as headroom below half the skin
        const double dnow = std::sqrt(bits_to_double(c.md_host[1]));
        const double reach = 2.0 * steps * dt * std::sqrt(bits_to_double(c.md_host[4]));
        using clk = std::chrono::steady_clock;
        const auto ta = clk::now();
        if (due || dnow + reach > half_skin) {
            md_rebuild(c, false);
            since_build = 0;
            ++r.rebuilds;
        }
        const auto tb = clk::now();
        md_prepare(c, steps, dt);
        const auto tc = clk::now();
        MDF_CUDA_TRY(cudaGraphLaunch(c.md_exec, c.stream));
        MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
        const auto td = clk::now();
        r.rebuild_s += std::chrono::duration<double>(tb - ta).count();
        r.record_s += std::chrono::duration<double>(tc - tb).count();
        r.wait_s += std::chrono::duration<double>(td - tc).count();
        check_host_status(c);
        if ((unsigned)c.md_host[2] & ST_OVERFLOW) throw ApiError(MDF_ERR_OVERFLOW, "kinetic energy out of range");
        done += steps;
        since_build += steps;
        if (std::sqrt(bits_to_double(c.md_host[1])) > half_skin)
            throw ApiError(MDF_ERR_STATE, "an atom moved more than half the skin between list builds by step " +
                                              std::to_string(done) + " (smaller time step or shorter chunks)");
        mdf_energies e;
        host_energies(c, MDF_COMPUTE_ENERGY, &e);
        const double ke = (double)(long long)c.md_host[0] * ENERGY_ISCALE;
        if (samples && nsamp < cap) {
            samples[3 * nsamp] = done * dt;
            samples[3 * nsamp + 1] = e.total;
            samples[3 * nsamp + 2] = ke;
        }
        if (nsamp == 0) {
            r.pe_first = e.total;
            r.ke_first = ke;
        }
        ++nsamp;
        r.pe_last = e.total;
        r.ke_last = ke;
        r.steps = done;
    }
    r.samples = nsamp;
    r.wall_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rep) *rep = r;
}

// ------------------------------------------------------------- minimiser
// Steepest descent with an adaptive step (the reference's intended use of
// calculate_forces, include/System/System.h:84,113): move every atom along
// its force, the largest move being `step`; keep the move and grow the step
// by 1.2 if the energy went down, else undo it and halve the step.  Stops at
// max |F| <= fmax_tol or after max_iter iterations.  The list is rebuilt
// before the accumulated largest move could pass a quarter of the skin.

__global__ void k_min_fmax(int n3, const double* __restrict__ f, unsigned long long* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double m = i < n3 ? fabs(f[i]) : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

__global__ void k_min_move(int n3, double* __restrict__ x, const double* __restrict__ f, double scale)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n3) x[i] += scale * f[i];
}

void minimize(Ctx& c, int max_iter, double fmax_tol, double max_step, mdf_min_report* rep)
{
    if (c.p.semantics != MDF_SEM_PHYSICAL) throw ApiError(MDF_ERR_UNSUPPORTED, "the minimiser needs PHYSICAL semantics");
    if (!c.have_positions) throw ApiError(MDF_ERR_STATE, "positions not set");
    if (!(max_step > 0.0)) max_step = 0.1;
    cudaStream_t s = c.stream;
    const int th = 256;
    const long long n3 = 3LL * c.N;
    md_words(c);
    c.min_x.alloc(n3);
    c.min_f.alloc(n3);
    auto evaluate = [&](double& e, double& fmax) {
        k_md_reset<<<1, 32, 0, s>>>(c.md_dev, 1u << 3);
        eval_async_impl(c, MDF_COMPUTE_ENERGY | MDF_COMPUTE_FORCES);
        k_min_fmax<<<grid_blocks(n3, th), th, 0, s>>>((int)n3, c.forces_out.p, c.md_dev + 3);
        k_md_publish<<<1, 32, 0, s>>>(c.md_dev, c.md_hmap);
        MDF_CUDA_TRY(cudaGetLastError());
        MDF_CUDA_TRY(cudaStreamSynchronize(s));
        check_host_status(c);
        mdf_energies en;
        host_energies(c, MDF_COMPUTE_ENERGY, &en);
        e = en.total;
        fmax = bits_to_double(c.md_host[3]);
    };
    mdf_min_report r;
    memset(&r, 0, sizeof(r));
    build_pairlist(c);
    double moved = 0.0, step = std::min(0.01, max_step);
    double e0, f0;
    evaluate(e0, f0);
    r.e_initial = e0;
    r.evaluations = 1;
    int it = 0;
    for (; it < max_iter && f0 > fmax_tol; ++it) {
        if (moved + step > 0.25 * c.p.skin) {
            build_pairlist(c);
            ++r.rebuilds;
            moved = 0.0;
            evaluate(e0, f0);   // the same positions on the new list
            ++r.evaluations;
        }
        MDF_CUDA_TRY(cudaMemcpyAsync(c.min_x.p, c.xyz.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
        MDF_CUDA_TRY(cudaMemcpyAsync(c.min_f.p, c.forces_out.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
        k_min_move<<<grid_blocks(n3, th), th, 0, s>>>((int)n3, c.xyz.p, c.forces_out.p, step / f0);
        MDF_CUDA_TRY(cudaGetLastError());
        double e1, f1;
        evaluate(e1, f1);
        ++r.evaluations;
        if (e1 < e0) {
            moved += step;
            e0 = e1;
            f0 = f1;
            step = std::min(step * 1.2, max_step);
        } else {
            MDF_CUDA_TRY(cudaMemcpyAsync(c.xyz.p, c.min_x.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
            MDF_CUDA_TRY(cudaMemcpyAsync(c.forces_out.p, c.min_f.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
            step *= 0.5;
            if (step < 1e-7) break;
        }
    }
    MDF_CUDA_TRY(cudaStreamSynchronize(s));
    r.iterations = it;
    r.e_final = e0;
    r.fmax_final = f0;
    c.md_ready = false;   // positions and list changed: dynamics restart from mdf_md_init
    md_drop_graph(c);
    if (rep) *rep = r;
}

// ------------------------------------------------------------- L-BFGS
// Limited-memory BFGS (Nocedal & Wright, Numerical Optimization, 2nd ed.,
// Algorithm 7.4 two-loop recursion and 7.5), the solver the reference names
// as the consumer of calculate_forces (include/System/System.h:84,113).
// Vectors live on the device; the recursion's scalars (alpha_i, beta,
// gamma) stay in device memory between its kernels, so a direction costs no
// host round trip.  Dot products are two-stage reductions with a fixed block
// count and order: runs are bit-reproducible.  Line search: backtracking
// from t = 1 (the step scaled so no atom moves more than max_step) with the
// Armijo condition, c1 = 1e-4 (where the energy change is below its
// resolution, a smaller largest force component decides).  A pair (s, y)
// with s.y <= 0 is not stored.
constexpr int LB_BLOCKS = 296;   // 2 x 148 SMs
constexpr int LB_THREADS = 256;

__global__ void __launch_bounds__(LB_THREADS) k_lb_dot_part(long long n, const double* __restrict__ a,
                                                            const double* __restrict__ b, double* __restrict__ part)
{
    __shared__ double w[LB_THREADS / 32];
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s = fma(a[i], b[i], s);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < LB_THREADS / 32; ++k) t += w[k];
        part[blockIdx.x] = t;
    }
}

// out = (sum of the partials) * (mul ? *mul : 1), in a fixed order
__global__ void k_lb_dot_final(int nb, const double* __restrict__ part, double* __restrict__ out,
                               const double* __restrict__ mul)
{
    if (threadIdx.x != 0) return;
    double t = 0.0;
    for (int k = 0; k < nb; ++k) t += part[k];
    *out = mul ? t * *mul : t;
}

__global__ void k_lb_set(long long n, double* __restrict__ out, const double* __restrict__ in, double scale)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = scale * in[i];
}

// y += sign * (*coef) * x
__global__ void k_lb_axpy(long long n, double* __restrict__ y, const double* __restrict__ x,
                          const double* __restrict__ coef, double sign)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = fma(sign * *coef, x[i], y[i]);
}

// r += (*a - *b) * s
__global__ void k_lb_axpy_diff(long long n, double* __restrict__ r, const double* __restrict__ s,
                               const double* __restrict__ a, const double* __restrict__ b)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = fma(*a - *b, s[i], r[i]);
}

// r *= (*num) / (*den)
__global__ void k_lb_scale(long long n, double* __restrict__ r, const double* __restrict__ num,
                           const double* __restrict__ den)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] *= *num / *den;
}

// x = x0 - t r (r approximates H g, so -r is the descent direction)
__global__ void k_lb_trial(long long n, double* __restrict__ x, const double* __restrict__ x0,
                           const double* __restrict__ r, double t)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = fma(-t, r[i], x0[i]);
}

// s = x - x0, y = g - g0 = F0 - F
__global__ void k_lb_pair(long long n, double* __restrict__ s, double* __restrict__ y, const double* __restrict__ x,
                          const double* __restrict__ x0, const double* __restrict__ f, const double* __restrict__ f0)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        s[i] = x[i] - x0[i];
        y[i] = f0[i] - f[i];
    }
}

__global__ void k_lb_recip(const double* __restrict__ in, double* __restrict__ out) { *out = 1.0 / *in; }

// largest per-atom norm of r (max of non-negative doubles through their bit patterns)
__global__ void k_lb_atom_max(int N, const double* __restrict__ r, unsigned long long* __restrict__ out)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0;
    if (a < N) m = sqrt(r[3 * a] * r[3 * a] + r[3 * a + 1] * r[3 * a + 1] + r[3 * a + 2] * r[3 * a + 2]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

void minimize_lbfgs(Ctx& c, int max_iter, double fmax_tol, double max_step, int m, mdf_min_report* rep)
{
    if (c.p.semantics != MDF_SEM_PHYSICAL) throw ApiError(MDF_ERR_UNSUPPORTED, "the minimiser needs PHYSICAL semantics");
    if (!c.have_positions) throw ApiError(MDF_ERR_STATE, "positions not set");
    if (m < 0 || m > 64) throw ApiError(MDF_ERR_INVALID, "history must be 0 (= 8) .. 64");
    if (m == 0) m = 8;
    if (!(max_step > 0.0)) max_step = 0.1;
    cudaStream_t s = c.stream;
    const int th = 256;
    const long long n3 = 3LL * c.N;
    const int nbv = grid_blocks(n3, th);
    md_words(c);
    c.min_x.alloc(n3);
    c.min_f.alloc(n3);
    c.lb_s.alloc((size_t)m * n3);
    c.lb_y.alloc((size_t)m * n3);
    c.lb_q.alloc(n3);
    c.lb_part.alloc(LB_BLOCKS);
    // scalars: alpha[m] | rho[m] | beta | sy | yy | gd | dmax bits
    c.lb_scal.alloc(2 * m + 5);
    double* alpha = c.lb_scal.p;
    double* rho = alpha + m;
    double* beta = rho + m;
    double* sy = beta + 1;
    double* yy = sy + 1;
    double* gd = yy + 1;
    unsigned long long* dmaxw = reinterpret_cast<unsigned long long*>(gd + 1);
    auto dot = [&](const double* a, const double* b, double* out, const double* mul) {
        k_lb_dot_part<<<LB_BLOCKS, LB_THREADS, 0, s>>>(n3, a, b, c.lb_part.p);
        k_lb_dot_final<<<1, 32, 0, s>>>(LB_BLOCKS, c.lb_part.p, out, mul);
    };
    auto evaluate = [&](double& e, double& fmax) {
        k_md_reset<<<1, 32, 0, s>>>(c.md_dev, 1u << 3);
        eval_async_impl(c, MDF_COMPUTE_ENERGY | MDF_COMPUTE_FORCES);
        k_min_fmax<<<grid_blocks(n3, th), th, 0, s>>>((int)n3, c.forces_out.p, c.md_dev + 3);
        k_md_publish<<<1, 32, 0, s>>>(c.md_dev, c.md_hmap);
        MDF_CUDA_TRY(cudaGetLastError());
        MDF_CUDA_TRY(cudaStreamSynchronize(s));
        check_host_status(c);
        mdf_energies en;
        host_energies(c, MDF_COMPUTE_ENERGY, &en);
        e = en.total;
        fmax = bits_to_double(c.md_host[3]);
    };
    auto read_scalars = [&](double& gdv, double& dmaxv) {
        double h[2];
        MDF_CUDA_TRY(cudaMemcpyAsync(h, gd, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        MDF_CUDA_TRY(cudaStreamSynchronize(s));
        gdv = h[0];
        unsigned long long u;
        memcpy(&u, &h[1], sizeof(u));
        dmaxv = bits_to_double(u);
    };
    mdf_min_report r;
    memset(&r, 0, sizeof(r));
    build_pairlist(c);
    double e0, f0;
    evaluate(e0, f0);
    r.e_initial = e0;
    r.evaluations = 1;
    int head = 0, count = 0;   // ring of stored pairs: newest at (head - 1) mod m
    double moved = 0.0;
    int it = 0;
    for (; it < max_iter && f0 > fmax_tol; ++it) {
        if (moved + max_step > 0.25 * c.p.skin) {
            build_pairlist(c);
            ++r.rebuilds;
            moved = 0.0;
            evaluate(e0, f0);   // the same positions on the new list
            ++r.evaluations;
        }
        // r = H g by the two-loop recursion, g = -F
        double* q = c.lb_q.p;
        k_lb_set<<<nbv, th, 0, s>>>(n3, q, c.forces_out.p, -1.0);
        for (int k = 0; k < count; ++k) {
            const int i = (head - 1 - k + m) % m;
            dot(c.lb_s.p + (size_t)i * n3, q, alpha + i, rho + i);
            k_lb_axpy<<<nbv, th, 0, s>>>(n3, q, c.lb_y.p + (size_t)i * n3, alpha + i, -1.0);
        }
        if (count > 0) k_lb_scale<<<nbv, th, 0, s>>>(n3, q, sy, yy);   // H0 = (s.y / y.y) I, newest pair
        for (int k = count - 1; k >= 0; --k) {
            const int i = (head - 1 - k + m) % m;
            dot(c.lb_y.p + (size_t)i * n3, q, beta, rho + i);
            k_lb_axpy_diff<<<nbv, th, 0, s>>>(n3, q, c.lb_s.p + (size_t)i * n3, alpha + i, beta);
        }
        // directional derivative g.d = F.r (d = -r) and the largest atom move of r
        dot(c.forces_out.p, q, gd, nullptr);
        MDF_CUDA_TRY(cudaMemsetAsync(dmaxw, 0, sizeof(unsigned long long), s));
        k_lb_atom_max<<<grid_blocks(c.N, th), th, 0, s>>>(c.N, q, dmaxw);
        MDF_CUDA_TRY(cudaGetLastError());
        double gdv, dmax;
        read_scalars(gdv, dmax);
        if (!(gdv < 0.0) || !(dmax > 0.0)) {   // not a descent direction: drop the history, use -g
            count = 0;
            k_lb_set<<<nbv, th, 0, s>>>(n3, q, c.forces_out.p, -1.0);
            dot(c.forces_out.p, q, gd, nullptr);
            MDF_CUDA_TRY(cudaMemsetAsync(dmaxw, 0, sizeof(unsigned long long), s));
            k_lb_atom_max<<<grid_blocks(c.N, th), th, 0, s>>>(c.N, q, dmaxw);
            read_scalars(gdv, dmax);
            if (!(gdv < 0.0) || !(dmax > 0.0)) break;   // zero gradient
        }
        // first step (no curvature yet): at most 0.01 A; afterwards the unit step, capped at max_step
        double t = count > 0 ? std::min(1.0, max_step / dmax) : std::min(0.01, max_step) / dmax;
        MDF_CUDA_TRY(cudaMemcpyAsync(c.min_x.p, c.xyz.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
        MDF_CUDA_TRY(cudaMemcpyAsync(c.min_f.p, c.forces_out.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
        bool accepted = false;
        double e1 = e0, f1 = f0;
        for (int ls = 0; ls < 30; ++ls) {
            k_lb_trial<<<nbv, th, 0, s>>>(n3, c.xyz.p, c.min_x.p, q, t);
            evaluate(e1, f1);
            ++r.evaluations;
            // Armijo; or, with the change at the energy's resolution (fixed-point
            // sums), a smaller largest force
            const bool flat = std::fabs(e1 - e0) <= 1e-9 * std::max(1.0, std::fabs(e0));
            if (e1 <= e0 + 1e-4 * t * gdv || (flat && f1 < f0)) {
                accepted = true;
                break;
            }
            t *= 0.5;
        }
        if (!accepted) {   // restore; with no history left to drop, stop
            MDF_CUDA_TRY(cudaMemcpyAsync(c.xyz.p, c.min_x.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
            MDF_CUDA_TRY(cudaMemcpyAsync(c.forces_out.p, c.min_f.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice,
                                         s));
            if (count == 0) break;
            count = 0;
            continue;
        }
        moved += t * dmax;
        // the new pair (s, y), kept when s.y > 0
        double* sn = c.lb_s.p + (size_t)head * n3;
        double* yn = c.lb_y.p + (size_t)head * n3;
        k_lb_pair<<<nbv, th, 0, s>>>(n3, sn, yn, c.xyz.p, c.min_x.p, c.forces_out.p, c.min_f.p);
        // staging: alpha[head] and beta are rewritten by the next recursion anyway
        double* sy_stage = alpha + head;
        double* yy_stage = beta;
        dot(sn, yn, sy_stage, nullptr);
        dot(yn, yn, yy_stage, nullptr);
        double syv = 0.0, yyv = 0.0;
        MDF_CUDA_TRY(cudaMemcpyAsync(&syv, sy_stage, sizeof(double), cudaMemcpyDeviceToHost, s));
        MDF_CUDA_TRY(cudaMemcpyAsync(&yyv, yy_stage, sizeof(double), cudaMemcpyDeviceToHost, s));
        MDF_CUDA_TRY(cudaStreamSynchronize(s));
        if (syv > 1e-12 * std::sqrt(yyv) && yyv > 0.0) {
            MDF_CUDA_TRY(cudaMemcpyAsync(sy, sy_stage, sizeof(double), cudaMemcpyDeviceToDevice, s));
            MDF_CUDA_TRY(cudaMemcpyAsync(yy, yy_stage, sizeof(double), cudaMemcpyDeviceToDevice, s));
            k_lb_recip<<<1, 1, 0, s>>>(sy_stage, rho + head);
            head = (head + 1) % m;
            count = std::min(count + 1, m);
        }
        e0 = e1;
        f0 = f1;
    }
    MDF_CUDA_TRY(cudaStreamSynchronize(s));
    r.iterations = it;
    r.e_final = e0;
    r.fmax_final = f0;
    c.md_ready = false;   // positions and list changed: dynamics restart from mdf_md_init
    md_drop_graph(c);
    if (rep) *rep = r;
}

void md_state(Ctx& c, double* xyz, double* vel)
{
    MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
    if (xyz) MDF_CUDA_TRY(cudaMemcpy(xyz, c.xyz.p, sizeof(double) * 3 * (size_t)c.N, cudaMemcpyDeviceToHost));
    if (vel) {
        if (!c.md_v.p) throw ApiError(MDF_ERR_STATE, "no velocities: mdf_md_init first");
        MDF_CUDA_TRY(cudaMemcpy(vel, c.md_v.p, sizeof(double) * 3 * (size_t)c.N, cudaMemcpyDeviceToHost));
    }
}

// Amber ASCII restart: title, natoms + time, coordinates 6 per line (12.7f),
// velocities in Amber units (A per 1/20.455 ps), box lengths and angles.
void md_write_rst7(Ctx& c, const char* path, const char* title, double time_ps)
{
    if (!path) throw ApiError(MDF_ERR_INVALID, "no path");
    std::vector<double> x(3 * (size_t)c.N), v(3 * (size_t)c.N);
    md_state(c, x.data(), v.data());
    FILE* f = std::fopen(path, "w");
    if (!f) throw ApiError(MDF_ERR_INVALID, std::string("cannot open ") + path);
    std::fprintf(f, "%s\n", title ? title : "md_b200 restart");
    std::fprintf(f, "%6d%15.7e\n", c.N, time_ps);
    auto block = [&](const std::vector<double>& a, double scale) {
        for (size_t k = 0; k < a.size(); ++k) {
            std::fprintf(f, "%12.7f", a[k] * scale);
            if (k % 6 == 5 || k + 1 == a.size()) std::fprintf(f, "\n");
        }
    };
    block(x, 1.0);
    block(v, 1.0 / AMBER_VEL);
    std::fprintf(f, "%12.7f%12.7f%12.7f%12.7f%12.7f%12.7f\n", c.box[0], c.box[1], c.box[2], 90.0, 90.0, 90.0);
    if (std::fclose(f) != 0) throw ApiError(MDF_ERR_INVALID, std::string("write failed: ") + path);
}

}  // namespace mdf
