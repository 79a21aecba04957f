// Bonded forces and energies without any device allocation.
//
// Some callers cannot let the library allocate device memory at call time:
// an MD driver that reserves the whole device up front for its own arena (a
// cudaMalloc would then fail, or push the driver's pool out of its budget),
// and a time-step loop that runs other streams concurrently, where
// cudaMalloc/cudaFree may synchronise the device and stall them.  This entry
// point therefore keeps its scratch - the int64 fixed-point force
// accumulators, the energy words and the status word - in one file-scope
// __device__ array of fixed size and allocates nothing: no cudaMalloc, no
// cudaFree, no pool or library routine that allocates.
//
// The array is one per device and shared by every context on it, so two calls
// that overlap in time race on it; callers must serialise them.
#include <mutex>

#include "mdf_device.cuh"
#include "mdf_internal.cuh"

namespace mdf {

constexpr int NOALLOC_MAX_ATOMS = MDF_NOALLOC_MAX_ATOMS;
constexpr size_t NOALLOC_FORCE_WORDS = 3 * (size_t)NOALLOC_MAX_ATOMS;
constexpr size_t NOALLOC_WORDS = NOALLOC_FORCE_WORDS + NUM_SCAL;
constexpr int NOALLOC_MAX_DEVICES = 64;

// [0, 3 * MAX_ATOMS): forces SoA x|y|z with stride natoms of the call;
// then NUM_SCAL words: energies + virial, pairs in cutoff, status.
static __device__ __align__(256) unsigned long long g_noalloc_scratch[NOALLOC_WORDS];

static std::mutex g_noalloc_mutex;
static unsigned long long* g_noalloc_ptr[NOALLOC_MAX_DEVICES];

// Device address of the scratch array on the current device, looked up once.
static unsigned long long* noalloc_scratch(int device)
{
    if (device < 0 || device >= NOALLOC_MAX_DEVICES)
        throw ApiError(MDF_ERR_UNSUPPORTED, "mdf_compute_bonded_noalloc: device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (rc != cudaSuccess || !p)
            throw ApiError(MDF_ERR_CUDA, std::string("mdf_compute_bonded_noalloc: scratch address lookup failed: ") +
                                             cudaGetErrorString(rc));
        g_noalloc_ptr[device] = static_cast<unsigned long long*>(p);
    }
    return g_noalloc_ptr[device];
}

__global__ void k_noalloc_forces(int N, const unsigned long long* __restrict__ f, double* __restrict__ out)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= N) return;
    for (int k = 0; k < 3; ++k) out[3 * a + k] = (double)(long long)f[(size_t)k * N + a] * FORCE_ISCALE;
}

// Forget the cached address of a device whose last context is gone: a caller
// may reset the device (cudaDeviceReset) before creating new contexts, and the
// module - with the array - is then loaded again, possibly elsewhere.
void noalloc_forget_device(int device)
{
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) return;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    g_noalloc_ptr[device] = nullptr;
}

static void bonded_noalloc(Ctx& c, uint32_t flags, double* d_forces, mdf_energies* e_out)
{
    if (!c.have_positions) throw ApiError(MDF_ERR_STATE, "positions not set");
    // the bonded lists are not split over ranks here: a rank's context would
    // return the whole bonded set, unlike mdf_compute
    if (distributed(c)) throw ApiError(MDF_ERR_UNSUPPORTED, "mdf_compute_bonded_noalloc: not available with nranks > 1");
    if (c.N > NOALLOC_MAX_ATOMS)
        throw ApiError(MDF_ERR_INVALID, "mdf_compute_bonded_noalloc: " + std::to_string(c.N) +
                                            " atoms exceed the static scratch limit of " +
                                            std::to_string(NOALLOC_MAX_ATOMS));
    const bool want_f = flags & MDF_COMPUTE_FORCES, want_e = flags & MDF_COMPUTE_ENERGY;
    if (want_f && !d_forces) throw ApiError(MDF_ERR_INVALID, "d_forces is NULL");
    unsigned long long* base = noalloc_scratch(c.device);
    unsigned long long* f = base;
    unsigned long long* scal = base + NOALLOC_FORCE_WORDS;
    unsigned* st = reinterpret_cast<unsigned*>(scal + NUM_ACC + 1);
    // The accumulators are summed into with atomics: the 3N force words and
    // the scalar block must start at zero.
    MDF_CUDA_TRY(cudaMemsetAsync(f, 0, sizeof(unsigned long long) * 3 * (size_t)c.N, c.stream));
    MDF_CUDA_TRY(cudaMemsetAsync(scal, 0, sizeof(unsigned long long) * NUM_SCAL, c.stream));
    launch_bonded_into(c, want_e, f, scal, st);
    if (want_f) {
        k_noalloc_forces<<<grid_blocks(c.N, 256), 256, 0, c.stream>>>(c.N, f, d_forces);
        MDF_CUDA_TRY(cudaGetLastError());
    }
    unsigned long long h[NUM_SCAL];
    MDF_CUDA_TRY(cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
    MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
    const unsigned status = (unsigned)h[NUM_ACC + 1];
    if (status & ST_NONFINITE) throw ApiError(MDF_ERR_NONFINITE, "non-finite bonded force or energy");
    if (status & ST_OVERFLOW) throw ApiError(MDF_ERR_OVERFLOW, "fixed-point accumulator range exceeded");
    if (e_out) {
        memset(e_out, 0, sizeof(*e_out));
        if (want_e) {
            const int terms[] = {MDF_E_BOND, MDF_E_ANGLE, MDF_E_DIHEDRAL, MDF_E_UB, MDF_E_IMPROPER, MDF_E_CMAP};
            double tot = 0;
            for (int k : terms) {
                e_out->e[k] = (double)(long long)h[k] * ENERGY_ISCALE;
                tot += e_out->e[k];
            }
            e_out->total = tot;
        }
    }
}

}  // namespace mdf

using namespace mdf;

extern "C" int mdf_compute_bonded_noalloc(mdf_ctx* ctx, uint32_t flags, double* d_forces, mdf_energies* energies)
{
    if (!ctx) return MDF_ERR_INVALID;
    Ctx& c = ctx->c;
    try {
        MDF_CUDA_TRY(cudaSetDevice(c.device));
        bonded_noalloc(c, flags, d_forces, energies);
        c.last_error.clear();
        return MDF_OK;
    } catch (const ApiError& e) {
        c.last_error = e.msg;
        return e.status;
    } catch (const CudaError& e) {
        c.last_error = e.msg;
        return MDF_ERR_CUDA;
    } catch (const std::exception& e) {
        c.last_error = e.what();
        return MDF_ERR_INVALID;
    }
}
