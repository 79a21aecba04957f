// Launch arguments of the evaluation kernels, one struct per kernel.
//
// Every kernel of an evaluation takes its arguments as one struct, so the same
// body serves two launch forms:
//   k_X(XArgs a)                 one system, the struct passed by value;
//   k_X_multi(const XArgs* as)   many systems in one launch: blockIdx.z picks
//                                the system's struct in device memory, and
//                                blocks past that system's own grid (gx, gy)
//                                return at once.
// A system's blocks run the same code on the same data in both forms, so a
// batch launch reproduces the single-system results bit for bit (energies
// included: each block, or each i cluster in the persistent pair kernels,
// sums the same terms in the same order).
#pragma once

#include "mdf_device.cuh"
#include "mdf_internal.cuh"
#include "nb_common.cuh"

namespace mdf {

// The blocks of a many-system launch: a one-dimensional grid of n blocks,
// block b running block map[b].y (linear in the system's own gx x gy grid)
// of system map[b].x.
struct BlockMap {
    const int2* map;
    int n;
};

// ---------------------------------------------------------------- pairlist
template <typename R>
struct PackArgs {
    int gx, gy;
    int nslots;
    const double* xyz;
    const double* q;
    const int* slot_atom;
    const double4* center;
    double L[3];
    typename V4<R>::type* xq;
    float4 *cur_lo, *cur_hi;
    const typename V4<R>::type* snap;   // self-pruning: positions of the last prune (nullptr: off)
    unsigned* disp;                     // largest squared displacement from snap (FP32 bits, atomicMax)
    unsigned* st;
};

struct PruneShifts {
    float v[27][6];
};

template <typename R>
struct PruneArgs {
    int gx, gy;
    int ncl;
    const ILRange* ilist;
    const PairEntry* plist;
    const typename V4<R>::type* xq;
    const float4 *centerf, *cur_lo, *cur_hi;
    PruneShifts shifts;
    float rcut2;
    ILRange* ilist_in;
    PairEntry* plist_in;
    // self-pruning: prune only when force is set or the displacement since the
    // last prune (written by the pack kernel) exceeds disp_thr2; a prune that
    // runs records the positions it used in snap
    typename V4<R>::type* snap;
    const unsigned* disp;
    float disp_thr2;
    int force;
};

// ------------------------------------------------------------- pair kernels
// Constants of the FP32 pair kernel, folded on the host.
struct PairConstF {
    float rc2;
    float kex;        // -alpha^2 log2(e): exp(-alpha^2 r^2) = 2^(kex r^2)
    float pa;         // 0.3275911 alpha (A&S 7.1.26 argument)
    float two_a_spi;  // 2 alpha / sqrt(pi)
    float inv_sw, rsw_inv;          // 1/(rc - rsw), rsw/(rc - rsw)
    float d30, d60;                 // -30, 60 times inv_sw (dS/dr = x^2 (d30 + x (d60 + x d30)))
    float uc6, uc12, rcf, rc2f;     // force-shifted LJ
};

struct PairF32Args {
    int gx, gy;
    int nlist;
    const ILRange* ilist;
    const PairEntry* plist;
    const float4* xq;
    const int* stype;
    const float4* centerf;
    const float4* lj4;
    int ntp;
    int lj_smem;
    float kc;
    PairConstF K;
    ShiftTable shifts;
    unsigned long long* fslot;
    int nslots;
    unsigned long long* acc;
    unsigned long long* npairs;
    unsigned long long* next;   // work counter of the persistent warps, zero at launch
    int persist;                // 1: persistent warps on the counter; 0: warp w takes item w
    int half;                   // items are half entries (the 4 x 8 kernel)
    unsigned* st;
};

// Constants and image offsets of the FP64 PHYSICAL pair kernel (the same
// structure as the FP32 kernel's, in double).
struct PairConstD {
    double rc2, alpha, two_a_spi;
    double inv_sw, rsw_inv, d30, d60;   // switch: x = r inv_sw - rsw_inv; dS/dr = x^2 (d30 + x (d60 + x d30))
    double uc6, uc12, rc;               // force-shifted LJ
};

struct ShiftTableD {
    double v[27][3];
};

struct PairF64Args {
    int gx, gy;
    int nlist;
    const ILRange* ilist;
    const PairEntry* plist;
    const double4* xq;
    const int* stype;
    const double4* center;
    const double4* lj4;     // (A, B, 12A, 6B) per type pair
    int ntp;
    int lj_smem;
    double kc;
    PairConstD K;
    ShiftTableD shifts;
    unsigned long long* fslot;
    int nslots;
    unsigned long long* acc;
    unsigned long long* npairs;
    unsigned long long* next;   // work counter of the persistent warps, zero at launch
    int persist;                // 1: persistent warps on the counter; 0: warp w takes item w
    int half;                   // items are half entries (the 4 x 8 kernel)
    unsigned* st;
};

template <typename R>
struct PairArgs {
    int gx, gy;
    int nlist;
    const ILRange* ilist;
    const PairEntry* plist;
    const typename V4<R>::type* xq;
    const int* stype;
    const double4* center;
    const typename V2<R>::type* ljAB;
    const int* ljvalid;
    NBParams P;
    unsigned long long* fslot;
    int nslots;
    unsigned long long* acc;
    unsigned long long* npairs;
    int count;
    unsigned* st;
};

struct ExclArgs {
    int gx, gy;
    int n;
    const int* pairs;
    const int* is14;
    const double* xyz;
    const double* q;
    NBParams P;
    int N;
    unsigned long long* fatom;
    unsigned long long* acc;
    unsigned* st;
};

struct Pair14Args {
    int gx, gy;
    int n;
    const int* pairs;
    const double2* scale;
    const double* xyz;
    const double* q;
    const int* type;
    const double2* lj14;
    const int* ljvalid;
    NBParams P;
    int N;
    unsigned long long* fatom;
    unsigned long long* acc;
    unsigned* st;
};

// ------------------------------------------------------------------ bonded
struct BondedArgs {
    int gx, gy;
    int n[6];        // end index per list: bonds, ub, angles, dihedrals, impropers, cmaps
    int lo[6];       // first index per list (a rank's share starts there)
    int blk0[7];     // first block of each segment (prefix)
    const int *bond_atoms, *ub_atoms, *angle_atoms, *dih_atoms, *imp_atoms, *cmap_atoms, *cmap_set;
    const double2 *bond_par, *ub_par, *angle_par, *imp_par;
    const double* dih_par;
    const double* cmap_coeff;
    int cmap_res;
    const double* xyz;
    int N;
    unsigned long long* f;
    unsigned long long* acc;
    unsigned* st;
};

// --------------------------------------------------------------------- PME
struct GridGeom {
    int K[3];
    double L[3];
    double scale[3];   // K/L
};

struct FFTDesc {
    int n;
    int nst;
    int radix[12];
    int ns[12];
    int toff[12];
    int ntab;
};

struct ConvParams {
    int K[3];
    double pa2;       // pi^2 / alpha^2 (virial factor)
    int reference;    // REFERENCE solve: no energy or virial
};

struct ZeroArgs {
    int gx, gy;
    unsigned long long* p;
    long long n;
};

struct SpreadArgs {
    int gx, gy;
    int s0, s1;
    const int* slot_atom;
    const double* xyz;
    const double* q;
    GridGeom g;
    unsigned long long* qgrid;
    unsigned* st;
    int win_lo, win_n;   // halo exchange: stencil bases must lie in win_lo .. +win_n-1 (mod K0); win_n = 0: any
};

template <typename R>
struct GatherArgs {
    int gx, gy;
    int s0, s1, nslots;
    const int* slot_atom;
    const double* xyz;
    const double* q;
    GridGeom g;
    const R* phi;
    unsigned long long* fslot;
    unsigned* st;
};

// z passes (r2c: charge grid -> half complex; c2r: half complex -> potential)
template <typename R>
struct FFTZArgs {
    int gx, gy;
    const unsigned long long* qgrid;              // r2c input
    typename V2<R>::type* cgrid;                   // r2c output / c2r input
    R* rgrid;                                      // c2r output
    int nlines;
    FFTDesc d;
    const typename V2<R>::type* tw;
    const int2* tab;
    int LP;
};

template <typename R>
struct FFTYArgs {
    int gx, gy;
    typename V2<R>::type* cgrid;
    int Kc;
    FFTDesc d;
    const typename V2<R>::type* tw;
    const int2* tab;
    int LP, lp_shift;
    int inverse;
};

template <typename R>
struct FFTXArgs {
    int gx, gy;
    typename V2<R>::type* cgrid;
    int K1, Kc;
    FFTDesc d;
    const typename V2<R>::type* tw;
    const int2* tab;
    int LP, lp_shift;
    ConvParams cp;
    const R* infl;
    const double *mx, *my, *mz;
    unsigned long long* acc;
    unsigned* st;
};

// One system's FFT chain: the five passes and their dynamic shared memory.
template <typename R>
struct FFTChain {
    FFTZArgs<R> zf, zi;
    FFTYArgs<R> yf, yi;
    FFTXArgs<R> x;
    size_t smz, smy, smx;
    bool energy;
};

// Many systems' chains: device arrays [nsys] of each pass's arguments ...
template <typename R>
struct FFTChainDev {
    const FFTZArgs<R>* zf;
    const FFTYArgs<R>* yf;
    const FFTXArgs<R>* x;
    const FFTYArgs<R>* yi;
    const FFTZArgs<R>* zi;
    BlockMap mz, my, mx;   // the blocks of the z, y and x passes (forward and inverse share them)
};

// ... and the largest shared memory of each pass over the systems.
struct FFTChainMax {
    size_t smz, smy, smx;
};

// --------------------------------------------------------------- finalize
struct FinalizeArgs {
    int gx, gy;
    int N, nslots;
    unsigned long long* fatom;
    unsigned long long* fslot;
    const int* atom_slot;
    double* out;
    unsigned long long* scal;
    unsigned long long* host_scal;
};

// ----------------------------------------------------- host-side builders
// The arguments of one system's launch (from its context) and the
// many-system launchers (device arrays of arguments, the largest grid).
template <typename R> PackArgs<R> make_pack_args(const Ctx& c);
template <typename R> void launch_pack_multi(const PackArgs<R>* d_args, BlockMap bm, cudaStream_t s);
template <typename R> PruneArgs<R> make_prune_args(const Ctx& c);
template <typename R> PruneArgs<R> make_prune_half_args(const Ctx& c);
void ensure_half_lists(Ctx& c);
template <typename R>
void launch_prune_multi(const PruneArgs<R>* d_args, int nsys, int gx, bool half, cudaStream_t s);
PairF32Args make_pair_f32_args(const Ctx& c, size_t* dyn);
void launch_pairs_f32_multi(const PairF32Args* d_args, int nsys, int gx, int threads, size_t dyn, bool energy,
                            bool use_switch, bool persist, bool half, bool lj_smem, cudaStream_t s);
template <typename R> PairArgs<R> make_pair_args(const Ctx& c, bool count);
PairF64Args make_pair_f64_args(const Ctx& c, size_t* dyn);
void launch_pairs_f64_multi(const PairF64Args* d_args, int nsys, int gx, int threads, size_t dyn, bool energy,
                            bool use_switch, bool persist, bool half, bool lj_smem, cudaStream_t s);
int pair_threads(const Ctx& c);
ExclArgs make_excl_args(const Ctx& c);
Pair14Args make_pair14_args(const Ctx& c);
void launch_exclusions_multi(const ExclArgs* d_excl, int gx_excl, const Pair14Args* d_14, int gx_14, int nsys,
                             bool energy, cudaStream_t s);
BondedArgs make_bonded_args(const Ctx& c, bool whole, unsigned long long* f, unsigned long long* acc, unsigned* st);
void launch_bonded_multi(const BondedArgs* d_args, int nsys, int gx, bool energy, cudaStream_t s);
template <typename R> FFTChain<R> make_fft_chain(const Ctx& c, bool energy);
SpreadArgs make_spread_args(const Ctx& c);
template <typename R> GatherArgs<R> make_gather_args(const Ctx& c);
template <typename R>
void launch_pme_multi(const ZeroArgs* d_zero, BlockMap mzero, const SpreadArgs* d_spread, BlockMap mspread,
                      const FFTChainDev<R>& D, const FFTChainMax& M, const GatherArgs<R>* d_gather, BlockMap mgather,
                      bool energy, cudaStream_t s);
FinalizeArgs make_finalize_args(const Ctx& c, double* d_forces);
void launch_finalize_multi(const FinalizeArgs* d_args, BlockMap bm, cudaStream_t s);

// The grid of a one-system launch from the struct's own extents.
template <typename A>
inline dim3 grid_of(const A& a)
{
    return dim3((unsigned)a.gx, (unsigned)a.gy, 1u);
}

}  // namespace mdf
