/*
 * mdf.h — C ABI of the B200 force/energy engine (libmdf.so).
 *
 * Drop-in for the CPU energy/force path of prateekbansal97/MD.  In the
 * reference that path is the private member functions of md::System
 * (include/System/System.h:78-170): calculate_energies()
 * (src/System/System.cpp:9-23), calculate_forces() (src/System/System.cpp:25-39),
 * the pairlist build (src/System/NonBondedUtils.cpp:185-282) and the PME chain
 * spread -> FFT -> solve -> FFT^-1 -> gather (src/System/PBC.cpp:183-653).  The
 * reference keeps an empty CUDA slot for it (src/cuda/nonbonded_cuda.cu,
 * CMakeLists.txt:140-160).
 *
 * Conventions (identical to the reference's):
 *   - lengths in Angstrom, energies in kcal/mol, forces in kcal/mol/Angstrom
 *     (forces, not gradients: System::forces_, include/System/System.h:175);
 *   - positions and forces are 3N doubles, atom-major (x0 y0 z0 x1 ...);
 *   - charges in the reference's internal unit, prmtop charge / 18.2206899283247
 *     (src/AmberTopology/TopologyParser.cpp:52), with the Coulomb constant
 *     passed in mdf_params.coulomb_const (18.2206899283247^2,
 *     src/NonBonded/CoulombicEE.cpp:12);
 *   - orthorhombic periodic box.
 *
 * Ownership: the caller owns every host array it passes; the library copies
 * what it needs during the call.  The library owns all device memory.
 * Threading: one context per host thread; a context is not internally
 * synchronised.  Errors: every entry point returns an mdf_status (0 = OK);
 * mdf_last_error() describes the last failure on that context.  There is no
 * CPU fallback: without a usable CUDA device mdf_create fails with
 * MDF_ERR_CUDA.
 */
#ifndef MDF_H
#define MDF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MDF_API_VERSION 1

typedef enum {
    MDF_OK = 0,
    MDF_ERR_INVALID = 1,     /* bad argument / inconsistent topology */
    MDF_ERR_CUDA = 2,        /* CUDA runtime error or no device */
    MDF_ERR_CAPACITY = 3,    /* a device list outgrew its buffer (retry grows it) */
    MDF_ERR_NONFINITE = 4,   /* non-finite position or force detected */
    MDF_ERR_OVERFLOW = 5,    /* fixed-point accumulator range exceeded */
    MDF_ERR_TIMEOUT = 6,     /* a bounded device wait gave up */
    MDF_ERR_STATE = 7,       /* call out of order (e.g. compute before positions) */
    MDF_ERR_NOMEM = 8,       /* device or host allocation failed */
    MDF_ERR_UNSUPPORTED = 9  /* option not supported by this build */
} mdf_status;

/* Which formulas to evaluate. */
typedef enum {
    /* The reference exactly as it runs: exclusion lists are whatever the host
     * passes (the reference's loader leaves them empty), switched LJ, plain
     * cutoff Coulomb forces, its torsion-force formulas, unwrapped improper
     * energy, and the reference's energy terms reported side by side. */
    MDF_SEM_REFERENCE = 0,
    /* Textbook Amber/CHARMM physics: prmtop exclusions, scaled 1-4 pairs,
     * -grad(E) torsion forces, erfc real-space Ewald + excluded-pair erf
     * corrections + self energy + smooth PME reciprocal sum. */
    MDF_SEM_PHYSICAL = 1
} mdf_semantics;

typedef enum {
    MDF_PREC_FP64 = 0,   /* every kernel in double */
    MDF_PREC_MIXED = 1   /* FP32 pair/spread/FFT/gather, int64 fixed-point forces,
                            FP64 bonded terms, corrections and energy sums */
} mdf_precision;

/* Energy terms.  Which ones are filled depends on the semantics:
 * REFERENCE: BOND..CMAP, VDW, EE (all-pairs plain Coulomb,
 *   src/System/NonBondedEnergy.cpp:133-174), EE_PAIRLIST (:176-204),
 *   EE_CUTOFF (:206-234), EE_DIRECT (:236-305), EE_SELF (:307-316).
 * PHYSICAL: BOND..CMAP, VDW, VDW14, EE_DIRECT (erfc real space), EE14,
 *   EE_EXCL (-erf correction over excluded pairs), EE_SELF, EE_RECIP. */
enum {
    MDF_E_BOND = 0, MDF_E_ANGLE, MDF_E_DIHEDRAL, MDF_E_UB, MDF_E_IMPROPER, MDF_E_CMAP,
    MDF_E_VDW, MDF_E_VDW14, MDF_E_EE, MDF_E_EE_PAIRLIST, MDF_E_EE_CUTOFF, MDF_E_EE_DIRECT,
    MDF_E_EE14, MDF_E_EE_EXCL, MDF_E_EE_SELF, MDF_E_EE_RECIP,
    MDF_E_COUNT
};

typedef struct {
    double e[MDF_E_COUNT];
    double total;        /* potential energy of the chosen semantics */
    double virial[9];    /* reciprocal-space virial (PHYSICAL), row-major */
} mdf_energies;

/* Flattened topology.  All indices 0-based.  Term parameters are resolved
 * per term (what the reference's term objects carry after
 * src/AmberTopology/CreateBondedFromParsed.cpp). */
typedef struct {
    int32_t natoms;
    const double *charge;          /* [natoms], internal charge unit */
    const int32_t *type;           /* [natoms], 0-based atom type */
    int32_t ntypes;                /* 1..8000 */
    const int32_t *nb_index;       /* [ntypes*ntypes] NONBONDED_PARM_INDEX, 1-based, 0 = none */
    int32_t n_ljpair;
    const double *lj_a, *lj_b;     /* [n_ljpair] */
    const double *lj14_a, *lj14_b; /* [n_ljpair] */

    int32_t n_bonds;  const int32_t *bond_atoms;     const double *bond_k, *bond_r0;        /* 2/term */
    int32_t n_ub;     const int32_t *ub_atoms;       const double *ub_k, *ub_r0;            /* 2/term */
    int32_t n_angles; const int32_t *angle_atoms;    const double *angle_k, *angle_theta0;  /* 3/term */
    int32_t n_dihedrals; const int32_t *dihedral_atoms;                                    /* 4/term */
    const double *dihedral_k, *dihedral_n, *dihedral_phase;
    int32_t n_impropers; const int32_t *improper_atoms;                                    /* 4/term */
    const double *improper_k, *improper_phase;
    int32_t n_cmaps;  const int32_t *cmap_atoms;     const int32_t *cmap_set;               /* 5/term, set 0-based */
    int32_t cmap_nsets, cmap_res;
    const double *cmap_coeff;      /* [nsets][res][res][16] bicubic coefficients
                                      (src/AmberTopology/CreateNonBondedFromParsed.cpp:46-117) */

    /* Pairs excluded from the ordinary nonbonded sum (i<j), and the subset
     * that receives the scaled 1-4 interaction.  pairs14 must be a subset of
     * excl_pairs. */
    int32_t n_excl;   const int32_t *excl_pairs;     /* 2/pair */
    int32_t n_pairs14; const int32_t *pairs14;       /* 2/pair */
    const double *scee14, *scnb14;                   /* [n_pairs14] */
} mdf_topology;

/* Run parameters; mdf_params_default() gives the reference's init() values
 * (src/System/init.cpp:15-23): cutoff 10, skin 2, switch 9, tolerance 1e-6. */
typedef struct {
    int32_t semantics;       /* mdf_semantics */
    int32_t precision;       /* mdf_precision */
    double box[3];
    double cutoff;           /* LJ and Coulomb cutoff (reference: lj_cutoff_ = ee_cutoff_) */
    double skin;             /* pairlist skin; list cutoff = cutoff + skin */
    double switch_radius;    /* LJ potential switch start; <= 0 selects force-shifted LJ */
    double ewald_tol;        /* alpha = sqrt(-ln(2 tol)) / cutoff (src/System/PBC.cpp:88-91); (0, 0.5) */
    double ewald_alpha;      /* > 0 overrides ewald_tol; alpha >= 1e-12 per Angstrom */
    int32_t grid[3];         /* PME mesh; 0 = the reference's formula (src/System/PBC.cpp:93-99) */
    int32_t pme_order;       /* PHYSICAL B-spline order (4); REFERENCE uses its order-5 chain */
    double coulomb_const;    /* 18.2206899283247^2 */
    int32_t device;          /* CUDA device ordinal */
    /* Dynamic pruning of the cluster-pair list: every prune_every evaluations
     * the entries whose closest atom pair lies beyond cutoff + prune_margin
     * are dropped from the list the pair kernel walks (the outer list keeps
     * them).  prune_every = 1, prune_margin = 0 prunes against the current
     * positions at every evaluation (exact); larger intervals need a margin
     * of at least twice the largest displacement between prunes.
     * prune_every < 0 (self-pruning): the pack kernel measures at every
     * evaluation the largest displacement of an atom since the last prune,
     * and the prune kernel runs only when it exceeds prune_margin / 2 (or the
     * list changed), so every pair within the cutoff stays in the list
     * without a host decision (dynamics graphs, batches); with nranks > 1 it
     * prunes at every evaluation.  prune_every = 0 disables pruning. */
    int32_t prune_every;
    double prune_margin;
    /* Launch shapes (results do not depend on them; mdf_batch_autotune picks
     * them): warps per block of the pair kernel (2, 4 or 8; 0 = 8) and FFT
     * lines per block (1, 2, 4, 8, 16 or 32; 0 = chosen per grid size: 4 for
     * 100 or 216 points, 16 for 32, so small grids keep every thread busy). */
    int32_t pair_warps;
    int32_t fft_lines;
    /* Work split over nranks contexts (one per GPU, PHYSICAL semantics; 0 or
     * 1 = one context does everything).  Every rank holds all positions;
     * rank r takes its share of the i clusters (prune + pair kernel: the
     * x-columns of atoms whose centres lie in its x-slab of the PME grid,
     * a band of space), of the exclusion, 1-4 and bonded lists and of the
     * PME spread and gather (its band's atoms); the
     * charge grid and the fixed-point force/energy accumulators are summed
     * over the ranks through the mdf_set_allreduce callback, so every rank
     * ends with the full forces and energies, bit-identical to one context. */
    int32_t rank;
    int32_t nranks;
    /* How the pair kernel's warps find their i clusters (results do not
     * depend on it): 0 = one warp per i cluster over a grid of all of them;
     * 1 = persistent warps, as many as stay resident, that take the next
     * i cluster from a work counter (no partial last wave, but they hold
     * every SM slot until the list is done, so kernels queued beside them
     * wait).  mdf_autotune picks. */
    int32_t pair_schedule;
    /* Unit of the pruned list the pair kernel walks (results do not depend
     * on it): 0 = whole 8 x 8 cluster pairs; 1 = half entries, each half of
     * an i cluster (atoms 0-3, 4-7) with the j clusters within the cutoff
     * of that half (fewer atom pairs outside the cutoff, more list work).
     * Needs pruning (prune_every > 0).  mdf_autotune picks. */
    int32_t pair_layout;
} mdf_params;

/* Sum of `count` 64-bit integers at d_buf (device memory of the context's
 * GPU) over all ranks, in place, ordered on `stream` (a cudaStream_t): work
 * queued on the stream before the call must be in the sum, work queued after
 * it must see the result.  Two's-complement wrap-around (an NCCL int64 sum,
 * for instance).  Returns 0 on success. */
typedef int (*mdf_allreduce_u64)(uint64_t *d_buf, int64_t count, void *stream, void *user);

/* The collectives of the distributed reciprocal space and force return
 * (mdf_set_collectives), all on device memory of the context's GPU, ordered on
 * `stream` like mdf_allreduce_u64, returning 0 on success:
 *   reduce-scatter  send holds nranks blocks of `count` int64 words; rank r
 *                   receives into recv the sum over ranks of block r
 *                   (ncclReduceScatter, ncclInt64, ncclSum);
 *   all-gather      rank r's `bytes` bytes of send land at recv + r * bytes on
 *                   every rank (ncclAllGather);
 *   all-to-all      send holds nranks blocks of `bytes` bytes, block k for rank
 *                   k; recv block k comes from rank k (grouped ncclSend /
 *                   ncclRecv). */
typedef int (*mdf_reduce_scatter_u64)(const uint64_t *d_send, uint64_t *d_recv, int64_t count, void *stream,
                                      void *user);
typedef int (*mdf_allgather_bytes)(const void *d_send, void *d_recv, int64_t bytes, void *stream, void *user);
typedef int (*mdf_alltoall_bytes)(const void *d_send, void *d_recv, int64_t bytes, void *stream, void *user);
/* All-to-all with per-rank sizes (mdf_set_halo_exchange), ordered on `stream`
 * like the others: send_bytes[k] bytes for rank k lie in send one after the
 * other in rank order, and recv receives recv_bytes[k] bytes from rank k the
 * same way (ncclSend / ncclRecv grouped, or MPI_Alltoallv).  Zero-size blocks
 * are frequent: a rank exchanges grid planes with its spatial neighbours
 * only.  send_bytes and recv_bytes are host arrays of nranks entries. */
typedef int (*mdf_alltoallv_bytes)(const void *d_send, const int64_t *send_bytes, void *d_recv,
                                   const int64_t *recv_bytes, void *stream, void *user);

/* Flags for mdf_compute. */
#define MDF_COMPUTE_ENERGY 1u
#define MDF_COMPUTE_FORCES 2u
/* REFERENCE semantics: also run the reference's order-5 PME chain and make its
 * forces available through mdf_get_pme_forces (the reference computes them in
 * init() and then discards them, src/System/init.cpp:59-64 + System.cpp:28). */
#define MDF_COMPUTE_PME_REFERENCE 4u

typedef struct mdf_ctx mdf_ctx;

/* Fill *p with the reference's defaults for the given box. */
void mdf_params_default(mdf_params *p);

/* Create a context on p->device and upload the topology. */
int mdf_create(const mdf_topology *top, const mdf_params *p, mdf_ctx **out);
void mdf_destroy(mdf_ctx *ctx);
const char *mdf_last_error(const mdf_ctx *ctx);
const char *mdf_status_string(int status);

/* Host positions, 3N doubles (replaces topology_.get_coordinates()). */
int mdf_set_positions(mdf_ctx *ctx, const double *xyz);
/* Device positions, 3N doubles already on ctx's device. */
int mdf_set_positions_device(mdf_ctx *ctx, const double *d_xyz);
int mdf_set_box(mdf_ctx *ctx, const double box[3]);
/* The collective a context with nranks > 1 sums through (required there;
 * called twice per evaluation: the PME charge grid, then the force and
 * energy accumulators).  Only mdf_compute / mdf_compute_async / mdf_fetch
 * support nranks > 1; the other evaluation entry points return
 * MDF_ERR_UNSUPPORTED. */
int mdf_set_allreduce(mdf_ctx *ctx, mdf_allreduce_u64 fn, void *user);
/* With nranks > 1, also register the collectives above (all three, or NULL
 * to go back to the all-reduce form): the reciprocal space is then
 * distributed as x-slabs of the PME grid - the charge grid is reduce-scattered
 * (each rank receives its slab of planes), every rank runs the z and y
 * passes of its slab, an all-to-all transposes to y-slabs for the x pass and
 * the convolution (each rank its y-range, energy and virial included), a
 * second all-to-all transposes back, and the potential slabs are all-gathered
 * for the force gather - and the forces come back by a reduce-scatter of the
 * fixed-point accumulators (each rank finalises its block of atom slots) and
 * an all-gather of the finished forces.  Every rank still ends with all
 * forces and energies, bit-identical to one context; the energy words and the
 * pair count are still summed by the all-reduce. */
int mdf_set_collectives(mdf_ctx *ctx, mdf_reduce_scatter_u64 reduce_scatter, mdf_allgather_bytes allgather,
                        mdf_alltoall_bytes alltoall, void *user);
/* With the collectives set, also register an all-to-all with per-rank sizes
 * (NULL to go back): the charge grid and the potential then cross between
 * ranks as halo planes instead of whole grids.  A split context gives rank r
 * the i clusters of the x-columns whose centres lie in its x-slab of the PME
 * grid, so its atoms' spread stencils reach only the planes of that slab and
 * a few around it (half the skin of drift and the stencil's reach); rank r
 * sends the planes it spread outside its slab to their owners, which add
 * them, and after the FFTs receives the potential of those planes back.  At
 * 960k atoms and 8 ranks that is ~6 MB per rank per evaluation instead of the
 * 80 MB reduce-scatter and 40 MB all-gather.  An atom farther than half the
 * skin outside its band since the last list build makes the evaluation fail
 * with MDF_ERR_STATE on the rank that owns it (rebuild the list, as for the
 * pair list itself).  Forces are still exact and identical to one context. */
int mdf_set_halo_exchange(mdf_ctx *ctx, mdf_alltoallv_bytes alltoallv, void *user);

/* Cell sort + cluster-pair list with exclusion masks (replaces
 * setup_pairlists / build_lj_pairlist, src/System/NonBondedUtils.cpp:49-57,185-282). */
int mdf_build_pairlist(mdf_ctx *ctx);

/* One evaluation.  forces_out: host 3N doubles or NULL (its content is
 * unspecified when the call fails); e_out: host or NULL.
 * Replaces calculate_forces() + calculate_energies() (+ the PME chain). */
int mdf_compute(mdf_ctx *ctx, uint32_t flags, double *forces_out, mdf_energies *e_out);

/* Same evaluation, enqueued on the context's stream without a host sync; the
 * results stay on the device until mdf_fetch / mdf_compute_device. */
int mdf_compute_async(mdf_ctx *ctx, uint32_t flags);
/* Wait for the last async evaluation and copy its results (either may be NULL). */
int mdf_fetch(mdf_ctx *ctx, double *forces_out, mdf_energies *e_out);
/* Pipelined evaluations from and to host memory, two in flight: mdf_submit
 * queues the copy of positions xyz (3N doubles, host) to the device on the
 * context's copy stream, the evaluation on its stream and the copy of the
 * forces back to forces_out (3N doubles, host, or NULL) on the copy stream,
 * and returns at once; mdf_collect waits for the oldest submitted evaluation,
 * checks its status and fills e_out (may be NULL).  The copies of one
 * evaluation overlap the computation of the other, so a caller that submits
 * evaluation k+1 before collecting k hides them.  xyz must stay unchanged and
 * forces_out untouched until the evaluation is collected; pinned host memory
 * (cudaHostAlloc) makes the copies asynchronous.  A third submit before a
 * collect returns MDF_ERR_STATE.  The results equal mdf_compute's bit for
 * bit; mdf_fetch does not see these evaluations.  Not available with
 * nranks > 1. */
int mdf_submit(mdf_ctx *ctx, uint32_t flags, const double *xyz, double *forces_out);
int mdf_collect(mdf_ctx *ctx, mdf_energies *e_out);
/* Device forces (3N doubles on ctx's device) of the last evaluation. */
int mdf_forces_device(mdf_ctx *ctx, double *d_forces_out);

/* REFERENCE semantics only: forces of the reference's order-5 PME chain from
 * the last evaluation that asked for MDF_COMPUTE_PME_REFERENCE. */
int mdf_get_pme_forces(mdf_ctx *ctx, double *forces_out);

/* Diagnostic: the PME mesh of the last evaluation.  grid_out (may be NULL)
 * receives K0, K1, K2; charge_grid [K0*K1*K2] the spread charges Q (x-major,
 * z fastest) and potential_grid [K0*K1*K2] the potential C*Q the gather reads
 * (the hand-written FFT's convolution with the influence function, unscaled
 * inverse transform), either may be NULL.  Lets a caller check the FFT chain
 * against another FFT (the tests use cuFFT through torch.fft). */
int mdf_pme_grids(mdf_ctx *ctx, int32_t grid_out[3], double *charge_grid, double *potential_grid);

/* Use an existing CUDA stream (cudaStream_t passed as void*); NULL = the
 * context's own stream. */
int mdf_set_stream(mdf_ctx *ctx, void *stream);

/* Sizes of the current pairlist: clusters, cluster pairs of the outer list,
 * cluster pairs kept by the last prune, and atom pairs within the cutoff as
 * counted by the first evaluation after the last pairlist build (-1 where
 * unknown).  Any pointer may be NULL. */
int mdf_pairlist_info(mdf_ctx *ctx, int64_t *n_clusters, int64_t *n_cluster_pairs,
                      int64_t *n_cluster_pairs_pruned, int64_t *n_pairs_in_cutoff);

/* Kernel timings of the last evaluation in milliseconds, recorded with CUDA
 * events when MDF timing is enabled (mdf_enable_timing). names[i] points to
 * static strings. Returns the number of entries written. */
int mdf_enable_timing(mdf_ctx *ctx, int enable);
/* Number of kernels this context has launched for evaluations so far. */
int64_t mdf_kernel_launches(const mdf_ctx *ctx);
int mdf_kernel_times(mdf_ctx *ctx, const char **names, float *ms, int max_entries);

/* Host-only utility: bicubic CMAP coefficients [nsets][res][res][16] from the
 * energy grids [nsets][res*res], the reference's table build
 * (src/AmberTopology/CreateNonBondedFromParsed.cpp:46-117). */
int mdf_cmap_coefficients(int nsets, int res, const double *grids, double *coeff);
/* Host-only utility, PHYSICAL semantics: the same table layout from C1
 * bicubic Hermite patches (corner values, periodic-cubic-spline first
 * derivatives and cross derivative, in grid-index units).  The reference's
 * patches match the grid at cell corners but not along cell edges, so its
 * CMAP energy jumps when a torsion crosses a grid line. */
int mdf_cmap_coefficients_spline(int nsets, int res, const double *grids, double *coeff);

/* Diagnostic: measured FMA throughput of the device's CUDA cores in TFLOP/s
 * (an FMA counts 2), precision MDF_PREC_MIXED for FP32, MDF_PREC_FP64 for
 * FP64.  The roofline denominator of the FP32-pipe-bound pair kernel. */
int mdf_probe_fma_tflops(int device, int precision, double *tflops);
/* Diagnostic: measured rate of int64 reductions (atomic adds) per second
 * into an L2-resident buffer of `words` 64-bit words on the device.
 * pattern 0 = four consecutive words per thread at scattered 32-byte rows
 * (the PME charge spread's access), 1 = 32 consecutive words per warp (the
 * most favourable form).  The roofline denominator of the charge spread,
 * whose fixed-point grid stays in L2. */
int mdf_probe_l2_reductions(int device, int64_t words, int pattern, double *per_s);

/* Replace the per-atom charges (internal unit, [natoms]) and/or the LJ A/B
 * coefficients ([n_ljpair], indexed by NONBONDED_PARM_INDEX - 1) of the
 * context; NULL keeps the current values (lj_a and lj_b go together).  The
 * 1-4 coefficients are kept.  Positions and the pairlist are unchanged. */
int mdf_set_parameters(mdf_ctx *ctx, const double *charge, const double *lj_a, const double *lj_b);

/* Backward (vector-Jacobian product) of one PHYSICAL evaluation at the
 * current positions: for a loss L(F, E) with dL_dF = dL/dF ([3N], forces as
 * mdf_compute returns them; NULL = 0) and dL_dE = dL/dE (total energy),
 * writes dL/dq ([natoms]), dL/dA and dL/dB ([n_ljpair], the main LJ table per
 * NONBONDED_PARM_INDEX - 1 entry).  Any output may be NULL.  The pair kernel is
 * recomputed; nothing from the forward evaluation is needed.  Positions and
 * bonded terms are constants here.  REFERENCE semantics return
 * MDF_ERR_UNSUPPORTED (their forces are not the gradient of their energy). */
int mdf_backward(mdf_ctx *ctx, const double *dL_dF, double dL_dE, double *dL_dq, double *dL_dA, double *dL_dB);

/* ---------------------------------------------------------------------------
 * Dynamics and minimisation (PHYSICAL semantics).  Units: A, A/ps, amu,
 * kcal/mol.  The reference has neither (apps/main.cpp stops after one
 * evaluation); its intended consumer of calculate_forces is a minimiser
 * (include/System/System.h:84,113) and its list rebuild test is
 * ljpairs_needs_rebuild (src/System/NonBondedUtils.cpp:87-100). */
typedef struct {
    int32_t iterations;
    int32_t rebuilds;
    double e_initial, e_final;   /* total potential energy, kcal/mol */
    double fmax_final;           /* largest force component at the end */
    int32_t evaluations;         /* energy + force evaluations, line-search trials included */
    int32_t reserved;
} mdf_min_report;
/* Steepest descent at the current positions, largest move per iteration
 * adaptive up to max_step (A); stops at max |F| <= fmax_tol (kcal/mol/A) or
 * after max_iter iterations.  The positions stay on the device
 * (mdf_md_state reads them); call mdf_md_init afterwards to start dynamics. */
int mdf_minimize(mdf_ctx *ctx, int32_t max_iter, double fmax_tol, double max_step, mdf_min_report *report);
/* L-BFGS (two-loop recursion, Nocedal & Wright Algorithm 7.4, `history`
 * pairs, 0 = 8) with a backtracking Armijo line search; no atom moves more
 * than max_step (A) per iteration.  Same stopping rule, list handling and
 * report as mdf_minimize; bit-reproducible run to run. */
int mdf_minimize_lbfgs(mdf_ctx *ctx, int32_t max_iter, double fmax_tol, double max_step, int32_t history,
                       mdf_min_report *report);

typedef struct {
    int64_t steps;        /* steps done */
    int64_t rebuilds;     /* list builds during the run */
    int64_t samples;      /* energy samples (one per chunk) */
    double wall_s;        /* host wall time of the run */
    double pe_first, ke_first;   /* potential / kinetic energy after the first chunk */
    double pe_last, ke_last;     /* ... after the last chunk */
    double rebuild_s;     /* host wall time in list rebuilds */
    double record_s;      /* host wall time recording / updating the chunk graphs */
    double wait_s;        /* host wall time waiting for the chunk graphs to finish */
} mdf_md_report;
/* masses [natoms] (amu); velocities [3N] (A/ps), or NULL to draw them from a
 * Maxwell-Boltzmann distribution at temperature (K) with the given seed
 * (centre-of-mass motion removed).  Builds the list and computes the forces. */
int mdf_md_init(mdf_ctx *ctx, const double *masses, const double *velocities, double temperature, uint64_t seed);
/* Velocity-Verlet NVE steps in CUDA-graph chunks of `chunk` steps (0 = 10).
 * The pairlist is rebuilt every rebuild_every steps, or with rebuild_every = 0
 * when the largest displacement since the last build, plus twice what the
 * fastest atom covers in a chunk, would pass half the skin; a displacement
 * past half the skin between builds is an error.  samples (may be NULL)
 * receives up to cap rows (t ps, potential, kinetic), one per chunk. */
int mdf_md_run(mdf_ctx *ctx, int64_t nsteps, double dt_ps, int32_t chunk, int32_t rebuild_every, double *samples,
               int64_t cap, mdf_md_report *report);
/* Current positions and velocities to host ([3N] each; either may be NULL). */
int mdf_md_state(mdf_ctx *ctx, double *xyz, double *velocities);
/* Amber ASCII restart (positions, velocities, box) of the current state. */
int mdf_md_write_rst7(mdf_ctx *ctx, const char *path, const char *title, double time_ps);

/* ---------------------------------------------------------------------------
 * Batches: many independent PHYSICAL systems (uneven atom counts, boxes and
 * PME grids) evaluated by one CUDA graph launch.  Positions and forces are
 * the systems' 3N arrays concatenated in system order.  Each system keeps
 * its own pairlist (built at the positions of mdf_batch_build_pairlists, or
 * at the first compute); evaluate within the skin of those positions, or
 * rebuild.  Not thread-safe; one batch per host thread. */
typedef struct mdf_batch mdf_batch;

typedef struct {
    int32_t pair_warps;   /* chosen launch shapes (see mdf_params) */
    int32_t fft_lines;
    int32_t prune_every;
    int32_t n_tried;      /* candidates timed */
    double best_ms;       /* one batch evaluation with the chosen shapes */
    double default_ms;    /* ... with the shapes the batch was created with */
    int32_t pair_schedule;
    int32_t pair_layout;
} mdf_tune_report;

int mdf_batch_create(int nsys, const mdf_topology *const *topos, const mdf_params *params, mdf_batch **out);
void mdf_batch_destroy(mdf_batch *b);
const char *mdf_batch_last_error(const mdf_batch *b);
/* Systems, total atoms, kernels in one graph launch (-1 before the first capture). */
int mdf_batch_info(const mdf_batch *b, int64_t *n_systems, int64_t *total_atoms, int64_t *graph_kernels);
/* Host positions [3 * total atoms]; copied at the call, uploaded inside the graph. */
int mdf_batch_set_positions(mdf_batch *b, const double *xyz);
/* The batch's own pinned host buffers ([3 * total atoms] each, system order):
 * the graph copies positions from the first and forces into the second, so a
 * caller that writes positions there (and passes that pointer to
 * mdf_batch_set_positions) and reads forces there (forces = NULL in
 * mdf_batch_compute / mdf_batch_fetch) moves no extra host copy.  Valid until
 * mdf_batch_destroy. */
int mdf_batch_host_buffers(mdf_batch *b, double **positions, double **forces);
int mdf_batch_build_pairlists(mdf_batch *b);
/* One batch evaluation; forces [3 * total atoms] and energies [nsys] to host
 * (either may be NULL).  Returns after the evaluation. */
int mdf_batch_compute(mdf_batch *b, uint32_t flags, double *forces, mdf_energies *energies);
/* The same split in two: launch (ordered after `stream` if non-NULL, and
 * `stream` after it) and fetch (waits, then copies out). */
int mdf_batch_launch(mdf_batch *b, uint32_t flags, void *stream);
int mdf_batch_fetch(mdf_batch *b, uint32_t flags, double *forces, mdf_energies *energies);
/* Pipelined batch evaluation: submit queues one evaluation of the positions
 * at xyz (all systems concatenated, 3 * total atoms doubles; pinned host
 * memory for asynchronous copies) and returns; the forces go to `forces`
 * (may be NULL).  At most two evaluations are in flight: the positions of
 * the next one go in on one copy stream and the forces of the previous one
 * come out on another while the GPU computes.  collect waits for the oldest
 * and writes its energies (one per system, may be NULL); xyz and forces of a
 * submission must stay valid until it is collected.  Needs the same launch
 * parameters (precision, switch, pruning, launch shapes) in every system.
 * The first submission builds the pairlists from its positions. */
int mdf_batch_submit(mdf_batch *b, uint32_t flags, const double *xyz, double *forces);
int mdf_batch_collect(mdf_batch *b, mdf_energies *energies);
/* Time every candidate launch shape on this batch (reps graph launches each)
 * and keep the fastest.  report may be NULL. */
int mdf_batch_autotune(mdf_batch *b, int reps, mdf_tune_report *report);
/* The same for one context: pair_warps {2, 4, 8} x fft_lines {2, 4, 8, 16} x
 * prune_every {0, 1} x pair_schedule {0, 1} x pair_layout {0, 1} (layout 1
 * only with pruning) at the current positions (reps energy + force
 * evaluations each, CUDA events on the context's stream); the fastest stays
 * in the context's parameters.  Forces do not depend on the choice.  Not
 * available with nranks > 1. */
int mdf_autotune(mdf_ctx *ctx, int reps, mdf_tune_report *report);

/* No counterpart in the reference.
 *
 * Bonded terms only (bond, Urey-Bradley, angle, dihedral, improper, CMAP) of
 * the context's current positions, computed without any device allocation:
 * the fixed-point force and energy accumulators live in one static device
 * array of the library, MDF_NOALLOC_MAX_ATOMS atoms at most (3 MiB of int64
 * plus the energy words).  A context with more atoms gets MDF_ERR_INVALID
 * before any device work.
 *
 * d_forces: device array [3 * natoms] (x,y,z per atom), overwritten; may be
 * NULL without MDF_COMPUTE_FORCES.  energies: host struct, may be NULL; the
 * bonded entries of e[] and their sum in total are set, the rest zeroed.
 * The call runs on the context's stream and returns after it has finished.
 *
 * The first call on a device looks up the static array's device address
 * (cudaGetSymbolAddress) and keeps it; make that first call before any
 * stream capture.  The address is kept while any context lives on that
 * device; destroying the device's last context forgets it, so a caller that
 * resets the device (cudaDeviceReset) after destroying its contexts gets a
 * fresh lookup on the next first call.  The array is shared by every context
 * on the device, so calls that overlap in time (other threads, other streams)
 * race and corrupt each other's results: serialise them.  A context with
 * nranks > 1 gets MDF_ERR_UNSUPPORTED (the bonded lists are not split over
 * the ranks here). */
#define MDF_NOALLOC_MAX_ATOMS 131072
int mdf_compute_bonded_noalloc(mdf_ctx *ctx, uint32_t flags, double *d_forces, mdf_energies *energies);

#ifdef __cplusplus
}
#endif
#endif
