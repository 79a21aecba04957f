/* O2: FP64 CPU restatement of the reference's energy/force path, both
 * semantics.  TEST INFRASTRUCTURE ONLY — the checker for libmdf, never the
 * thing measured or shipped.  Built into oracle/_ref/liboracle.so. */
#ifndef MDF_ORACLE_H
#define MDF_ORACLE_H
#include "../include/mdf.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int semantics;          /* MDF_SEM_* */
    double box[3];
    double cutoff;          /* energy/force cutoff */
    double list_cutoff;     /* REFERENCE: pairlist cutoff (cutoff + skin) */
    double switch_radius;   /* <= 0: force-shifted LJ */
    double alpha;
    double kc;              /* Coulomb constant */
    int grid[3];
    int pme_order;          /* PHYSICAL */
    int do_allpairs;        /* REFERENCE: all-pairs EE term */
    int do_recip;           /* PHYSICAL: reciprocal sum */
} oracle_params;

/* One evaluation.  f: 3N forces (may be NULL), e: MDF_E_COUNT energies,
 * virial: 9 (reciprocal, PHYSICAL) or NULL, f_pme_ref: 3N forces of the
 * reference's order-5 PME chain (REFERENCE) or NULL, npairs: pairs within the
 * cutoff that the pair kernel evaluates (or NULL). Returns 0 on success. */
int oracle_eval(const mdf_topology *t, const oracle_params *p, const double *x,
                double *f, double *e, double *virial, double *f_pme_ref, long *npairs);

/* Reference order-5 PME chain pieces: the spread grid (K^3) and the potential
 * grid after the backward transform (K^3). */
int oracle_pme_ref_grids(const mdf_topology *t, const oracle_params *p, const double *x,
                         double *grid_q, double *grid_phi);

/* Smooth PME (PHYSICAL) energy, forces (3N, added) and virial. */
double oracle_pme_recip(const mdf_topology *t, const oracle_params *p, const double *x,
                        double *f, double *virial);

/* Plain Ewald reciprocal sum over |m_d| <= kmax (validation of PME). */
double oracle_ewald_recip_exact(int n, const double *q, const double *x, const double box[3],
                                double alpha, double kc, int kmax, double *f);

/* Bicubic CMAP coefficient table from energy grids, the reference's scheme
 * (src/AmberTopology/CreateNonBondedFromParsed.cpp:46-117). grids: [nsets][res*res]. */
void oracle_cmap_coeff(int nsets, int res, const double *grids, double *coeff);

#ifdef __cplusplus
}
#endif
#endif
