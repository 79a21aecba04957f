/*
 * O2 — FP64 CPU restatement of the reference's energy/force path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for libmdf: tests,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may call it; the
 * product library never links or calls it.
 *
 * REFERENCE semantics follow the reference function by function:
 *   bonded energies   src/System/BondedEnergy.cpp:10-166, src/System/Metrics.cpp:12-82,
 *                     src/Bonded/{HarmonicBond,harmonicUB,HarmonicAngle,CosineDihedral,
 *                     HarmonicImproper}.cpp:6-12, src/Bonded/CMapGroup.cpp:82-144
 *   bonded forces     src/System/BondedForces.cpp:10-479, CMapGroup.cpp:148-237
 *   pairlist set      src/System/NonBondedUtils.cpp:185-282 (a<b, r^2 <= (rc+skin)^2,
 *                     r^2 > 1e-12, nb != 0, excluded-and-not-1-4 skipped)
 *   LJ                src/System/NonBondedEnergy.cpp:79-131, NonBondedForces.cpp:92-155,
 *                     NonBondedUtils.cpp:117-132 (switch), :162-183 (shift tables),
 *                     src/NonBonded/LennardJones.cpp:9-26
 *   Coulomb           src/System/NonBondedEnergy.cpp:133-316, NonBondedForces.cpp:207-241,
 *                     src/NonBonded/CoulombicEE.cpp:10-44
 *   PME chain         src/System/PBC.cpp:183-250 (spread), :329-401 (weights),
 *                     :455-490 (moduli), :501-564 (solve), :576-653 (gather)
 * PHYSICAL semantics: same bonded energies (improper difference wrapped),
 * forces = -grad E, erfc real-space Ewald with excluded-pair erf corrections,
 * scaled 1-4 pairs, self energy, and smooth PME (Essmann et al., J. Chem.
 * Phys. 103, 8577 (1995)) with its reciprocal energy and virial.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "mdf_oracle.h"
#include "fft_ref.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef long double acc_t;

static double min_image_1d(double d, double L) { return d - L * round(d / L); }
static double wrapx(double x, double L) { return x - L * floor(x / L); }

static void mic(const oracle_params *p, double *d)
{
    d[0] = min_image_1d(d[0], p->box[0]);
    d[1] = min_image_1d(d[1], p->box[1]);
    d[2] = min_image_1d(d[2], p->box[2]);
}

/* ---------------------------------------------------------------- lookups */

static int cmp_u64(const void *a, const void *b)
{
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : x > y;
}

static uint64_t pkey(int a, int b)
{
    if (a > b) { int t = a; a = b; b = t; }
    return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
}

typedef struct {
    uint64_t *excl;  long nexcl;
    uint64_t *p14;   long np14;   /* sorted keys */
    long *p14_idx;                /* original index of sorted key */
} pairsets;

static void build_sets(const mdf_topology *t, pairsets *s)
{
    s->nexcl = t->n_excl;
    s->excl = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(t->n_excl + 1));
    for (long i = 0; i < t->n_excl; ++i) s->excl[i] = pkey(t->excl_pairs[2 * i], t->excl_pairs[2 * i + 1]);
    qsort(s->excl, (size_t)s->nexcl, sizeof(uint64_t), cmp_u64);
    s->np14 = t->n_pairs14;
    s->p14 = (uint64_t *)malloc(sizeof(uint64_t) * 2 * (size_t)(t->n_pairs14 + 1));
    /* pack (key, index) pairs to sort together */
    for (long i = 0; i < t->n_pairs14; ++i) {
        s->p14[2 * i] = pkey(t->pairs14[2 * i], t->pairs14[2 * i + 1]);
        s->p14[2 * i + 1] = (uint64_t)i;
    }
    qsort(s->p14, (size_t)s->np14, 2 * sizeof(uint64_t), cmp_u64);
    s->p14_idx = (long *)malloc(sizeof(long) * (size_t)(s->np14 + 1));
    for (long i = 0; i < s->np14; ++i) s->p14_idx[i] = (long)s->p14[2 * i + 1];
    for (long i = 0; i < s->np14; ++i) s->p14[i] = s->p14[2 * i];
}

static void free_sets(pairsets *s) { free(s->excl); free(s->p14); free(s->p14_idx); }

static int in_excl(const pairsets *s, uint64_t k)
{
    return s->nexcl && bsearch(&k, s->excl, (size_t)s->nexcl, sizeof(uint64_t), cmp_u64) != NULL;
}

static long find14(const pairsets *s, uint64_t k)
{
    if (!s->np14) return -1;
    const uint64_t *r = (const uint64_t *)bsearch(&k, s->p14, (size_t)s->np14, sizeof(uint64_t), cmp_u64);
    return r ? s->p14_idx[r - s->p14] : -1;
}

/* ------------------------------------------------------- pair enumeration */

typedef void (*pair_fn)(void *ctx, int a, int b, const double *d, double r2);

/* Visit each unordered pair (a<b) whose min-image distance^2 <= rmax^2 once. */
static void for_pairs(const oracle_params *p, int n, const double *x, double rmax, pair_fn fn, void *ctx)
{
    int nc[3];
    for (int k = 0; k < 3; ++k) {
        nc[k] = (int)floor(p->box[k] / rmax);
        if (nc[k] < 1) nc[k] = 1;
    }
    double r2max = rmax * rmax;
    if (nc[0] < 3 || nc[1] < 3 || nc[2] < 3) {
        for (int a = 0; a < n; ++a)
            for (int b = a + 1; b < n; ++b) {
                double d[3] = {x[3 * a] - x[3 * b], x[3 * a + 1] - x[3 * b + 1], x[3 * a + 2] - x[3 * b + 2]};
                mic(p, d);
                double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                if (r2 <= r2max) fn(ctx, a, b, d, r2);
            }
        return;
    }
    int ncell = nc[0] * nc[1] * nc[2];
    int *head = (int *)malloc(sizeof(int) * (size_t)ncell), *next = (int *)malloc(sizeof(int) * (size_t)n);
    for (int c = 0; c < ncell; ++c) head[c] = -1;
    for (int i = n - 1; i >= 0; --i) {
        int ci[3];
        for (int k = 0; k < 3; ++k) {
            double w = wrapx(x[3 * i + k], p->box[k]);
            ci[k] = (int)(w * nc[k] / p->box[k]);
            if (ci[k] >= nc[k]) ci[k] = nc[k] - 1;
            if (ci[k] < 0) ci[k] = 0;
        }
        int c = ci[0] + nc[0] * (ci[1] + nc[1] * ci[2]);
        next[i] = head[c];
        head[c] = i;
    }
    for (int cz = 0; cz < nc[2]; ++cz)
        for (int cy = 0; cy < nc[1]; ++cy)
            for (int cx = 0; cx < nc[0]; ++cx) {
                int c1 = cx + nc[0] * (cy + nc[1] * cz);
                for (int dz = -1; dz <= 1; ++dz)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx) {
                            int jx = (cx + dx + nc[0]) % nc[0], jy = (cy + dy + nc[1]) % nc[1], jz = (cz + dz + nc[2]) % nc[2];
                            int c2 = jx + nc[0] * (jy + nc[1] * jz);
                            if (c2 < c1) continue;
                            for (int i = head[c1]; i >= 0; i = next[i])
                                for (int j = head[c2]; j >= 0; j = next[j]) {
                                    if (c1 == c2 && j <= i) continue;
                                    int a = i < j ? i : j, b = i < j ? j : i;
                                    double d[3] = {x[3 * a] - x[3 * b], x[3 * a + 1] - x[3 * b + 1], x[3 * a + 2] - x[3 * b + 2]};
                                    mic(p, d);
                                    double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                                    if (r2 <= r2max) fn(ctx, a, b, d, r2);
                                }
                        }
            }
    free(head);
    free(next);
}

/* ------------------------------------------------------------- nonbonded */

static void lj_switch(const oracle_params *p, double r, double *S, double *dS)
{
    /* src/System/NonBondedUtils.cpp:117-132 */
    if (!(p->switch_radius > 0.0) || r <= p->switch_radius) { *S = 1.0; *dS = 0.0; return; }
    if (r >= p->cutoff) { *S = 0.0; *dS = 0.0; return; }
    double inv = 1.0 / (p->cutoff - p->switch_radius);
    double xx = (r - p->switch_radius) * inv;
    double x2 = xx * xx, x3 = x2 * xx, x4 = x2 * x2, x5 = x4 * xx;
    *S = 1.0 - 10.0 * x3 + 15.0 * x4 - 6.0 * x5;
    *dS = (-30.0 * x2 + 60.0 * x3 - 30.0 * x4) * inv;
}

static double lj_u(double r2, double A, double B)
{
    double i2 = 1.0 / r2, i6 = i2 * i2 * i2, i12 = i6 * i6;
    return A * i12 - B * i6;
}

static double lj_g(double r2, double A, double B)
{
    double i2 = 1.0 / r2, i4 = i2 * i2, i6 = i4 * i2, i8 = i4 * i4, i12 = i6 * i6, i14 = i12 * i2;
    return 12.0 * A * i14 - 6.0 * B * i8;
}

typedef struct {
    const mdf_topology *t;
    const oracle_params *p;
    const pairsets *s;
    double *f;
    acc_t e[MDF_E_COUNT];
    long npairs;
} nbctx;

/* LJ energy/gradient for a pair, switched or force-shifted; returns energy,
 * *g = scalar with F_a = g * d. */
static double lj_pair(const nbctx *c, double r2, double r, double A, double B, double *g)
{
    const oracle_params *p = c->p;
    double U = lj_u(r2, A, B), G = lj_g(r2, A, B);
    if (p->switch_radius > 0.0) {
        double S, dS;
        lj_switch(p, r, &S, &dS);
        *g = S * G - (U / r) * dS;
        return U * S;
    }
    double rc2 = p->cutoff * p->cutoff;
    double Ucut = lj_u(rc2, A, B), Gcut = lj_g(rc2, A, B);
    *g = G - Gcut * (p->cutoff / r);
    return U - Ucut + (r - p->cutoff) * (Gcut * p->cutoff);
}

static void ref_pair(void *vc, int a, int b, const double *d, double r2)
{
    nbctx *c = (nbctx *)vc;
    const mdf_topology *t = c->t;
    const oracle_params *p = c->p;
    double kc = p->kc, qa = t->charge[a], qb = t->charge[b];
    uint64_t key = pkey(a, b);
    int is14 = 0;
    double scee = 1.0;
    if (in_excl(c->s, key)) {
        long k = find14(c->s, key);
        if (k < 0) return;              /* excluded and not 1-4 */
        is14 = 1;
        scee = t->scee14[k];
    }
    double rc2 = p->cutoff * p->cutoff;
    if (r2 > rc2 || r2 < 1e-12) return;
    double r = sqrt(r2);
    /* all-pairs Coulomb (no nb test), src/System/NonBondedEnergy.cpp:133-174 */
    if (p->do_allpairs) c->e[MDF_E_EE] += (1.0 / scee) * ((qa * qb) / r) * kc;
    int nb = t->nb_index[t->type[a] * t->ntypes + t->type[b]];
    if (nb == 0) return;
    int pi = nb - 1;
    c->npairs++;
    double A = is14 ? t->lj14_a[pi] : t->lj_a[pi];
    double B = is14 ? t->lj14_b[pi] : t->lj_b[pi];
    double g;
    c->e[MDF_E_VDW] += lj_pair(c, r2, r, A, B, &g);
    double ecoul = ((qa * qb) / r) * kc;
    c->e[MDF_E_EE_PAIRLIST] += (1.0 / scee) * ecoul;
    c->e[MDF_E_EE_CUTOFF] += (1.0 / scee) * ((qa * qb) * kc) * (1.0 / r - 1.0 / p->cutoff);
    if (is14) /* CalculateEnergyEwaldDirectTerm_14 with erf(r) (src/NonBonded/CoulombicEE.cpp:38-44) */
        c->e[MDF_E_EE_DIRECT] += (1.0 / (scee * r) - erf(r) / r) * ((qa * qb) * kc);
    else
        c->e[MDF_E_EE_DIRECT] += ((qa * qb) / r) * erfc(p->alpha * r) * kc;
    /* forces: switched LJ + plain Coulomb k q q / r^3 (src/System/NonBondedForces.cpp:207-241) */
    double gc = (1.0 / scee) * ((qa * qb) / (r2 * r)) * kc;
    double gt = g + gc;
    if (c->f) {
        for (int k = 0; k < 3; ++k) {
            c->f[3 * a + k] += gt * d[k];
            c->f[3 * b + k] -= gt * d[k];
        }
    }
}

static void phys_pair(void *vc, int a, int b, const double *d, double r2)
{
    nbctx *c = (nbctx *)vc;
    const mdf_topology *t = c->t;
    const oracle_params *p = c->p;
    if (r2 > p->cutoff * p->cutoff || r2 < 1e-12) return;
    if (in_excl(c->s, pkey(a, b))) return;
    c->npairs++;
    double r = sqrt(r2);
    double qq = t->charge[a] * t->charge[b] * p->kc;
    int nb = t->nb_index[t->type[a] * t->ntypes + t->type[b]];
    double g = 0.0;
    if (nb > 0) {
        double glj;
        c->e[MDF_E_VDW] += lj_pair(c, r2, r, t->lj_a[nb - 1], t->lj_b[nb - 1], &glj);
        g += glj;
    }
    double ar = p->alpha * r;
    double ec = qq * erfc(ar) / r;
    c->e[MDF_E_EE_DIRECT] += ec;
    g += (ec + qq * (2.0 * p->alpha / sqrt(M_PI)) * exp(-ar * ar)) / r2;
    if (c->f)
        for (int k = 0; k < 3; ++k) {
            c->f[3 * a + k] += g * d[k];
            c->f[3 * b + k] -= g * d[k];
        }
}

/* ----------------------------------------------------------------- bonded */

static double dihedral_angle(const double *x1, const double *x2, const double *x3, const double *x4)
{
    /* src/System/Metrics.cpp:42-82 */
    double b1[3], b2[3], b3[3], n1[3], n2[3];
    for (int k = 0; k < 3; ++k) { b1[k] = x2[k] - x1[k]; b2[k] = x3[k] - x2[k]; b3[k] = x4[k] - x3[k]; }
    n1[0] = b1[1] * b2[2] - b1[2] * b2[1];
    n1[1] = b2[0] * b1[2] - b1[0] * b2[2];
    n1[2] = b1[0] * b2[1] - b1[1] * b2[0];
    n2[0] = b2[1] * b3[2] - b2[2] * b3[1];
    n2[1] = b3[0] * b2[2] - b2[0] * b3[2];
    n2[2] = b2[0] * b3[1] - b2[1] * b3[0];
    double m1 = n1[0] * n1[0] + n1[1] * n1[1] + n1[2] * n1[2];
    double m2 = n2[0] * n2[0] + n2[1] * n2[1] + n2[2] * n2[2];
    double mb = sqrt(b2[0] * b2[0] + b2[1] * b2[1] + b2[2] * b2[2]);
    if (m1 < 1e-28 || m2 < 1e-28 || mb < 1e-14) return NAN;
    double xx = n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2];
    double yy = (b1[0] * n2[0] + b1[1] * n2[1] + b1[2] * n2[2]) * mb;
    return atan2(yy, xx);
}

static double angle_value(const double *x1, const double *x2, const double *x3)
{
    /* src/System/Metrics.cpp:20-40 */
    double a[3], c[3];
    for (int k = 0; k < 3; ++k) { a[k] = x1[k] - x2[k]; c[k] = x3[k] - x2[k]; }
    double dot = a[0] * c[0] + a[1] * c[1] + a[2] * c[2];
    double m1 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2], m2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
    if (m1 < 1e-14 || m2 < 1e-14) return NAN;
    double cc = dot * (1.0 / sqrt(m1 * m2));
    if (cc < -1.0) cc = -1.0;
    if (cc > 1.0) cc = 1.0;
    return acos(cc);
}

/* Torsion forces for dE/dphi on atoms (1,2,3,4).  physical=0 reproduces the
 * reference's formulas (src/System/BondedForces.cpp:193-239); physical=1 is
 * -grad E: with s1 = dphi/dr1 = -|cb|/|m|^2 m and s4 = +|cb|/|n|^2 n,
 * s2 = -(1 + ba.cb/|cb|^2) s1 + (dc.cb/|cb|^2) s4 and
 * s3 = (ba.cb/|cb|^2) s1 - (1 + dc.cb/|cb|^2) s4. */
static void torsion_forces(const double *x1, const double *x2, const double *x3, const double *x4,
                           double dEdphi, int physical, double *f1, double *f2, double *f3, double *f4, int *ok)
{
    double ba[3], cb[3], dc[3], m[3], n[3];
    for (int k = 0; k < 3; ++k) { ba[k] = x1[k] - x2[k]; cb[k] = x2[k] - x3[k]; dc[k] = x3[k] - x4[k]; }
    m[0] = ba[1] * cb[2] - ba[2] * cb[1]; m[1] = ba[2] * cb[0] - ba[0] * cb[2]; m[2] = ba[0] * cb[1] - ba[1] * cb[0];
    n[0] = cb[1] * dc[2] - cb[2] * dc[1]; n[1] = cb[2] * dc[0] - cb[0] * dc[2]; n[2] = cb[0] * dc[1] - cb[1] * dc[0];
    double mm = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
    double nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
    double bb = cb[0] * cb[0] + cb[1] * cb[1] + cb[2] * cb[2];
    *ok = !(mm < 1e-24 || nn < 1e-24 || bb < 1e-24);
    if (!*ok) return;
    double b = sqrt(bb);
    double dab = ba[0] * cb[0] + ba[1] * cb[1] + ba[2] * cb[2];
    double ddc = dc[0] * cb[0] + dc[1] * cb[1] + dc[2] * cb[2];
    double tau = -dEdphi;
    double sgn = physical ? -1.0 : 1.0;
    for (int k = 0; k < 3; ++k) {
        double fa = sgn * tau * b / mm * m[k];
        double fd = -sgn * tau * b / nn * n[k];
        f1[k] = fa;
        f4[k] = fd;
        if (!physical) {
            f2[k] = (dab / bb - 1) * fa - ddc / bb * fd;
            f3[k] = (ddc / bb - 1) * fd - dab / bb * fa;
        } else {
            f2[k] = (-1.0 - dab / bb) * fa + ddc / bb * fd;
            f3[k] = dab / bb * fa + (-1.0 - ddc / bb) * fd;
        }
    }
}

static void cmap_eval(const mdf_topology *t, int set, double phi, double psi, double *E, double *dphi, double *dpsi)
{
    /* src/Bonded/CMapGroup.cpp:82-237 */
    int res = t->cmap_res;
    double ph = phi, ps = psi;
    while (ph <= -M_PI) ph += 2.0 * M_PI;
    while (ph > M_PI) ph -= 2.0 * M_PI;
    while (ps <= -M_PI) ps += 2.0 * M_PI;
    while (ps > M_PI) ps -= 2.0 * M_PI;
    ph += M_PI;
    ps += M_PI;
    double sp = (2.0 * M_PI) / res;
    double gp = ph / sp, gs = ps / sp;
    int row = (int)gp, col = (int)gs;
    double u = gp - (double)row, v = gs - (double)col;
    row %= res; col %= res;
    if (row < 0) row += res;
    if (col < 0) col += res;
    const double *c = t->cmap_coeff + ((long)set * res * res + (long)row * res + col) * 16;
    double up[4] = {1.0, u, u * u, u * u * u}, vp[4] = {1.0, v, v * v, v * v * v};
    double dup[4] = {0.0, 1.0, 2.0 * u, 3.0 * u * u}, dvp[4] = {0.0, 1.0, 2.0 * v, 3.0 * v * v};
    double e = 0, du = 0, dv = 0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double cc = c[i * 4 + j];
            e += cc * up[i] * vp[j];
            du += cc * dup[i] * vp[j];
            dv += cc * up[i] * dvp[j];
        }
    double inv = 1.0 / sp;
    *E = e;
    *dphi = du * inv;
    *dpsi = dv * inv;
}

static void add3(double *f, int i, const double *v)
{
    f[3 * i] += v[0]; f[3 * i + 1] += v[1]; f[3 * i + 2] += v[2];
}

static void bonded(const mdf_topology *t, const oracle_params *p, const double *x, double *f, acc_t *e)
{
    int phys = p->semantics == MDF_SEM_PHYSICAL;
    /* bonds and UB: E = k (r - r0)^2, F_a = -2k (r - r0) d / r */
    for (int pass = 0; pass < 2; ++pass) {
        int n = pass ? t->n_ub : t->n_bonds;
        const int32_t *at = pass ? t->ub_atoms : t->bond_atoms;
        const double *K = pass ? t->ub_k : t->bond_k, *R0 = pass ? t->ub_r0 : t->bond_r0;
        for (int i = 0; i < n; ++i) {
            int a = at[2 * i], b = at[2 * i + 1];
            double d[3] = {x[3 * a] - x[3 * b], x[3 * a + 1] - x[3 * b + 1], x[3 * a + 2] - x[3 * b + 2]};
            double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            e[pass ? MDF_E_UB : MDF_E_BOND] += K[i] * (r - R0[i]) * (r - R0[i]);
            if (!f || r < 1e-12) continue;
            double fm = -2 * K[i] * (r - R0[i]);
            for (int k = 0; k < 3; ++k) {
                double fa = fm * d[k] / r;
                f[3 * a + k] += fa;
                f[3 * b + k] -= fa;
            }
        }
    }
    /* angles (src/System/BondedForces.cpp:73-153) */
    for (int i = 0; i < t->n_angles; ++i) {
        int a = t->angle_atoms[3 * i], b = t->angle_atoms[3 * i + 1], c = t->angle_atoms[3 * i + 2];
        const double *x1 = x + 3 * a, *x2 = x + 3 * b, *x3 = x + 3 * c;
        double th = angle_value(x1, x2, x3);
        double K = t->angle_k[i], t0 = t->angle_theta0[i];
        e[MDF_E_ANGLE] += K * (th - t0) * (th - t0);
        if (!f) continue;
        double ba[3], bc[3];
        for (int k = 0; k < 3; ++k) { ba[k] = x1[k] - x2[k]; bc[k] = x3[k] - x2[k]; }
        double ab2 = ba[0] * ba[0] + ba[1] * ba[1] + ba[2] * ba[2], ab = sqrt(ab2);
        if (ab < 1e-12) continue;
        double dot = ba[0] * bc[0] + ba[1] * bc[1] + ba[2] * bc[2];
        double pa[3] = {dot * ba[0] - ab2 * bc[0], dot * ba[1] - ab2 * bc[1], dot * ba[2] - ab2 * bc[2]};
        double mpa = sqrt(pa[0] * pa[0] + pa[1] * pa[1] + pa[2] * pa[2]);
        if (mpa < 1e-12) continue;
        double bc2 = bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2], cbm = sqrt(bc2);
        if (cbm < 1e-12) continue;
        double pc[3] = {dot * bc[0] - bc2 * ba[0], dot * bc[1] - bc2 * ba[1], dot * bc[2] - bc2 * ba[2]};
        double mpc = sqrt(pc[0] * pc[0] + pc[1] * pc[1] + pc[2] * pc[2]);
        if (mpc < 1e-12) continue;
        double fm = -2 * K * (th - t0);
        for (int k = 0; k < 3; ++k) {
            double fa = fm / ab * (pa[k] / mpa), fc = fm / cbm * (pc[k] / mpc);
            f[3 * a + k] += fa;
            f[3 * c + k] += fc;
            f[3 * b + k] += -fa - fc;
        }
    }
    /* cosine dihedrals */
    for (int i = 0; i < t->n_dihedrals; ++i) {
        const int32_t *at = t->dihedral_atoms + 4 * i;
        const double *x1 = x + 3 * at[0], *x2 = x + 3 * at[1], *x3 = x + 3 * at[2], *x4 = x + 3 * at[3];
        double phi = dihedral_angle(x1, x2, x3, x4);
        double K = t->dihedral_k[i], n = t->dihedral_n[i], dl = t->dihedral_phase[i];
        e[MDF_E_DIHEDRAL] += K * (1.0 + cos(n * phi - dl));
        if (!f) continue;
        double f1[3], f2[3], f3[3], f4[3];
        int ok;
        torsion_forces(x1, x2, x3, x4, -K * n * sin(n * phi - dl), phys, f1, f2, f3, f4, &ok);
        if (!ok) continue;
        add3(f, at[0], f1); add3(f, at[1], f2); add3(f, at[2], f3); add3(f, at[3], f4);
    }
    /* harmonic impropers: energy without wrap (REFERENCE, src/Bonded/HarmonicImproper.cpp:6-12),
     * force with wrap (src/System/BondedForces.cpp:281-284) */
    for (int i = 0; i < t->n_impropers; ++i) {
        const int32_t *at = t->improper_atoms + 4 * i;
        const double *x1 = x + 3 * at[0], *x2 = x + 3 * at[1], *x3 = x + 3 * at[2], *x4 = x + 3 * at[3];
        double psi = dihedral_angle(x1, x2, x3, x4);
        double K = t->improper_k[i], p0 = t->improper_phase[i];
        double dw = psi - p0;
        while (dw <= -M_PI) dw += 2.0 * M_PI;
        while (dw > M_PI) dw -= 2.0 * M_PI;
        double de = phys ? dw : psi - p0;
        e[MDF_E_IMPROPER] += K * de * de;
        if (!f) continue;
        double f1[3], f2[3], f3[3], f4[3];
        int ok;
        torsion_forces(x1, x2, x3, x4, 2.0 * K * dw, phys, f1, f2, f3, f4, &ok);
        if (!ok) continue;
        add3(f, at[0], f1); add3(f, at[1], f2); add3(f, at[2], f3); add3(f, at[3], f4);
    }
    /* CMAP (src/System/BondedEnergy.cpp:124-166, BondedForces.cpp:334-479) */
    for (int i = 0; i < t->n_cmaps; ++i) {
        const int32_t *at = t->cmap_atoms + 5 * i;
        const double *x1 = x + 3 * at[0], *x2 = x + 3 * at[1], *x3 = x + 3 * at[2], *x4 = x + 3 * at[3],
                     *x5 = x + 3 * at[4];
        double phi = dihedral_angle(x1, x2, x3, x4), psi = dihedral_angle(x2, x3, x4, x5);
        double E, dphi, dpsi;
        cmap_eval(t, t->cmap_set[i], phi, psi, &E, &dphi, &dpsi);
        e[MDF_E_CMAP] += E;
        if (!f) continue;
        /* the reference skips the whole term when any of its five norms is tiny */
        double ed[3], o[3], dc[3];
        for (int k = 0; k < 3; ++k) { ed[k] = x4[k] - x5[k]; dc[k] = x3[k] - x4[k]; }
        o[0] = dc[1] * ed[2] - dc[2] * ed[1]; o[1] = dc[2] * ed[0] - dc[0] * ed[2]; o[2] = dc[0] * ed[1] - dc[1] * ed[0];
        double oo = o[0] * o[0] + o[1] * o[1] + o[2] * o[2];
        double cd2 = dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2];
        double f1[3], f2[3], f3[3], f4[3], g2[3], g3[3], g4[3], g5[3];
        int ok1, ok2;
        torsion_forces(x1, x2, x3, x4, dphi, phys, f1, f2, f3, f4, &ok1);
        torsion_forces(x2, x3, x4, x5, dpsi, phys, g2, g3, g4, g5, &ok2);
        if (!ok1 || !ok2 || oo < 1e-24 || cd2 < 1e-24) continue;
        add3(f, at[0], f1); add3(f, at[1], f2); add3(f, at[2], f3); add3(f, at[3], f4);
        add3(f, at[1], g2); add3(f, at[2], g3); add3(f, at[3], g4); add3(f, at[4], g5);
    }
}

/* --------------------------------------------------------- reference PME */

static void ref_bspline5(double u, double *th, double *dth)
{
    /* src/System/PBC.cpp:329-401, including its order-3 weight (1+u) */
    double c0 = 1.0 - u, c1 = u;
    double w0 = 0.5 * (1.0 - u) * c0;
    double w1 = 0.5 * ((1.0 + u) * c0 + (2.0 - u) * c1);
    double w2 = 0.5 * (1.0 + u) * c1;
    double d4 = 1.0 / 3.0;
    double x0 = d4 * (1.0 - u) * w0;
    double x1 = d4 * ((2.0 + u) * w0 + (2.0 - u) * w1);
    double x2 = d4 * ((1.0 + u) * w1 + (3.0 - u) * w2);
    double x3 = d4 * (2.0 + u) * w2;
    th[0] = 0.25 * (1.0 - u) * x0;
    th[1] = 0.25 * ((3.0 + u) * x0 + (2.0 - u) * x1);
    th[2] = 0.25 * ((2.0 + u) * x1 + (3.0 - u) * x2);
    th[3] = 0.25 * ((1.0 + u) * x2 + (4.0 - u) * x3);
    th[4] = 0.25 * (3.0 + u) * x3;
    if (dth) {
        dth[0] = -x0; dth[1] = x0 - x1; dth[2] = x1 - x2; dth[3] = x2 - x3; dth[4] = x3;
    }
}

static void ref_bspline5_spread(double u, double *th)
{
    /* the spread path uses (1/2)((1-u) c0) etc. in this exact operation order */
    double c0 = 1.0 - u, c1 = u;
    double w0 = (1.0 / 2.0) * ((1.0 - u) * c0);
    double w1 = (1.0 / 2.0) * ((1.0 + u) * c0 + (2.0 - u) * c1);
    double w2 = (1.0 / 2.0) * ((1.0 + u) * c1);
    double x0 = (1.0 / 3.0) * ((1.0 - u) * w0);
    double x1 = (1.0 / 3.0) * ((2.0 + u) * w0 + (2.0 - u) * w1);
    double x2 = (1.0 / 3.0) * ((1.0 + u) * w1 + (3.0 - u) * w2);
    double x3 = (1.0 / 3.0) * ((2.0 + u) * w2);
    th[0] = (1.0 / 4.0) * ((1.0 - u) * x0);
    th[1] = (1.0 / 4.0) * ((3.0 + u) * x0 + (2.0 - u) * x1);
    th[2] = (1.0 / 4.0) * ((2.0 + u) * x1 + (3.0 - u) * x2);
    th[3] = (1.0 / 4.0) * ((1.0 + u) * x2 + (4.0 - u) * x3);
    th[4] = (1.0 / 4.0) * ((3.0 + u) * x3);
}

static void ref_moduli(int K, double *mod)
{
    double th[5];
    ref_bspline5_spread(0.0, th);
    double *rd = (double *)calloc((size_t)K, sizeof(double));
    double *co = (double *)calloc(2 * (size_t)(K / 2 + 1), sizeof(double));
    rd[0] = th[2]; rd[1] = th[3]; rd[2] = th[4]; rd[K - 1] = th[1]; rd[K - 2] = th[0];
    fft_ref_r2c_1d(rd, co, K);
    for (int i = 0; i < K / 2 + 1; ++i) {
        double m2 = co[2 * i] * co[2 * i] + co[2 * i + 1] * co[2 * i + 1];
        mod[i] = m2;
        if (i > 0 && i < (K + 1) / 2) mod[K - i] = m2;
    }
    free(rd);
    free(co);
}

static void ref_pme(const mdf_topology *t, const oracle_params *p, const double *x, double *fpme,
                    double *grid_q_out, double *grid_phi_out)
{
    int Kx = p->grid[0], Ky = p->grid[1], Kz = p->grid[2];
    long ntot = (long)Kx * Ky * Kz;
    double sx = Kx / p->box[0], sy = Ky / p->box[1], sz = Kz / p->box[2];
    double *Q = (double *)calloc((size_t)ntot, sizeof(double));
    for (int i = 0; i < t->natoms; ++i) {
        double q = t->charge[i];
        if (q == 0.0) continue;
        double ux = wrapx(x[3 * i], p->box[0]) * sx, uy = wrapx(x[3 * i + 1], p->box[1]) * sy,
               uz = wrapx(x[3 * i + 2], p->box[2]) * sz;
        int ix = (int)floor(ux), iy = (int)floor(uy), iz = (int)floor(uz);
        double tx[5], ty[5], tz[5];
        ref_bspline5_spread(ux - ix, tx);
        ref_bspline5_spread(uy - iy, ty);
        ref_bspline5_spread(uz - iz, tz);
        for (int a = 0; a < 5; ++a) {
            int kx = ((ix - 2 + a) % Kx + Kx) % Kx;
            for (int b = 0; b < 5; ++b) {
                int ky = ((iy - 2 + b) % Ky + Ky) % Ky;
                double wxy = tx[a] * ty[b];
                for (int c = 0; c < 5; ++c) {
                    int kz = ((iz - 2 + c) % Kz + Kz) % Kz;
                    Q[(long)kx * Ky * Kz + (long)ky * Kz + kz] += q * wxy * tz[c];
                }
            }
        }
    }
    if (grid_q_out) memcpy(grid_q_out, Q, sizeof(double) * (size_t)ntot);
    int Kzc = Kz / 2 + 1;
    double *C = (double *)malloc(sizeof(double) * 2 * (size_t)Kx * Ky * Kzc);
    fft_ref_r2c_3d(Q, C, Kx, Ky, Kz);
    double *mx = (double *)malloc(sizeof(double) * Kx), *my = (double *)malloc(sizeof(double) * Ky),
           *mz = (double *)malloc(sizeof(double) * Kz);
    ref_moduli(Kx, mx); ref_moduli(Ky, my); ref_moduli(Kz, mz);
    double V = p->box[0] * p->box[1] * p->box[2];
    double pre = 4.0 * M_PI / V, bsq = -1.0 / (4.0 * p->alpha * p->alpha), norm = 1.0 / (double)ntot;
    for (int i = 0; i < Kx; ++i) {
        int mi = (i <= Kx / 2) ? i : i - Kx;
        double kx = 2.0 * M_PI * mi / p->box[0];
        for (int j = 0; j < Ky; ++j) {
            int mj = (j <= Ky / 2) ? j : j - Ky;
            double ky = 2.0 * M_PI * mj / p->box[1];
            for (int k = 0; k < Kzc; ++k) {
                double kz = 2.0 * M_PI * k / p->box[2];
                double ksq = kx * kx + ky * ky + kz * kz;
                long idx = ((long)i * Ky + j) * Kzc + k;
                if (ksq < 1e-10) { C[2 * idx] = 0; C[2 * idx + 1] = 0; continue; }
                double infl = pre * exp(ksq * bsq) / ksq;
                double bc = 1.0 / (mx[i] * my[j] * mz[k]);
                double s = infl * bc * norm;
                C[2 * idx] *= s;
                C[2 * idx + 1] *= s;
            }
        }
    }
    fft_ref_c2r_3d(C, Q, Kx, Ky, Kz);
    if (grid_phi_out) memcpy(grid_phi_out, Q, sizeof(double) * (size_t)ntot);
    if (fpme) {
        for (int i = 0; i < t->natoms; ++i) {
            double q = t->charge[i];
            if (q == 0.0) continue;
            double ux = wrapx(x[3 * i], p->box[0]) * sx, uy = wrapx(x[3 * i + 1], p->box[1]) * sy,
                   uz = wrapx(x[3 * i + 2], p->box[2]) * sz;
            int ix = (int)floor(ux), iy = (int)floor(uy), iz = (int)floor(uz);
            double tx[5], ty[5], tz[5], dx[5], dy[5], dz[5];
            ref_bspline5(ux - ix, tx, dx);
            ref_bspline5(uy - iy, ty, dy);
            ref_bspline5(uz - iz, tz, dz);
            double fx = 0, fy = 0, fz = 0;
            for (int a = 0; a < 5; ++a) {
                int kx = (ix - 2 + a) % Kx; if (kx < 0) kx += Kx;
                for (int b = 0; b < 5; ++b) {
                    int ky = (iy - 2 + b) % Ky; if (ky < 0) ky += Ky;
                    for (int c = 0; c < 5; ++c) {
                        int kz = (iz - 2 + c) % Kz; if (kz < 0) kz += Kz;
                        double pot = Q[(long)kx * Ky * Kz + (long)ky * Kz + kz];
                        fx -= q * pot * dx[a] * ty[b] * tz[c] * sx;
                        fy -= q * pot * tx[a] * dy[b] * tz[c] * sy;
                        fz -= q * pot * tx[a] * ty[b] * dz[c] * sz;
                    }
                }
            }
            fpme[3 * i] += fx; fpme[3 * i + 1] += fy; fpme[3 * i + 2] += fz;
        }
    }
    free(Q); free(C); free(mx); free(my); free(mz);
}

/* ------------------------------------------------------------ smooth PME */

/* Cardinal B-spline weights of order n at fractional offset w in [0,1):
 * th[j] = M_n(w + n - 1 - j), dth[j] = d/dw of it (Essmann et al. eq. 4.1-4.2). */
static void bspline(int n, double w, double *th, double *dth)
{
    double m[16];
    /* order 2 */
    m[0] = 1.0 - w; m[1] = w;
    for (int k = 3; k <= n; ++k) {
        double div = 1.0 / (k - 1);
        if (k == n && dth) {
            /* derivative from order n-1: dM_n(x)/dx = M_{n-1}(x) - M_{n-1}(x-1) */
            dth[0] = -m[0];
            for (int j = 1; j < k - 1; ++j) dth[j] = m[j - 1] - m[j];
            dth[k - 1] = m[k - 2];
        }
        /* m[j] = M_{k-1}(w + k-2-j), j = 0..k-2; recursion
         * M_k(x) = x/(k-1) M_{k-1}(x) + (k-x)/(k-1) M_{k-1}(x-1) */
        double nm[16];
        nm[0] = div * (1.0 - w) * m[0];
        for (int j = 1; j < k - 1; ++j)
            nm[j] = div * ((w + k - 1 - j) * m[j - 1] + (1.0 - w + j) * m[j]);
        nm[k - 1] = div * w * m[k - 2];
        for (int j = 0; j < k; ++j) m[j] = nm[j];
    }
    for (int j = 0; j < n; ++j) th[j] = m[j];
}

double oracle_pme_recip(const mdf_topology *t, const oracle_params *p, const double *x, double *f, double *virial)
{
    int n = p->pme_order;
    int K[3] = {p->grid[0], p->grid[1], p->grid[2]};
    long ntot = (long)K[0] * K[1] * K[2];
    int Kzc = K[2] / 2 + 1;
    double *Q = (double *)calloc((size_t)ntot, sizeof(double));
    int N = t->natoms;
    int *base = (int *)malloc(sizeof(int) * 3 * (size_t)N);
    double *th = (double *)malloc(sizeof(double) * 3 * (size_t)N * n);
    double *dth = (double *)malloc(sizeof(double) * 3 * (size_t)N * n);
    int shift = n / 2 - 1;   /* grid point of weight j: base - shift + j */
    for (int i = 0; i < N; ++i) {
        for (int d = 0; d < 3; ++d) {
            double u = wrapx(x[3 * i + d], p->box[d]) * (K[d] / p->box[d]);
            if (u >= K[d]) u -= K[d];
            int b = (int)floor(u);
            base[3 * i + d] = b;
            bspline(n, u - b, th + (3 * (long)i + d) * n, dth + (3 * (long)i + d) * n);
        }
        double q = t->charge[i];
        const double *tx = th + (3 * (long)i) * n, *ty = tx + n, *tz = ty + n;
        for (int a = 0; a < n; ++a) {
            int kx = ((base[3 * i] - shift + a) % K[0] + K[0]) % K[0];
            for (int b = 0; b < n; ++b) {
                int ky = ((base[3 * i + 1] - shift + b) % K[1] + K[1]) % K[1];
                for (int c = 0; c < n; ++c) {
                    int kz = ((base[3 * i + 2] - shift + c) % K[2] + K[2]) % K[2];
                    Q[((long)kx * K[1] + ky) * K[2] + kz] += q * tx[a] * ty[b] * tz[c];
                }
            }
        }
    }
    double *S = (double *)malloc(sizeof(double) * 2 * (size_t)K[0] * K[1] * Kzc);
    fft_ref_r2c_3d(Q, S, K[0], K[1], K[2]);
    /* B-spline moduli: D(m) = |sum_{k=0}^{n-2} M_n(k+1) exp(2 pi i m k / K)|^2, B = 1/D */
    double Mk[16], dummy[16];
    bspline(n, 0.0, Mk, dummy);    /* Mk[j] = M_n(n-1-j) at w=0 */
    double *Bd[3];
    for (int d = 0; d < 3; ++d) {
        Bd[d] = (double *)malloc(sizeof(double) * K[d]);
        for (int m = 0; m < K[d]; ++m) {
            double sr = 0, si = 0;
            for (int k = 0; k <= n - 2; ++k) {
                double v = Mk[n - 2 - k];          /* M_n(k+1) */
                double a = 2.0 * M_PI * m * k / K[d];
                sr += v * cos(a);
                si += v * sin(a);
            }
            Bd[d][m] = sr * sr + si * si;
        }
        for (int m = 0; m < K[d]; ++m)
            if (Bd[d][m] < 1e-7) Bd[d][m] = 0.5 * (Bd[d][(m - 1 + K[d]) % K[d]] + Bd[d][(m + 1) % K[d]]);
    }
    double V = p->box[0] * p->box[1] * p->box[2];
    double fac = p->kc / (M_PI * V), pa2 = M_PI * M_PI / (p->alpha * p->alpha);
    acc_t E = 0, W[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < K[0]; ++i) {
        double mx = ((i <= K[0] / 2) ? i : i - K[0]) / p->box[0];
        for (int j = 0; j < K[1]; ++j) {
            double my = ((j <= K[1] / 2) ? j : j - K[1]) / p->box[1];
            for (int k = 0; k < Kzc; ++k) {
                double mz = k / p->box[2];
                long idx = ((long)i * K[1] + j) * Kzc + k;
                double m2 = mx * mx + my * my + mz * mz;
                if (i == 0 && j == 0 && k == 0) { S[2 * idx] = S[2 * idx + 1] = 0; continue; }
                double c = fac * exp(-pa2 * m2) / m2 / (Bd[0][i] * Bd[1][j] * Bd[2][k]);
                double s2 = S[2 * idx] * S[2 * idx] + S[2 * idx + 1] * S[2 * idx + 1];
                double wgt = (k == 0 || (K[2] % 2 == 0 && k == K[2] / 2)) ? 1.0 : 2.0;
                double em = 0.5 * c * s2 * wgt;
                E += em;
                double vf = 2.0 * (1.0 + pa2 * m2) / m2;
                double mv[3] = {mx, my, mz};
                int q = 0;
                for (int a = 0; a < 3; ++a)
                    for (int b = a; b < 3; ++b)
                        W[q++] += em * ((a == b ? 1.0 : 0.0) - vf * mv[a] * mv[b]);
                S[2 * idx] *= c;
                S[2 * idx + 1] *= c;
            }
        }
    }
    if (virial) {
        virial[0] = (double)W[0]; virial[1] = (double)W[1]; virial[2] = (double)W[2];
        virial[3] = (double)W[1]; virial[4] = (double)W[3]; virial[5] = (double)W[4];
        virial[6] = (double)W[2]; virial[7] = (double)W[4]; virial[8] = (double)W[5];
    }
    if (f) {
        fft_ref_c2r_3d(S, Q, K[0], K[1], K[2]);     /* Phi = dE/dQ */
        for (int i = 0; i < N; ++i) {
            double q = t->charge[i];
            const double *tx = th + (3 * (long)i) * n, *ty = tx + n, *tz = ty + n;
            const double *dx = dth + (3 * (long)i) * n, *dy = dx + n, *dz = dy + n;
            double gx = 0, gy = 0, gz = 0;
            for (int a = 0; a < n; ++a) {
                int kx = ((base[3 * i] - shift + a) % K[0] + K[0]) % K[0];
                for (int b = 0; b < n; ++b) {
                    int ky = ((base[3 * i + 1] - shift + b) % K[1] + K[1]) % K[1];
                    for (int c = 0; c < n; ++c) {
                        int kz = ((base[3 * i + 2] - shift + c) % K[2] + K[2]) % K[2];
                        double ph = Q[((long)kx * K[1] + ky) * K[2] + kz];
                        gx += dx[a] * ty[b] * tz[c] * ph;
                        gy += tx[a] * dy[b] * tz[c] * ph;
                        gz += tx[a] * ty[b] * dz[c] * ph;
                    }
                }
            }
            f[3 * i] -= q * gx * K[0] / p->box[0];
            f[3 * i + 1] -= q * gy * K[1] / p->box[1];
            f[3 * i + 2] -= q * gz * K[2] / p->box[2];
        }
    }
    free(Q); free(S); free(base); free(th); free(dth);
    for (int d = 0; d < 3; ++d) free(Bd[d]);
    return (double)E;
}

double oracle_ewald_recip_exact(int n, const double *q, const double *x, const double box[3],
                                double alpha, double kc, int kmax, double *f)
{
    double V = box[0] * box[1] * box[2];
    double pa2 = M_PI * M_PI / (alpha * alpha);
    acc_t E = 0;
    double *cs = (double *)malloc(sizeof(double) * (size_t)n), *sn = (double *)malloc(sizeof(double) * (size_t)n);
    for (int a = -kmax; a <= kmax; ++a)
        for (int b = -kmax; b <= kmax; ++b)
            for (int c = -kmax; c <= kmax; ++c) {
                if (!a && !b && !c) continue;
                double m[3] = {a / box[0], b / box[1], c / box[2]};
                double m2 = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
                double sr = 0, si = 0;
                for (int i = 0; i < n; ++i) {
                    double ph = 2.0 * M_PI * (m[0] * x[3 * i] + m[1] * x[3 * i + 1] + m[2] * x[3 * i + 2]);
                    cs[i] = cos(ph); sn[i] = sin(ph);
                    sr += q[i] * cs[i];
                    si += q[i] * sn[i];
                }
                double g = kc / (2.0 * M_PI * V) * exp(-pa2 * m2) / m2;
                E += g * (sr * sr + si * si);
                if (f)
                    for (int i = 0; i < n; ++i) {
                        /* dE/dx_i = g * 2 * q_i * 2 pi m (-sin * sr + cos * si) */
                        double t = g * 2.0 * q[i] * 2.0 * M_PI * (-sn[i] * sr + cs[i] * si);
                        f[3 * i] -= t * m[0]; f[3 * i + 1] -= t * m[1]; f[3 * i + 2] -= t * m[2];
                    }
            }
    free(cs); free(sn);
    return (double)E;
}

/* ------------------------------------------------------------------- CMAP */

/* The reference's 16x16 integer interpolation table (it defines the
 * interpolant and is not a plain bicubic: rows 9-13 do not sum to zero). */
static const signed char CMAP_M[16][16] = {
    {0, 0, 0, 0, 0, 16, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, -8, 0, 8, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, 16, -40, 32, -8, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, -8, 24, -24, 8, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, -8, 0, 0, 0, 0, 0, 0, 0, 8, 0, 0, 0, 0, 0, 0},
    {0, -4, 0, 0, -4, 4, 0, 0, 0, 0, 4, 0, 0, 0, 0, 0},
    {0, 32, -20, 0, 8, -4, -4, 0, 0, -24, 16, -4, 0, 0, 0, 0},
    {0, -20, 12, 0, -4, 0, 4, 0, 0, 16, -12, 4, 0, 0, 0, 0},
    {0, 16, 0, 0, 0, -40, 0, 0, 0, 32, 0, 0, 0, -8, 0, 0},
    {0, 8, 0, 0, 32, -4, -24, 0, -20, -4, 0, 0, 0, 0, -4, 0},
    {0, -64, 40, 0, -64, 96, -68, 24, 40, -68, -16, -16, 0, 24, -16, 0},
    {0, 40, -24, 0, 32, -52, 52, -24, -20, 40, 16, 16, 0, -16, 12, 0},
    {0, -8, 0, 0, 0, 24, 0, 0, 0, -24, 0, 0, 0, 8, 0, 4},
    {0, -4, 0, 0, -20, 0, 16, 0, 12, 4, -12, 0, 0, 0, 4, -4},
    {0, 32, -20, 0, 40, -52, 40, -16, -24, 52, -52, 12, 0, -24, 16, -4},
    {0, -20, 12, 0, -20, 28, -32, 16, 12, -32, 40, -12, 0, 16, -12, 4}};

void oracle_cmap_coeff(int nsets, int res, const double *grids, double *coeff)
{
    for (int s = 0; s < nsets; ++s) {
        const double *g = grids + (long)s * res * res;
        for (int r = 0; r < res; ++r)
            for (int c = 0; c < res; ++c) {
                double e16[16];
                int k = 0;
                for (int dc = -1; dc <= 2; ++dc)
                    for (int dr = -1; dr <= 2; ++dr) {
                        int rr = r + dr, cc = c + dc;
                        if (rr < 0) rr += res; else if (rr >= res) rr -= res;
                        if (cc < 0) cc += res; else if (cc >= res) cc -= res;
                        e16[k++] = g[rr * res + cc];
                    }
                double *out = coeff + (((long)s * res + r) * res + c) * 16;
                for (int row = 0; row < 16; ++row) {
                    double acc = 0.0;
                    for (int col = 0; col < 16; ++col) acc += CMAP_M[row][col] * e16[col] / 16;
                    out[row] = acc;
                }
            }
    }
}

/* ------------------------------------------------------------------- main */

int oracle_pme_ref_grids(const mdf_topology *t, const oracle_params *p, const double *x, double *grid_q,
                         double *grid_phi)
{
    ref_pme(t, p, x, NULL, grid_q, grid_phi);
    return 0;
}

int oracle_eval(const mdf_topology *t, const oracle_params *p, const double *x, double *f, double *e,
                double *virial, double *f_pme_ref, long *npairs)
{
    int N = t->natoms;
    if (f) memset(f, 0, sizeof(double) * 3 * (size_t)N);
    if (virial) memset(virial, 0, sizeof(double) * 9);
    pairsets ps;
    build_sets(t, &ps);
    nbctx c;
    memset(&c, 0, sizeof(c));
    c.t = t; c.p = p; c.s = &ps; c.f = f;
    bonded(t, p, x, f, c.e);
    int phys = p->semantics == MDF_SEM_PHYSICAL;
    if (!phys) {
        for_pairs(p, N, x, p->cutoff, ref_pair, &c);
        /* excluded non-1-4 pairs: -k q q erf(alpha r)/r, src/System/NonBondedEnergy.cpp:271-304 */
        for (long i = 0; i < t->n_excl; ++i) {
            int a = t->excl_pairs[2 * i], b = t->excl_pairs[2 * i + 1];
            if (a > b) { int tt = a; a = b; b = tt; }
            if (find14(&ps, pkey(a, b)) >= 0) continue;
            double d[3] = {x[3 * a] - x[3 * b], x[3 * a + 1] - x[3 * b + 1], x[3 * a + 2] - x[3 * b + 2]};
            mic(p, d);
            double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            c.e[MDF_E_EE_DIRECT] += -p->kc * (t->charge[a] * t->charge[b] / r) * erf(p->alpha * r);
        }
        /* self term, src/System/NonBondedEnergy.cpp:307-316 */
        for (int i = 0; i < N; ++i)
            c.e[MDF_E_EE_SELF] += -p->kc * (p->alpha / sqrt(M_PI)) * (t->charge[i] * t->charge[i]);
        if (f_pme_ref) {
            memset(f_pme_ref, 0, sizeof(double) * 3 * (size_t)N);
            ref_pme(t, p, x, f_pme_ref, NULL, NULL);
        }
    } else {
        for_pairs(p, N, x, p->cutoff, phys_pair, &c);
        /* excluded pairs: -k q q erf(alpha r)/r and its force, min image, no cutoff */
        for (long i = 0; i < t->n_excl; ++i) {
            int a = t->excl_pairs[2 * i], b = t->excl_pairs[2 * i + 1];
            double d[3] = {x[3 * a] - x[3 * b], x[3 * a + 1] - x[3 * b + 1], x[3 * a + 2] - x[3 * b + 2]};
            mic(p, d);
            double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2], r = sqrt(r2);
            double qq = t->charge[a] * t->charge[b] * p->kc;
            double ar = p->alpha * r;
            double ee = -qq * erf(ar) / r;
            c.e[MDF_E_EE_EXCL] += ee;
            /* F_a = -dE/dr d/r, dE/dr = -qq (2a/sqrt(pi) e^{-a^2r^2}/r - erf/r^2) */
            double g = (ee + qq * (2.0 * p->alpha / sqrt(M_PI)) * exp(-ar * ar)) / r2;
            if (f)
                for (int k = 0; k < 3; ++k) { f[3 * a + k] += g * d[k]; f[3 * b + k] -= g * d[k]; }
        }
        /* scaled 1-4 pairs: k q q /(scee r) + (A14/r^12 - B14/r^6)/scnb, min image, no cutoff */
        for (long i = 0; i < t->n_pairs14; ++i) {
            int a = t->pairs14[2 * i], b = t->pairs14[2 * i + 1];
            double d[3] = {x[3 * a] - x[3 * b], x[3 * a + 1] - x[3 * b + 1], x[3 * a + 2] - x[3 * b + 2]};
            mic(p, d);
            double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2], r = sqrt(r2);
            double qq = t->charge[a] * t->charge[b] * p->kc / t->scee14[i];
            double ec = qq / r;
            c.e[MDF_E_EE14] += ec;
            double g = ec / r2;
            int nb = t->nb_index[t->type[a] * t->ntypes + t->type[b]];
            if (nb > 0) {
                double A = t->lj14_a[nb - 1] / t->scnb14[i], B = t->lj14_b[nb - 1] / t->scnb14[i];
                c.e[MDF_E_VDW14] += lj_u(r2, A, B);
                g += lj_g(r2, A, B);
            }
            if (f)
                for (int k = 0; k < 3; ++k) { f[3 * a + k] += g * d[k]; f[3 * b + k] -= g * d[k]; }
        }
        acc_t q2 = 0, qt = 0;
        for (int i = 0; i < N; ++i) { q2 += t->charge[i] * t->charge[i]; qt += t->charge[i]; }
        c.e[MDF_E_EE_SELF] = -p->kc * (p->alpha / sqrt(M_PI)) * q2;
        if (p->do_recip) {
            double V = p->box[0] * p->box[1] * p->box[2];
            c.e[MDF_E_EE_RECIP] = oracle_pme_recip(t, p, x, f, virial);
            /* neutralising-background term for a net charge */
            c.e[MDF_E_EE_RECIP] += -p->kc * M_PI * (double)(qt * qt) / (2.0 * V * p->alpha * p->alpha);
        }
    }
    for (int k = 0; k < MDF_E_COUNT; ++k) e[k] = (double)c.e[k];
    if (npairs) *npairs = c.npairs;
    free_sets(&ps);
    return 0;
}
