// Bonded terms in one launch: bond, Urey-Bradley, angle, cosine dihedral,
// harmonic improper, CMAP.  FP64 in both precision modes (bond stretches of
// ~1 A with k ~ 450 make FP32 coordinate rounding visible in the forces).
//
// Replaces src/System/BondedEnergy.cpp:10-166 and
// src/System/BondedForces.cpp:10-479 (geometry from src/System/Metrics.cpp,
// term energies from src/Bonded/*.cpp, CMAP from src/Bonded/CMapGroup.cpp).
// REFERENCE semantics keep the reference's torsion-force formulas and its
// unwrapped improper energy; PHYSICAL semantics use -grad E and wrap the
// improper difference into (-pi, pi].
#include <cmath>

#include "kargs.cuh"
#include "mdf_device.cuh"
#include "mdf_internal.cuh"

namespace mdf {


__device__ __forceinline__ void ld3(const double* x, int a, double p[3])
{
    p[0] = x[3 * a]; p[1] = x[3 * a + 1]; p[2] = x[3 * a + 2];
}

__device__ __forceinline__ void fadd3(unsigned long long* f, int N, int a, const double v[3], unsigned* st)
{
    fx_add(f + a, v[0], FORCE_SCALE, st);
    fx_add(f + N + a, v[1], FORCE_SCALE, st);
    fx_add(f + 2 * N + a, v[2], FORCE_SCALE, st);
}

// Metrics::dihedral (src/System/Metrics.cpp:42-82)
__device__ double dihedral_angle(const double x1[3], const double x2[3], const double x3[3], const double x4[3])
{
    double b1[3], b2[3], b3[3];
    for (int k = 0; k < 3; ++k) { b1[k] = x2[k] - x1[k]; b2[k] = x3[k] - x2[k]; b3[k] = x4[k] - x3[k]; }
    double n1[3] = {b1[1] * b2[2] - b1[2] * b2[1], b2[0] * b1[2] - b1[0] * b2[2], b1[0] * b2[1] - b1[1] * b2[0]};
    double n2[3] = {b2[1] * b3[2] - b2[2] * b3[1], b3[0] * b2[2] - b2[0] * b3[2], b2[0] * b3[1] - b2[1] * b3[0]};
    double m1 = n1[0] * n1[0] + n1[1] * n1[1] + n1[2] * n1[2];
    double m2 = n2[0] * n2[0] + n2[1] * n2[1] + n2[2] * n2[2];
    double mb = sqrt(b2[0] * b2[0] + b2[1] * b2[1] + b2[2] * b2[2]);
    if (m1 < 1e-28 || m2 < 1e-28 || mb < 1e-14) return nan("");
    double xx = n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2];
    double yy = (b1[0] * n2[0] + b1[1] * n2[1] + b1[2] * n2[2]) * mb;
    return atan2(yy, xx);
}

// Torsion forces for a given dE/dphi.  PHYS=false: the reference's formulas
// (src/System/BondedForces.cpp:193-239).  PHYS=true: -grad E with
// dphi/dr1 = -|cb|/|m|^2 m, dphi/dr4 = |cb|/|n|^2 n and the middle atoms from
// translational and rotational invariance.
template <bool PHYS>
__device__ bool torsion_forces(const double x1[3], const double x2[3], const double x3[3], const double x4[3],
                               double dEdphi, double f1[3], double f2[3], double f3[3], double f4[3])
{
    double ba[3], cb[3], dc[3];
    for (int k = 0; k < 3; ++k) { ba[k] = x1[k] - x2[k]; cb[k] = x2[k] - x3[k]; dc[k] = x3[k] - x4[k]; }
    double m[3] = {ba[1] * cb[2] - ba[2] * cb[1], ba[2] * cb[0] - ba[0] * cb[2], ba[0] * cb[1] - ba[1] * cb[0]};
    double n[3] = {cb[1] * dc[2] - cb[2] * dc[1], cb[2] * dc[0] - cb[0] * dc[2], cb[0] * dc[1] - cb[1] * dc[0]};
    double mm = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
    double nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
    double bb = cb[0] * cb[0] + cb[1] * cb[1] + cb[2] * cb[2];
    if (mm < 1e-24 || nn < 1e-24 || bb < 1e-24) return false;
    double b = sqrt(bb);
    double dab = ba[0] * cb[0] + ba[1] * cb[1] + ba[2] * cb[2];
    double ddc = dc[0] * cb[0] + dc[1] * cb[1] + dc[2] * cb[2];
    double tau = -dEdphi;
    for (int k = 0; k < 3; ++k) {
        if (!PHYS) {
            double fa = tau * b / mm * m[k], fd = -tau * b / nn * n[k];
            f1[k] = fa;
            f4[k] = fd;
            f2[k] = (dab / bb - 1) * fa - ddc / bb * fd;
            f3[k] = (ddc / bb - 1) * fd - dab / bb * fa;
        } else {
            double fa = -tau * b / mm * m[k], fd = tau * b / nn * n[k];
            f1[k] = fa;
            f4[k] = fd;
            f2[k] = (-1.0 - dab / bb) * fa + ddc / bb * fd;
            f3[k] = dab / bb * fa + (-1.0 - ddc / bb) * fd;
        }
    }
    return true;
}

// CMapGroup::return_energy_bicubic / return_gradient_bicubic
// (src/Bonded/CMapGroup.cpp:82-237)
__device__ void cmap_eval(const double* __restrict__ coeff, int res, int set, double phi, double psi, double& E,
                          double& dphi, double& dpsi)
{
    const double PI = 3.14159265358979323846;
    double ph = phi, ps = psi;
    while (ph <= -PI) ph += 2.0 * PI;
    while (ph > PI) ph -= 2.0 * PI;
    while (ps <= -PI) ps += 2.0 * PI;
    while (ps > PI) ps -= 2.0 * PI;
    ph += PI;
    ps += PI;
    double sp = (2.0 * PI) / res;
    double gp = ph / sp, gs = ps / sp;
    int row = (int)gp, col = (int)gs;
    double u = gp - (double)row, v = gs - (double)col;
    row %= res;
    col %= res;
    if (row < 0) row += res;
    if (col < 0) col += res;
    const double* c = coeff + ((long long)set * res * res + (long long)row * res + col) * 16;
    double up[4] = {1.0, u, u * u, u * u * u}, vp[4] = {1.0, v, v * v, v * v * v};
    double dup[4] = {0.0, 1.0, 2.0 * u, 3.0 * u * u}, dvp[4] = {0.0, 1.0, 2.0 * v, 3.0 * v * v};
    double e = 0, du = 0, dv = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double cc = __ldg(c + i * 4 + j);
            e += cc * up[i] * vp[j];
            du += cc * dup[i] * vp[j];
            dv += cc * up[i] * dvp[j];
        }
    double inv = 1.0 / sp;
    E = e;
    dphi = du * inv;
    dpsi = dv * inv;
}

template <bool PHYS, bool ENERGY>
__device__ __forceinline__ void bonded_dev(const BondedArgs& A)
{
    unsigned long long* __restrict__ f = A.f;
    unsigned long long* __restrict__ acc = A.acc;
    unsigned* st = A.st;
    const double PI = 3.14159265358979323846;
    int seg = 0;
    while (seg < 5 && (int)blockIdx.x >= A.blk0[seg + 1]) ++seg;
    int i = A.lo[seg] + ((int)blockIdx.x - A.blk0[seg]) * blockDim.x + threadIdx.x;
    const double* x = A.xyz;
    double e = 0.0;
    int eidx = MDF_E_BOND;
    if (seg == 0 || seg == 1) {
        eidx = seg == 0 ? MDF_E_BOND : MDF_E_UB;
        if (i < A.n[seg]) {
            const int* at = seg == 0 ? A.bond_atoms : A.ub_atoms;
            double2 kp = seg == 0 ? A.bond_par[i] : A.ub_par[i];
            int a = at[2 * i], b = at[2 * i + 1];
            double pa[3], pb[3];
            ld3(x, a, pa);
            ld3(x, b, pb);
            double d[3] = {pa[0] - pb[0], pa[1] - pb[1], pa[2] - pb[2]};
            double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            e = kp.x * (r - kp.y) * (r - kp.y);
            if (r >= 1e-12) {
                double fm = -2 * kp.x * (r - kp.y);
                double fa[3] = {fm * d[0] / r, fm * d[1] / r, fm * d[2] / r};
                double fb[3] = {-fa[0], -fa[1], -fa[2]};
                fadd3(f, A.N, a, fa, st);
                fadd3(f, A.N, b, fb, st);
            }
        }
    } else if (seg == 2) {
        eidx = MDF_E_ANGLE;
        if (i < A.n[2]) {
            int a = A.angle_atoms[3 * i], b = A.angle_atoms[3 * i + 1], c = A.angle_atoms[3 * i + 2];
            double2 kp = A.angle_par[i];
            double x1[3], x2[3], x3[3];
            ld3(x, a, x1);
            ld3(x, b, x2);
            ld3(x, c, x3);
            double ba[3], bc[3];
            for (int k = 0; k < 3; ++k) { ba[k] = x1[k] - x2[k]; bc[k] = x3[k] - x2[k]; }
            double dot = ba[0] * bc[0] + ba[1] * bc[1] + ba[2] * bc[2];
            double ab2 = ba[0] * ba[0] + ba[1] * ba[1] + ba[2] * ba[2];
            double bc2 = bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2];
            double th;
            if (ab2 < 1e-14 || bc2 < 1e-14) {
                th = nan("");
            } else {
                double cc = dot * (1.0 / sqrt(ab2 * bc2));
                cc = fmin(1.0, fmax(-1.0, cc));
                th = acos(cc);
            }
            e = kp.x * (th - kp.y) * (th - kp.y);
            // forces (src/System/BondedForces.cpp:73-153)
            double ab = sqrt(ab2), cbm = sqrt(bc2);
            double pa[3] = {dot * ba[0] - ab2 * bc[0], dot * ba[1] - ab2 * bc[1], dot * ba[2] - ab2 * bc[2]};
            double pc[3] = {dot * bc[0] - bc2 * ba[0], dot * bc[1] - bc2 * ba[1], dot * bc[2] - bc2 * ba[2]};
            double mpa = sqrt(pa[0] * pa[0] + pa[1] * pa[1] + pa[2] * pa[2]);
            double mpc = sqrt(pc[0] * pc[0] + pc[1] * pc[1] + pc[2] * pc[2]);
            if (ab >= 1e-12 && mpa >= 1e-12 && cbm >= 1e-12 && mpc >= 1e-12) {
                double fm = -2 * kp.x * (th - kp.y);
                double fa[3], fc[3], fb[3];
                for (int k = 0; k < 3; ++k) {
                    fa[k] = fm / ab * (pa[k] / mpa);
                    fc[k] = fm / cbm * (pc[k] / mpc);
                    fb[k] = -fa[k] - fc[k];
                }
                fadd3(f, A.N, a, fa, st);
                fadd3(f, A.N, c, fc, st);
                fadd3(f, A.N, b, fb, st);
            }
        }
    } else if (seg == 3 || seg == 4) {
        eidx = seg == 3 ? MDF_E_DIHEDRAL : MDF_E_IMPROPER;
        if (i < A.n[seg]) {
            const int* at = (seg == 3 ? A.dih_atoms : A.imp_atoms) + 4 * i;
            double x1[3], x2[3], x3[3], x4[3];
            ld3(x, at[0], x1);
            ld3(x, at[1], x2);
            ld3(x, at[2], x3);
            ld3(x, at[3], x4);
            double phi = dihedral_angle(x1, x2, x3, x4);
            double dEdphi;
            if (seg == 3) {
                double K = A.dih_par[3 * i], n = A.dih_par[3 * i + 1], dl = A.dih_par[3 * i + 2];
                e = K * (1.0 + cos(n * phi - dl));
                dEdphi = -K * n * sin(n * phi - dl);
            } else {
                double2 kp = A.imp_par[i];
                double dw = phi - kp.y;
                while (dw <= -PI) dw += 2.0 * PI;
                while (dw > PI) dw -= 2.0 * PI;
                double de = PHYS ? dw : phi - kp.y;
                e = kp.x * de * de;
                dEdphi = 2.0 * kp.x * dw;
            }
            double f1[3], f2[3], f3[3], f4[3];
            if (torsion_forces<PHYS>(x1, x2, x3, x4, dEdphi, f1, f2, f3, f4)) {
                fadd3(f, A.N, at[0], f1, st);
                fadd3(f, A.N, at[1], f2, st);
                fadd3(f, A.N, at[2], f3, st);
                fadd3(f, A.N, at[3], f4, st);
            }
        }
    } else {
        eidx = MDF_E_CMAP;
        if (i < A.n[5]) {
            const int* at = A.cmap_atoms + 5 * i;
            double x1[3], x2[3], x3[3], x4[3], x5[3];
            ld3(x, at[0], x1);
            ld3(x, at[1], x2);
            ld3(x, at[2], x3);
            ld3(x, at[3], x4);
            ld3(x, at[4], x5);
            double phi = dihedral_angle(x1, x2, x3, x4), psi = dihedral_angle(x2, x3, x4, x5);
            double dphi, dpsi;
            cmap_eval(A.cmap_coeff, A.cmap_res, A.cmap_set[i], phi, psi, e, dphi, dpsi);
            double f1[3], f2[3], f3[3], f4[3], g2[3], g3[3], g4[3], g5[3];
            bool ok1 = torsion_forces<PHYS>(x1, x2, x3, x4, dphi, f1, f2, f3, f4);
            bool ok2 = torsion_forces<PHYS>(x2, x3, x4, x5, dpsi, g2, g3, g4, g5);
            if (ok1 && ok2) {
                for (int k = 0; k < 3; ++k) {
                    f2[k] += g2[k];
                    f3[k] += g3[k];
                    f4[k] += g4[k];
                }
                fadd3(f, A.N, at[0], f1, st);
                fadd3(f, A.N, at[1], f2, st);
                fadd3(f, A.N, at[2], f3, st);
                fadd3(f, A.N, at[3], f4, st);
                fadd3(f, A.N, at[4], g5, st);
            }
        }
    }
    if (ENERGY) {
        const double v[1] = {e};
        const int idx[1] = {eidx};
        block_acc_fixed<1>(v, acc, idx, ENERGY_SCALE, st);
    }
}

template <bool PHYS, bool ENERGY>
__global__ void __launch_bounds__(256) k_bonded(BondedArgs A)
{
    bonded_dev<PHYS, ENERGY>(A);
}

template <bool PHYS, bool ENERGY>
__global__ void __launch_bounds__(256) k_bonded_multi(const BondedArgs* __restrict__ As)
{
    const BondedArgs& A = As[blockIdx.z];
    if ((int)blockIdx.x >= A.gx) return;
    bonded_dev<PHYS, ENERGY>(A);
}

// The six term lists in one launch: this rank's share of each (all of them
// with one rank, or with whole = true), accumulated into f / acc / st.
BondedArgs make_bonded_args(const Ctx& c, bool whole, unsigned long long* f, unsigned long long* acc, unsigned* st)
{
    BondedArgs A;
    const int total[6] = {c.n_bonds, c.n_ub, c.n_angles, c.n_dih, c.n_imp, c.n_cmap};
    const int th = 256;
    A.blk0[0] = 0;
    for (int s = 0; s < 6; ++s) {
        long long lo = 0, hi = total[s];
        if (!whole) rank_slice(c, total[s], lo, hi);
        A.lo[s] = (int)lo;
        A.n[s] = (int)hi;
        A.blk0[s + 1] = A.blk0[s] + (int)((hi - lo + th - 1) / th);
    }
    A.gx = A.blk0[6];
    A.gy = 1;
    A.bond_atoms = c.bond_atoms.p; A.ub_atoms = c.ub_atoms.p; A.angle_atoms = c.angle_atoms.p;
    A.dih_atoms = c.dih_atoms.p; A.imp_atoms = c.imp_atoms.p; A.cmap_atoms = c.cmap_atoms.p;
    A.cmap_set = c.cmap_set.p;
    A.bond_par = c.bond_par.p; A.ub_par = c.ub_par.p; A.angle_par = c.angle_par.p; A.imp_par = c.imp_par.p;
    A.dih_par = c.dih_par.p; A.cmap_coeff = c.cmap_coeff.p; A.cmap_res = c.cmap_res;
    A.xyz = c.xyz.p;
    A.N = c.N;
    A.f = f;
    A.acc = acc;
    A.st = st;
    return A;
}

static void launch_bonded_args(const Ctx& c, const BondedArgs& A, bool energy)
{
    if (A.gx == 0) return;
    const int th = 256;
    if (c.p.semantics == MDF_SEM_PHYSICAL) {
        if (energy) k_bonded<true, true><<<grid_of(A), th, 0, c.stream>>>(A);
        else k_bonded<true, false><<<grid_of(A), th, 0, c.stream>>>(A);
    } else {
        if (energy) k_bonded<false, true><<<grid_of(A), th, 0, c.stream>>>(A);
        else k_bonded<false, false><<<grid_of(A), th, 0, c.stream>>>(A);
    }
    MDF_CUDA_TRY(cudaGetLastError());
}

void launch_bonded(Ctx& c, bool energy)
{
    const BondedArgs A = make_bonded_args(c, false, c.f_atom.p, c.acc.p, c.status.p);
    if (A.gx == 0) return;
    launch_bonded_args(c, A, energy);
    c.launches += 1;
}

void launch_bonded_into(Ctx& c, bool energy, unsigned long long* f, unsigned long long* acc, unsigned* st)
{
    launch_bonded_args(c, make_bonded_args(c, true, f, acc, st), energy);
}

void launch_bonded_multi(const BondedArgs* d_args, int nsys, int gx, bool energy, cudaStream_t s)
{
    if (gx == 0) return;
    if (energy) k_bonded_multi<true, true><<<dim3(gx, 1, nsys), 256, 0, s>>>(d_args);
    else k_bonded_multi<true, false><<<dim3(gx, 1, nsys), 256, 0, s>>>(d_args);
    MDF_CUDA_TRY(cudaGetLastError());
}

}  // namespace mdf
