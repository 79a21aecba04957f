// Host-side CMAP coefficient table for the C ABI (mdf_cmap_coefficients).
//
// The reference builds, for every grid cell, 16 coefficients c_ij of
// E(u, v) = sum_ij c_ij u^i v^j from the 4x4 neighbourhood of grid energies
// through a fixed 16x16 integer matrix divided by 16
// (src/AmberTopology/CreateNonBondedFromParsed.cpp:46-117).  That matrix
// defines the interpolant the reference evaluates (it is not a plain bicubic:
// several rows do not sum to zero, so a constant grid does not interpolate to
// a constant), so it is reproduced entry for entry.
#include <vector>

#include "../../include/mdf.h"

namespace {
const signed char kCmapMatrix[16][16] = {
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
}  // namespace

extern "C" int mdf_cmap_coefficients(int nsets, int res, const double* grids, double* coeff)
{
    if (nsets < 0 || res <= 0 || (nsets > 0 && (!grids || !coeff))) return MDF_ERR_INVALID;
    for (int s = 0; s < nsets; ++s) {
        const double* g = grids + (long long)s * res * res;
        for (int row = 0; row < res; ++row)
            for (int col = 0; col < res; ++col) {
                // neighbourhood ordered column offset outer, row offset inner,
                // each offset in -1..2 with periodic wrap
                double e16[16];
                int k = 0;
                for (int dc = -1; dc <= 2; ++dc)
                    for (int dr = -1; dr <= 2; ++dr) {
                        int r = (row + dr + res) % res, c = (col + dc + res) % res;
                        e16[k++] = g[r * res + c];
                    }
                double* out = coeff + (((long long)s * res + row) * res + col) * 16;
                for (int i = 0; i < 16; ++i) {
                    double acc = 0.0;
                    for (int j = 0; j < 16; ++j) acc += kCmapMatrix[i][j] * e16[j] / 16;
                    out[i] = acc;
                }
            }
    }
    return MDF_OK;
}

// PHYSICAL semantics: a C1 bicubic interpolant.  The reference's patches
// agree with the grid at the cell corners but not along the cell edges (the
// energy jumps by up to the grid's amplitude when phi or psi crosses a grid
// line), which no time integrator can conserve.  Here every cell is the
// bicubic Hermite patch of the corner values, the first derivatives of the
// periodic cubic splines through the grid rows and columns, and the cross
// derivative (the column spline's derivative of the row derivatives), all in
// grid-index units, so neighbouring patches share values and first
// derivatives along their common edge.  Same layout as the reference table:
// cell (row, col) starts at grid point (row, col), u along rows (phi), v along
// columns (psi), E = sum_ij c[i*4+j] u^i v^j.
namespace {

// Derivatives (per grid index) of the periodic cubic spline through f[0..n):
// d[i-1] + 4 d[i] + d[i+1] = 3 (f[i+1] - f[i-1]), solved as a dense cyclic
// system (n is a CMAP resolution, a few dozen).
void spline_derivative(int n, const double* f, int stride, double* d, int dstride)
{
    if (n < 3) {
        for (int i = 0; i < n; ++i) d[i * dstride] = 0.0;
        return;
    }
    std::vector<double> A((size_t)n * n, 0.0), b(n);
    for (int i = 0; i < n; ++i) {
        A[(size_t)i * n + i] = 4.0;
        A[(size_t)i * n + (i + n - 1) % n] += 1.0;
        A[(size_t)i * n + (i + 1) % n] += 1.0;
        b[i] = 3.0 * (f[((i + 1) % n) * stride] - f[((i + n - 1) % n) * stride]);
    }
    // Gaussian elimination; the matrix is strictly diagonally dominant
    for (int k = 0; k < n; ++k) {
        const double piv = A[(size_t)k * n + k];
        for (int i = k + 1; i < n; ++i) {
            const double m = A[(size_t)i * n + k] / piv;
            if (m == 0.0) continue;
            for (int j = k; j < n; ++j) A[(size_t)i * n + j] -= m * A[(size_t)k * n + j];
            b[i] -= m * b[k];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        double acc = b[i];
        for (int j = i + 1; j < n; ++j) acc -= A[(size_t)i * n + j] * b[j];
        b[i] = acc / A[(size_t)i * n + i];
    }
    for (int i = 0; i < n; ++i) d[i * dstride] = b[i];
}

// Hermite basis polynomials (coefficients of 1, t, t^2, t^3): value at 0,
// value at 1, slope at 0, slope at 1.
const double kH[4][4] = {{1, 0, -3, 2}, {0, 0, 3, -2}, {0, 1, -2, 1}, {0, 0, -1, 1}};

}  // namespace

extern "C" int mdf_cmap_coefficients_spline(int nsets, int res, const double* grids, double* coeff)
{
    if (nsets < 0 || res <= 0 || (nsets > 0 && (!grids || !coeff))) return MDF_ERR_INVALID;
    const int n = res;
    std::vector<double> fu((size_t)n * n), fv((size_t)n * n), fuv((size_t)n * n);
    for (int s = 0; s < nsets; ++s) {
        const double* g = grids + (long long)s * n * n;
        for (int c = 0; c < n; ++c) spline_derivative(n, g + c, n, fu.data() + c, n);      // d/du along rows
        for (int r = 0; r < n; ++r) spline_derivative(n, g + (size_t)r * n, 1, fv.data() + (size_t)r * n, 1);
        for (int r = 0; r < n; ++r)
            spline_derivative(n, fu.data() + (size_t)r * n, 1, fuv.data() + (size_t)r * n, 1);
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) {
                double* out = coeff + (((long long)s * n + r) * n + c) * 16;
                for (int k = 0; k < 16; ++k) out[k] = 0.0;
                for (int a = 0; a < 2; ++a)
                    for (int b = 0; b < 2; ++b) {
                        const size_t idx = (size_t)((r + a) % n) * n + (c + b) % n;
                        // value, d/du, d/dv, d2/dudv at corner (a, b)
                        const double data[4] = {g[idx], fu[idx], fv[idx], fuv[idx]};
                        const double* bu[2] = {kH[a], kH[2 + a]};   // value / slope basis in u
                        const double* bv[2] = {kH[b], kH[2 + b]};
                        for (int q = 0; q < 4; ++q) {
                            const double* pu = bu[q & 1];
                            const double* pv = bv[q >> 1];
                            const double w = data[q];
                            for (int i = 0; i < 4; ++i)
                                for (int j = 0; j < 4; ++j) out[i * 4 + j] += w * pu[i] * pv[j];
                        }
                    }
            }
    }
    return MDF_OK;
}

