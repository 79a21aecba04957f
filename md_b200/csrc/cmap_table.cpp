// Host-side CMAP coefficient table for the C ABI (mdf_cmap_coefficients).
//
// The reference builds, for every grid cell, 16 coefficients c_ij of
// E(u, v) = sum_ij c_ij u^i v^j from the 4x4 neighbourhood of grid energies
// through a fixed 16x16 integer matrix divided by 16
// (src/AmberTopology/CreateNonBondedFromParsed.cpp:46-117).  That matrix
// defines the interpolant the reference evaluates (it is not a plain bicubic:
// several rows do not sum to zero, so a constant grid does not interpolate to
// a constant), so it is reproduced entry for entry.
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
