// Cluster sort and cluster-pair list (replaces the reference's linked-list
// cell pairlist, src/System/NonBondedUtils.cpp:185-282).
//
// Atoms are binned into x-y columns whose cross-section holds about one
// cluster-height of atoms, sorted by z inside each column, and cut into
// clusters of 8.  Every i cluster then gets the list of j clusters (j >= i,
// half list) whose bounding boxes, in some periodic image, come within the
// list cutoff (cutoff + skin).  Each entry carries a 64-bit mask of the atom
// pairs that interact: padding slots, the lower triangle of the self pair and
// excluded pairs are cleared.
#include <algorithm>
#include <cmath>

#include "mdf_device.cuh"
#include "mdf_internal.cuh"

namespace mdf {

int grid_blocks(long long n, int threads)
{
    long long b = (n + threads - 1) / threads;
    return (int)std::max(1LL, b);
}

// ------------------------------------------------------------------ scan
// Single-block exclusive scan; n up to a few million.
__global__ void k_scan_1block(const int* __restrict__ in, int* __restrict__ out, int n, int* total)
{
    __shared__ int part[1024];
    int tid = threadIdx.x;
    int per = (n + blockDim.x - 1) / blockDim.x;
    int b0 = tid * per, b1 = min(n, b0 + per);
    int s = 0;
    for (int i = b0; i < b1; ++i) s += in[i];
    part[tid] = s;
    __syncthreads();
    // Hillis-Steele inclusive scan over the block partials
    for (int o = 1; o < blockDim.x; o <<= 1) {
        int v = tid >= o ? part[tid - o] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    int run = tid ? part[tid - 1] : 0;
    for (int i = b0; i < b1; ++i) {
        int v = in[i];
        out[i] = run;
        run += v;
    }
    if (tid == blockDim.x - 1 && total) *total = part[tid];
}

void exclusive_scan_int(const int* d_in, int* d_out, int n, int* d_total_out, cudaStream_t s)
{
    k_scan_1block<<<1, 1024, 0, s>>>(d_in, d_out, n, d_total_out);
    MDF_CUDA_TRY(cudaGetLastError());
}

// ------------------------------------------------------------- binning
__global__ void k_assign_columns(int N, const double* __restrict__ xyz, double Lx, double Ly, int ncx, int ncy,
                                 int* __restrict__ atom_col, int* __restrict__ col_count, unsigned* st)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    if (!isfinite(x) || !isfinite(y) || !isfinite(z)) {
        status_set(st, ST_NONFINITE);
        x = y = 0.0;
    }
    x = wrap_coord(x, Lx);
    y = wrap_coord(y, Ly);
    int cx = (int)(x * ncx / Lx), cy = (int)(y * ncy / Ly);
    cx = min(max(cx, 0), ncx - 1);
    cy = min(max(cy, 0), ncy - 1);
    int col = cx + ncx * cy;
    atom_col[i] = col;
    atomicAdd(&col_count[col], 1);
}

__global__ void k_clusters_per_column(int ncols, const int* __restrict__ cnt, int* __restrict__ ncl)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < ncols) ncl[c] = (cnt[c] + CLUSTER - 1) / CLUSTER;
}

__global__ void k_bucket(int N, const int* __restrict__ atom_col, const int* __restrict__ col_start,
                         int* __restrict__ col_fill, int* __restrict__ col_atoms)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int col = atom_col[i];
    int pos = col_start[col] + atomicAdd(&col_fill[col], 1);
    col_atoms[pos] = i;
}

constexpr int COL_MAX = 2048;   // atoms per column handled by the in-block sort

// One block (1024 threads) per column: bitonic sort of (z, atom) keys, then
// cut into clusters of 8.
__global__ void __launch_bounds__(1024) k_sort_columns(const double* __restrict__ xyz, double Lz,
                                                       const int* __restrict__ col_count,
                                                       const int* __restrict__ col_start,
                                                       const int* __restrict__ col_cstart,
                                                       const int* __restrict__ col_atoms,
                                                       int* __restrict__ slot_atom, int* __restrict__ atom_slot,
                                                       int* __restrict__ cluster_col, unsigned* st)
{
    __shared__ unsigned long long key[COL_MAX];
    int col = blockIdx.x, tid = threadIdx.x;
    int n = col_count[col];
    if (n > COL_MAX) {
        if (tid == 0) status_set(st, ST_CAPACITY_COLUMN);
        return;
    }
    int s0 = col_start[col];
    // pad to the next power of two >= n (at least 2)
    int m = 2;
    while (m < n) m <<= 1;
    for (int k = tid; k < m; k += blockDim.x) {
        unsigned long long kk = ~0ull;
        if (k < n) {
            int a = col_atoms[s0 + k];
            double zw = wrap_coord(xyz[3 * a + 2], Lz);
            float zf = (float)zw;
            if (!(zf >= 0.0f)) zf = 0.0f;
            kk = ((unsigned long long)__float_as_uint(zf) << 32) | (unsigned)a;
        }
        key[k] = kk;
    }
    for (int size = 2; size <= m; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            __syncthreads();
            for (int t = tid; t < (m >> 1); t += blockDim.x) {
                int i = 2 * t - (t & (stride - 1));
                int j = i + stride;
                bool asc = (i & size) == 0;
                unsigned long long a = key[i], b = key[j];
                if ((a > b) == asc) {
                    key[i] = b;
                    key[j] = a;
                }
            }
        }
    }
    __syncthreads();
    int c0 = col_cstart[col];
    int ncl = (n + CLUSTER - 1) / CLUSTER;
    for (int k = tid; k < ncl * CLUSTER; k += blockDim.x) {
        int cl = c0 + k / CLUSTER;
        int slot = cl * CLUSTER + (k % CLUSTER);
        if (k < n) {
            int a = (int)(key[k] & 0xffffffffu);
            slot_atom[slot] = a;
            atom_slot[a] = slot;
        } else {
            slot_atom[slot] = -1;
        }
        if ((k % CLUSTER) == 0) cluster_col[cl] = col;
    }
}

// Cluster bounding boxes (wrapped coordinates) and centres; center.w = number
// of real atoms in the cluster.
__global__ void k_cluster_geom(int ncl, const double* __restrict__ xyz, double Lx, double Ly, double Lz,
                               double quantum, const int* __restrict__ slot_atom, double4* __restrict__ center,
                               float4* __restrict__ centerf, float4* __restrict__ bb_lo, float4* __restrict__ bb_hi)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncl) return;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    int nv = 0;
    for (int k = 0; k < CLUSTER; ++k) {
        int a = slot_atom[c * CLUSTER + k];
        if (a < 0) continue;
        ++nv;
        double p[3] = {wrap_coord(xyz[3 * a], Lx), wrap_coord(xyz[3 * a + 1], Ly), wrap_coord(xyz[3 * a + 2], Lz)};
        for (int d = 0; d < 3; ++d) {
            lo[d] = fmin(lo[d], p[d]);
            hi[d] = fmax(hi[d], p[d]);
        }
    }
    if (nv == 0) {
        for (int d = 0; d < 3; ++d) lo[d] = hi[d] = 0.0;
    }
    // centres on a 2^-k grid fine enough that they are exact in FP32, so the
    // FP32 pair kernel forms centre differences without rounding
    double cc[3];
    for (int d = 0; d < 3; ++d) cc[d] = rint(0.5 * (lo[d] + hi[d]) / quantum) * quantum;
    center[c] = make_double4(cc[0], cc[1], cc[2], (double)nv);
    centerf[c] = make_float4((float)cc[0], (float)cc[1], (float)cc[2], (float)nv);
    bb_lo[c] = make_float4(__double2float_rd(lo[0]), __double2float_rd(lo[1]), __double2float_rd(lo[2]), 0.f);
    bb_hi[c] = make_float4(__double2float_ru(hi[0]), __double2float_ru(hi[1]), __double2float_ru(hi[2]), 0.f);
}

// Per-evaluation packing: cluster-ordered offsets from the cluster centre
// (min image, so atoms crossing the box edge between rebuilds stay whole)
// plus charge, in the working precision.
// Also the cluster's current bounding box in its own frame (FP32, rounded
// outward) for the prune's box test.  blockDim.x must be a multiple of 32.
template <typename R>
__global__ void k_pack(int nslots, const double* __restrict__ xyz, const double* __restrict__ q,
                       const int* __restrict__ slot_atom, const double4* __restrict__ center, double Lx, double Ly,
                       double Lz, typename V4<R>::type* __restrict__ xq, float4* __restrict__ cur_lo,
                       float4* __restrict__ cur_hi, unsigned* st)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool inside = s < nslots;
    const int a = inside ? slot_atom[s] : -1;
    typename V4<R>::type v;
    float lo[3] = {3.0e38f, 3.0e38f, 3.0e38f}, hi[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
    if (a < 0) {
        v.x = v.y = v.z = v.w = (R)0;
    } else {
        double4 c = center[s / CLUSTER];
        double d[3] = {min_image(xyz[3 * a] - c.x, Lx), min_image(xyz[3 * a + 1] - c.y, Ly),
                       min_image(xyz[3 * a + 2] - c.z, Lz)};
        if (!isfinite(d[0] + d[1] + d[2])) status_set(st, ST_NONFINITE);
        v.x = (R)d[0];
        v.y = (R)d[1];
        v.z = (R)d[2];
        v.w = (R)q[a];
        for (int k = 0; k < 3; ++k) {
            lo[k] = __double2float_rd(d[k]);
            hi[k] = __double2float_ru(d[k]);
        }
    }
    if (inside) xq[s] = v;
    // min/max over the 8 slots of the cluster (8 consecutive lanes)
#pragma unroll
    for (int o = 1; o < CLUSTER; o <<= 1)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
    if (inside && (s % CLUSTER) == 0) {
        cur_lo[s / CLUSTER] = make_float4(lo[0], lo[1], lo[2], 0.f);
        cur_hi[s / CLUSTER] = make_float4(hi[0], hi[1], hi[2], 0.f);
    }
}

__global__ void k_slot_type(int nslots, const int* __restrict__ slot_atom, const int* __restrict__ type, int pad_type,
                            int* __restrict__ slot_type)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    int a = slot_atom[s];
    slot_type[s] = a < 0 ? pad_type : type[a];
}

// -------------------------------------------------------- pair search
struct SearchGeom {
    double L[3];
    double colw[3];
    int ncx, ncy;
    int Rx, Ry;
    float rlist2;
    float rlist;
};

__device__ __forceinline__ unsigned long long entry_mask(int nvi, int nvj, bool self_pair)
{
    unsigned long long row = (nvj >= 8) ? 0xffull : ((1ull << nvj) - 1ull);
    unsigned long long m = 0;
    for (int ii = 0; ii < nvi; ++ii) {
        unsigned long long r = row;
        if (self_pair) r &= ~((2ull << ii) - 1ull);   // keep jj > ii
        m |= r << (8 * ii);
    }
    return m;
}

// One warp per i cluster.  FILL=false: count entries into icount[i];
// FILL=true: write them at ilist[i].start (deterministic lane-major order).
template <bool FILL>
__global__ void __launch_bounds__(256) k_pair_search(int ncl, SearchGeom g, const int* __restrict__ cluster_col,
                                                     const int* __restrict__ col_cstart,
                                                     const float4* __restrict__ bb_lo, const float4* __restrict__ bb_hi,
                                                     const double4* __restrict__ center, int* __restrict__ icount,
                                                     const int* __restrict__ istart, PairEntry* __restrict__ out,
                                                     long long cap, ILRange* __restrict__ ilist, unsigned* st)
{
    int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (I >= ncl) return;
    int col = cluster_col[I];
    int cx = col % g.ncx, cy = col / g.ncx;
    float4 lo = bb_lo[I], hi = bb_hi[I];
    int nvi = (int)center[I].w;
    int nxc = 2 * g.Rx + 1, nyc = 2 * g.Ry + 1;
    int ncombo = nxc * nyc * 3;
    float Lx = (float)g.L[0], Ly = (float)g.L[1], Lz = (float)g.L[2];
    int cnt = 0;
    long long base = 0;
    // FILL runs two sweeps: count this lane's entries, then write them after
    // the lane-exclusive prefix
    for (int sweep = FILL ? 0 : 1; sweep < 2; ++sweep) {
        if (FILL && sweep == 1) {
            // lane-exclusive prefix
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            base = (long long)istart[I] + (incl - cnt);
            if (lane == 31) {
                ILRange r;
                r.i = I;
                r.start = istart[I];
                r.count = incl;
                r.pad = 0;
                ilist[I] = r;
            }
            cnt = 0;
        }
        for (int combo = lane; combo < ncombo; combo += 32) {
            int szi = combo % 3;
            int rest = combo / 3;
            int dcx = rest % nxc - g.Rx;
            int dcy = rest / nxc - g.Ry;
            int jx = cx + dcx, jy = cy + dcy;
            int sx = jx < 0 ? -1 : (jx >= g.ncx ? 1 : 0);
            int sy = jy < 0 ? -1 : (jy >= g.ncy ? 1 : 0);
            jx -= sx * g.ncx;
            jy -= sy * g.ncy;
            int sz = szi - 1;
            float cxl = (float)(jx * g.colw[0] + sx * g.L[0]), cxh = (float)((jx + 1) * g.colw[0] + sx * g.L[0]);
            float cyl = (float)(jy * g.colw[1] + sy * g.L[1]), cyh = (float)((jy + 1) * g.colw[1] + sy * g.L[1]);
            float gx = fmaxf(0.f, fmaxf(cxl - hi.x, lo.x - cxh));
            float gy = fmaxf(0.f, fmaxf(cyl - hi.y, lo.y - cyh));
            if (gx * gx + gy * gy > g.rlist2) continue;
            float zmin = lo.z - g.rlist - sz * Lz, zmax = hi.z + g.rlist - sz * Lz;
            if (zmax < -1.0f || zmin > Lz + 1.0f) continue;
            int jcol = jx + g.ncx * jy;
            int c0 = col_cstart[jcol], c1 = col_cstart[jcol + 1];
            // first cluster whose hi.z >= zmin
            int a = c0, b = c1;
            while (a < b) {
                int mid = (a + b) >> 1;
                if (bb_hi[mid].z < zmin) a = mid + 1;
                else b = mid;
            }
            for (int J = a; J < c1; ++J) {
                float4 jl = bb_lo[J], jh = bb_hi[J];
                if (jl.z > zmax) break;
                float ox = sx * Lx, oy = sy * Ly, oz = sz * Lz;
                float dx = fmaxf(0.f, fmaxf(jl.x + ox - hi.x, lo.x - (jh.x + ox)));
                float dy = fmaxf(0.f, fmaxf(jl.y + oy - hi.y, lo.y - (jh.y + oy)));
                float dz = fmaxf(0.f, fmaxf(jl.z + oz - hi.z, lo.z - (jh.z + oz)));
                if (dx * dx + dy * dy + dz * dz > g.rlist2) continue;
                int code = (sx + 1) + 3 * (sy + 1) + 9 * (sz + 1);
                if (J < I || (J == I && code < 13)) continue;
                if (FILL && sweep == 1) {
                    long long pos = base + cnt;
                    if (pos < cap) {
                        PairEntry e;
                        e.j = J;
                        e.shift = code;
                        e.mask = entry_mask(nvi, (int)center[J].w, J == I && code == 13);
                        out[pos] = e;
                    } else {
                        status_set(st, ST_CAPACITY_PAIRS);
                    }
                }
                ++cnt;
            }
        }
    }
    if (!FILL) {
        int tot = cnt;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
        if (lane == 0) icount[I] = tot;
    }
}

// Clear the mask bit of every excluded pair in the entry that holds it.
__global__ void k_exclusion_masks(int nexcl, const int* __restrict__ excl, const int* __restrict__ atom_slot,
                                  const double* __restrict__ xyz, const double4* __restrict__ center, double Lx,
                                  double Ly, double Lz, const ILRange* __restrict__ ilist,
                                  PairEntry* __restrict__ plist)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nexcl) return;
    int a = excl[2 * k], b = excl[2 * k + 1];
    int sa = atom_slot[a], sb = atom_slot[b];
    int Ia = sa / CLUSTER, la = sa % CLUSTER, Ib = sb / CLUSTER, lb = sb % CLUSTER;
    double4 ca = center[Ia], cb = center[Ib];
    // list-geometry positions: centre + min-image offset
    double pa[3] = {ca.x + min_image(xyz[3 * a] - ca.x, Lx), ca.y + min_image(xyz[3 * a + 1] - ca.y, Ly),
                    ca.z + min_image(xyz[3 * a + 2] - ca.z, Lz)};
    double pb[3] = {cb.x + min_image(xyz[3 * b] - cb.x, Lx), cb.y + min_image(xyz[3 * b + 1] - cb.y, Ly),
                    cb.z + min_image(xyz[3 * b + 2] - cb.z, Lz)};
    // J atoms sit at p + s L in I's frame: s = round((p_I - p_J) / L)
    int s[3] = {(int)round((pa[0] - pb[0]) / Lx), (int)round((pa[1] - pb[1]) / Ly), (int)round((pa[2] - pb[2]) / Lz)};
    if (s[0] < -1 || s[0] > 1 || s[1] < -1 || s[1] > 1 || s[2] < -1 || s[2] > 1) return;  // never listed
    int I, J, bit;
    int code = (s[0] + 1) + 3 * (s[1] + 1) + 9 * (s[2] + 1);
    if (Ia < Ib) {
        I = Ia; J = Ib; bit = la * 8 + lb;
    } else if (Ia > Ib) {
        I = Ib; J = Ia; bit = lb * 8 + la; code = 26 - code;
    } else {
        I = J = Ia;
        if (code == 13) bit = min(la, lb) * 8 + max(la, lb);
        else if (code > 13) bit = la * 8 + lb;
        else { bit = lb * 8 + la; code = 26 - code; }
    }
    ILRange r = ilist[I];
    for (int e = r.start; e < r.start + r.count; ++e) {
        if (plist[e].j == J && plist[e].shift == code) {
            atomicAnd(&plist[e].mask, ~(1ull << bit));
            break;
        }
    }
}

// ------------------------------------------------------------- pruning
// Two levels, one lane per outer entry.  Level 1 rejects the entry when the
// current bounding boxes of the two clusters (k_pack) are rcut apart.  Level 2
// loads the entry's eight j atoms (independent loads, all in flight at once),
// skips every j atom farther than rcut from the i cluster's box, and tests the
// rest against the eight i atoms (held in registers by every lane), stopping
// at the first unmasked pair inside rcut.  Kept entries are compacted, in
// list order, into the same offsets of the pruned list.  Image offsets use the
// exact-FP32 centres plus the hi/lo shift table.
struct PruneShifts {
    float v[27][6];
};

// Dynamic pruning: keep the outer-list entries that have at least one atom
// pair within the prune radius at the current positions.  Warp per i cluster.
// The warp loads 32 entries at once (one per lane), drops those whose current
// cluster boxes are farther apart than the radius, and checks the remaining
// candidates four at a time with lane = (candidate, j atom): each lane tests
// its j atom against the eight i atoms held in registers, and one ballot gives
// the four keep flags.  The test ignores the entry's exclusion mask (an entry
// whose only close pairs are excluded is kept; the pair kernel applies the
// mask), so it keeps a superset of the exact set.  Distances use
// |a - b|^2 = |a|^2 + |b|^2 - 2 a.b: three FMAs and a min per pair, the
// rounding (~1e-4 A^2 at these magnitudes) far inside the radius' margin.
// Kept entries are written in order, packed from the i cluster's start offset
// in the outer list.
template <typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 3) k_prune(
    int ncl, const ILRange* __restrict__ ilist, const PairEntry* __restrict__ plist,
    const typename V4<R>::type* __restrict__ xq, const float4* __restrict__ centerf,
    const float4* __restrict__ cur_lo, const float4* __restrict__ cur_hi, PruneShifts shifts, float rcut2,
    ILRange* __restrict__ ilist_in, PairEntry* __restrict__ plist_in, unsigned long long* __restrict__ n_in)
{
    using V4t = typename V4<R>::type;
    __shared__ float sh[27][6];
    for (int k = threadIdx.x; k < 27 * 6; k += blockDim.x) sh[k / 6][k % 6] = shifts.v[k / 6][k % 6];
    __syncthreads();
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;   // index into this launch's ilist range
    const int lane = threadIdx.x & 31;
    if (w >= ncl) return;
    const unsigned below = (1u << lane) - 1u;
    const ILRange L = ilist[w];
    const int I = L.i;
    R ax[CLUSTER], ay[CLUSTER], az[CLUSTER], an[CLUSTER];   // -2 x_i and |x_i|^2
#pragma unroll
    for (int k = 0; k < CLUSTER; ++k) {
        const V4t v = xq[I * CLUSTER + k];
        ax[k] = (R)-2 * v.x; ay[k] = (R)-2 * v.y; az[k] = (R)-2 * v.z;
        an[k] = v.x * v.x + v.y * v.y + v.z * v.z;
    }
    const float4 cI = centerf[I], ilo = cur_lo[I], ihi = cur_hi[I];
    const R rc2 = (R)rcut2;
    int kept = 0;
    for (int base = 0; base < L.count; base += 32) {
        const bool have = base + lane < L.count;
        PairEntry my;
        my.j = I; my.shift = 13; my.mask = 0ull;
        if (have) my = plist[L.start + base + lane];
        // this lane's entry: J's frame origin seen from I's frame, and the box test
        const float4 cJ = centerf[my.j], jlo = cur_lo[my.j], jhi = cur_hi[my.j];
        const float* s6 = sh[my.shift];
        const float ox = -(((cI.x - cJ.x) - s6[0]) - s6[3]);
        const float oy = -(((cI.y - cJ.y) - s6[1]) - s6[4]);
        const float oz = -(((cI.z - cJ.z) - s6[2]) - s6[5]);
        const float gx = fmaxf(0.f, fmaxf(jlo.x + ox - ihi.x, ilo.x - (jhi.x + ox)));
        const float gy = fmaxf(0.f, fmaxf(jlo.y + oy - ihi.y, ilo.y - (jhi.y + oy)));
        const float gz = fmaxf(0.f, fmaxf(jlo.z + oz - ihi.z, ilo.z - (jhi.z + oz)));
        const bool cand = have && my.mask != 0ull && gx * gx + gy * gy + gz * gz < rcut2;
        unsigned keepmask;
        if constexpr (sizeof(R) == 4) {
            // FP32: this lane's entry against all 64 atom pairs, two j atoms at
            // a time (loads issued together), until one pair is in range
            bool keep = false;
            if (cand) {
                const R px = (R)ox, py = (R)oy, pz = (R)oz;
                const V4t* __restrict__ xj = xq + (size_t)my.j * CLUSTER;
#pragma unroll 1
                for (int j = 0; j < CLUSTER && !keep; j += 2) {
                    V4t v[2];
                    v[0] = xj[j];
                    v[1] = xj[j + 1];
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        const R qx = v[u].x + px, qy = v[u].y + py, qz = v[u].z + pz;
                        const R thr = rc2 - (qx * qx + qy * qy + qz * qz);
                        R m = fma(ax[0], qx, fma(ay[0], qy, fma(az[0], qz, an[0])));
#pragma unroll
                        for (int ii = 1; ii < CLUSTER; ++ii)
                            m = fmin(m, fma(ax[ii], qx, fma(ay[ii], qy, fma(az[ii], qz, an[ii]))));
                        keep = keep || m < thr;
                    }
                }
            }
            keepmask = __ballot_sync(0xffffffffu, keep);
        } else {
            // FP64 (half-rate arithmetic: idle lanes cost more than bookkeeping):
            // the pending candidates four at a time, eight lanes (one j atom
            // each) per candidate
            const int slot = lane >> 3, jj = lane & 7;
            unsigned todo = __ballot_sync(0xffffffffu, cand);
            unsigned mine = 0u;
            while (todo) {
                // this lane's candidate: the (slot+1)-th lowest pending entry
                unsigned x = todo;
                if (slot >= 1) x &= x - 1u;
                if (slot >= 2) x &= x - 1u;
                if (slot >= 3) x &= x - 1u;
                const bool valid = x != 0u;
                const int sl = valid ? __ffs(x) - 1 : 0;
                const int j = __shfl_sync(0xffffffffu, my.j, sl);
                const R px = (R)__shfl_sync(0xffffffffu, ox, sl), py = (R)__shfl_sync(0xffffffffu, oy, sl),
                        pz = (R)__shfl_sync(0xffffffffu, oz, sl);
                const V4t vj = xq[j * CLUSTER + jj];
                const R qx = vj.x + px, qy = vj.y + py, qz = vj.z + pz;
                const R thr = rc2 - (qx * qx + qy * qy + qz * qz);
                R m = fma(ax[0], qx, fma(ay[0], qy, fma(az[0], qz, an[0])));
#pragma unroll
                for (int ii = 1; ii < CLUSTER; ++ii)
                    m = fmin(m, fma(ax[ii], qx, fma(ay[ii], qy, fma(az[ii], qz, an[ii]))));
                const unsigned bal = __ballot_sync(0xffffffffu, valid && m < thr);
                // lane L's own entry, if pending and among the four: its rank is its slot
                const unsigned rank = __popc(todo & below);
                if (((todo >> lane) & 1u) && rank < 4u && ((bal >> (8u * rank)) & 0xffu)) mine = 1u;
                todo &= todo - 1u;
                todo &= todo - 1u;
                todo &= todo - 1u;
                todo &= todo - 1u;
            }
            keepmask = __ballot_sync(0xffffffffu, mine != 0u);
        }
        if ((keepmask >> lane) & 1u) plist_in[L.start + kept + __popc(keepmask & below)] = my;
        kept += __popc(keepmask);
    }
    if (lane == 0) {
        ILRange r;
        r.i = I; r.start = L.start; r.count = kept; r.pad = 0;
        ilist_in[w] = r;
        if (kept) atomicAdd(n_in, (unsigned long long)kept);
    }
}

void prune_pairlist(Ctx& c)
{
    const int th = 256;
    // a hair above the cutoff so working-precision rounding never drops a pair at r ~ rc
    double rc = c.p.cutoff + std::max(0.0, c.p.prune_margin) + 0.02;
    PruneShifts sh;
    for (int code = 0; code < 27; ++code) {
        int sv[3] = {code % 3 - 1, (code / 3) % 3 - 1, code / 9 - 1};
        for (int d = 0; d < 3; ++d) {
            double v = sv[d] * c.box[d];
            float hi = (float)v;
            sh.v[code][d] = hi;
            sh.v[code][3 + d] = (float)(v - (double)hi);
        }
    }
    MDF_CUDA_TRY(cudaMemsetAsync(c.n_in.p, 0, sizeof(unsigned long long), c.stream));
    long long lo, hi;
    rank_slice(c, c.n_clusters, lo, hi);   // this rank's i clusters
    const int ncl = (int)(hi - lo);
    int blocks = grid_blocks((long long)ncl * 32, th);
    if (ncl > 0) {
        if (c.p.precision == MDF_PREC_MIXED)
            k_prune<float><<<blocks, th, 0, c.stream>>>(ncl, c.ilist.p + lo, c.plist.p, c.xq_f.p, c.centerf.p,
                                                       c.cur_lo.p, c.cur_hi.p, sh, (float)(rc * rc),
                                                       c.ilist_in.p + lo, c.plist_in.p, c.n_in.p);
        else
            k_prune<double><<<blocks, th, 0, c.stream>>>(ncl, c.ilist.p + lo, c.plist.p, c.xq_d.p, c.centerf.p,
                                                        c.cur_lo.p, c.cur_hi.p, sh, (float)(rc * rc),
                                                        c.ilist_in.p + lo, c.plist_in.p, c.n_in.p);
    }
    MDF_CUDA_TRY(cudaGetLastError());
    c.launches += 1;
    c.pruned_valid = true;
}

// ------------------------------------------------------------------ host
static double atom_density(const Ctx& c)
{
    return (double)c.N / (c.box[0] * c.box[1] * c.box[2]);
}

void pack_positions(Ctx& c)
{
    int th = 256;
    if (c.p.precision == MDF_PREC_MIXED) {
        k_pack<float><<<grid_blocks(c.n_slots, th), th, 0, c.stream>>>(c.n_slots, c.xyz.p, c.q.p, c.slot_atom.p,
                                                                         c.center.p, c.box[0], c.box[1], c.box[2],
                                                                         c.xq_f.p, c.cur_lo.p, c.cur_hi.p, c.status.p);
    } else {
        k_pack<double><<<grid_blocks(c.n_slots, th), th, 0, c.stream>>>(c.n_slots, c.xyz.p, c.q.p, c.slot_atom.p,
                                                                          c.center.p, c.box[0], c.box[1], c.box[2],
                                                                          c.xq_d.p, c.cur_lo.p, c.cur_hi.p,
                                                                          c.status.p);
    }
    MDF_CUDA_TRY(cudaGetLastError());
    c.launches += 1;
}

void build_pairlist(Ctx& c)
{
    c.npairs_dev.alloc(1);
    c.count_next = true;
    c.counted = false;
    cudaStream_t s = c.stream;
    const int th = 256;
    double rlist = c.p.cutoff + c.p.skin;
    for (int d = 0; d < 3; ++d)
        if (!(c.box[d] >= 2.0 * c.p.cutoff))
            throw ApiError(MDF_ERR_INVALID, "box edge shorter than twice the cutoff (minimum image undefined)");
    // column cross-section ~ one cluster of atoms per column-height cube
    double rho = atom_density(c);
    double side = std::cbrt((double)CLUSTER / std::max(rho, 1e-6));
    for (int attempt = 0; attempt < 6; ++attempt) {
        c.ncol_x = std::max(1, (int)std::floor(c.box[0] / side));
        c.ncol_y = std::max(1, (int)std::floor(c.box[1] / side));
        // The one-image search visits the +-R columns around a column (R =
        // floor(rlist / width) + 1), which must be distinct: R < columns.
        // Sparse systems start from wide columns; add columns until it holds.
        auto reach = [&](double L, int nc) { return (int)std::floor(rlist / (L / nc)) + 1; };
        while (reach(c.box[0], c.ncol_x) >= c.ncol_x && c.ncol_x < 4096) ++c.ncol_x;
        while (reach(c.box[1], c.ncol_y) >= c.ncol_y && c.ncol_y < 4096) ++c.ncol_y;
        const int Rx = reach(c.box[0], c.ncol_x), Ry = reach(c.box[1], c.ncol_y);
        if (Rx >= c.ncol_x || Ry >= c.ncol_y) throw ApiError(MDF_ERR_INVALID, "box too small for the list cutoff");
        c.ncols = c.ncol_x * c.ncol_y;
        c.col_count.alloc(c.ncols + 1);
        c.col_start.alloc(c.ncols + 1);
        c.col_cstart.alloc(c.ncols + 1);
        c.scan_tmp.alloc(c.ncols + 1);
        c.atom_col.alloc(c.N);
        c.col_atoms.alloc(c.N);
        c.atom_slot.alloc(c.N);
        MDF_CUDA_TRY(cudaMemsetAsync(c.col_count.p, 0, sizeof(int) * (c.ncols + 1), s));
        MDF_CUDA_TRY(cudaMemsetAsync(c.status.p, 0, sizeof(unsigned), s));
        k_assign_columns<<<grid_blocks(c.N, th), th, 0, s>>>(c.N, c.xyz.p, c.box[0], c.box[1], c.ncol_x, c.ncol_y,
                                                             c.atom_col.p, c.col_count.p, c.status.p);
        exclusive_scan_int(c.col_count.p, c.col_start.p, c.ncols + 1, nullptr, s);
        k_clusters_per_column<<<grid_blocks(c.ncols + 1, th), th, 0, s>>>(c.ncols + 1, c.col_count.p, c.scan_tmp.p);
        exclusive_scan_int(c.scan_tmp.p, c.col_cstart.p, c.ncols + 1, nullptr, s);
        int ncl = 0;
        MDF_CUDA_TRY(cudaMemcpyAsync(&ncl, c.col_cstart.p + c.ncols, sizeof(int), cudaMemcpyDeviceToHost, s));
        MDF_CUDA_TRY(cudaMemsetAsync(c.scan_tmp.p, 0, sizeof(int) * (c.ncols + 1), s));
        k_bucket<<<grid_blocks(c.N, th), th, 0, s>>>(c.N, c.atom_col.p, c.col_start.p, c.scan_tmp.p, c.col_atoms.p);
        MDF_CUDA_TRY(cudaStreamSynchronize(s));
        c.n_clusters = ncl;
        c.n_slots = ncl * CLUSTER;
        c.slot_atom.alloc(c.n_slots);
        c.cluster_col.alloc(ncl);
        k_sort_columns<<<c.ncols, 1024, 0, s>>>(c.xyz.p, c.box[2], c.col_count.p, c.col_start.p, c.col_cstart.p,
                                                c.col_atoms.p, c.slot_atom.p, c.atom_slot.p, c.cluster_col.p,
                                                c.status.p);
        unsigned st = 0;
        MDF_CUDA_TRY(cudaMemcpyAsync(&st, c.status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        MDF_CUDA_TRY(cudaStreamSynchronize(s));
        if (st & ST_NONFINITE) throw ApiError(MDF_ERR_NONFINITE, "non-finite position");
        if (st & ST_CAPACITY_COLUMN) {
            side *= 0.7;   // too many atoms in a column: thinner columns
            if (attempt == 5) throw ApiError(MDF_ERR_CAPACITY, "column too populated for the in-block sort");
            continue;
        }
        // geometry
        c.center.alloc(ncl);
        c.bb_lo.alloc(ncl);
        c.bb_hi.alloc(ncl);
        c.cur_lo.alloc(ncl);
        c.cur_hi.alloc(ncl);
        c.centerf.alloc(ncl);
        {
            // largest power-of-two quantum keeping every centre exact in FP32 (24-bit significand)
            double lmax = std::max(c.box[0], std::max(c.box[1], c.box[2]));
            c.center_quantum = std::ldexp(1.0, (int)std::ceil(std::log2(lmax + 1.0)) - 24);
        }
        k_cluster_geom<<<grid_blocks(ncl, th), th, 0, s>>>(ncl, c.xyz.p, c.box[0], c.box[1], c.box[2],
                                                           c.center_quantum, c.slot_atom.p, c.center.p, c.centerf.p,
                                                           c.bb_lo.p, c.bb_hi.p);
        c.slot_type.alloc(c.n_slots);
        k_slot_type<<<grid_blocks(c.n_slots, th), th, 0, s>>>(c.n_slots, c.slot_atom.p, c.type.p, c.ntp - 1,
                                                              c.slot_type.p);
        if (c.p.precision == MDF_PREC_MIXED) c.xq_f.alloc(c.n_slots);
        else c.xq_d.alloc(c.n_slots);
        MDF_CUDA_TRY(cudaGetLastError());

        SearchGeom g;
        for (int d = 0; d < 3; ++d) g.L[d] = c.box[d];
        g.colw[0] = c.box[0] / c.ncol_x;
        g.colw[1] = c.box[1] / c.ncol_y;
        g.colw[2] = c.box[2];
        g.ncx = c.ncol_x;
        g.ncy = c.ncol_y;
        g.Rx = Rx;
        g.Ry = Ry;
        // bounding boxes are rounded outward to float; pad the list radius a hair
        g.rlist = (float)(rlist * (1.0 + 1e-6));
        g.rlist2 = g.rlist * g.rlist;
        c.icount.alloc(ncl + 1);
        c.ilist.alloc(ncl);
        MDF_CUDA_TRY(cudaMemsetAsync(c.icount.p, 0, sizeof(int) * (ncl + 1), s));
        int wblocks = grid_blocks((long long)ncl * 32, th);
        k_pair_search<false><<<wblocks, th, 0, s>>>(ncl, g, c.cluster_col.p, c.col_cstart.p, c.bb_lo.p, c.bb_hi.p,
                                                    c.center.p, c.icount.p, nullptr, nullptr, 0, nullptr, c.status.p);
        c.scan_tmp.alloc(ncl + 1);
        exclusive_scan_int(c.icount.p, c.scan_tmp.p, ncl + 1, nullptr, s);
        int total = 0;
        MDF_CUDA_TRY(cudaMemcpyAsync(&total, c.scan_tmp.p + ncl, sizeof(int), cudaMemcpyDeviceToHost, s));
        MDF_CUDA_TRY(cudaStreamSynchronize(s));
        c.n_entries = total;
        c.plist.alloc((size_t)total + 1);
        k_pair_search<true><<<wblocks, th, 0, s>>>(ncl, g, c.cluster_col.p, c.col_cstart.p, c.bb_lo.p, c.bb_hi.p,
                                                   c.center.p, nullptr, c.scan_tmp.p, c.plist.p, total, c.ilist.p,
                                                   c.status.p);
        if (c.n_excl > 0)
            k_exclusion_masks<<<grid_blocks(c.n_excl, th), th, 0, s>>>(c.n_excl, c.excl_pairs.p, c.atom_slot.p,
                                                                      c.xyz.p, c.center.p, c.box[0], c.box[1],
                                                                      c.box[2], c.ilist.p, c.plist.p);
        MDF_CUDA_TRY(cudaGetLastError());
        MDF_CUDA_TRY(cudaMemcpyAsync(&st, c.status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        MDF_CUDA_TRY(cudaStreamSynchronize(s));
        if (st & ST_CAPACITY_PAIRS) throw ApiError(MDF_ERR_CAPACITY, "pair list capacity exceeded");
        c.f_slot.alloc((size_t)3 * c.n_slots);
        c.need_clear = true;   // slot layout changed: clear the accumulators before the next evaluation
        c.plist_in.alloc((size_t)total + 1);
        c.ilist_in.alloc(ncl);
        c.n_in.alloc(1);
        c.pruned_valid = false;
        c.since_prune = 0;
        c.have_list = true;
        return;
    }
}

}  // namespace mdf
