// Cluster sort and cluster-pair list (replaces the reference's linked-list
// cell pairlist, src/System/NonBondedUtils.cpp:185-282).
//
// Atoms are binned into x-y columns whose cross-section holds about one
// cluster-height of atoms, sorted by z inside each column, and cut into
// clusters of 8; columns are numbered x-major (y fastest), so consecutive
// clusters sweep a band of x.  Every i cluster then gets the list of j clusters (j >= i,
// half list) whose bounding boxes, in some periodic image, come within the
// list cutoff (cutoff + skin).  Each entry carries a 64-bit mask of the atom
// pairs that interact: padding slots, the lower triangle of the self pair and
// excluded pairs are cleared.
#include <algorithm>
#include <cmath>

#include "bands.hpp"
#include "kargs.cuh"
#include "mdf_device.cuh"
#include "mdf_internal.cuh"

namespace mdf {

int grid_blocks(long long n, int threads)
{
    long long b = (n + threads - 1) / threads;
    return (int)std::max(1LL, b);
}

// ------------------------------------------------------------------ scan
// Column table in one block: exclusive scans of the atom counts (col_start)
// and of the cluster counts (col_cstart, ceil(count / 8) per column), and the
// cluster total at col_cstart[ncols].  A column above COL_MAX atoms (the
// in-block sort's limit) sets ST_CAPACITY_COLUMN.  ncols is at most a few
// thousand, so each thread takes a contiguous chunk.
constexpr int COL_MAX = 2048;   // atoms per column handled by the in-block sort

__global__ void __launch_bounds__(1024) k_column_table(int ncols, const int* __restrict__ cnt,
                                                       int* __restrict__ col_start, int* __restrict__ col_cstart,
                                                       unsigned* st)
{
    __shared__ int part_a[1024], part_c[1024];
    const int tid = threadIdx.x, per = (ncols + blockDim.x - 1) / blockDim.x;
    const int b0 = min(ncols, tid * per), b1 = min(ncols, b0 + per);
    int sa = 0, sc = 0;
    bool over = false;
    for (int i = b0; i < b1; ++i) {
        const int n = cnt[i];
        sa += n;
        sc += (n + CLUSTER - 1) / CLUSTER;
        over = over || n > COL_MAX;
    }
    if (over) status_set(st, ST_CAPACITY_COLUMN);
    part_a[tid] = sa;
    part_c[tid] = sc;
    __syncthreads();
    for (int o = 1; o < blockDim.x; o <<= 1) {   // Hillis-Steele inclusive scan of the partials
        const int va = tid >= o ? part_a[tid - o] : 0, vc = tid >= o ? part_c[tid - o] : 0;
        __syncthreads();
        part_a[tid] += va;
        part_c[tid] += vc;
        __syncthreads();
    }
    int ra = tid ? part_a[tid - 1] : 0, rc = tid ? part_c[tid - 1] : 0;
    for (int i = b0; i < b1; ++i) {
        const int n = cnt[i];
        col_start[i] = ra;
        col_cstart[i] = rc;
        ra += n;
        rc += (n + CLUSTER - 1) / CLUSTER;
    }
    if (tid == blockDim.x - 1) {
        col_start[ncols] = part_a[tid];
        col_cstart[ncols] = part_c[tid];
    }
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
    // x-major: consecutive columns run along y, so a contiguous range of
    // clusters is a band of x (a split evaluation's share of space)
    int col = cy + ncy * cx;
    atom_col[i] = col;
    atomicAdd(&col_count[col], 1);
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
    int s0 = col_start[col];
    if (n > COL_MAX) {
        // The build restarts with thinner columns; until then this column's
        // clusters are left empty and its atoms point at slot 0, so the
        // kernels queued after this one only touch valid memory.
        if (tid == 0) status_set(st, ST_CAPACITY_COLUMN);
        const int c0 = col_cstart[col], ncl = (n + CLUSTER - 1) / CLUSTER;
        for (int k = tid; k < ncl * CLUSTER; k += blockDim.x) {
            slot_atom[c0 * CLUSTER + k] = -1;
            if ((k % CLUSTER) == 0) cluster_col[c0 + k / CLUSTER] = col;
        }
        for (int k = tid; k < n; k += blockDim.x) atom_slot[col_atoms[s0 + k]] = 0;
        return;
    }
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
// Launched over the cluster capacity; the clusters the column table made
// (*d_ncl) are the ones with work.
__global__ void k_cluster_geom(const int* __restrict__ d_ncl, const double* __restrict__ xyz, double Lx, double Ly,
                               double Lz, double quantum, const int* __restrict__ slot_atom,
                               double4* __restrict__ center, float4* __restrict__ centerf, float4* __restrict__ bb_lo,
                               float4* __restrict__ bb_hi)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= *d_ncl) return;
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
__device__ __forceinline__ void pack_dev(const PackArgs<R>& A, int bx, int by)
{
    const int nslots = A.nslots;
    const double* __restrict__ xyz = A.xyz;
    const double* __restrict__ q = A.q;
    const int* __restrict__ slot_atom = A.slot_atom;
    const double4* __restrict__ center = A.center;
    const double Lx = A.L[0], Ly = A.L[1], Lz = A.L[2];
    typename V4<R>::type* __restrict__ xq = A.xq;
    float4* __restrict__ cur_lo = A.cur_lo;
    float4* __restrict__ cur_hi = A.cur_hi;
    unsigned* st = A.st;
    const int s = bx * blockDim.x + threadIdx.x;
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
    if (A.snap) {
        // self-pruning: the largest squared displacement since the last prune
        float d2 = 0.f;
        if (a >= 0) {
            const typename V4<R>::type o = A.snap[s];
            const double ex = (double)v.x - (double)o.x, ey = (double)v.y - (double)o.y, ez = (double)v.z - (double)o.z;
            d2 = __double2float_ru(ex * ex + ey * ey + ez * ez);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d2 = fmaxf(d2, __shfl_xor_sync(0xffffffffu, d2, o));
        if ((threadIdx.x & 31) == 0 && d2 > 0.f) atomicMax(A.disp, __float_as_uint(d2));
    }
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

template <typename R>
__global__ void k_pack(PackArgs<R> A)
{
    pack_dev(A, blockIdx.x, 0);
}

template <typename R>
__global__ void k_pack_multi(const PackArgs<R>* __restrict__ As, const int2* __restrict__ bmap)
{
    const int2 m = bmap[blockIdx.x];
    pack_dev(As[m.x], m.y, 0);
}

__global__ void k_slot_type(const int* __restrict__ d_ncl, const int* __restrict__ slot_atom,
                            const int* __restrict__ type, int pad_type, int* __restrict__ slot_type)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= *d_ncl * CLUSTER) return;
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

// One warp per i cluster (launched over the cluster capacity; clusters at or
// above *d_ncl return).  Two sweeps over the same candidates: the first counts
// this lane's entries, then lane 0 claims the cluster's range of the list with
// one atomicAdd on *d_total and the second sweep writes the entries there
// after the lane-exclusive prefix.  The order inside an i cluster's range is
// fixed (lane-major over the column/image candidates), so every evaluation
// sums the same terms in the same order; only the ranges' positions in the
// list depend on the order the warps ran in.  Entries past `cap` are counted
// but not written (ST_CAPACITY_PAIRS: the host grows the list and searches
// again).
__global__ void __launch_bounds__(256) k_pair_search(const int* __restrict__ d_ncl, SearchGeom g,
                                                     const int* __restrict__ cluster_col,
                                                     const int* __restrict__ col_cstart,
                                                     const float4* __restrict__ bb_lo, const float4* __restrict__ bb_hi,
                                                     const double4* __restrict__ center, int* __restrict__ d_total,
                                                     PairEntry* __restrict__ out, long long cap,
                                                     ILRange* __restrict__ ilist, unsigned* st)
{
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (I >= *d_ncl) return;
    const int col = cluster_col[I];
    const int cx = col / g.ncy, cy = col % g.ncy;
    const float4 lo = bb_lo[I], hi = bb_hi[I];
    const int nvi = (int)center[I].w;
    const int nxc = 2 * g.Rx + 1, nyc = 2 * g.Ry + 1;
    const int ncombo = nxc * nyc * 3;
    const float Lx = (float)g.L[0], Ly = (float)g.L[1], Lz = (float)g.L[2];
    int cnt = 0;
    long long base = 0;
    for (int sweep = 0; sweep < 2; ++sweep) {
        if (sweep == 1) {
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const int tot = __shfl_sync(0xffffffffu, incl, 31);
            int start = 0;
            if (lane == 0) start = atomicAdd(d_total, tot);
            start = __shfl_sync(0xffffffffu, start, 0);
            if (lane == 0) {
                ILRange r;
                r.i = I;
                r.start = start;
                r.count = tot;
                r.pad = 0;
                ilist[I] = r;
                if ((long long)start + tot > cap) status_set(st, ST_CAPACITY_PAIRS);
            }
            base = (long long)start + (incl - cnt);
            cnt = 0;
        }
        for (int combo = lane; combo < ncombo; combo += 32) {
            const int szi = combo % 3;
            const int rest = combo / 3;
            const int dcx = rest % nxc - g.Rx;
            const int dcy = rest / nxc - g.Ry;
            int jx = cx + dcx, jy = cy + dcy;
            const int sx = jx < 0 ? -1 : (jx >= g.ncx ? 1 : 0);
            const int sy = jy < 0 ? -1 : (jy >= g.ncy ? 1 : 0);
            jx -= sx * g.ncx;
            jy -= sy * g.ncy;
            const int sz = szi - 1;
            const float cxl = (float)(jx * g.colw[0] + sx * g.L[0]), cxh = (float)((jx + 1) * g.colw[0] + sx * g.L[0]);
            const float cyl = (float)(jy * g.colw[1] + sy * g.L[1]), cyh = (float)((jy + 1) * g.colw[1] + sy * g.L[1]);
            const float gx = fmaxf(0.f, fmaxf(cxl - hi.x, lo.x - cxh));
            const float gy = fmaxf(0.f, fmaxf(cyl - hi.y, lo.y - cyh));
            if (gx * gx + gy * gy > g.rlist2) continue;
            const float zmin = lo.z - g.rlist - sz * Lz, zmax = hi.z + g.rlist - sz * Lz;
            if (zmax < -1.0f || zmin > Lz + 1.0f) continue;
            const int jcol = jy + g.ncy * jx;
            const int c0 = col_cstart[jcol], c1 = col_cstart[jcol + 1];
            // first cluster whose hi.z >= zmin
            int a = c0, b = c1;
            while (a < b) {
                const int mid = (a + b) >> 1;
                if (bb_hi[mid].z < zmin) a = mid + 1;
                else b = mid;
            }
            for (int J = a; J < c1; ++J) {
                const float4 jl = bb_lo[J], jh = bb_hi[J];
                if (jl.z > zmax) break;
                const float ox = sx * Lx, oy = sy * Ly, oz = sz * Lz;
                const float dx = fmaxf(0.f, fmaxf(jl.x + ox - hi.x, lo.x - (jh.x + ox)));
                const float dy = fmaxf(0.f, fmaxf(jl.y + oy - hi.y, lo.y - (jh.y + oy)));
                const float dz = fmaxf(0.f, fmaxf(jl.z + oz - hi.z, lo.z - (jh.z + oz)));
                if (dx * dx + dy * dy + dz * dz > g.rlist2) continue;
                const int code = (sx + 1) + 3 * (sy + 1) + 9 * (sz + 1);
                if (J < I || (J == I && code < 13)) continue;
                if (sweep == 1) {
                    const long long pos = base + cnt;
                    if (pos < cap) {
                        PairEntry e;
                        e.j = J;
                        e.shift = code;
                        e.mask = entry_mask(nvi, (int)center[J].w, J == I && code == 13);
                        out[pos] = e;
                    }
                }
                ++cnt;
            }
        }
    }
}

// Clear the mask bit of every excluded pair in the entry that holds it.  One
// warp per excluded pair: the warp locates the (I, J, image) entry in I's
// range 32 entries at a time (coalesced 16-byte loads) and one lane clears
// the bit.
__global__ void k_exclusion_masks(int nexcl, const int* __restrict__ excl, const int* __restrict__ atom_slot,
                                  const double* __restrict__ xyz, const double4* __restrict__ center, double Lx,
                                  double Ly, double Lz, const ILRange* __restrict__ ilist,
                                  PairEntry* __restrict__ plist, long long cap)
{
    const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (k >= nexcl) return;
    const int a = excl[2 * k], b = excl[2 * k + 1];
    const int sa = atom_slot[a], sb = atom_slot[b];
    const int Ia = sa / CLUSTER, la = sa % CLUSTER, Ib = sb / CLUSTER, lb = sb % CLUSTER;
    const double4 ca = center[Ia], cb = center[Ib];
    // list-geometry positions: centre + min-image offset
    const double pa[3] = {ca.x + min_image(xyz[3 * a] - ca.x, Lx), ca.y + min_image(xyz[3 * a + 1] - ca.y, Ly),
                          ca.z + min_image(xyz[3 * a + 2] - ca.z, Lz)};
    const double pb[3] = {cb.x + min_image(xyz[3 * b] - cb.x, Lx), cb.y + min_image(xyz[3 * b + 1] - cb.y, Ly),
                          cb.z + min_image(xyz[3 * b + 2] - cb.z, Lz)};
    // J atoms sit at p + s L in I's frame: s = round((p_I - p_J) / L)
    const int s[3] = {(int)round((pa[0] - pb[0]) / Lx), (int)round((pa[1] - pb[1]) / Ly),
                      (int)round((pa[2] - pb[2]) / Lz)};
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
    const ILRange r = ilist[I];
    const long long end = min((long long)r.start + r.count, cap);
    for (long long e0 = r.start; e0 < end; e0 += 32) {
        const long long e = e0 + lane;
        const bool hit = e < end && plist[e].j == J && plist[e].shift == code;
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (m) {
            if (lane == __ffs(m) - 1) atomicAnd(&plist[e].mask, ~(1ull << bit));
            return;
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
__device__ __forceinline__ void prune_dev(const PruneArgs<R>& A)
{
    const int ncl = A.ncl;
    const ILRange* __restrict__ ilist = A.ilist;
    const PairEntry* __restrict__ plist = A.plist;
    const typename V4<R>::type* __restrict__ xq = A.xq;
    const float4* __restrict__ centerf = A.centerf;
    const float4* __restrict__ cur_lo = A.cur_lo;
    const float4* __restrict__ cur_hi = A.cur_hi;
    const PruneShifts& shifts = A.shifts;
    const float rcut2 = A.rcut2;
    ILRange* __restrict__ ilist_in = A.ilist_in;
    PairEntry* __restrict__ plist_in = A.plist_in;
    using V4t = typename V4<R>::type;
    // self-pruning: the list pruned last time still holds every pair within the cutoff
    if (!A.force && __uint_as_float(*A.disp) <= A.disp_thr2) return;
    __shared__ float sh[27][6];
    for (int k = threadIdx.x; k < 27 * 6; k += blockDim.x) sh[k / 6][k % 6] = shifts.v[k / 6][k % 6];
    __syncthreads();
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;   // index into this launch's ilist range
    const int lane = threadIdx.x & 31;
    if (w >= ncl) return;
    const unsigned below = (1u << lane) - 1u;
    const ILRange L = ilist[w];
    const int I = L.i;
    if (A.snap && lane < CLUSTER) A.snap[I * CLUSTER + lane] = xq[I * CLUSTER + lane];
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
    }
}

// Half prune (the 4 x 8 pair layout): the same box test, then each half of
// the i cluster (atoms 0-3, 4-7) is tested on its own; an entry goes to the
// list of every half that has an atom pair within the radius.  One lane per
// outer entry, two j atoms at a time, stopping once both halves are found.
// The outer range [start, start + count) of i cluster I owns the slots
// [2 start + h count, 2 start + (h + 1) count) of the half list; item 2 w + h
// of this launch describes half h (ILRange.pad = h).
template <typename R>
__device__ __forceinline__ void prune_half_dev(const PruneArgs<R>& A)
{
    using V4t = typename V4<R>::type;
    if (!A.force && __uint_as_float(*A.disp) <= A.disp_thr2) return;   // self-pruning: the lists still hold
    __shared__ float sh[27][6];
    for (int k = threadIdx.x; k < 27 * 6; k += blockDim.x) sh[k / 6][k % 6] = A.shifts.v[k / 6][k % 6];
    __syncthreads();
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= A.ncl) return;
    const unsigned below = (1u << lane) - 1u;
    const ILRange L = A.ilist[w];
    const int I = L.i;
    const V4t* __restrict__ xq = A.xq;
    if (A.snap && lane < CLUSTER) A.snap[I * CLUSTER + lane] = xq[I * CLUSTER + lane];
    R ax[CLUSTER], ay[CLUSTER], az[CLUSTER], an[CLUSTER];   // -2 x_i and |x_i|^2
#pragma unroll
    for (int k = 0; k < CLUSTER; ++k) {
        const V4t v = xq[I * CLUSTER + k];
        ax[k] = (R)-2 * v.x; ay[k] = (R)-2 * v.y; az[k] = (R)-2 * v.z;
        an[k] = v.x * v.x + v.y * v.y + v.z * v.z;
    }
    const float4 cI = A.centerf[I], ilo = A.cur_lo[I], ihi = A.cur_hi[I];
    const R rc2 = (R)A.rcut2;
    const long long out0 = 2LL * L.start, out1 = 2LL * L.start + L.count;
    int kept0 = 0, kept1 = 0;
    for (int base = 0; base < L.count; base += 32) {
        const bool have = base + lane < L.count;
        PairEntry my;
        my.j = I; my.shift = 13; my.mask = 0ull;
        if (have) my = A.plist[L.start + base + lane];
        const float4 cJ = A.centerf[my.j], jlo = A.cur_lo[my.j], jhi = A.cur_hi[my.j];
        const float* s6 = sh[my.shift];
        const float ox = -(((cI.x - cJ.x) - s6[0]) - s6[3]);
        const float oy = -(((cI.y - cJ.y) - s6[1]) - s6[4]);
        const float oz = -(((cI.z - cJ.z) - s6[2]) - s6[5]);
        const float gx = fmaxf(0.f, fmaxf(jlo.x + ox - ihi.x, ilo.x - (jhi.x + ox)));
        const float gy = fmaxf(0.f, fmaxf(jlo.y + oy - ihi.y, ilo.y - (jhi.y + oy)));
        const float gz = fmaxf(0.f, fmaxf(jlo.z + oz - ihi.z, ilo.z - (jhi.z + oz)));
        const bool cand = have && my.mask != 0ull && gx * gx + gy * gy + gz * gz < A.rcut2;
        bool k0 = false, k1 = false;
        if (cand) {
            const R px = (R)ox, py = (R)oy, pz = (R)oz;
            const V4t* __restrict__ xj = xq + (size_t)my.j * CLUSTER;
#pragma unroll 1
            for (int j = 0; j < CLUSTER && !(k0 && k1); j += 2) {
                V4t v[2];
                v[0] = xj[j];
                v[1] = xj[j + 1];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const R qx = v[u].x + px, qy = v[u].y + py, qz = v[u].z + pz;
                    const R thr = rc2 - (qx * qx + qy * qy + qz * qz);
                    R m0 = fma(ax[0], qx, fma(ay[0], qy, fma(az[0], qz, an[0])));
                    R m1 = fma(ax[4], qx, fma(ay[4], qy, fma(az[4], qz, an[4])));
#pragma unroll
                    for (int ii = 1; ii < 4; ++ii) {
                        m0 = fmin(m0, fma(ax[ii], qx, fma(ay[ii], qy, fma(az[ii], qz, an[ii]))));
                        m1 = fmin(m1, fma(ax[ii + 4], qx, fma(ay[ii + 4], qy, fma(az[ii + 4], qz, an[ii + 4]))));
                    }
                    k0 = k0 || m0 < thr;
                    k1 = k1 || m1 < thr;
                }
            }
        }
        const unsigned b0 = __ballot_sync(0xffffffffu, k0), b1 = __ballot_sync(0xffffffffu, k1);
        if (k0) A.plist_in[out0 + kept0 + __popc(b0 & below)] = my;
        if (k1) A.plist_in[out1 + kept1 + __popc(b1 & below)] = my;
        kept0 += __popc(b0);
        kept1 += __popc(b1);
    }
    if (lane == 0) {
        ILRange r;
        r.i = I; r.start = (int)out0; r.count = kept0; r.pad = 0;
        A.ilist_in[2 * w] = r;
        r.start = (int)out1; r.count = kept1; r.pad = 1;
        A.ilist_in[2 * w + 1] = r;
    }
}

template <typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 3) k_prune_half(PruneArgs<R> A)
{
    prune_half_dev(A);
}

template <typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 3) k_prune_half_multi(const PruneArgs<R>* __restrict__ As)
{
    const PruneArgs<R>& A = As[blockIdx.z];
    if ((int)blockIdx.x >= A.gx) return;
    prune_half_dev(A);
}

template <typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 3) k_prune(PruneArgs<R> A)
{
    prune_dev(A);
}

template <typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 3) k_prune_multi(const PruneArgs<R>* __restrict__ As)
{
    const PruneArgs<R>& A = As[blockIdx.z];
    if ((int)blockIdx.x >= A.gx) return;
    prune_dev(A);
}

// Prune arguments for this rank's i clusters (ncl = 0: nothing to do).
template <typename R>
PruneArgs<R> make_prune_args(const Ctx& c)
{
    PruneArgs<R> A;
    // a hair above the cutoff so working-precision rounding never drops a pair at r ~ rc
    const double rc = c.p.cutoff + std::max(0.0, c.p.prune_margin) + 0.02;
    for (int code = 0; code < 27; ++code) {
        int sv[3] = {code % 3 - 1, (code / 3) % 3 - 1, code / 9 - 1};
        for (int d = 0; d < 3; ++d) {
            double v = sv[d] * c.box[d];
            float hi = (float)v;
            A.shifts.v[code][d] = hi;
            A.shifts.v[code][3 + d] = (float)(v - (double)hi);
        }
    }
    long long lo, hi;
    cluster_share(c, lo, hi);   // this rank's i clusters
    A.ncl = (int)(hi - lo);
    A.gx = grid_blocks((long long)A.ncl * 32, 256);
    A.gy = 1;
    A.ilist = c.ilist.p + lo;
    A.plist = c.plist.p;
    A.xq = reinterpret_cast<const typename V4<R>::type*>(sizeof(R) == 4 ? (const void*)c.xq_f.p : (const void*)c.xq_d.p);
    A.centerf = c.centerf.p;
    A.cur_lo = c.cur_lo.p;
    A.cur_hi = c.cur_hi.p;
    A.rcut2 = (float)(rc * rc);
    A.ilist_in = c.ilist_in.p + lo;
    A.plist_in = c.plist_in.p;
    const bool selfp = self_pruning(c);
    A.snap = selfp ? reinterpret_cast<typename V4<R>::type*>(c.xq_snap.p) : nullptr;
    A.disp = reinterpret_cast<const unsigned*>(c.scal.p + SCAL_DISP);
    const float half_margin = (float)(0.5 * std::max(0.0, c.p.prune_margin));
    A.disp_thr2 = half_margin * half_margin;
    A.force = (!selfp || !c.pruned_valid) ? 1 : 0;
    return A;
}

// The half-layout lists (two items per i cluster, twice the outer capacity).
void ensure_half_lists(Ctx& c)
{
    c.ilist_h.alloc(2 * (size_t)std::max(c.n_clusters, 1));
    c.plist_h.alloc(2 * (size_t)std::max<size_t>(c.plist.n, 1));
}

// Prune arguments writing the half lists (item 2 w + h of this rank's range).
template <typename R>
PruneArgs<R> make_prune_half_args(const Ctx& c)
{
    PruneArgs<R> A = make_prune_args<R>(c);
    long long lo, hi;
    cluster_share(c, lo, hi);
    A.ilist_in = c.ilist_h.p + 2 * lo;
    A.plist_in = c.plist_h.p;
    return A;
}
template PruneArgs<float> make_prune_half_args<float>(const Ctx&);
template PruneArgs<double> make_prune_half_args<double>(const Ctx&);
template PruneArgs<float> make_prune_args<float>(const Ctx&);
template PruneArgs<double> make_prune_args<double>(const Ctx&);

template <typename R>
void launch_prune_multi(const PruneArgs<R>* d_args, int nsys, int gx, bool half, cudaStream_t s)
{
    if (half) k_prune_half_multi<R><<<dim3(gx, 1, nsys), 256, 0, s>>>(d_args);
    else k_prune_multi<R><<<dim3(gx, 1, nsys), 256, 0, s>>>(d_args);
    MDF_CUDA_TRY(cudaGetLastError());
}
template void launch_prune_multi<float>(const PruneArgs<float>*, int, int, bool, cudaStream_t);
template void launch_prune_multi<double>(const PruneArgs<double>*, int, int, bool, cudaStream_t);

// whole_entries: build the 8 x 8 pruned list even in the half layout (the
// adjoint walks whole entries); it also prunes unconditionally.
void prune_pairlist(Ctx& c, bool whole_entries)
{
    if (whole_entries) c.pruned_valid = false;   // a self-pruning launch prunes when the list is not valid
    const bool half = half_layout(c) && !whole_entries;
    if (half) ensure_half_lists(c);
    if (c.p.precision == MDF_PREC_MIXED) {
        const PruneArgs<float> A = half ? make_prune_half_args<float>(c) : make_prune_args<float>(c);
        if (A.ncl > 0) {
            if (half) k_prune_half<float><<<grid_of(A), 256, 0, c.stream>>>(A);
            else k_prune<float><<<grid_of(A), 256, 0, c.stream>>>(A);
        }
    } else {
        const PruneArgs<double> A = half ? make_prune_half_args<double>(c) : make_prune_args<double>(c);
        if (A.ncl > 0) {
            if (half) k_prune_half<double><<<grid_of(A), 256, 0, c.stream>>>(A);
            else k_prune<double><<<grid_of(A), 256, 0, c.stream>>>(A);
        }
    }
    MDF_CUDA_TRY(cudaGetLastError());
    c.launches += 1;
    c.pruned_valid = true;
    c.pruned_half = half;
}

// ------------------------------------------------------------------ host
static double atom_density(const Ctx& c)
{
    return (double)c.N / (c.box[0] * c.box[1] * c.box[2]);
}

template <typename R>
PackArgs<R> make_pack_args(const Ctx& c)
{
    PackArgs<R> A;
    A.nslots = c.n_slots;
    A.gx = grid_blocks(c.n_slots, 256);
    A.gy = 1;
    A.xyz = c.xyz.p;
    A.q = c.q.p;
    A.slot_atom = c.slot_atom.p;
    A.center = c.center.p;
    for (int d = 0; d < 3; ++d) A.L[d] = c.box[d];
    A.xq = reinterpret_cast<typename V4<R>::type*>(sizeof(R) == 4 ? (void*)c.xq_f.p : (void*)c.xq_d.p);
    A.cur_lo = c.cur_lo.p;
    A.cur_hi = c.cur_hi.p;
    A.snap = self_pruning(c) ? reinterpret_cast<const typename V4<R>::type*>(c.xq_snap.p) : nullptr;
    A.disp = reinterpret_cast<unsigned*>(c.scal.p + SCAL_DISP);
    A.st = c.status.p;
    return A;
}
template PackArgs<float> make_pack_args<float>(const Ctx&);
template PackArgs<double> make_pack_args<double>(const Ctx&);

template <typename R>
void launch_pack_multi(const PackArgs<R>* d_args, BlockMap bm, cudaStream_t s)
{
    if (bm.n <= 0) return;
    k_pack_multi<R><<<bm.n, 256, 0, s>>>(d_args, bm.map);
    MDF_CUDA_TRY(cudaGetLastError());
}
template void launch_pack_multi<float>(const PackArgs<float>*, BlockMap, cudaStream_t);
template void launch_pack_multi<double>(const PackArgs<double>*, BlockMap, cudaStream_t);

void pack_positions(Ctx& c)
{
    if (c.p.precision == MDF_PREC_MIXED) {
        const PackArgs<float> A = make_pack_args<float>(c);
        k_pack<float><<<grid_of(A), 256, 0, c.stream>>>(A);
    } else {
        const PackArgs<double> A = make_pack_args<double>(c);
        k_pack<double><<<grid_of(A), 256, 0, c.stream>>>(A);
    }
    MDF_CUDA_TRY(cudaGetLastError());
    c.launches += 1;
}

// Bands of a split evaluation (the arithmetic in bands.hpp): this rank's
// clusters, its stencil window and its halo plane lists, uploaded once per
// build.
void build_bands(Ctx& c)
{
    const int P = c.p.nranks, me = c.p.rank, K0 = c.K[0];
    const int ncy = c.ncol_y;
    std::vector<int> cst(c.ncols + 1);
    MDF_CUDA_TRY(cudaMemcpyAsync(cst.data(), c.col_cstart.p, sizeof(int) * (c.ncols + 1), cudaMemcpyDeviceToHost,
                                 c.stream));
    MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));
    const BandPlan B = plan_bands(P, K0, c.ncol_x, c.box[0], c.p.skin);
    c.band_cl.assign(P + 1, 0);
    for (int t = 0; t <= P; ++t) c.band_cl[t] = cst[B.first[t] * ncy];
    c.win_lo = B.win_lo;
    c.win_n = B.win_n;
    const HaloLists H = halo_lists(B, P, me, K0);
    auto upload = [&](DevBuf<int>& d, const std::vector<int>& h) {
        d.alloc(std::max<size_t>(1, h.size()));
        if (!h.empty())
            MDF_CUDA_TRY(cudaMemcpyAsync(d.p, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, c.stream));
    };
    upload(c.halo_send_pl, H.send);
    upload(c.halo_recv_pl, H.recv);
    upload(c.halo_local_pl, H.local);
    c.halo_send_n = H.send_n;
    c.halo_recv_n = H.recv_n;
    c.halo_n_send = (int)H.send.size();
    c.halo_n_recv = (int)H.recv.size();
    c.halo_n_local = (int)H.local.size();
    for (int k = 0; k < 2; ++k)
        for (int l = 0; l < 2; ++l) c.halo_rng[k][l] = H.rng[k][l];
    MDF_CUDA_TRY(cudaStreamSynchronize(c.stream));   // the host lists are freed on return
}


// The whole build is queued on the context's stream without a host round trip
// in between: every buffer the build kernels write is sized from bounds known
// on the host (clusters <= ceil(N/8) + columns; the list from a density
// estimate or the last build), the kernels read the cluster count from the
// device, and one synchronisation at the end returns the cluster and entry
// counts with the status word.  A list that outgrew its capacity is grown and
// searched again; a column above the sort's limit restarts with thinner
// columns.
void build_pairlist(Ctx& c)
{
    c.npairs_dev.alloc(1);
    c.count_next = true;
    c.counted = false;
    cudaStream_t s = c.stream;
    const int th = 256;
    const double rlist = c.p.cutoff + c.p.skin;
    for (int d = 0; d < 3; ++d)
        if (!(c.box[d] >= 2.0 * c.p.cutoff))
            throw ApiError(MDF_ERR_INVALID, "box edge shorter than twice the cutoff (minimum image undefined)");
    if (!c.h_build) MDF_CUDA_TRY(cudaHostAlloc((void**)&c.h_build, 4 * sizeof(int), cudaHostAllocDefault));
    c.d_build.alloc(4);
    // column cross-section ~ one cluster of atoms per column-height cube
    const double rho = atom_density(c);
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
        // every column wastes at most one partly filled cluster
        const long long ncl_cap = ((long long)c.N + CLUSTER - 1) / CLUSTER + c.ncols;
        if (ncl_cap * CLUSTER > INT32_MAX / 3) throw ApiError(MDF_ERR_CAPACITY, "too many atoms for one context");
        c.col_count.alloc(c.ncols + 1);
        c.col_start.alloc(c.ncols + 1);
        c.col_cstart.alloc(c.ncols + 1);
        c.scan_tmp.alloc(c.ncols + 1);
        c.atom_col.alloc(c.N);
        c.col_atoms.alloc(c.N);
        c.atom_slot.alloc(c.N);
        c.slot_atom.alloc(ncl_cap * CLUSTER);
        c.slot_type.alloc(ncl_cap * CLUSTER);
        c.cluster_col.alloc(ncl_cap);
        c.center.alloc(ncl_cap);
        c.centerf.alloc(ncl_cap);
        c.bb_lo.alloc(ncl_cap);
        c.bb_hi.alloc(ncl_cap);
        c.ilist.alloc(ncl_cap);
        if (!c.plist.p) {
            // list estimate: half the clusters within rlist + one cluster extent, 30% over
            const double ext = rlist + side;
            const double per = 0.5 * (rho / CLUSTER) * (4.0 / 3.0) * M_PI * ext * ext * ext * 1.3;
            c.plist.alloc((size_t)(ncl_cap * std::max(32.0, per)) + 1024);
        }
        {
            // largest power-of-two quantum keeping every centre exact in FP32 (24-bit significand)
            const double lmax = std::max(c.box[0], std::max(c.box[1], c.box[2]));
            c.center_quantum = std::ldexp(1.0, (int)std::ceil(std::log2(lmax + 1.0)) - 24);
        }
        const int* d_ncl = c.col_cstart.p + c.ncols;   // cluster count, written by k_column_table
        MDF_CUDA_TRY(cudaMemsetAsync(c.col_count.p, 0, sizeof(int) * (c.ncols + 1), s));
        MDF_CUDA_TRY(cudaMemsetAsync(c.scan_tmp.p, 0, sizeof(int) * (c.ncols + 1), s));
        MDF_CUDA_TRY(cudaMemsetAsync(c.status.p, 0, sizeof(unsigned), s));
        k_assign_columns<<<grid_blocks(c.N, th), th, 0, s>>>(c.N, c.xyz.p, c.box[0], c.box[1], c.ncol_x, c.ncol_y,
                                                             c.atom_col.p, c.col_count.p, c.status.p);
        k_column_table<<<1, 1024, 0, s>>>(c.ncols, c.col_count.p, c.col_start.p, c.col_cstart.p, c.status.p);
        k_bucket<<<grid_blocks(c.N, th), th, 0, s>>>(c.N, c.atom_col.p, c.col_start.p, c.scan_tmp.p, c.col_atoms.p);
        k_sort_columns<<<c.ncols, 1024, 0, s>>>(c.xyz.p, c.box[2], c.col_count.p, c.col_start.p, c.col_cstart.p,
                                                c.col_atoms.p, c.slot_atom.p, c.atom_slot.p, c.cluster_col.p,
                                                c.status.p);
        k_cluster_geom<<<grid_blocks(ncl_cap, th), th, 0, s>>>(d_ncl, c.xyz.p, c.box[0], c.box[1], c.box[2],
                                                               c.center_quantum, c.slot_atom.p, c.center.p,
                                                               c.centerf.p, c.bb_lo.p, c.bb_hi.p);
        k_slot_type<<<grid_blocks(ncl_cap * CLUSTER, th), th, 0, s>>>(d_ncl, c.slot_atom.p, c.type.p, c.ntp - 1,
                                                                      c.slot_type.p);
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
        unsigned st = 0;
        for (int search = 0; search < 3; ++search) {
            const long long cap = (long long)c.plist.n;
            MDF_CUDA_TRY(cudaMemsetAsync(c.d_build.p, 0, sizeof(int) * 4, s));
            k_pair_search<<<grid_blocks(ncl_cap * 32, th), th, 0, s>>>(d_ncl, g, c.cluster_col.p, c.col_cstart.p,
                                                                       c.bb_lo.p, c.bb_hi.p, c.center.p, c.d_build.p,
                                                                       c.plist.p, cap, c.ilist.p, c.status.p);
            if (c.n_excl > 0)
                k_exclusion_masks<<<grid_blocks((long long)c.n_excl * 32, th), th, 0, s>>>(
                    c.n_excl, c.excl_pairs.p, c.atom_slot.p, c.xyz.p, c.center.p, c.box[0], c.box[1], c.box[2],
                    c.ilist.p, c.plist.p, cap);
            MDF_CUDA_TRY(cudaGetLastError());
            MDF_CUDA_TRY(cudaMemcpyAsync(c.h_build, d_ncl, sizeof(int), cudaMemcpyDeviceToHost, s));
            MDF_CUDA_TRY(cudaMemcpyAsync(c.h_build + 1, c.d_build.p, sizeof(int), cudaMemcpyDeviceToHost, s));
            MDF_CUDA_TRY(cudaMemcpyAsync(c.h_build + 2, c.status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
            MDF_CUDA_TRY(cudaStreamSynchronize(s));
            st = (unsigned)c.h_build[2];
            if (st & (ST_NONFINITE | ST_CAPACITY_COLUMN)) break;
            if (!(st & ST_CAPACITY_PAIRS)) break;
            // the list outgrew its buffer: grow to the count found (+1/8) and search again
            c.plist.alloc((size_t)c.h_build[1] + 1);
            MDF_CUDA_TRY(cudaMemsetAsync(c.status.p, 0, sizeof(unsigned), s));
        }
        if (st & ST_NONFINITE) throw ApiError(MDF_ERR_NONFINITE, "non-finite position");
        if (st & ST_CAPACITY_COLUMN) {
            side *= 0.7;   // too many atoms in a column: thinner columns
            if (attempt == 5) throw ApiError(MDF_ERR_CAPACITY, "column too populated for the in-block sort");
            continue;
        }
        if (st & ST_CAPACITY_PAIRS) throw ApiError(MDF_ERR_CAPACITY, "pair list capacity exceeded");
        const int ncl = c.h_build[0];
        c.n_clusters = ncl;
        c.n_slots = ncl * CLUSTER;
        c.n_entries = c.h_build[1];
        c.cur_lo.alloc(ncl);
        c.cur_hi.alloc(ncl);
        if (c.p.precision == MDF_PREC_MIXED) c.xq_f.alloc(c.n_slots);
        else c.xq_d.alloc(c.n_slots);
        if (c.p.prune_every < 0)
            c.xq_snap.alloc((c.p.precision == MDF_PREC_MIXED ? sizeof(float4) : sizeof(double4)) * (size_t)c.n_slots);
        if (half_layout(c)) ensure_half_lists(c);   // sized here, not inside a later stream capture
        c.f_slot.alloc((size_t)3 * c.n_slots);
        c.need_clear = true;   // slot layout changed: clear the accumulators before the next evaluation
        c.plist_in.alloc(c.plist.n);
        c.ilist_in.alloc(ncl);
        c.pruned_valid = false;
        c.since_prune = 0;
        if (distributed(c)) build_bands(c);
        c.have_list = true;
        return;
    }
}

}  // namespace mdf
