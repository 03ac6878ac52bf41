// Dimer/trimer enumeration on the GPU, reproducing the reference's lists.
//
// The reference (systools::AddClusters, bblock/sys_tools.cpp:472-592) builds a
// kd-tree over the monomers' first atoms wrapped into the central cell plus
// seven periodic copies of every point (kdutils::XyzToCloud,
// kdtree/kdtree_utils.h:196-278), radius-searches each local monomer i with a
// strict d^2 < cutoff^2 test (kdtree/nanoflann.hpp:166-167), and accepts
//   dimer (i, j)    if tag_i < tag_j,
//   trimer (i,j,k)  for every pair of i's matches (j, k distinct, neither i)
//                   if |q_j - q_k|^2 > cutoff^2 or tag_i < min(tag_j, tag_k),
// where q are the matched cloud points (images near i).
//
// Here the same cloud is built explicitly (k_cloud), monomers are binned into
// a cell grid over fractional coordinates (k_cells*), every local monomer
// collects its matches from the 27 surrounding cells by testing all eight
// cloud points of each candidate (k_neighbors), and the dimer and trimer rules
// run on those matches (k_dimers, k_trimers).  Every distance that decides
// membership is computed with explicitly rounded operations in the
// reference's operand order, so the sets are bit-for-bit the reference's.
//
// Accepted n-mers are written to per-type buckets, already in evaluator
// (holder) order with the slot of the original first monomer, which is the
// image anchor (GetCloseDimerImage/GetCloseTrimerImage image relative to it).
#include <cuda_runtime.h>
#include <stdint.h>

#include "holder_common.cuh"
#include "nmer_build.h"

namespace {

__device__ __forceinline__ double dist2_rn(double a0, double a1, double a2, double b0, double b1, double b2) {
    const double d0 = __dsub_rn(a0, b0), d1 = __dsub_rn(a1, b1), d2 = __dsub_rn(a2, b2);
    return __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
}

// GetFractionalCoordinates (kdtree/kdtree_utils.h:165-190); only the signs of
// its results matter (they choose which periodic copies exist).
__device__ void frac_coords(const double* box, const double (&pt)[3], double (&c)[3]) {
    const double A = box[0];
    const double B = sqrt(box[3] * box[3] + box[4] * box[4]);
    const double C = sqrt(box[6] * box[6] + box[7] * box[7] + box[8] * box[8]);
    const double AdotB = box[0] * box[3], AdotC = box[0] * box[6], BdotC = box[3] * box[6] + box[4] * box[7];
    const double gamma = acos(AdotB / A / B), beta = acos(AdotC / A / C), alpha = acos(BdotC / B / C);
    const double ca = cos(alpha), cb = cos(beta), cg = cos(gamma), sg = sin(gamma);
    const double omega = A * B * C * sqrt(1 - ca * ca - cb * cb - cg * cg + 2 * ca * cb * cg);
    c[0] = 1 / A * pt[0] - cg / A / sg * pt[1] + B * C * (ca * cg - cb) / omega / sg * pt[2];
    c[1] = 1 / B / sg * pt[1] + A * C * (cb * cg - ca) / omega / sg * pt[2];
    c[2] = A * B * sg / omega * pt[2];
}

}  // namespace

// FixMonomerCoordinates (bblock/sys_tools.cpp:257-320), in place.
__global__ void k_fix_monomers(double* __restrict__ xyz, const int* __restrict__ first_index,
                               const int* __restrict__ nat, int nmon, BoxParams bp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nmon) return;
    double* p = xyz + 3 * (size_t)first_index[i];
    double q[3] = {p[0], p[1], p[2]}, f0[3];
    to_frac_rn(bp.inv, q, f0);
    f0[0] = __dsub_rn(f0[0], floor(__dadd_rn(f0[0], 0.5)));
    f0[1] = __dsub_rn(f0[1], floor(__dadd_rn(f0[1], 0.5)));
    f0[2] = __dsub_rn(f0[2], floor(__dadd_rn(f0[2], 0.5)));
    to_cart_rn(bp.box, f0, q);
    p[0] = q[0]; p[1] = q[1]; p[2] = q[2];
    for (int j = 1; j < nat[i]; ++j) {
        double a[3] = {p[3 * j], p[3 * j + 1], p[3 * j + 2]}, f[3];
        to_frac_rn(bp.inv, a, f);
        f[0] = __dsub_rn(f[0], floor(__dadd_rn(__dsub_rn(f[0], f0[0]), 0.5)));
        f[1] = __dsub_rn(f[1], floor(__dadd_rn(__dsub_rn(f[1], f0[1]), 0.5)));
        f[2] = __dsub_rn(f[2], floor(__dadd_rn(__dsub_rn(f[2], f0[2]), 0.5)));
        to_cart_rn(bp.box, f, a);
        p[3 * j] = a[0]; p[3 * j + 1] = a[1]; p[3 * j + 2] = a[2];
    }
}

// Cloud points of every monomer in the search: slot 0 is the wrapped first
// atom, slots 1..7 its periodic copies in the reference's shift categories
// (m,n,l nonzero pattern: 1 = z, 2 = y, 3 = x, 4 = xyz, 5 = yz, 6 = xz, 7 = xy).
// Also assigns the monomer's cell.
namespace {

// Cloud point q (monomer i) in the grid cg of box bp; returns its cell, and
// in dir the directions of its periodic copies (bit a set: the copies along
// axis a are at +1 box, else at -1).
__device__ __forceinline__ int cloud_point(const double* __restrict__ xyz, const int* __restrict__ first_index, int i,
                                           int q, const BoxParams& bp, const CellGrid& cg,
                                           double* __restrict__ cloud, int& dir) {
    dir = 0;
    const double* p0 = xyz + 3 * (size_t)first_index[i];
    double p[3] = {p0[0], p0[1], p0[2]};
    double* out = cloud + (size_t)q * 24;
    double fr[3];
    if (bp.use_pbc) {
        double f[3];
        to_frac_rn(bp.inv, p, f);
        f[0] = __dsub_rn(f[0], floor(__dadd_rn(f[0], 0.5)));
        f[1] = __dsub_rn(f[1], floor(__dadd_rn(f[1], 0.5)));
        f[2] = __dsub_rn(f[2], floor(__dadd_rn(f[2], 0.5)));
        to_cart_rn(bp.box, f, p);
        double uvw[3];
        frac_coords(bp.box, p, uvw);
        // per axis: the copy at -1 exists if uvw > 0, at +1 if uvw < 0; at
        // uvw == 0 both are made and the +1 copy overwrites (loop order 0,-1,1)
        int sgn[3];
        for (int a = 0; a < 3; ++a) sgn[a] = (uvw[a] > 0.0) ? -1 : 1;
        dir = (sgn[0] > 0 ? 1 : 0) | (sgn[1] > 0 ? 2 : 0) | (sgn[2] > 0 ? 4 : 0);
        for (int cat = 1; cat < 8; ++cat) {
            // category -> which axes are shifted
            const int mx = (cat == 3 || cat == 4 || cat == 6 || cat == 7);
            const int my = (cat == 2 || cat == 4 || cat == 5 || cat == 7);
            const int mz = (cat == 1 || cat == 4 || cat == 5 || cat == 6);
            const double m = mx ? sgn[0] : 0, n = my ? sgn[1] : 0, l = mz ? sgn[2] : 0;
            const double sx = __dadd_rn(__dadd_rn(__dmul_rn(m, bp.box[0]), __dmul_rn(n, bp.box[3])),
                                        __dmul_rn(l, bp.box[6]));
            const double sy = __dadd_rn(__dadd_rn(__dmul_rn(m, bp.box[1]), __dmul_rn(n, bp.box[4])),
                                        __dmul_rn(l, bp.box[7]));
            const double sz = __dadd_rn(__dadd_rn(__dmul_rn(m, bp.box[2]), __dmul_rn(n, bp.box[5])),
                                        __dmul_rn(l, bp.box[8]));
            out[3 * cat + 0] = __dadd_rn(p[0], sx);
            out[3 * cat + 1] = __dadd_rn(p[1], sy);
            out[3 * cat + 2] = __dadd_rn(p[2], sz);
        }
        fr[0] = f[0] + 0.5; fr[1] = f[1] + 0.5; fr[2] = f[2] + 0.5;   // in [0, 1)
    } else {
        for (int cat = 1; cat < 8; ++cat) {
            out[3 * cat] = out[3 * cat + 1] = out[3 * cat + 2] = 1e300;   // no copies without PBC
        }
        fr[0] = fr[1] = fr[2] = 0.0;
    }
    out[0] = p[0]; out[1] = p[1]; out[2] = p[2];
    int c[3];
    for (int a = 0; a < 3; ++a) {
        if (bp.use_pbc) {
            const int v = (int)floor(fr[a] * cg.n[a]);
            c[a] = v < 0 ? 0 : (v >= cg.n[a] ? cg.n[a] - 1 : v);
        } else {
            // hashed grid: cells of edge rc, indices taken modulo n
            const double f = floor(p[a] * cg.inv_extent[a]);
            const long long v = (long long)fmod(f, (double)cg.n[a]);
            c[a] = (int)((v + cg.n[a]) % cg.n[a]);
        }
    }
    return (c[2] * cg.n[1] + c[1]) * cg.n[0] + c[0];
}

}  // namespace

__global__ void k_cloud(const double* __restrict__ xyz, const int* __restrict__ first_index,
                        const int* __restrict__ members, int nmem, BoxParams bp, CellGrid cg,
                        double* __restrict__ cloud, int* __restrict__ cell_of, int* __restrict__ copy_dir) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nmem) return;
    int dir;
    cell_of[q] = cloud_point(xyz, first_index, members[q], q, bp, cg, cloud, dir);
    copy_dir[q] = dir;
}

__global__ void k_cloud_batch(const double* __restrict__ xyz, const int* __restrict__ first_index, int nmem,
                              const int* __restrict__ conf_of, const BatchGrid* __restrict__ grids,
                              double* __restrict__ cloud, int* __restrict__ cell_of, int* __restrict__ copy_dir) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nmem) return;
    const BatchGrid& G = grids[conf_of[q]];
    int dir;
    cell_of[q] = G.cell_off + cloud_point(xyz, first_index, q, q, G.bp, G.cg, cloud, dir);
    copy_dir[q] = dir;
}


__global__ void k_cell_count(const int* __restrict__ cell_of, int nmem, int* __restrict__ cell_count) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < nmem) atomicAdd(cell_count + cell_of[q], 1);
}

// Exclusive scan of the cell counts in one block (cell grids here are small).
__global__ void k_cell_scan(const int* __restrict__ cell_count, int ncell, int* __restrict__ cell_start,
                            int* __restrict__ cell_fill) {
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < ncell; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < ncell ? cell_count[i] : 0;
        int x = v;
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[w] = x;
        __syncthreads();
        if (w == 0) {
            int s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            warp_sums[lane] = s;
        }
        __syncthreads();
        const int excl = carry + (w ? warp_sums[w - 1] : 0) + x - v;
        if (i < ncell) {
            cell_start[i] = excl;
            cell_fill[i] = excl;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) cell_start[ncell] = carry;
}

__global__ void k_cell_fill(const int* __restrict__ cell_of, int nmem, int* __restrict__ cell_fill,
                            int* __restrict__ cell_items) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < nmem) cell_items[atomicAdd(cell_fill + cell_of[q], 1)] = q;
}

// The items of every cell in ascending order (k_cell_fill places them in
// atomic order): the neighbour lists, and with them the slot order of every
// n-mer, are then the same from run to run.  One warp per cell; an item's
// place is the number of smaller items of its cell (all items differ).
__global__ void k_cell_sort(const int* __restrict__ cell_start, int ncell, const int* __restrict__ items,
                            int* __restrict__ sorted) {
    const int lane = threadIdx.x & 31;
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= ncell) return;
    const int b = cell_start[c], n = cell_start[c + 1] - b;
    for (int i0 = 0; i0 < n; i0 += 32) {
        const int i = i0 + lane;
        const int v = i < n ? items[b + i] : 0;
        int rank = 0;
        for (int j = 0; j < n; ++j) rank += items[b + j] < v;
        if (i < n) sorted[b + rank] = v;
    }
}

// Matches of one query monomer: NW warps of a block split the 27 surrounding
// cells (each warp a contiguous run of them, in the order below), stage their
// hits in shared memory and write them out in cell order, so the list is the
// same as a single warp scanning all cells.  A query with more than `cap`
// matches sets MBX_STATUS_NB_OVERFLOW and its count in status[1].
namespace {

template <int NW, int U>
__device__ __forceinline__ void neighbors_block(const double* __restrict__ cloud, const int* __restrict__ copy_dir,
                            const int* __restrict__ cell_of,
                            const int* __restrict__ cell_start, const int* __restrict__ cell_items,
                            const int* __restrict__ query, int nquery, const CellGrid& cg, int use_pbc,
                            int cell_off, double rc2, int cap, int* __restrict__ nb_count, NbEntry* __restrict__ nb,
                            int* __restrict__ status, NbEntry* stage, int* wcount) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int wq = blockIdx.x;
    if (wq >= nquery) return;
    const int qi = query[wq];
    const double* pi = cloud + (size_t)qi * 24;
    const double x0 = pi[0], x1 = pi[1], x2 = pi[2];
    const int c = cell_of[qi] - cell_off;   // the cell in the query's own grid
    const int cx = c % cg.n[0], cy = (c / cg.n[0]) % cg.n[1], cz = c / (cg.n[0] * cg.n[1]);
    // neighbouring cells; an axis with fewer than 3 cells is scanned once
    const int rx = cg.n[0] >= 3 ? 1 : 0, ry = cg.n[1] >= 3 ? 1 : 0, rz = cg.n[2] >= 3 ? 1 : 0;
    const int sx = cg.n[0] >= 3 ? 3 : cg.n[0], sy = cg.n[1] >= 3 ? 3 : cg.n[1], sz = cg.n[2] >= 3 ? 3 : cg.n[2];
    const int ncell = sx * sy * sz;
    const int k0 = w * ncell / NW, k1 = (w + 1) * ncell / NW;
    const int ncopy = use_pbc ? 8 : 1;
    // One copy per member (cg.one_copy): a point within the cutoff of the
    // query lies in the 3 x 3 x 3 block of cells around it in real space
    // (every cell is wider than the cutoff), so a member of a scanned cell can
    // only match through the copy that moves it into that block, the one the
    // cell's wrap names (-1 / 0 / +1 box per axis); if the member has no copy
    // in that direction, it cannot match at all.  The hits, and their order,
    // are those of the full eight-point test.
    const bool one = use_pbc && cg.one_copy;
    const int npts = one ? 1 : ncopy;
    // cloud category of a shift pattern (x, y, z shifted) -> copy index (k_cloud's order)
    const int cat_of[8] = {0, 1, 2, 5, 3, 6, 7, 4};
    NbEntry* mine = stage + (size_t)w * cap;
    int count = 0;
    for (int k = k0; k < k1; ++k) {
        const int dx = k % sx, dy = (k / sx) % sy, dz = k / (sx * sy);
        // periodic in index space both with PBC and for the hashed grid
        // without PBC (n >= 3 there, so the 27 cells are distinct)
        int ax = rx ? cx + dx - 1 : dx, ay = ry ? cy + dy - 1 : dy, az = rz ? cz + dz - 1 : dz;
        // wrap of the cell in real space (one-copy mode: n >= 3, rx = ry = rz = 1)
        const int tx = ax < 0 ? -1 : (ax >= cg.n[0] ? 1 : 0);
        const int ty = ay < 0 ? -1 : (ay >= cg.n[1] ? 1 : 0);
        const int tz = az < 0 ? -1 : (az >= cg.n[2] ? 1 : 0);
        const int need = (tx != 0 ? 1 : 0) | (ty != 0 ? 2 : 0) | (tz != 0 ? 4 : 0);   // axes that must be shifted
        const int dirs = (tx > 0 ? 1 : 0) | (ty > 0 ? 2 : 0) | (tz > 0 ? 4 : 0);       // and their directions
        const int cat = cat_of[(tx != 0 ? 4 : 0) | (ty != 0 ? 2 : 0) | (tz != 0 ? 1 : 0)];
        ax = (ax + cg.n[0]) % cg.n[0];
        ay = (ay + cg.n[1]) % cg.n[1];
        az = (az + cg.n[2]) % cg.n[2];
        const int cell = cell_off + (az * cg.n[1] + ay) * cg.n[0] + ax;
        const int b = cell_start[cell], e = cell_start[cell + 1];
        // the cell's items in chunks of 32 (one load per lane, then shuffled);
        // its (item, copy) points in item-major order, lanes over consecutive
        // points (coalesced cloud loads), U independent 32-point blocks at a time
        for (int c0 = b; c0 < e; c0 += 32) {
            const int nit = e - c0 < 32 ? e - c0 : 32;
            const int my_item = lane < nit ? cell_items[c0 + lane] : 0;
            const int total = nit * npts;
            for (int base = 0; base < total; base += 32 * U) {
                bool hit[U];
                NbEntry ent[U];
#pragma unroll
                for (int h = 0; h < U; ++h) {
                    const int t = base + 32 * h + lane;
                    const int it = t < total ? t / npts : 0;
                    const int qj = __shfl_sync(0xffffffffu, my_item, it);
                    const bool ok = t < total && (!one || (copy_dir[qj] & need) == dirs);
                    hit[h] = false;
                    if (ok) {
                        const int s = one ? cat : t - it * npts;
                        const double* pj = cloud + (size_t)qj * 24 + 3 * s;
                        const double d2 = dist2_rn(x0, x1, x2, pj[0], pj[1], pj[2]);
                        if (d2 < rc2) {
                            hit[h] = true;
                            ent[h].member = qj;
                            ent[h].copy = s;
                            ent[h].d2 = d2;
                        }
                    }
                }
#pragma unroll
                for (int h = 0; h < U; ++h) {
                    const unsigned m = __ballot_sync(0xffffffffu, hit[h]);
                    if (hit[h]) {
                        const int pos = count + __popc(m & ((1u << lane) - 1u));
                        if (pos < cap) mine[pos] = ent[h];
                    }
                    count += __popc(m);
                }
            }
        }
    }
    if (lane == 0) wcount[w] = count;
    __syncthreads();
    int off = 0, total = 0;
    for (int j = 0; j < NW; ++j) {
        off += j < w ? wcount[j] : 0;
        total += wcount[j];
    }
    NbEntry* out = nb + (size_t)wq * cap;
    const int lim = count < cap ? count : cap;
    for (int i = lane; i < lim && off + i < cap; i += 32) out[off + i] = mine[i];
    if (threadIdx.x == 0) {
        nb_count[wq] = total < cap ? total : cap;
        if (total > cap) {
            atomicOr(status, MBX_STATUS_NB_OVERFLOW);
            atomicMax(status + 1, total);
        }
    }
}

}  // namespace

template <int NW, int U>
__global__ void __launch_bounds__(NW * 32) k_neighbors(const double* __restrict__ cloud,
                                                       const int* __restrict__ copy_dir,
                                                       const int* __restrict__ cell_of,
                                                       const int* __restrict__ cell_start,
                                                       const int* __restrict__ cell_items,
                                                       const int* __restrict__ query, int nquery, CellGrid cg,
                                                       int use_pbc, double rc2, int cap, int* __restrict__ nb_count,
                                                       NbEntry* __restrict__ nb, int* __restrict__ status) {
    extern __shared__ unsigned char smem[];
    __shared__ int wcount[NW];
    neighbors_block<NW, U>(cloud, copy_dir, cell_of, cell_start, cell_items, query, nquery, cg, use_pbc, 0, rc2, cap,
                           nb_count, nb, status, reinterpret_cast<NbEntry*>(smem), wcount);
}

// The same over a batch: each query searches its own configuration's grid.
template <int NW, int U>
__global__ void __launch_bounds__(NW * 32) k_neighbors_batch(const double* __restrict__ cloud,
                                                             const int* __restrict__ copy_dir,
                                                             const int* __restrict__ cell_of,
                                                             const int* __restrict__ cell_start,
                                                             const int* __restrict__ cell_items,
                                                             const int* __restrict__ query, int nquery,
                                                             const int* __restrict__ conf_of,
                                                             const BatchGrid* __restrict__ grids, double rc2, int cap,
                                                             int* __restrict__ nb_count, NbEntry* __restrict__ nb,
                                                             int* __restrict__ status) {
    extern __shared__ unsigned char smem[];
    __shared__ int wcount[NW];
    if (blockIdx.x >= nquery) return;
    const BatchGrid& G = grids[conf_of[query[blockIdx.x]]];
    neighbors_block<NW, U>(cloud, copy_dir, cell_of, cell_start, cell_items, query, nquery, G.cg, G.bp.use_pbc,
                           G.cell_off, rc2, cap, nb_count, nb, status, reinterpret_cast<NbEntry*>(smem), wcount);
}

// Host side: one block of `warps` warps per query (1 or 4), U = `unroll`
// independent 32-point blocks per iteration (1, 2 or 4); the hits of each
// warp are staged in warps x cap NbEntry of dynamic shared memory.
int launch_neighbors(int warps, int unroll, const double* cloud, const int* copy_dir, const int* cell_of,
                     const int* cell_start, const int* cell_items, const int* query, int nquery, CellGrid cg,
                     int use_pbc, double rc2, int cap, int* nb_count, NbEntry* nb, int* status, cudaStream_t s) {
    if (nquery <= 0) return 0;
    const size_t smem = (size_t)warps * cap * sizeof(NbEntry);
    if (smem > 227 * 1024) return (int)cudaErrorInvalidValue;
#define MBX_NB_CASE(NW, UU)                                                                                      \
    if (warps == NW && unroll == UU) {                                                                           \
        if (smem > 48 * 1024) {                                                                                  \
            cudaError_t e = cudaFuncSetAttribute(k_neighbors<NW, UU>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                                 (int)smem);                                                    \
            if (e != cudaSuccess) return (int)e;                                                                 \
        }                                                                                                        \
        k_neighbors<NW, UU><<<nquery, NW * 32, smem, s>>>(cloud, copy_dir, cell_of, cell_start, cell_items, query, \
                                                           nquery,                                                \
                                                           cg, use_pbc, rc2, cap, nb_count, nb, status);          \
        return (int)cudaGetLastError();                                                                          \
    }
    MBX_NB_CASE(4, 1)
    MBX_NB_CASE(4, 2)
    MBX_NB_CASE(4, 4)
    MBX_NB_CASE(1, 1)
    MBX_NB_CASE(1, 2)
    MBX_NB_CASE(1, 4)
#undef MBX_NB_CASE
    return (int)cudaErrorInvalidValue;
}

int launch_neighbors_batch(int warps, int unroll, const double* cloud, const int* copy_dir, const int* cell_of,
                           const int* cell_start,
                           const int* cell_items, const int* query, int nquery, const int* conf_of,
                           const BatchGrid* grids, double rc2, int cap, int* nb_count, NbEntry* nb, int* status,
                           cudaStream_t s) {
    if (nquery <= 0) return 0;
    const size_t smem = (size_t)warps * cap * sizeof(NbEntry);
    if (smem > 227 * 1024) return (int)cudaErrorInvalidValue;
#define MBX_NB_CASE(NW, UU)                                                                                      \
    if (warps == NW && unroll == UU) {                                                                           \
        if (smem > 48 * 1024) {                                                                                  \
            cudaError_t e = cudaFuncSetAttribute(k_neighbors_batch<NW, UU>,                                      \
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);       \
            if (e != cudaSuccess) return (int)e;                                                                 \
        }                                                                                                        \
        k_neighbors_batch<NW, UU><<<nquery, NW * 32, smem, s>>>(cloud, copy_dir, cell_of, cell_start, cell_items, \
                                                                 query,                                          \
                                                                 nquery, conf_of, grids, rc2, cap, nb_count, nb, \
                                                                 status);                                        \
        return (int)cudaGetLastError();                                                                          \
    }
    MBX_NB_CASE(4, 1)
    MBX_NB_CASE(4, 2)
    MBX_NB_CASE(4, 4)
    MBX_NB_CASE(1, 1)
    MBX_NB_CASE(1, 2)
    MBX_NB_CASE(1, 4)
#undef MBX_NB_CASE
    return (int)cudaErrorInvalidValue;
}

namespace {

// A match of a trimer query staged in shared memory: its cloud point, the
// squared distance to the query, the member index and its monomer, tag, type.
struct TriMatch {
    double p[3];
    double d2;
    int member, m, tag, type;
};
static_assert(sizeof(TriMatch) == MBX_TRIMATCH_BYTES, "TriMatch layout");

// One slot per lane that wants one, in counters[key]: lanes with the same key
// share one atomicAdd.  Called by all 32 lanes of the warp.
__device__ __forceinline__ int warp_reserve(int* counters, int key, bool want) {
    const int lane = threadIdx.x & 31;
    const unsigned act = __ballot_sync(0xffffffffu, want);
    int pos = -1;
    if (want) {
        const unsigned peers = __match_any_sync(act, key);
        const int leader = __ffs(peers) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(counters + key, __popc(peers));
        base = __shfl_sync(peers, base, leader);
        pos = base + __popc(peers & ((1u << lane) - 1u));
    }
    return pos;
}

// Same for one 64-bit counter.
__device__ __forceinline__ long long warp_reserve_ull(unsigned long long* counter, bool want) {
    const int lane = threadIdx.x & 31;
    const unsigned act = __ballot_sync(0xffffffffu, want);
    unsigned long long base = 0;
    if (lane == 0 && act) base = atomicAdd(counter, (unsigned long long)__popc(act));
    base = __shfl_sync(0xffffffffu, base, 0);
    return want ? (long long)(base + __popc(act & ((1u << lane) - 1u))) : -1;
}

}  // namespace

// Dimers from the matches: (i, j) with d^2 < rc2 and tag_i < tag_j.  One warp
// per query monomer, lanes over its matches.
__global__ void k_dimers(const int* __restrict__ query, int nquery, const int* __restrict__ members,
                         const int* __restrict__ tag, const int* __restrict__ type, const int* __restrict__ nb_count,
                         const NbEntry* __restrict__ nb, int cap, double rc2, DimerRules R,
                         unsigned long long* __restrict__ listed, int4* __restrict__ list, long list_cap,
                         int4* __restrict__ bucket_data, int* __restrict__ bucket_count,
                         int* __restrict__ status) {
    const int lane = threadIdx.x & 31;
    const int wq = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wq >= nquery) return;
    const int qi = query[wq];
    const int mi = members[qi];
    const int ti = tag[mi];
    const int n = nb_count[wq];
    const NbEntry* e = nb + (size_t)wq * cap;
    unsigned long long mine = 0;
    for (int base = 0; base < n; base += 32) {
        const int a = base + lane;
        bool keep = false;
        int mj = 0, b = -1;
        double d2 = 0.0;
        if (a < n) {
            const NbEntry ea = e[a];
            d2 = ea.d2;
            mj = members[ea.member];
            keep = d2 < rc2 && ti < tag[mj];
        }
        mine += keep;
        if (list) {
            const long long pos = warp_reserve_ull(listed + 1, keep);
            if (keep && pos < list_cap) list[pos] = make_int4(mi, mj, -1, 0);
        }
        int code = 0;
        if (keep) {
            code = type[mi] * MBX_MAX_TYPES + type[mj];
            b = R.bucket[code];
            if (b >= 0 && d2 > R.pre2[b]) b = -1;   // cannot pass the evaluator's own cutoff
            if (b >= 0 && d2 < R.split2[b]) b = R.near[b];   // mixed mode: short-range share
        }
        const bool ins = b >= 0;
        const int pos = warp_reserve(bucket_count, ins ? b : 0, ins);
        if (ins) {
            if (pos < R.cap[b]) {
                bucket_data[R.offset[b] + pos] = R.swap[code] ? make_int4(mj, mi, -1, 1) : make_int4(mi, mj, -1, 0);
            } else {
                atomicOr(status, MBX_STATUS_BUCKET_OVERFLOW);
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if (lane == 0 && mine) atomicAdd(listed, mine);
}

// Trimers: a block of warps per query monomer i.  Its matches within rc are
// staged in shared memory with everything the rules read (cloud point,
// member, tag, type), then the block's lanes run over the pairs of matches.
__global__ void __launch_bounds__(256) k_trimers(const int* __restrict__ query, int nquery,
                          const int* __restrict__ members,
                          const int* __restrict__ tag, const int* __restrict__ type, const double* __restrict__ cloud,
                          const int* __restrict__ nb_count, const NbEntry* __restrict__ nb, int cap, double rc2,
                          TrimerRules R, unsigned long long* __restrict__ listed, int4* __restrict__ list,
                          long list_cap, int4* __restrict__ bucket_data, int* __restrict__ bucket_count,
                          int* __restrict__ status) {
    extern __shared__ unsigned char smem[];
    TriMatch* sh = reinterpret_cast<TriMatch*>(smem);
    __shared__ int s_n;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int wq = blockIdx.x;
    if (wq >= nquery) return;
    const int qi = query[wq];
    const int mi = members[qi];
    const int ti = tag[mi];
    if (w == 0) {
        // compact this query's matches with d^2 < rc2 (other monomers only)
        const int n0 = nb_count[wq];
        const NbEntry* e = nb + (size_t)wq * cap;
        int n = 0;
        for (int base = 0; base < n0; base += 32) {
            const int a = base + lane;
            bool keep = false;
            NbEntry ea;
            if (a < n0) {
                ea = e[a];
                keep = ea.d2 < rc2 && ea.member != qi;
            }
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                TriMatch t;
                const double* p = cloud + (size_t)ea.member * 24 + 3 * ea.copy;
                t.p[0] = p[0];
                t.p[1] = p[1];
                t.p[2] = p[2];
                t.d2 = ea.d2;
                t.member = ea.member;
                t.m = members[ea.member];
                t.tag = tag[t.m];
                t.type = type[t.m];
                sh[n + __popc(m & ((1u << lane) - 1u))] = t;
            }
            n += __popc(m);
        }
        if (lane == 0) s_n = n;
    }
    __syncthreads();
    const int n = s_n;
    const long npair = (long)n * (n - 1) / 2;
    unsigned long long mine = 0;
    for (long base = 32L * w; base < npair; base += blockDim.x) {
        const long p = base + lane;
        bool keep = false;
        int mj = 0, mk = 0, bk = -1, code = 0;
        if (p < npair) {
            // pair index -> (a, b), a < b
            int a = (int)((2.0 * n - 1 - sqrt((2.0 * n - 1) * (2.0 * n - 1) - 8.0 * p)) / 2.0);
            if (a < 0) a = 0;
            while ((long)(a + 1) * (2 * n - a - 2) / 2 <= p) ++a;
            while ((long)a * (2 * n - a - 1) / 2 > p) --a;
            const int b = (int)(p - (long)a * (2 * n - a - 1) / 2) + a + 1;
            const TriMatch& ea = sh[a];
            const TriMatch& eb = sh[b];
            if (ea.member != eb.member) {
                const double djk = dist2_rn(ea.p[0], ea.p[1], ea.p[2], eb.p[0], eb.p[1], eb.p[2]);
                mj = ea.m;
                mk = eb.m;
                keep = djk > rc2 || (ti < ea.tag && ti < eb.tag);
                if (keep) {
                    code = (type[mi] * MBX_MAX_TYPES + ea.type) * MBX_MAX_TYPES + eb.type;
                    bk = R.bucket[code];
                    if (bk >= 0) {
                        // pre-filter with the evaluator's skip rule on the cloud distances
                        const double rf2 = R.pre2[bk];
                        const int nfar = (ea.d2 > rf2) + (eb.d2 > rf2) + (djk > rf2);
                        if ((R.skip[bk] == 1 && nfar >= 2) || (R.skip[bk] == 2 && nfar == 3)) bk = -1;
                    }
                }
            }
        }
        mine += keep;
        if (list) {
            const long long pos = warp_reserve_ull(listed + 1, keep);
            if (keep && pos < list_cap) list[pos] = make_int4(mi, mj, mk, 0);
        }
        const bool ins = bk >= 0;
        const int pos = warp_reserve(bucket_count, ins ? bk : 0, ins);
        if (ins) {
            if (pos < R.cap[bk]) {
                const int perm = R.perm[code];   // slot s of the holder takes original slot (perm >> 2s) & 3
                const int orig[3] = {mi, mj, mk};
                const int s0 = perm & 3, s1 = (perm >> 2) & 3, s2 = (perm >> 4) & 3;
                int anchor = 0;
                if (s1 == 0) anchor = 1;
                if (s2 == 0) anchor = 2;
                bucket_data[R.offset[bk] + pos] = make_int4(orig[s0], orig[s1], orig[s2], anchor);
            } else {
                atomicOr(status, MBX_STATUS_BUCKET_OVERFLOW);
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if (lane == 0 && mine) atomicAdd(listed, mine);
}
