// Device octree construction: Box, Morton keys, adaptive refinement, and the
// lists the evaluation needs -- all on the GPU.
//
// Refinement reproduces OctreeNode::refine (partition.hpp:47-61, 93-143)
// level-synchronously: at level l every node with more than max_ppn points
// (and l < max_level) is split by a STABLE partition of its point segment on
// the 3-bit child digit of the level-20 Morton key.  Starting from the
// identity order and partitioning stably at every level leaves each leaf's
// points in ascending original index -- the order the reference's
// sort-by-(key, index) subdivide produces -- and children in Morton order,
// so node keys per level come out sorted (the reference's _c_node).
//
// Per level: tiles of 2048 points (a segment owns >= 1 tile), digit
// histograms per tile, one exclusive scan over the [digit][tile] table,
// per-node child counts, then a stable scatter (warp match + inter-warp
// prefix) that writes points of still-splitting children to the next work
// buffer and points of new leaves straight to the final order.
//
// By default every level, the colleague lists and the leaf numbering run in
// ONE cooperative launch (k_refine) whose steps are separated by grid
// barriers; the per-level launch chain (k_ntiles ... k_scatter, k_colleagues,
// k_leafflag / k_leafids) is the fallback for devices without cooperative
// launch, and both give the same tree bit for bit.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "fmm_internal.cuh"

namespace sfmm {
namespace {

constexpr int kTileThreads = 256;
constexpr int kTileItems = 8;
constexpr int kTile = kTileThreads * kTileItems;
constexpr int kBoxBlocks = 1024;

struct I3 { int x, y, z; };

__device__ __host__ inline I3 key_ijk(uint64_t k)
{
    return {static_cast<int>(compact3(k)), static_cast<int>(compact3(k >> 1)), static_cast<int>(compact3(k >> 2))};
}

__device__ inline int slot_of(int dx, int dy, int dz) { return (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1); }

// ------------------------------------------------------------------ box
__global__ void k_minmax(const double* __restrict__ xyz, int64_t n, BoxDev b, double* __restrict__ partial)
{
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        double r[3];
        box_rotate(b, xyz + 3 * i, r);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lo[a] = fmin(lo[a], r[a]);
            hi[a] = fmax(hi[a], r[a]);
        }
    }
    __shared__ double s[6][32];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        for (int a = 0; a < 3; ++a) { s[a][w] = lo[a]; s[3 + a][w] = hi[a]; }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int nw = blockDim.x >> 5;
        double v = s[threadIdx.x][0];
        for (int k = 1; k < nw; ++k) v = threadIdx.x < 3 ? fmin(v, s[threadIdx.x][k]) : fmax(v, s[threadIdx.x][k]);
        partial[blockIdx.x * 6 + threadIdx.x] = v;
    }
}

// box.hpp:96-106 evaluated with the same double operations, after the block
// partials are reduced by the whole block (min / max: exact in any order).
constexpr int kBoxFinalThreads = 256;
__global__ void __launch_bounds__(kBoxFinalThreads) k_box_final(const double* __restrict__ partial, int nb, BoxDev b,
                                                                BoxDev* out)
{
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = threadIdx.x; k < nb; k += blockDim.x)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lo[a] = fmin(lo[a], partial[6 * k + a]);
            hi[a] = fmax(hi[a], partial[6 * k + 3 + a]);
        }
    __shared__ double s[6][kBoxFinalThreads / 32];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        for (int a = 0; a < 3; ++a) {
            s[a][w] = lo[a];
            s[3 + a][w] = hi[a];
        }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int k = 1; k < static_cast<int>(blockDim.x >> 5); ++k)
        for (int a = 0; a < 3; ++a) {
            lo[a] = fmin(lo[a], s[a][k]);
            hi[a] = fmax(hi[a], s[3 + a][k]);
        }
    double dl[3], c[3];
    for (int a = 0; a < 3; ++a) {
        dl[a] = hi[a] - lo[a];
        c[a] = (hi[a] + lo[a]) / 2;
    }
    double dmax = dl[0];
    dmax = dmax > dl[1] ? dmax : dl[1];
    dmax = dmax > dl[2] ? dmax : dl[2];
    const double margin = 1 + 2 * 1e-3;
    double width = margin * dl[2];
    b.status = FMM_OK;
    if (!(width > 0) && dmax > 0) {
        b.status = FMM_ERR_DEGENERATE_INPUT;   // the reference's doubling loop never ends
    } else {
        while (width < dmax) {
            c[2] += width / 2;
            width *= 2;
        }
    }
    b.width = width;
    for (int a = 0; a < 3; ++a) b.corner[a] = c[a] - width / 2;
    *out = b;
}

// box.hpp:58-63 + 119-122 at level 20; coarser keys are shifts of it
// (truncating u * 2^l is exact for a power of two scale).
__global__ void k_keys(const double* __restrict__ xyz, int64_t n, const BoxDev* __restrict__ bp,
                       uint64_t* __restrict__ key, int32_t* __restrict__ ord)
{
    const BoxDev b = *bp;
    const int imax = (1 << kKeyLevel) - 1;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        double r[3];
        box_rotate(b, xyz + 3 * i, r);
        uint64_t k = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double u = (r[a] - b.corner[a]) / b.width;
            int ia = __double2int_rz(u * double(1 << kKeyLevel));
            ia = ia < 0 ? 0 : (ia > imax ? imax : ia);
            k |= spread3(static_cast<uint32_t>(ia)) << a;
        }
        key[i] = k;
        ord[i] = static_cast<int32_t>(i);
    }
}

__global__ void k_iota(int32_t* a, int64_t n)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        a[i] = static_cast<int32_t>(i);
}

// ------------------------------------------------------------------ refinement
__device__ inline int find_seg(const int32_t* __restrict__ off, int S, int t)
{
    int lo = 0, hi = S - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void k_ntiles(const int32_t* __restrict__ sp, int S, const int32_t* __restrict__ pbeg,
                         const int32_t* __restrict__ pend, int32_t* __restrict__ ntile)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < S) {
        const int g = sp[s];
        ntile[s] = (pend[g] - pbeg[g] + kTile - 1) / kTile;
    }
}

__global__ void k_hist(const int32_t* __restrict__ sp, int S, const int32_t* __restrict__ tile_off, int T,
                       const int32_t* __restrict__ pbeg, const int32_t* __restrict__ pend,
                       const uint64_t* __restrict__ key, int shift, int32_t* __restrict__ hist)
{
    __shared__ int cnt[8];
    if (threadIdx.x < 8) cnt[threadIdx.x] = 0;
    __syncthreads();
    const int t = blockIdx.x;
    const int s = find_seg(tile_off, S, t);
    const int g = sp[s];
    const int b = pbeg[g] + (t - tile_off[s]) * kTile;
    const int e = min(pend[g], b + kTile);
    for (int i = b + threadIdx.x; i < e; i += blockDim.x) atomicAdd(&cnt[(key[i] >> shift) & 7], 1);
    __syncthreads();
    if (threadIdx.x < 8) hist[threadIdx.x * T + t] = cnt[threadIdx.x];
}

__global__ void k_nodestats(int S, const int32_t* __restrict__ tile_off, int T, const int32_t* __restrict__ pre,
                            int ppn, int child_may_split, int32_t* __restrict__ cnt, int32_t* __restrict__ offs,
                            int32_t* __restrict__ nch, int32_t* __restrict__ nsp)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const int f = tile_off[s], l = tile_off[s + 1];
    int off = 0, a = 0, b = 0;
    for (int d = 0; d < 8; ++d) {
        const int c = pre[d * T + l] - pre[d * T + f];
        cnt[8 * s + d] = c;
        offs[8 * s + d] = off;
        off += c;
        a += c > 0;
        b += (c > ppn && child_may_split);
    }
    nch[s] = a;
    nsp[s] = b;
}

__global__ void k_children(const int32_t* __restrict__ sp, int S, int64_t child_level_off,
                           const int32_t* __restrict__ child_base, const int32_t* __restrict__ split_base,
                           const int32_t* __restrict__ cnt, const int32_t* __restrict__ offs, int ppn, int child_may_split,
                           uint64_t* __restrict__ key, int32_t* __restrict__ pbeg, int32_t* __restrict__ pend,
                           int32_t* __restrict__ parent, int32_t* __restrict__ child_beg, int32_t* __restrict__ nchild,
                           int32_t* __restrict__ next_sp)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const int g = sp[s];
    const uint64_t k = key[g];
    const int cb = static_cast<int>(child_level_off) + child_base[s];
    int r = 0, rs = split_base[s];
    for (int d = 0; d < 8; ++d) {
        const int c = cnt[8 * s + d];
        if (!c) continue;
        const int h = cb + r++;
        key[h] = (k << 3) | uint64_t(d);
        pbeg[h] = pbeg[g] + offs[8 * s + d];
        pend[h] = pbeg[h] + c;
        parent[h] = g;
        child_beg[h] = -1;
        nchild[h] = 0;
        if (c > ppn && child_may_split) next_sp[rs++] = h;
    }
    child_beg[g] = cb;
    nchild[g] = r;
}

__global__ void __launch_bounds__(kTileThreads) k_scatter(
    const int32_t* __restrict__ sp, int S, const int32_t* __restrict__ tile_off, int T,
    const int32_t* __restrict__ pbeg, const int32_t* __restrict__ pend, const int32_t* __restrict__ pre,
    const int32_t* __restrict__ cnt, const int32_t* __restrict__ offs, int ppn, int child_may_split, int shift,
    const uint64_t* __restrict__ key_in, const int32_t* __restrict__ ord_in,
    uint64_t* __restrict__ key_out, int32_t* __restrict__ ord_out, int32_t* __restrict__ final_ord)
{
    __shared__ int base[8];
    __shared__ int splits[8];
    __shared__ int running[8];
    __shared__ int roundtot[8];
    __shared__ int wcnt[kTileThreads / 32][8];
    const int t = blockIdx.x;
    const int s = find_seg(tile_off, S, t);
    const int g = sp[s];
    const int f = tile_off[s];
    const int b = pbeg[g] + (t - f) * kTile;
    const int e = min(pend[g], b + kTile);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x < 8) {
        const int d = threadIdx.x;
        base[d] = pbeg[g] + offs[8 * s + d] + (pre[d * T + t] - pre[d * T + f]);
        splits[d] = cnt[8 * s + d] > ppn && child_may_split;
        running[d] = 0;
        for (int k = 0; k < kTileThreads / 32; ++k) wcnt[k][d] = 0;
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    for (int r = 0; r < kTileItems; ++r) {
        const int i = b + r * kTileThreads + threadIdx.x;
        const bool valid = i < e;
        uint64_t k = 0;
        int o = 0;
        int d = 8;
        if (valid) {
            k = key_in[i];
            o = ord_in[i];
            d = static_cast<int>((k >> shift) & 7);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & lt);
        if (valid && rank == 0) wcnt[w][d] = __popc(peers);
        __syncthreads();
        if (threadIdx.x < 8) {
            int run = 0;
            for (int k2 = 0; k2 < kTileThreads / 32; ++k2) {
                const int tmp = wcnt[k2][threadIdx.x];
                wcnt[k2][threadIdx.x] = run;
                run += tmp;
            }
            roundtot[threadIdx.x] = run;
        }
        __syncthreads();
        if (valid) {
            const int pos = base[d] + running[d] + wcnt[w][d] + rank;
            if (splits[d]) {
                key_out[pos] = k;
                ord_out[pos] = o;
            } else {
                final_ord[pos] = o;
            }
        }
        __syncthreads();
        if (threadIdx.x < 8) {
            running[threadIdx.x] += roundtot[threadIdx.x];
            for (int k2 = 0; k2 < kTileThreads / 32; ++k2) wcnt[k2][threadIdx.x] = 0;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ post-processing
__global__ void k_leafflag(const int32_t* __restrict__ nchild, int64_t nn, int32_t* __restrict__ flag)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nn; i += int64_t(gridDim.x) * blockDim.x)
        flag[i] = nchild[i] == 0;
}

__global__ void k_leafids(const int32_t* __restrict__ nchild, const int32_t* __restrict__ scan, int64_t nn,
                          int32_t* __restrict__ leaf_id, int32_t* __restrict__ leaf_node)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nn; i += int64_t(gridDim.x) * blockDim.x) {
        if (nchild[i] == 0) {
            leaf_id[i] = scan[i];
            leaf_node[scan[i]] = static_cast<int32_t>(i);
        } else {
            leaf_id[i] = -1;
        }
    }
}

__global__ void k_gather_points(const double* __restrict__ xyz, const int32_t* __restrict__ ord, int64_t n,
                                const BoxDev* __restrict__ bp, double* __restrict__ pts, double* __restrict__ rpts)
{
    const BoxDev b = *bp;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const double* v = xyz + 3 * int64_t(ord[i]);
        pts[i] = v[0];
        pts[n + i] = v[1];
        pts[2 * n + i] = v[2];
        if (rpts) {
            double r[3];
            box_rotate(b, v, r);
            rpts[i] = r[0];
            rpts[n + i] = r[1];
            rpts[2 * n + i] = r[2];
        }
    }
}

// Same-level neighbours (clipped 3x3x3, self included; tree.hpp:66-119) in a
// slot per offset: children of the parent's neighbours that are adjacent.
__global__ void k_colleagues(int64_t off, int64_t cnt, int level, const uint64_t* __restrict__ key,
                             const int32_t* __restrict__ parent, const int32_t* __restrict__ child_beg,
                             const int32_t* __restrict__ nchild, int32_t* __restrict__ col)
{
    const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (i >= cnt) return;
    const int64_t g = off + i;
    int32_t* my = col + 27 * g;
    for (int s = 0; s < 27; ++s) my[s] = -1;
    if (level == 0) {
        my[13] = static_cast<int32_t>(g);
        return;
    }
    const I3 me = key_ijk(key[g]);
    const int32_t* pc = col + 27 * int64_t(parent[g]);
    for (int ps = 0; ps < 27; ++ps) {
        const int P = pc[ps];
        if (P < 0) continue;
        const int cb = child_beg[P], nc = nchild[P];
        for (int c = cb; c < cb + nc; ++c) {
            const I3 o = key_ijk(key[c]);
            const int dx = o.x - me.x, dy = o.y - me.y, dz = o.z - me.z;
            if (abs(dx) <= 1 && abs(dy) <= 1 && abs(dz) <= 1) my[slot_of(dx, dy, dz)] = c;
        }
    }
}

// Parent's neighbours sorted by node index (= key order): their children
// then come out sorted too, the row order CSRP::finish gives (csr.hpp:48-56).
__device__ inline int sorted_parent_colleagues(const int32_t* __restrict__ pc, int* out)
{
    int m = 0;
    for (int s = 0; s < 27; ++s) {
        const int v = pc[s];
        if (v < 0) continue;
        int j = m++;
        while (j > 0 && out[j - 1] > v) { out[j] = out[j - 1]; --j; }
        out[j] = v;
    }
    return m;
}

// partition.hpp:283-297 / tree.hpp:122-174: children of the parent's
// neighbours that exist and are not adjacent; dijk = source - target.  A warp
// per node: lane a holds the parent's a-th neighbour in node order (= key
// order, so the children come out in the row order CSRP::finish gives,
// csr.hpp:48-56); the candidates (neighbour, child) are taken 32 at a time in
// that order and the kept ones written contiguously (ballot + prefix).
template<bool kFill>
__global__ void k_ilist(int64_t off, int64_t cnt, const uint64_t* __restrict__ key, const int32_t* __restrict__ parent,
                        const int32_t* __restrict__ child_beg, const int32_t* __restrict__ nchild,
                        const int32_t* __restrict__ col, int32_t* __restrict__ count_or_ptr,
                        int32_t* __restrict__ src, int32_t* __restrict__ code)
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < cnt; i += nw) {
        const int64_t g = off + i;
        const I3 me = key_ijk(key[g]);
        const int v = lane < 27 ? col[27 * int64_t(parent[g]) + lane] : -1;
        int rank = 0;                                  // neighbours are distinct nodes
        for (int j = 0; j < 27; ++j) {
            const int u = __shfl_sync(full, v, j);
            rank += u >= 0 && u < v;
        }
        int P = -1;                                    // the lane-th neighbour in node order
        for (int j = 0; j < 27; ++j) {
            const int u = __shfl_sync(full, v, j), r = __shfl_sync(full, rank, j);
            if (u >= 0 && r == lane) P = u;
        }
        const int m = __popc(__ballot_sync(full, v >= 0));
        int cb = 0, nc = 0;
        if (lane < m) {
            cb = child_beg[P];
            nc = nchild[P];
        }
        int pos = kFill ? count_or_ptr[g] : 0;
        for (int j0 = 0; j0 < 8 * m; j0 += 32) {
            const int j = j0 + lane, a = (j >> 3) & 31, ci = j & 7;
            const int cbj = __shfl_sync(full, cb, a), ncj = __shfl_sync(full, nc, a);
            bool take = false;
            int c = 0, cd = 0;
            if ((j >> 3) < m && ci < ncj) {
                c = cbj + ci;
                const I3 o = key_ijk(key[c]);
                const int dx = o.x - me.x, dy = o.y - me.y, dz = o.z - me.z;
                take = abs(dx) > 1 || abs(dy) > 1 || abs(dz) > 1;
                cd = (dx + 3) | ((dy + 3) << 3) | ((dz + 3) << 6);
            }
            const unsigned tm = __ballot_sync(full, take);
            if (kFill && take) {
                const int r = pos + __popc(tm & lt);
                src[r] = c;
                code[r] = cd;
            }
            pos += __popc(tm);
        }
        if (!kFill && lane == 0) count_or_ptr[g] = pos;
    }
}

// Near-field source point ranges of one leaf: the point sets of its _nlist
// row (partition.hpp:343-366) -- leaves among every ancestor's neighbours,
// and the whole subtree of every same-level neighbour (self included).  A
// warp per leaf, a lane per neighbour slot: ranges are kept in slot order,
// ancestors from the parent up, then the leaf's own neighbours.
template<bool kFill>
__global__ void k_near(int64_t n_leaves, const int32_t* __restrict__ leaf_node, const int32_t* __restrict__ parent,
                       const int32_t* __restrict__ nchild, const int32_t* __restrict__ pbeg,
                       const int32_t* __restrict__ pend, const int32_t* __restrict__ col,
                       int32_t* __restrict__ count_or_ptr, int2* __restrict__ ranges, unsigned long long* __restrict__ pairs)
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t f = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; f < n_leaves; f += nw) {
        const int g = leaf_node[f];
        int pos = kFill ? count_or_ptr[f] : 0;
        long long npts = 0;
        // ancestors (take their leaf neighbours), then the leaf itself (all)
        for (int a = parent[g], self = 0; a >= 0 || !self;) {
            const int node = a >= 0 ? a : g;
            const int c = lane < 27 ? col[27 * int64_t(node) + lane] : -1;
            int b = 0, e = 0;
            bool take = false;
            if (c >= 0) {
                b = pbeg[c];
                e = pend[c];
                take = a < 0 || nchild[c] == 0;
            }
            const unsigned tm = __ballot_sync(full, take);
            if (kFill && take) ranges[pos + __popc(tm & lt)] = make_int2(b, e);
            if (take) npts += e - b;
            pos += __popc(tm);
            if (a >= 0) a = parent[a];
            else self = 1;
        }
        if (!kFill) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) npts += __shfl_xor_sync(full, npts, o);
            if (lane == 0) {
                count_or_ptr[f] = pos;
                const long long t = pend[g] - pbeg[g];
                atomicAdd(pairs, static_cast<unsigned long long>(t * npts - t));
            }
        }
    }
}

// ------------------------------------------------------------------ nlist export
__device__ inline int lower_bound_u64(const uint64_t* __restrict__ a, int n, uint64_t v)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

struct LevelTabs {
    int64_t lvl_off[kKeyLevel + 2];
    int64_t leaf_off[kKeyLevel + 2];
    int depth;
};

// One row of the reference's _nlist: (level, leaf) pairs sorted by level,
// then leaf (partition.hpp:343-366 with CSRP row sorting).
template<bool kFill>
__global__ void k_nlist(int level, LevelTabs L, const uint64_t* __restrict__ key, const int32_t* __restrict__ parent,
                        const int32_t* __restrict__ nchild, const int32_t* __restrict__ leaf_node,
                        const int32_t* __restrict__ leafscan, const int32_t* __restrict__ col,
                        int32_t* __restrict__ count_or_ptr, int2* __restrict__ out)
{
    const int64_t nl = L.leaf_off[level + 1] - L.leaf_off[level];
    const int64_t f = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (f >= nl) return;
    const int g = leaf_node[L.leaf_off[level] + f];
    int pos = kFill ? count_or_ptr[f] : 0;
    int anc[kKeyLevel + 1];
    {
        int a = g;
        for (int l = level; l >= 0; --l) { anc[l] = a; a = parent[a]; }
    }
    int sorted[27];
    for (int l = 0; l < level; ++l) {
        const int m = sorted_parent_colleagues(col + 27 * int64_t(anc[l]), sorted);
        for (int k = 0; k < m; ++k) {
            const int c = sorted[k];
            if (nchild[c] == 0) {
                if (kFill) out[pos] = make_int2(l, leafscan[c] - static_cast<int>(L.leaf_off[l]));
                ++pos;
            }
        }
    }
    const int m = sorted_parent_colleagues(col + 27 * int64_t(g), sorted);
    for (int l2 = level; l2 <= L.depth; ++l2) {
        const int sh = 3 * (l2 - level);
        const uint64_t* keys = key + L.lvl_off[l2];
        const int nk = static_cast<int>(L.lvl_off[l2 + 1] - L.lvl_off[l2]);
        for (int k = 0; k < m; ++k) {
            const uint64_t kc = key[sorted[k]];
            const int lo = lower_bound_u64(keys, nk, kc << sh);
            const int hi = lower_bound_u64(keys, nk, (kc + 1) << sh);
            const int a0 = leafscan[L.lvl_off[l2] + lo], a1 = leafscan[L.lvl_off[l2] + hi];
            for (int q = a0; q < a1; ++q) {
                if (kFill) out[pos] = make_int2(l2, q - static_cast<int>(L.leaf_off[l2]));
                ++pos;
            }
        }
    }
    if (!kFill) count_or_ptr[f] = pos;
}

// ------------------------------------------------------------------ single-launch refinement
// The refinement above, the colleague lists and the leaf numbering in ONE
// cooperative launch (every block resident at once), the steps separated by
// grid barriers instead of kernel boundaries and host reads of counts.  Per
// level (S splitting nodes in `sp`, T tiles of at most kWTile points):
//   A  colleagues of the level's nodes; tile counts of the splitting nodes,
//      one partial sum per block over its contiguous range of nodes
//   B  tile offsets (each block adds up the partials before its range); T
//   C  digit histogram of every tile (a warp per tile, tiles in contiguous
//      ranges per block), the block's per-digit totals, and per-node digit
//      counts by integer atomics (exact whatever the order)
//   D  per-digit exclusive prefixes over the tiles (the [digit][tile] scan of
//      the level path, row by row); child counts per node, block totals
//   E  child numbering, the children's node fields, and the stable scatter:
//      a warp takes a tile's points in index order, 32 at a time, and places
//      each after the earlier points of its digit (match + 8 ballots)
// and after the last level the leaf numbering (two steps).  The partition,
// node numbering and lists are the level path's, bit for bit.
//
// A level that needs more node slots than allocated ends the launch at its
// start with kRefGrow; the host grows the node arrays and launches again from
// that level.  Each barrier wait is bounded (%globaltimer, about two seconds,
// and an iteration cap); a wait that runs out sets an abort flag that every
// other waiting block sees, and the launch ends with kRefTimeout.
constexpr int kRefThreads = 256;
constexpr int kRefWarps = kRefThreads / 32;
constexpr int kWTile = 1024;                  // points per tile (one warp)
constexpr int kParts = 12;                    // partial sums per block
constexpr unsigned long long kBarrierNs = 2000000000ull;

enum { kRefDone = 0, kRefGrow = 1, kRefTimeout = 2, kRefOverflow = 3 };

struct RefineState {
    unsigned bar_count;
    unsigned bar_gen;
    int abort;
    int status;
    int level;                       // level whose splitting nodes come next
    int S;                           // their number
    int cur;                         // which sp / point buffers hold them
    int need;                        // children of that level (kRefGrow)
    int gate;                        // set by nothing: the wait of the stall test
    long long total;                 // nodes so far
    long long lvl_off[kKeyLevel + 3];
    int leaf_off[kKeyLevel + 3];
};

struct RefineArgs {
    uint64_t* key;
    int32_t *pbeg, *pend, *parent, *child_beg, *nchild, *col, *leaf_id, *leaf_node;
    long long cap;
    uint64_t* pkey[2];
    int32_t* pord[2];
    int32_t* final_ord;
    int32_t* sp[2];
    int32_t *tile_off, *hist, *pre, *ncnt, *offs, *nch, *nsp, *part;
    int smax, tmax;
    int max_level, ppn;
    int stall;                       // test switch: block 0 waits on `gate` (never set)
    RefineState* st;
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid barrier (sense by generation).  Returns false when this block must
// leave: its wait ran out or another block's did.
__device__ bool grid_barrier(RefineState* st)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile int* abort = &st->abort;
        if (*abort) {
            ok = 0;
        } else {
            const unsigned gen = ld_acquire_u32(&st->bar_gen);
            __threadfence();
            if (atomicAdd(&st->bar_count, 1u) == gridDim.x - 1) {
                atomicExch(&st->bar_count, 0u);
                __threadfence();
                st_release_u32(&st->bar_gen, gen + 1);
            } else {
                const unsigned long long t0 = global_ns();
                unsigned spins = 0, nap = 32;
                while (ld_acquire_u32(&st->bar_gen) == gen) {
                    if (*abort || ++spins > (1u << 25) || global_ns() - t0 > kBarrierNs) {
                        atomicExch(&st->abort, 1);
                        ok = 0;
                        break;
                    }
                    __nanosleep(nap);
                    if (nap < 256) nap *= 2;
                }
            }
            __threadfence();
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Exclusive sum over the block of one value per thread; *tot = block total.
__device__ int block_excl(int v, int* tot, int* sh)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        int y = lane < kRefWarps ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < kRefWarps; o <<= 1) {
            const int z = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += z;
        }
        if (lane < kRefWarps) sh[lane] = y;
    }
    __syncthreads();
    const int before = (w ? sh[w - 1] : 0) + x - v;
    *tot = sh[kRefWarps - 1];
    __syncthreads();
    return before;
}

__device__ int block_sum(int v, int* sh)
{
    int tot;
    block_excl(v, &tot, sh);
    return tot;
}

// Field f of the per-block partials: the sum over blocks before this one and
// over all blocks.
__device__ void parts_sums(const int32_t* part, int f, int* before, int* all, int* sh)
{
    int x = 0, y = 0;
    for (int k = threadIdx.x; k < static_cast<int>(gridDim.x); k += blockDim.x) {
        const int v = part[k * kParts + f];
        y += v;
        if (k < static_cast<int>(blockIdx.x)) x += v;
    }
    *before = block_sum(x, sh);
    *all = block_sum(y, sh);
}

__device__ __forceinline__ int tile_count(const RefineArgs& a, const int32_t* sp, int s)
{
    const int g = sp[s];
    return (a.pend[g] - a.pbeg[g] + kWTile - 1) / kWTile;
}

// first tile of the warp: binary search; later (larger) tiles: walk on
__device__ __forceinline__ int seg_of(const int32_t* tile_off, int S, int t, int s)
{
    if (s < 0) return find_seg(tile_off, S, t);
    while (s + 1 < S && tile_off[s + 1] <= t) ++s;
    return s;
}

__global__ void __launch_bounds__(kRefThreads) k_refine(RefineArgs a)
{
    __shared__ int sh[kRefWarps];
    __shared__ int s_dig[8];
    __shared__ long long s_lvl[kKeyLevel + 3];
    RefineState* st = a.st;
    const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t gthreads = int64_t(G) * kRefThreads, gtid = int64_t(b) * kRefThreads + tid;
    if (a.stall && b == 0) {
        // test of the bounded waits: block 0 never reaches the first barrier;
        // its thread 0 waits on a flag nothing sets, then raises the abort
        // that ends every other block's barrier wait
        if (tid == 0) {
            const unsigned long long t0 = global_ns();
            unsigned spins = 0;
            while (!*reinterpret_cast<volatile int*>(&st->gate)) {
                if (++spins > (1u << 25) || global_ns() - t0 > kBarrierNs) break;
                __nanosleep(256);
            }
            atomicExch(&st->abort, 1);
        }
        return;
    }
    int level = st->level, S = st->S, cur = st->cur;
    int64_t lo = st->lvl_off[level], total = st->total;
    int status = kRefDone, need = 0;

    for (;;) {
        const int32_t* sp = cur ? a.sp[1] : a.sp[0];
        int32_t* spn = cur ? a.sp[0] : a.sp[1];
        const uint64_t* kin = cur ? a.pkey[1] : a.pkey[0];
        uint64_t* kout = cur ? a.pkey[0] : a.pkey[1];
        const int32_t* oin = cur ? a.pord[1] : a.pord[0];
        int32_t* oout = cur ? a.pord[0] : a.pord[1];
        const int child_may_split = (level + 1) < a.max_level;

        // ---- A: colleagues of this level (a warp per node, a lane per
        //      neighbour of the parent); tile counts
        for (int64_t g = lo + (gtid >> 5); g < total; g += gthreads >> 5) {
            int32_t* my = a.col + 27 * g;
            if (lane < 27) my[lane] = (level == 0 && lane == 13) ? static_cast<int32_t>(g) : -1;
            if (level == 0) continue;
            __syncwarp();
            const I3 me = key_ijk(a.key[g]);
            const int P = lane < 27 ? a.col[27 * int64_t(a.parent[g]) + lane] : -1;
            if (P >= 0) {
                const int cb = a.child_beg[P], nc = a.nchild[P];
                uint64_t kc[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) kc[j] = j < nc ? a.key[cb + j] : 0;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    if (j >= nc) break;
                    const I3 o = key_ijk(kc[j]);
                    const int dx = o.x - me.x, dy = o.y - me.y, dz = o.z - me.z;
                    if (abs(dx) <= 1 && abs(dy) <= 1 && abs(dz) <= 1) my[slot_of(dx, dy, dz)] = cb + j;
                }
            }
            __syncwarp();
        }
        if (S == 0) break;
        const int cs = (S + G - 1) / G, s0 = min(S, b * cs), s1 = min(S, s0 + cs);
        {
            int mine = 0;
            for (int s = s0 + tid; s < s1; s += kRefThreads) {
                mine += tile_count(a, sp, s);
#pragma unroll
                for (int d = 0; d < 8; ++d) a.ncnt[8 * s + d] = 0;
            }
            const int tot = block_sum(mine, sh);
            if (tid == 0) a.part[b * kParts] = tot;
        }
        if (!grid_barrier(st)) return;

        // ---- B: tile offsets
        int T;
        {
            int before;
            parts_sums(a.part, 0, &before, &T, sh);
            if (T > a.tmax) {
                status = kRefOverflow;
                break;
            }
            int carry = before;
            for (int base = s0; base < s1; base += kRefThreads) {
                const int s = base + tid;
                const int v = s < s1 ? tile_count(a, sp, s) : 0;
                int tot;
                const int ex = block_excl(v, &tot, sh);
                if (s < s1) a.tile_off[s] = carry + ex;
                carry += tot;
            }
        }
        if (!grid_barrier(st)) return;

        // ---- C: digit histograms
        const int shift = 3 * (kKeyLevel - 1 - level);
        const int ct = (T + G - 1) / G, t0 = min(T, b * ct), t1 = min(T, t0 + ct);
        if (tid < 8) s_dig[tid] = 0;
        __syncthreads();
        {
            int s = -1;
            for (int t = t0 + warp; t < t1; t += kRefWarps) {
                s = seg_of(a.tile_off, S, t, s);
                const int g = sp[s];
                const int pb = a.pbeg[g] + (t - a.tile_off[s]) * kWTile;
                const int pe = min(a.pend[g], pb + kWTile);
                int c = 0;                                   // lane d < 8: points of digit d
                for (int i0 = pb; i0 < pe; i0 += 128) {
                    int dg[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int i = i0 + 32 * u + lane;
                        dg[u] = i < pe ? static_cast<int>((kin[i] >> shift) & 7) : 8;
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u)
#pragma unroll
                        for (int d = 0; d < 8; ++d) {
                            const unsigned m = __ballot_sync(0xffffffffu, dg[u] == d);
                            if (lane == d) c += __popc(m);
                        }
                }
                if (lane < 8) {
                    a.hist[int64_t(lane) * T + t] = c;
                    if (c) {
                        atomicAdd(&a.ncnt[8 * s + lane], c);
                        atomicAdd(&s_dig[lane], c);
                    }
                }
            }
        }
        __syncthreads();
        if (tid < 8) a.part[b * kParts + 1 + tid] = s_dig[tid];
        if (!grid_barrier(st)) return;

        // ---- D: per-digit tile prefixes (warp d); node statistics
        {
            const int d = warp;                               // 8 warps, one per digit
            int base = 0;
            for (int k = lane; k < b; k += 32) base += a.part[k * kParts + 1 + d];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) base += __shfl_xor_sync(0xffffffffu, base, o);
            for (int t = t0; t < t1; t += 32) {
                const int tt = t + lane;
                const int v = tt < t1 ? a.hist[int64_t(d) * T + tt] : 0;
                int x = v;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= o) x += y;
                }
                if (tt < t1) a.pre[int64_t(d) * T + tt] = base + x - v;
                base += __shfl_sync(0xffffffffu, x, 31);
            }
        }
        {
            int mc = 0, ms = 0;
            for (int s = s0 + tid; s < s1; s += kRefThreads) {
                int off = 0, nc = 0, ns = 0;
#pragma unroll
                for (int d = 0; d < 8; ++d) {
                    const int c = a.ncnt[8 * s + d];
                    a.offs[8 * s + d] = off;
                    off += c;
                    nc += c > 0;
                    ns += (c > a.ppn && child_may_split);
                }
                a.nch[s] = nc;
                a.nsp[s] = ns;
                mc += nc;
                ms += ns;
            }
            mc = block_sum(mc, sh);
            ms = block_sum(ms, sh);
            if (tid == 0) {
                a.part[b * kParts + 9] = mc;
                a.part[b * kParts + 10] = ms;
            }
        }
        if (!grid_barrier(st)) return;

        // ---- E: children and the scatter
        int NC, NS;
        {
            int cbefore, sbefore;
            parts_sums(a.part, 9, &cbefore, &NC, sh);
            parts_sums(a.part, 10, &sbefore, &NS, sh);
            if (total + NC > a.cap) {
                status = kRefGrow;
                need = NC;
                break;
            }
            if (NS > a.smax) {
                status = kRefOverflow;
                break;
            }
            int cc = cbefore, sc = sbefore;
            for (int base = s0; base < s1; base += kRefThreads) {
                const int s = base + tid;
                const int nc = s < s1 ? a.nch[s] : 0, ns = s < s1 ? a.nsp[s] : 0;
                int tc, ts;
                const int exc = block_excl(nc, &tc, sh);
                const int exs = block_excl(ns, &ts, sh);
                if (s < s1) {
                    const int g = sp[s];
                    const uint64_t k = a.key[g];
                    const int cb = static_cast<int>(total) + cc + exc;
                    int r = 0, rs = sc + exs;
                    for (int d = 0; d < 8; ++d) {
                        const int c = a.ncnt[8 * s + d];
                        if (!c) continue;
                        const int h = cb + r++;
                        a.key[h] = (k << 3) | uint64_t(d);
                        a.pbeg[h] = a.pbeg[g] + a.offs[8 * s + d];
                        a.pend[h] = a.pbeg[h] + c;
                        a.parent[h] = g;
                        a.child_beg[h] = -1;
                        a.nchild[h] = 0;
                        if (c > a.ppn && child_may_split) spn[rs++] = h;
                    }
                    a.child_beg[g] = cb;
                    a.nchild[g] = r;
                }
                cc += tc;
                sc += ts;
            }
        }
        {
            int s = -1;
            for (int t = t0 + warp; t < t1; t += kRefWarps) {
                s = seg_of(a.tile_off, S, t, s);
                const int g = sp[s];
                const int f = a.tile_off[s];
                const int pb = a.pbeg[g] + (t - f) * kWTile;
                const int pe = min(a.pend[g], pb + kWTile);
                int pos_d = 0, split_d = 0;                   // lane d < 8: next slot of digit d
                if (lane < 8) {
                    pos_d = a.pbeg[g] + a.offs[8 * s + lane] + (a.pre[int64_t(lane) * T + t] - a.pre[int64_t(lane) * T + f]);
                    split_d = a.ncnt[8 * s + lane] > a.ppn && child_may_split;
                }
                const unsigned splits = __ballot_sync(0xffffffffu, split_d);
                for (int i0 = pb; i0 < pe; i0 += 128) {
                    uint64_t kk[4];
                    int oo[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int i = i0 + 32 * u + lane;
                        kk[u] = i < pe ? kin[i] : 0;
                        oo[u] = i < pe ? oin[i] : 0;
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const bool valid = i0 + 32 * u + lane < pe;
                        const int dg = valid ? static_cast<int>((kk[u] >> shift) & 7) : 8;
                        const unsigned peers = __match_any_sync(0xffffffffu, dg);
                        const int pos = __shfl_sync(0xffffffffu, pos_d, dg & 7) + __popc(peers & lt);
                        if (valid) {
                            if ((splits >> dg) & 1u) {
                                kout[pos] = kk[u];
                                oout[pos] = oo[u];
                            } else {
                                a.final_ord[pos] = oo[u];
                            }
                        }
#pragma unroll
                        for (int d = 0; d < 8; ++d) {
                            const unsigned m = __ballot_sync(0xffffffffu, dg == d);
                            if (lane == d) pos_d += __popc(m);
                        }
                    }
                }
            }
        }
        if (b == 0 && tid == 0) st->lvl_off[level + 2] = total + NC;
        if (!grid_barrier(st)) return;
        lo = total;
        total += NC;
        ++level;
        S = NS;
        cur ^= 1;
    }

    if (status == kRefDone) {
        // ---- leaves in node order: ids, nodes, first leaf of every level
        const int64_t cn = (total + G - 1) / G, n0 = total < b * cn ? total : b * cn, n1 = total < n0 + cn ? total : n0 + cn;
        {
            int mine = 0;
            for (int64_t g = n0 + tid; g < n1; g += kRefThreads) mine += a.nchild[g] == 0;
            const int tot = block_sum(mine, sh);
            if (tid == 0) a.part[b * kParts + 11] = tot;
        }
        if (!grid_barrier(st)) return;
        int before, nleaves;
        parts_sums(a.part, 11, &before, &nleaves, sh);
        if (tid <= level + 1) s_lvl[tid] = reinterpret_cast<volatile long long*>(st->lvl_off)[tid];
        __syncthreads();
        int carry = before;
        for (int64_t base = n0; base < n1; base += kRefThreads) {
            const int64_t g = base + tid;
            const int leaf = g < n1 && a.nchild[g] == 0;
            int tot;
            const int id = carry + block_excl(leaf, &tot, sh);
            if (g < n1) {
                a.leaf_id[g] = leaf ? id : -1;
                if (leaf) a.leaf_node[id] = static_cast<int32_t>(g);
                for (int l = 0; l <= level; ++l)
                    if (s_lvl[l] == g) st->leaf_off[l] = id;
            }
            carry += tot;
        }
        if (b == 0 && tid == 0) st->leaf_off[level + 1] = nleaves;
    }
    if (b == 0 && tid == 0) {
        st->status = status;
        st->level = level;
        st->S = S;
        st->cur = cur;
        st->need = need;
        st->total = total;
    }
}

template<typename T>
std::vector<T> to_host(const T* d, size_t n, cudaStream_t s)
{
    std::vector<T> h(n);
    if (n) SFMM_CUDA(cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
    SFMM_CUDA(cudaStreamSynchronize(s));
    return h;
}

template<typename T>
T read_one(const T* d, cudaStream_t s)
{
    T v;
    SFMM_CUDA(cudaMemcpyAsync(&v, d, sizeof(T), cudaMemcpyDeviceToHost, s));
    SFMM_CUDA(cudaStreamSynchronize(s));
    return v;
}

// Two device values read back together: the stream drains once, for the first
// copy; the second follows it directly.
template<typename T>
void read_two(const T* d0, const T* d1, T& v0, T& v1, cudaStream_t s)
{
    SFMM_CUDA(cudaMemcpyAsync(&v0, d0, sizeof(T), cudaMemcpyDeviceToHost, s));
    SFMM_CUDA(cudaMemcpyAsync(&v1, d1, sizeof(T), cudaMemcpyDeviceToHost, s));
    SFMM_CUDA(cudaStreamSynchronize(s));
}

// The single-launch refinement unless SFMM_TREE_REFINE=levels asks for the
// level-by-level launches (the tests run both), the device cannot launch
// cooperatively, or the tile table would not fit 32-bit counts.
bool single_launch_refinement(int64_t n, int ppn)
{
    const char* m = std::getenv("SFMM_TREE_REFINE");
    if (m && std::strcmp(m, "levels") == 0) return false;
    int dev = 0, coop = 0;
    SFMM_CUDA(cudaGetDevice(&dev));
    SFMM_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    const int64_t smax = std::max<int64_t>(1, n / (int64_t(ppn) + 1));
    return coop && 8 * (n / kWTile + smax + 1) < (int64_t(1) << 31);
}

}  // namespace

void build_tree(Tree& t, const double* xyz, int max_level, int max_ppn, int vertical_axis, double phideg,
                const double* corner3, double width)
{
    cudaStream_t st = t.ctx->stream;
    const int64_t n = t.n;
    SFMM_REQUIRE(n > 0 && n < (int64_t(1) << 31) - 1, FMM_ERR_INVALID_ARGUMENT, "n must be in [1, 2^31 - 2]");
    SFMM_REQUIRE(vertical_axis >= 0 && vertical_axis < 3, FMM_ERR_INVALID_ARGUMENT, "vertical_axis must be 0, 1 or 2");
    SFMM_REQUIRE(max_level >= 0, FMM_ERR_INVALID_ARGUMENT, "max_level must be >= 0");
    SFMM_REQUIRE(max_ppn >= 0, FMM_ERR_INVALID_ARGUMENT, "max_particles_per_node must be >= 0");
    max_level = std::min(max_level, kKeyLevel);
    t.max_level = max_level;
    t.max_ppn = max_ppn;
    t.vertical_axis = vertical_axis;
    t.phideg = phideg;

    // events at the phase boundaries: start, keys, refinement, leaves and
    // points, colleagues, interaction lists, near-field lists (the end)
    struct Events {
        cudaEvent_t e[7] = {};
        ~Events()
        {
            for (auto& x : e)
                if (x) cudaEventDestroy(x);
        }
    } ev;
    for (auto& x : ev.e) SFMM_CUDA(cudaEventCreate(&x));
    cudaEvent_t e0 = ev.e[0], e1 = ev.e[6];
    SFMM_CUDA(cudaEventRecord(e0, st));

    // --- box (box.hpp:84-107)
    BoxDev b{};
    b.X = (vertical_axis + 1) % 3;
    b.Y = (vertical_axis + 2) % 3;
    b.Z = vertical_axis;
    const double phi = phideg * (M_PI / 180);
    b.rotated = phideg != 0.0;
    b.cphi = std::cos(phi);
    b.sphi = std::sin(phi);
    if (corner3) {
        // explicit cube: corner in the (rotated) key frame, as the reference stores it
        SFMM_REQUIRE(width > 0 && std::isfinite(width), FMM_ERR_INVALID_ARGUMENT, "box width must be positive");
        b.width = width;
        for (int a = 0; a < 3; ++a) b.corner[a] = corner3[a];
        b.status = FMM_OK;
        t.d_box.alloc(1, st);
        SFMM_CUDA(cudaMemcpyAsync(t.d_box.ptr, &b, sizeof(b), cudaMemcpyHostToDevice, st));
    } else {
        const int nb = static_cast<int>(std::min<int64_t>(kBoxBlocks, (n + 255) / 256));
        DevBuf<double> partial;
        partial.alloc(6 * nb, st);
        t.d_box.alloc(1, st);
        k_minmax<<<nb, 256, 0, st>>>(xyz, n, b, partial.ptr);
        SFMM_CHECK_LAUNCH();
        k_box_final<<<1, kBoxFinalThreads, 0, st>>>(partial.ptr, nb, b, t.d_box.ptr);
        SFMM_CHECK_LAUNCH();
    }

    // --- keys + refinement
    DevBuf<uint64_t> keyA, keyB;
    DevBuf<int32_t> ordA, ordB;
    keyA.alloc(n, st);
    keyB.alloc(n, st);
    ordA.alloc(n, st);
    ordB.alloc(n, st);
    t.order.alloc(n, st);
    k_keys<<<blocks_for(n, 256, 8192), 256, 0, st>>>(xyz, n, t.d_box.ptr, keyA.ptr, ordA.ptr);
    SFMM_CHECK_LAUNCH();
    SFMM_CUDA(cudaEventRecord(ev.e[1], st));
    t.box = read_one(t.d_box.ptr, st);
    SFMM_REQUIRE(t.box.status == FMM_OK, FMM_ERR_DEGENERATE_INPUT,
                 "all points share the vertical coordinate: the reference's box loop would never end");

    size_t cap = std::max<int64_t>(1024, n / 8);
    auto grow_nodes = [&](size_t need, size_t keep) {
        if (need <= cap && t.key.count) return;
        size_t nc = std::max(need, cap * 2);
        t.key.grow(nc, keep, st);
        t.pbeg.grow(nc, keep, st);
        t.pend.grow(nc, keep, st);
        t.parent.grow(nc, keep, st);
        t.child_beg.grow(nc, keep, st);
        t.nchild.grow(nc, keep, st);
        cap = nc;
    };
    grow_nodes(cap, 0);
    {
        const uint64_t k0 = 0;
        const int32_t z = 0, nn = static_cast<int32_t>(n), m1 = -1;
        SFMM_CUDA(cudaMemcpyAsync(t.key.ptr, &k0, 8, cudaMemcpyHostToDevice, st));
        SFMM_CUDA(cudaMemcpyAsync(t.pbeg.ptr, &z, 4, cudaMemcpyHostToDevice, st));
        SFMM_CUDA(cudaMemcpyAsync(t.pend.ptr, &nn, 4, cudaMemcpyHostToDevice, st));
        SFMM_CUDA(cudaMemcpyAsync(t.parent.ptr, &m1, 4, cudaMemcpyHostToDevice, st));
        SFMM_CUDA(cudaMemcpyAsync(t.child_beg.ptr, &m1, 4, cudaMemcpyHostToDevice, st));
        SFMM_CUDA(cudaMemcpyAsync(t.nchild.ptr, &z, 4, cudaMemcpyHostToDevice, st));
    }
    t.lvl_off.assign(1, 0);
    t.lvl_off.push_back(1);
    int64_t total = 1;

    DevBuf<int32_t> sp, sp_next;
    sp.alloc(1, st);
    const bool root_splits = n > max_ppn && 0 < max_level;
    int S = 0;
    if (root_splits) {
        const int32_t z = 0;
        SFMM_CUDA(cudaMemcpyAsync(sp.ptr, &z, 4, cudaMemcpyHostToDevice, st));
        S = 1;
    } else {
        k_iota<<<blocks_for(n, 256, 8192), 256, 0, st>>>(t.order.ptr, n);
        SFMM_CHECK_LAUNCH();
    }

    int level = 0;
    const bool single = single_launch_refinement(n, max_ppn);
    if (single) {
        // one cooperative launch: all levels, the colleague lists, the leaves
        const int64_t smax = std::max<int64_t>(1, n / (int64_t(max_ppn) + 1));
        const int64_t tmax = n / kWTile + smax + 1;
        int dev = 0, sms = 0, occ = 0;
        SFMM_CUDA(cudaGetDevice(&dev));
        SFMM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        SFMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_refine, kRefThreads, 0));
        SFMM_REQUIRE(occ > 0, FMM_ERR_UNSUPPORTED, "the refinement kernel cannot be resident");
        // two root tiles per block, at least 32 blocks (small trees: the colleague
        // and list steps are chains of dependent loads, one warp per node)
        const int G = static_cast<int>(std::min<int64_t>(int64_t(occ) * sms, std::max<int64_t>(32, (n + 2 * kWTile - 1) / (2 * kWTile))));
        DevBuf<int32_t> sp0, sp1, tile_off, hist, pre, ncnt, offs, nch, nsp, part;
        DevBuf<RefineState> dst;
        sp0.alloc(smax, st);
        sp1.alloc(smax, st);
        tile_off.alloc(smax, st);
        ncnt.alloc(8 * smax, st);
        offs.alloc(8 * smax, st);
        nch.alloc(smax, st);
        nsp.alloc(smax, st);
        hist.alloc(8 * tmax, st);
        pre.alloc(8 * tmax, st);
        part.alloc(size_t(kParts) * G, st);
        dst.alloc(1, st);
        if (S) {
            const int32_t z = 0;
            SFMM_CUDA(cudaMemcpyAsync(sp0.ptr, &z, 4, cudaMemcpyHostToDevice, st));
        }
        t.colleague.alloc(27 * cap, st);
        t.leaf_id.alloc(cap, st);
        t.leaf_node.alloc(cap, st);
        // SFMM_TREE_TEST_STALL=1: the test of the bounded waits (the build
        // then fails with FMM_ERR_TIMEOUT after about two seconds)
        const char* stall_env = std::getenv("SFMM_TREE_TEST_STALL");
        const int stall_test = stall_env && std::strcmp(stall_env, "1") == 0;
        RefineState h{};
        h.S = S;
        h.total = 1;
        h.lvl_off[1] = 1;
        for (;;) {
            RefineArgs ra{};
            ra.key = t.key.ptr;
            ra.pbeg = t.pbeg.ptr;
            ra.pend = t.pend.ptr;
            ra.parent = t.parent.ptr;
            ra.child_beg = t.child_beg.ptr;
            ra.nchild = t.nchild.ptr;
            ra.col = t.colleague.ptr;
            ra.leaf_id = t.leaf_id.ptr;
            ra.leaf_node = t.leaf_node.ptr;
            ra.cap = static_cast<long long>(cap);
            ra.pkey[0] = keyA.ptr;
            ra.pkey[1] = keyB.ptr;
            ra.pord[0] = ordA.ptr;
            ra.pord[1] = ordB.ptr;
            ra.final_ord = t.order.ptr;
            ra.sp[0] = sp0.ptr;
            ra.sp[1] = sp1.ptr;
            ra.tile_off = tile_off.ptr;
            ra.hist = hist.ptr;
            ra.pre = pre.ptr;
            ra.ncnt = ncnt.ptr;
            ra.offs = offs.ptr;
            ra.nch = nch.ptr;
            ra.nsp = nsp.ptr;
            ra.part = part.ptr;
            ra.smax = static_cast<int>(smax);
            ra.tmax = static_cast<int>(tmax);
            ra.max_level = max_level;
            ra.ppn = max_ppn;
            ra.stall = stall_test;
            ra.st = dst.ptr;
            SFMM_CUDA(cudaMemcpyAsync(dst.ptr, &h, sizeof(h), cudaMemcpyHostToDevice, st));
            void* params[] = {&ra};
            SFMM_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_refine), dim3(G), dim3(kRefThreads),
                                                  params, 0, st));
            SFMM_CHECK_LAUNCH();
            SFMM_CUDA(cudaMemcpyAsync(&h, dst.ptr, sizeof(h), cudaMemcpyDeviceToHost, st));
            SFMM_CUDA(cudaStreamSynchronize(st));
            if (h.abort) throw Error(FMM_ERR_TIMEOUT, "the tree refinement gave up waiting at a grid barrier");
            if (h.status == kRefGrow) {
                // more node slots: keep the nodes so far and their colleagues
                const int64_t keep = h.total;
                grow_nodes(keep + h.need, keep);
                t.colleague.grow(27 * cap, 27 * keep, st);
                t.leaf_id.alloc(cap, st);
                t.leaf_node.alloc(cap, st);
                h.status = kRefDone;
                continue;
            }
            SFMM_REQUIRE(h.status == kRefDone, FMM_ERR_UNSUPPORTED, "tree refinement: work exceeded its bounds");
            break;
        }
        level = h.level;
        total = h.total;
        t.lvl_off.assign(h.lvl_off, h.lvl_off + level + 2);
        t.leaf_off.assign(h.leaf_off, h.leaf_off + level + 2);
        t.n_leaves = h.leaf_off[level + 1];
        S = 0;
    }
    DevBuf<int32_t> ntile, tile_off, hist, pre, cnt, offs, nch, nsp, child_base, split_base;
    while (S > 0) {
        const int child_may_split = (level + 1) < max_level;
        const int shift = 3 * (kKeyLevel - 1 - level);
        ntile.alloc(S, st);
        tile_off.alloc(S + 1, st);
        k_ntiles<<<blocks_for(S, 256), 256, 0, st>>>(sp.ptr, S, t.pbeg.ptr, t.pend.ptr, ntile.ptr);
        SFMM_CHECK_LAUNCH();
        exclusive_scan_i32(ntile.ptr, tile_off.ptr, S, st);
        const int T = read_one(tile_off.ptr + S, st);
        hist.alloc(size_t(8) * T, st);
        pre.alloc(size_t(8) * T + 1, st);
        k_hist<<<T, kTileThreads, 0, st>>>(sp.ptr, S, tile_off.ptr, T, t.pbeg.ptr, t.pend.ptr, keyA.ptr, shift, hist.ptr);
        SFMM_CHECK_LAUNCH();
        exclusive_scan_i32(hist.ptr, pre.ptr, int64_t(8) * T, st);
        cnt.alloc(size_t(8) * S, st);
        offs.alloc(size_t(8) * S, st);
        nch.alloc(S, st);
        nsp.alloc(S, st);
        k_nodestats<<<blocks_for(S, 256), 256, 0, st>>>(S, tile_off.ptr, T, pre.ptr, max_ppn, child_may_split,
                                                          cnt.ptr, offs.ptr, nch.ptr, nsp.ptr);
        SFMM_CHECK_LAUNCH();
        child_base.alloc(S + 1, st);
        split_base.alloc(S + 1, st);
        exclusive_scan_i32(nch.ptr, child_base.ptr, S, st);
        exclusive_scan_i32(nsp.ptr, split_base.ptr, S, st);
        int NC = 0, NS = 0;
        read_two(child_base.ptr + S, split_base.ptr + S, NC, NS, st);
        grow_nodes(total + NC, total);
        sp_next.alloc(std::max(NS, 1), st);
        k_children<<<blocks_for(S, 256), 256, 0, st>>>(sp.ptr, S, total, child_base.ptr, split_base.ptr, cnt.ptr, offs.ptr,
                                                        max_ppn, child_may_split, t.key.ptr, t.pbeg.ptr, t.pend.ptr,
                                                        t.parent.ptr, t.child_beg.ptr, t.nchild.ptr, sp_next.ptr);
        SFMM_CHECK_LAUNCH();
        k_scatter<<<T, kTileThreads, 0, st>>>(sp.ptr, S, tile_off.ptr, T, t.pbeg.ptr, t.pend.ptr, pre.ptr, cnt.ptr,
                                               offs.ptr, max_ppn, child_may_split, shift, keyA.ptr, ordA.ptr, keyB.ptr,
                                               ordB.ptr, t.order.ptr);
        SFMM_CHECK_LAUNCH();
        std::swap(keyA, keyB);
        std::swap(ordA, ordB);
        std::swap(sp, sp_next);
        total += NC;
        t.lvl_off.push_back(total);
        ++level;
        S = NS;
    }
    t.depth = level;
    t.n_nodes = total;
    t.single_refine = single;
    SFMM_CUDA(cudaEventRecord(ev.e[2], st));

    // --- leaves (per level in key order: the reference's _i_leaf)
    if (!single) {
        DevBuf<int32_t> flag, scan;
        flag.alloc(total, st);
        scan.alloc(total + 1, st);
        k_leafflag<<<blocks_for(total, 256, 8192), 256, 0, st>>>(t.nchild.ptr, total, flag.ptr);
        SFMM_CHECK_LAUNCH();
        exclusive_scan_i32(flag.ptr, scan.ptr, total, st);
        const std::vector<int32_t> hs = to_host(scan.ptr, total + 1, st);
        t.n_leaves = hs[total];
        t.leaf_off.clear();
        for (int l = 0; l <= t.depth + 1; ++l) t.leaf_off.push_back(hs[t.lvl_off[l]]);
        t.leaf_id.alloc(total, st);
        t.leaf_node.alloc(std::max<int64_t>(t.n_leaves, 1), st);
        k_leafids<<<blocks_for(total, 256, 8192), 256, 0, st>>>(t.nchild.ptr, scan.ptr, total, t.leaf_id.ptr, t.leaf_node.ptr);
        SFMM_CHECK_LAUNCH();
    }

    // --- points in leaf order (original frame for the near field, rotated
    //     frame for the expansions; the rotation is an axis permutation
    //     unless phideg != 0)
    t.pts.alloc(3 * n, st);
    if (t.box.rotated) t.rpts.alloc(3 * n, st);
    k_gather_points<<<blocks_for(n, 256, 8192), 256, 0, st>>>(xyz, t.order.ptr, n, t.d_box.ptr, t.pts.ptr,
                                                                t.box.rotated ? t.rpts.ptr : nullptr);
    SFMM_CHECK_LAUNCH();
    if (t.box.rotated) {
        t.far_x = t.rpts.ptr;
        t.far_y = t.rpts.ptr + n;
        t.far_z = t.rpts.ptr + 2 * n;
    } else {
        t.far_x = t.pts.ptr + t.box.X * n;
        t.far_y = t.pts.ptr + t.box.Y * n;
        t.far_z = t.pts.ptr + t.box.Z * n;
    }

    SFMM_CUDA(cudaEventRecord(ev.e[3], st));

    // --- colleagues, level by level
    if (!single) t.colleague.alloc(27 * total, st);
    for (int l = 0; !single && l <= t.depth; ++l) {
        const int64_t c = t.lvl_off[l + 1] - t.lvl_off[l];
        k_colleagues<<<blocks_for(c, 128), 128, 0, st>>>(t.lvl_off[l], c, l, t.key.ptr, t.parent.ptr, t.child_beg.ptr,
                                                          t.nchild.ptr, t.colleague.ptr);
        SFMM_CHECK_LAUNCH();
    }

    SFMM_CUDA(cudaEventRecord(ev.e[4], st));

    // --- interaction lists (levels >= 2)
    {
        DevBuf<int32_t> icnt;
        icnt.alloc(total, st);
        SFMM_CUDA(cudaMemsetAsync(icnt.ptr, 0, total * 4, st));
        // every level >= 2 at once: nodes are stored level after level, and a
        // node's list depends only on its parent's colleagues
        const int64_t i0 = t.depth >= 2 ? t.lvl_off[2] : total, ic = total - i0;
        if (ic > 0) {
            k_ilist<false><<<blocks_for(32 * ic, 256, 16384), 256, 0, st>>>(i0, ic, t.key.ptr, t.parent.ptr, t.child_beg.ptr,
                                                                t.nchild.ptr, t.colleague.ptr, icnt.ptr, nullptr, nullptr);
            SFMM_CHECK_LAUNCH();
        }
        t.il_ptr.alloc(total + 1, st);
        DevBuf<int64_t> tot;
        tot.alloc(1, st);
        exclusive_scan_i32(icnt.ptr, t.il_ptr.ptr, total, st, tot.ptr);
        t.il_nnz = read_one(tot.ptr, st);
        require_i32_total(t.il_nnz, "the interaction list");
        t.il_src.alloc(std::max<int64_t>(t.il_nnz, 1), st);
        t.il_code.alloc(std::max<int64_t>(t.il_nnz, 1), st);
        if (ic > 0) {
            k_ilist<true><<<blocks_for(32 * ic, 256, 16384), 256, 0, st>>>(i0, ic, t.key.ptr, t.parent.ptr, t.child_beg.ptr,
                                                               t.nchild.ptr, t.colleague.ptr, t.il_ptr.ptr, t.il_src.ptr,
                                                               t.il_code.ptr);
            SFMM_CHECK_LAUNCH();
        }
    }

    SFMM_CUDA(cudaEventRecord(ev.e[5], st));

    // --- near-field ranges per leaf
    {
        DevBuf<int32_t> ncnt;
        DevBuf<unsigned long long> pairs;
        const int64_t L = t.n_leaves;
        ncnt.alloc(L, st);
        pairs.alloc(1, st);
        SFMM_CUDA(cudaMemsetAsync(pairs.ptr, 0, 8, st));
        k_near<false><<<blocks_for(32 * L, 256, 16384), 256, 0, st>>>(L, t.leaf_node.ptr, t.parent.ptr, t.nchild.ptr, t.pbeg.ptr,
                                                           t.pend.ptr, t.colleague.ptr, ncnt.ptr, nullptr, pairs.ptr);
        SFMM_CHECK_LAUNCH();
        t.nr_ptr.alloc(L + 1, st);
        DevBuf<int64_t> tot;
        tot.alloc(1, st);
        exclusive_scan_i32(ncnt.ptr, t.nr_ptr.ptr, L, st, tot.ptr);
        t.nr_nnz = read_one(tot.ptr, st);
        require_i32_total(t.nr_nnz, "the near-field range list");
        t.near_pairs = static_cast<int64_t>(read_one(pairs.ptr, st));
        t.nr.alloc(std::max<int64_t>(t.nr_nnz, 1), st);
        k_near<true><<<blocks_for(32 * L, 256, 16384), 256, 0, st>>>(L, t.leaf_node.ptr, t.parent.ptr, t.nchild.ptr, t.pbeg.ptr,
                                                          t.pend.ptr, t.colleague.ptr, t.nr_ptr.ptr, t.nr.ptr, nullptr);
        SFMM_CHECK_LAUNCH();
    }

    SFMM_CUDA(cudaEventRecord(e1, st));
    SFMM_CUDA(cudaEventSynchronize(e1));
    check_scan_error();
    SFMM_CUDA(cudaEventElapsedTime(&t.build_ms, e0, e1));
    for (int k = 0; k < 6; ++k) SFMM_CUDA(cudaEventElapsedTime(&t.phase_ms[k], ev.e[k], ev.e[k + 1]));
}

// Algorithmic device-memory bytes of each build phase (what the phase's
// kernels must read and write at least once), for the achieved-bandwidth
// figures beside phase_ms:
//   keys        min/max read 24 B and key kernel read 24 B + write 12 B per point
//   refinement  per level, each point of a splitting node: the histogram reads
//               its 8 B key, the scatter reads and writes key + index (24 B);
//               the final order is written once (4 B per point)
//   leaves      points gathered into leaf order: read 24 B + 4 B index, write 24 B
//               (twice when the frame is rotated); leaf ids 16 B per node
//   colleagues  27 int32 per node written, parent/child fields read (12 B)
//               (the single-launch refinement counts leaf ids and colleagues
//               in its own phase)
//   ilist       both passes read the 27 colleagues and 16 B of node fields per
//               node; the entries (src, code) are written once, 8 B each
//   near lists  both passes read the 27 colleagues per leaf's node; the ranges
//               are written once (int2), the row pointers once
void tree_phase_bytes(const Tree& t, double* bytes6)
{
    cudaStream_t st = t.ctx->stream;
    const auto nch = to_host(t.nchild.ptr, t.n_nodes, st);
    const auto pb = to_host(t.pbeg.ptr, t.n_nodes, st);
    const auto pe = to_host(t.pend.ptr, t.n_nodes, st);
    double active = 0;                           // sum over levels of points in splitting nodes
    for (int64_t g = 0; g < t.n_nodes; ++g)
        if (nch[g] > 0) active += double(pe[g] - pb[g]);
    const double n = double(t.n), nodes = double(t.n_nodes), L = double(t.n_leaves);
    const double leaf_b = 16.0 * nodes, col_b = (27.0 * 4 + 12.0) * nodes;
    bytes6[0] = 60.0 * n;
    bytes6[1] = 32.0 * active + 4.0 * n + (t.single_refine ? leaf_b + col_b : 0.0);
    bytes6[2] = (t.box.rotated ? 76.0 : 52.0) * n + (t.single_refine ? 0.0 : leaf_b);
    bytes6[3] = t.single_refine ? 0.0 : col_b;
    bytes6[4] = 2 * (27.0 * 4 + 16.0) * nodes + 8.0 * double(t.il_nnz) + 4.0 * nodes;
    bytes6[5] = 2 * 27.0 * 4 * L + 8.0 * double(t.nr_nnz) + 4.0 * L;
}

// ------------------------------------------------------------------ exports
int64_t tree_export(const Tree& t, int l, int what, void* out)
{
    cudaStream_t st = t.ctx->stream;
    if (what == FMM_EXPORT_PARTITIONS) {
        if (out) {
            const auto order = to_host(t.order.ptr, t.n, st);
            const auto pb = to_host(t.pbeg.ptr, t.n_nodes, st);
            const auto pe = to_host(t.pend.ptr, t.n_nodes, st);
            const auto ln = to_host(t.leaf_node.ptr, t.n_leaves, st);
            int32_t* o = static_cast<int32_t*>(out);
            for (int lv = 0; lv <= t.depth; ++lv)
                for (int64_t f = t.leaf_off[lv]; f < t.leaf_off[lv + 1]; ++f) {
                    const int g = ln[f];
                    for (int i = pb[g]; i < pe[g]; ++i) {
                        o[2 * int64_t(order[i])] = lv;
                        o[2 * int64_t(order[i]) + 1] = static_cast<int32_t>(f - t.leaf_off[lv]);
                    }
                }
        }
        return 2 * t.n;
    }
    if (l < 0 || l > t.depth) return -1;
    const int64_t n0 = t.lvl_off[l], nn = t.lvl_off[l + 1] - n0;
    const int64_t f0 = t.leaf_off[l], nf = t.leaf_off[l + 1] - f0;
    switch (what) {
    case FMM_EXPORT_NODE_KEYS:
        if (out && nn) {
            SFMM_CUDA(cudaMemcpyAsync(out, t.key.ptr + n0, nn * 8, cudaMemcpyDeviceToHost, st));
            SFMM_CUDA(cudaStreamSynchronize(st));
        }
        return nn;
    case FMM_EXPORT_LEAF_NODES:
        if (out && nf) {
            const auto ln = to_host(t.leaf_node.ptr + f0, nf, st);
            for (int64_t f = 0; f < nf; ++f) static_cast<int32_t*>(out)[f] = static_cast<int32_t>(ln[f] - n0);
        }
        return nf;
    case FMM_EXPORT_INDEX_PTR:
    case FMM_EXPORT_INDEX: {
        const auto ln = to_host(t.leaf_node.ptr + f0, nf, st);
        const auto pb = to_host(t.pbeg.ptr, t.n_nodes, st);
        const auto pe = to_host(t.pend.ptr, t.n_nodes, st);
        int64_t nnz = 0;
        for (int64_t f = 0; f < nf; ++f) nnz += pe[ln[f]] - pb[ln[f]];
        if (what == FMM_EXPORT_INDEX_PTR) {
            if (out) {
                int32_t* o = static_cast<int32_t*>(out);
                o[0] = 0;
                for (int64_t f = 0; f < nf; ++f) o[f + 1] = o[f] + (pe[ln[f]] - pb[ln[f]]);
            }
            return nf + 1;
        }
        if (out) {
            const auto order = to_host(t.order.ptr, t.n, st);
            int32_t* o = static_cast<int32_t*>(out);
            for (int64_t f = 0; f < nf; ++f)
                for (int i = pb[ln[f]]; i < pe[ln[f]]; ++i) *o++ = order[i];
        }
        return nnz;
    }
    case FMM_EXPORT_ILIST_PTR:
    case FMM_EXPORT_ILIST: {
        if (l < 2) return -1;
        const auto ptr = to_host(t.il_ptr.ptr + n0, nn + 1, st);
        if (what == FMM_EXPORT_ILIST_PTR) {
            if (out) for (int64_t i = 0; i <= nn; ++i) static_cast<int32_t*>(out)[i] = ptr[i] - ptr[0];
            return nn + 1;
        }
        const int64_t nnz = ptr[nn] - ptr[0];
        if (out && nnz) {
            const auto src = to_host(t.il_src.ptr + ptr[0], nnz, st);
            const auto code = to_host(t.il_code.ptr + ptr[0], nnz, st);
            int32_t* o = static_cast<int32_t*>(out);
            for (int64_t e = 0; e < nnz; ++e) {
                o[4 * e] = static_cast<int32_t>(src[e] - n0);
                o[4 * e + 1] = (code[e] & 7) - 3;
                o[4 * e + 2] = ((code[e] >> 3) & 7) - 3;
                o[4 * e + 3] = ((code[e] >> 6) & 7) - 3;
            }
        }
        return 4 * nnz;
    }
    case FMM_EXPORT_CLIST_PTR:
    case FMM_EXPORT_CLIST: {
        if (l >= t.depth) return -1;
        const auto cb = to_host(t.child_beg.ptr + n0, nn, st);
        const auto nc = to_host(t.nchild.ptr + n0, nn, st);
        int64_t nnz = 0;
        for (int64_t i = 0; i < nn; ++i) nnz += nc[i];
        if (what == FMM_EXPORT_CLIST_PTR) {
            if (out) {
                int32_t* o = static_cast<int32_t*>(out);
                o[0] = 0;
                for (int64_t i = 0; i < nn; ++i) o[i + 1] = o[i] + nc[i];
            }
            return nn + 1;
        }
        if (out) {
            const int64_t c0 = t.lvl_off[l + 1];
            const auto keys = to_host(t.key.ptr + c0, t.lvl_off[l + 2] - c0, st);
            int64_t* o = static_cast<int64_t*>(out);
            for (int64_t i = 0; i < nn; ++i)
                for (int c = cb[i]; c < cb[i] + nc[i]; ++c) {
                    *o++ = c - c0;
                    *o++ = static_cast<int64_t>(keys[c - c0]);
                }
        }
        return 2 * nnz;
    }
    case FMM_EXPORT_PLIST: {
        if (l < 1) return -1;
        if (out) {
            const auto par = to_host(t.parent.ptr + n0, nn, st);
            const auto keys = to_host(t.key.ptr + n0, nn, st);
            int64_t* o = static_cast<int64_t*>(out);
            for (int64_t i = 0; i < nn; ++i) {
                o[2 * i] = par[i] - t.lvl_off[l - 1];
                o[2 * i + 1] = static_cast<int64_t>(keys[i]);
            }
        }
        return 2 * nn;
    }
    case FMM_EXPORT_NLIST_PTR:
    case FMM_EXPORT_NLIST: {
        LevelTabs L{};
        for (int k = 0; k <= t.depth + 1; ++k) { L.lvl_off[k] = t.lvl_off[k]; L.leaf_off[k] = t.leaf_off[k]; }
        L.depth = t.depth;
        DevBuf<int32_t> cntb, ptr, leafscan;
        DevBuf<int2> rows;
        cntb.alloc(std::max<int64_t>(nf, 1), st);
        ptr.alloc(nf + 1, st);
        // leafscan[g] = number of leaves before node g (sentinel at n_nodes)
        leafscan.alloc(t.n_nodes + 1, st);
        {
            DevBuf<int32_t> flag;
            flag.alloc(t.n_nodes, st);
            k_leafflag<<<blocks_for(t.n_nodes, 256, 8192), 256, 0, st>>>(t.nchild.ptr, t.n_nodes, flag.ptr);
            SFMM_CHECK_LAUNCH();
            exclusive_scan_i32(flag.ptr, leafscan.ptr, t.n_nodes, st);
        }
        k_nlist<false><<<blocks_for(nf, 64), 64, 0, st>>>(l, L, t.key.ptr, t.parent.ptr, t.nchild.ptr, t.leaf_node.ptr,
                                                           leafscan.ptr, t.colleague.ptr, cntb.ptr, nullptr);
        SFMM_CHECK_LAUNCH();
        exclusive_scan_i32(cntb.ptr, ptr.ptr, nf, st);
        const auto hp = to_host(ptr.ptr, nf + 1, st);
        if (what == FMM_EXPORT_NLIST_PTR) {
            if (out) std::copy(hp.begin(), hp.end(), static_cast<int32_t*>(out));
            return nf + 1;
        }
        const int64_t nnz = hp[nf];
        if (out && nnz) {
            rows.alloc(nnz, st);
            k_nlist<true><<<blocks_for(nf, 64), 64, 0, st>>>(l, L, t.key.ptr, t.parent.ptr, t.nchild.ptr, t.leaf_node.ptr,
                                                              leafscan.ptr, t.colleague.ptr, ptr.ptr, rows.ptr);
            SFMM_CHECK_LAUNCH();
            SFMM_CUDA(cudaMemcpyAsync(out, rows.ptr, nnz * 8, cudaMemcpyDeviceToHost, st));
            SFMM_CUDA(cudaStreamSynchronize(st));
        }
        return 2 * nnz;
    }
    default:
        return -1;
    }
}

}  // namespace sfmm
