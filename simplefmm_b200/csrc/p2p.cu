// P2P (fmm.hpp:773-809) for the FP64 path: the near field of every leaf over
// its neighbour-list point ranges, with the reference's self exclusion
// (is_self: i == j, fmm.hpp:786, 880).
//
// Warp per work item: a leaf's targets against all of its near field, or,
// for a leaf with a large near field, against one part of it (work items
// below).  Sources are packed records (x y z q0 | q1 q2, leaf
// order) and an item's near-field ranges are staged into full shared tiles of
// kChunk sources by asynchronous 16-byte copies, two tiles per warp: the
// copies of tile c + 1 are in flight while tile c is summed, so the gathers'
// L2 / DRAM latency hides behind the arithmetic.  The item's ranges are read
// 32 at a time into registers (lane k holds range k) and walked with
// shuffles.  Lanes are (target group, source slice): tg targets per pass and
// 32/tg slices, with tg chosen per leaf so that at most kMaxPass passes cover
// its targets; every source read from shared memory is applied to the lane's
// target of every pass (register blocking over passes).  Slices of a target
// are summed with xor shuffles at the end.
#include "eval_util.cuh"

namespace sfmm {
namespace {

constexpr int kWarps = 8;
constexpr int kChunk = 128;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem) : "memory");
}
// Bulk (TMA engine) copies of contiguous source runs into a warp's tile,
// completed on the tile buffer's mbarrier (one arrival per fill plus the
// bytes in flight).  Waits are bounded: an expired wait records an error that
// the host reports (FMM_ERR_TIMEOUT).
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void tile_bar_init(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tile_expect(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tile_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool tile_wait(uint64_t* bar, uint32_t parity, int* err)
{
    for (long it = 0; it < (1L << 22); ++it) {
        uint32_t ok;
        asm volatile("{\n.reg .pred q;\nmbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\nselp.u32 %0, 1, 0, q;\n}\n"
                     : "=r"(ok)
                     : "r"(smem_u32(bar)), "r"(parity)
                     : "memory");
        if (ok) return true;
    }
    if (err) atomicExch(err, 1);
    return false;
}

// ---------------------------------------------------------------- work items
// A coarse leaf beside a dense region can hold most of the points in its
// near field (on 4M Plummer points eight leaves have ~500k near sources each,
// ten times one warp's share of the whole near field), so one warp per leaf
// leaves a few warps working long after the rest.  A leaf whose
// targets x sources exceeds kPartCost is split into parts of consecutive near
// sources of equal size, each part a work item; a split leaf's parts write
// rows of partial sums that k_p2p_reduce adds in part order, so the result
// does not depend on which warp ran which item.  Warps take items from a
// counter, in leaf order (coarse leaves, the split ones among them, first).
constexpr int64_t kPartCost = 131072;

__global__ void k_p2p_cost(const int32_t* __restrict__ nr_ptr, const int2* __restrict__ nr,
                           const int32_t* __restrict__ pbeg, const int32_t* __restrict__ pend,
                           const int32_t* __restrict__ leaf_node, int64_t n_leaves, int32_t* __restrict__ parts,
                           int32_t* __restrict__ rows, int32_t* __restrict__ psize, int32_t* __restrict__ nsrc)
{
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t f = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; f < n_leaves; f += stride) {
        const int g = leaf_node[f];
        const int nt = pend[g] - pbeg[g];
        const int r0 = nr_ptr[f], r1 = nr_ptr[f + 1];
        int64_t ns = 0;
        for (int r = r0 + lane; r < r1; r += 32) ns += nr[r].y - nr[r].x;
        for (int o = 16; o; o >>= 1) ns += __shfl_xor_sync(0xffffffffu, ns, o);
        if (lane == 0) {
            const int64_t cost = int64_t(nt) * ns;
            int64_t np = 1, S = ns;
            if (cost > kPartCost && ns > 1) {
                np = ns < (cost + kPartCost - 1) / kPartCost ? ns : (cost + kPartCost - 1) / kPartCost;
                S = (ns + np - 1) / np;
                np = (ns + S - 1) / S;
            }
            parts[f] = static_cast<int>(np);
            rows[f] = np > 1 ? static_cast<int>(np) * nt : 0;
            psize[f] = static_cast<int>(S);
            nsrc[f] = static_cast<int>(ns);
        }
    }
}

// Warp per leaf: the items of its parts.  Part k starts at source k * S of
// the leaf's near field; the range holding it is found from a warp prefix
// sum over 32 ranges at a time.
__global__ void k_p2p_items(const int32_t* __restrict__ nr_ptr, const int2* __restrict__ nr,
                            const int32_t* __restrict__ pbeg, const int32_t* __restrict__ pend,
                            const int32_t* __restrict__ leaf_node, int64_t n_leaves, const int32_t* __restrict__ parts,
                            const int32_t* __restrict__ psize, const int32_t* __restrict__ nsrc,
                            const int32_t* __restrict__ item_off, const int32_t* __restrict__ row_off,
                            int4* __restrict__ item, int32_t* __restrict__ row)
{
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t f = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; f < n_leaves; f += stride) {
        const int np = parts[f], off = item_off[f], ns = nsrc[f];
        const int r0 = nr_ptr[f], r1 = nr_ptr[f + 1];
        if (np == 1) {
            if (lane == 0) {
                item[off] = make_int4(static_cast<int>(f), r0, 0, ns);
                row[off] = -1;
            }
            continue;
        }
        const int g = leaf_node[f];
        const int nt = pend[g] - pbeg[g];
        const int64_t S = psize[f];
        const int rb = row_off[f];
        int64_t base = 0;
        for (int c0 = r0; c0 < r1; c0 += 32) {
            const int ri = c0 + lane;
            const int len = ri < r1 ? nr[ri].y - nr[ri].x : 0;
            int cum = len;
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, cum, o);
                if (lane >= o) cum += v;
            }
            const int64_t lo = base + cum - len, hi = base + cum;
            for (int64_t k = (lo + S - 1) / S; k < np && k * S < hi; ++k) {
                item[off + k] = make_int4(static_cast<int>(f), ri, static_cast<int>(k * S - lo),
                                          static_cast<int>(S < ns - k * S ? S : ns - k * S));
                row[off + k] = rb + static_cast<int>(k) * nt;
            }
            base += __shfl_sync(0xffffffffu, cum, 31);
        }
    }
}

// Sums the parts of every split leaf, in part order, into out2.
__global__ void k_p2p_reduce(EvalArgs a)
{
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t f = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; f < a.n_leaves; f += stride) {
        const int np = a.p2p_parts[f];
        if (np <= 1 || (a.own_leaf && !a.own_leaf[f])) continue;
        const int g = a.leaf_node[f];
        const int t0 = a.pbeg[g], nt = a.pend[g] - t0;
        const int64_t rb = a.p2p_rowoff[f];
        for (int e = lane; e < nt * a.K; e += 32) {
            const int t = e / a.K, o = e - t * a.K;
            double v = 0;
            for (int k = 0; k < np; ++k) v += a.p2p_part[(rb + int64_t(k) * nt + t) * a.K + o];
            a.out2[int64_t(o) * a.n + t0 + t] = v;
        }
    }
}

__device__ __forceinline__ int next_item(int* ctr, int lane)
{
    int it = 0;
    if (lane == 0) it = atomicAdd(ctr, 1);
    return __shfl_sync(0xffffffffu, it, 0);
}

// One target's sum of component comp: into out2, or into the item's rows.
__device__ __forceinline__ void put_near(const EvalArgs& a, int row, int t0, int i, int comp, double v)
{
    if (row < 0)
        a.out2[int64_t(comp) * a.n + i] = v;
    else
        a.p2p_part[(int64_t(row) + (i - t0)) * a.K + comp] = v;
}

template<int QD>
struct P2PSmem {
    static constexpr int tile = kChunk * (32 + (QD > 1 ? 16 : 0));   // double4 (+ double2) per source
    static constexpr int per_warp = 2 * tile + 16;                    // two tiles, their two mbarriers
    static constexpr int total = kWarps * per_warp;
};

// Cursor over a leaf's near ranges [r0, r1): lane k of the warp holds range
// base + k; every lane walks the same sequence.
struct RangeWalk {
    int ri, r1, base, roff, rem;
    int2 mine;

    // item: (leaf, first range, offset in it, sources); r_end: the leaf's
    // end of ranges
    __device__ __forceinline__ void start(const int2* __restrict__ nr, int4 item, int r_end, int lane)
    {
        ri = item.y;
        r1 = r_end;
        base = item.y;
        roff = item.z;
        rem = item.w;
        mine = ri + lane < r_end ? nr[ri + lane] : make_int2(0, 0);
    }

    // Issues the copies of the next tile (at most kChunk sources) into t4 / t2;
    // returns its fill and the one segment that overlaps the target leaf's own
    // points [t0, t1) (near ranges are disjoint and one of them holds the leaf
    // itself, so at most one segment of a tile overlaps it).
    template<int QD>
    __device__ __forceinline__ int fill_tile(const int2* __restrict__ nr, const double4* __restrict__ src4,
                                             const double2* __restrict__ src2, double4* t4, double2* t2, int lane,
                                             int t0, int t1, int& self_s0, int& self_j0, int& self_len, uint64_t* bar)
    {
        int fill = 0;
        // the buffer was last read by this warp's generic loads (ordered by the
        // caller's __syncwarp); order those before the bulk copies' writes
        if (lane == 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        self_s0 = 0;
        self_j0 = 0;
        self_len = 0;
        while (rem > 0 && ri < r1 && fill < kChunk) {
            if (ri - base >= 32) {
                base = ri;
                mine = ri + lane < r1 ? nr[ri + lane] : make_int2(0, 0);
            }
            const int rx = __shfl_sync(0xffffffffu, mine.x, ri - base);
            const int ry = __shfl_sync(0xffffffffu, mine.y, ri - base);
            const int j0 = rx + roff;
            const int len = min(min(ry - j0, kChunk - fill), rem);
            if (lane == 0) {
                // one bulk copy per run: len packed 32-byte records (and their 16-byte extra charges)
                tile_expect(bar, uint32_t(len) * (QD > 1 ? 48u : 32u));
                bulk_copy(t4 + fill, src4 + j0, uint32_t(len) * 32u, bar);
                if (QD > 1) bulk_copy(t2 + fill, src2 + j0, uint32_t(len) * 16u, bar);
            }
            if (j0 < t1 && j0 + len > t0) {
                self_s0 = fill;
                self_j0 = j0;
                self_len = len;
            }
            fill += len;
            roff += len;
            rem -= len;
            if (j0 + len == ry) {
                ++ri;
                roff = 0;
            }
        }
        if (lane == 0) tile_arrive(bar);
        return fill;
    }
};

template<int QD, bool POT, bool FLD, int kMaxPass, int MINB>
__global__ void __launch_bounds__(kWarps * 32, MINB) k_p2p(EvalArgs a)
{
    constexpr int kTargetsPerBlock = 32 * kMaxPass;
    constexpr int NO = (POT ? QD : 0) + (FLD ? 3 : 0);
    extern __shared__ __align__(16) unsigned char sm[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* mine = sm + w * P2PSmem<QD>::per_warp;
    double4* t4[2];
    double2* t2[2];
#pragma unroll
    for (int b = 0; b < 2; ++b) {
        t4[b] = reinterpret_cast<double4*>(mine + b * P2PSmem<QD>::tile);
        t2[b] = reinterpret_cast<double2*>(mine + b * P2PSmem<QD>::tile + kChunk * 32);
    }
    uint64_t* bars = reinterpret_cast<uint64_t*>(mine + 2 * P2PSmem<QD>::tile);
    if (lane == 0) {
        tile_bar_init(bars);
        tile_bar_init(bars + 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    uint32_t par = 0;                                   // bit b: parity of the next wait on tile buffer b
    bool broken = false;                                // a wait expired: stop (the host reports it)

    for (int it = next_item(a.p2p_ctr, lane); it < a.p2p_items; it = next_item(a.p2p_ctr, lane)) {
        const int4 item = a.p2p_item[it];
        if (a.own_leaf && !a.own_leaf[item.x]) continue;        // another shard's leaf
        const int row = a.p2p_row[it];
        const int g = a.leaf_node[item.x];
        const int t0 = a.pbeg[g], t1 = a.pend[g];
        const int r1 = a.nr_ptr[item.x + 1];
        for (int tb = t0; tb < t1; tb += kTargetsPerBlock) {
            const int nt = min(kTargetsPerBlock, t1 - tb);
            int tg = 1;
            while (tg < 32 && tg * kMaxPass < nt) tg <<= 1;
            const int slices = 32 / tg;
            const int passes = (nt + tg - 1) / tg;
            const int ti = lane / slices, s = lane - ti * slices;
            RangeWalk wk;
            wk.start(a.nr, item, r1, lane);
            int cs0, cj0, clen;
            int fill = wk.fill_tile<QD>(a.nr, a.src4, a.src2, t4[0], t2[0], lane, t0, t1, cs0, cj0, clen, bars);
            double xi[kMaxPass], yi[kMaxPass], zi[kMaxPass];
            int ii[kMaxPass];
            double acc[kMaxPass][NO > 0 ? NO : 1];
#pragma unroll
            for (int p = 0; p < kMaxPass; ++p) {
                const int t = p * tg + ti;
                const bool on = p < passes && t < nt;
                ii[p] = on ? tb + t : -1;
                const double4 v = a.src4[on ? tb + t : tb];
                xi[p] = v.x;
                yi[p] = v.y;
                zi[p] = v.z;
#pragma unroll
                for (int o = 0; o < NO; ++o) acc[p][o] = 0;
            }
            int buf = 0;
            for (;;) {
                // every fill of a buffer (the last one is empty) is waited for once
                const bool got = tile_wait(bars + buf, (par >> buf) & 1u, a.wait_err);
                if (!__all_sync(0xffffffffu, got)) {
                    broken = true;
                    tile_wait(bars + (buf ^ 1), (par >> (buf ^ 1)) & 1u, nullptr);   // a copy of the other buffer in flight
                    break;
                }
                par ^= 1u << buf;
                if (fill == 0) break;
                int ns0, nj0, nlen;
                const int nfill = wk.fill_tile<QD>(a.nr, a.src4, a.src2, t4[buf ^ 1], t2[buf ^ 1], lane, t0, t1, ns0, nj0,
                                                   nlen, bars + (buf ^ 1));
                // slot of the lane's own target in this tile, if it is here
                int ks[kMaxPass];
#pragma unroll
                for (int p = 0; p < kMaxPass; ++p) {
                    const unsigned d = static_cast<unsigned>(ii[p] - cj0);
                    ks[p] = ii[p] >= 0 && d < static_cast<unsigned>(clen) ? cs0 + static_cast<int>(d) : -1;
                }
                const double4* sx = t4[buf];
                const double2* sq = t2[buf];
#pragma unroll 2
                for (int k = s; k < fill; k += slices) {
                    const double4 v = sx[k];
                    double2 qq = make_double2(0, 0);
                    if (QD > 1) qq = sq[k];
#pragma unroll
                    for (int p = 0; p < kMaxPass; ++p) {
                        if (p >= passes) break;
                        const double dx = xi[p] - v.x, dy = yi[p] - v.y, dz = zi[p] - v.z;
                        const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
                        const double ir = k == ks[p] ? 0.0 : rsqrt(r2);
                        int o = 0;
                        if (POT) {
                            acc[p][o++] = fma(v.w, ir, acc[p][0]);
                            if (QD > 1) acc[p][o++] = fma(qq.x, ir, acc[p][1]);
                            if (QD > 2) acc[p][o++] = fma(qq.y, ir, acc[p][2]);
                        }
                        if (FLD) {
                            const double ir3 = ir * ir * ir;
                            if (QD == 1) {
                                const double cq = v.w * ir3;
                                acc[p][o] = fma(cq, dx, acc[p][o]);
                                acc[p][o + 1] = fma(cq, dy, acc[p][o + 1]);
                                acc[p][o + 2] = fma(cq, dz, acc[p][o + 2]);
                            } else {
                                const double qa = v.w, qb = qq.x, qc = qq.y;
                                acc[p][o] = fma((qb * dz - qc * dy), ir3, acc[p][o]);
                                acc[p][o + 1] = fma((qc * dx - qa * dz), ir3, acc[p][o + 1]);
                                acc[p][o + 2] = fma((qa * dy - qb * dx), ir3, acc[p][o + 2]);
                            }
                        }
                    }
                }
                __syncwarp();
                buf ^= 1;
                fill = nfill;
                cs0 = ns0;
                cj0 = nj0;
                clen = nlen;
            }
            if (broken) break;
            // sum the slices of each target (consecutive lanes)
#pragma unroll
            for (int p = 0; p < kMaxPass; ++p)
#pragma unroll
                for (int o = 0; o < NO; ++o)
                    for (int off = slices >> 1; off; off >>= 1) acc[p][o] += __shfl_xor_sync(0xffffffffu, acc[p][o], off);
            if (s == 0) {
#pragma unroll
                for (int p = 0; p < kMaxPass; ++p) {
                    if (ii[p] < 0) continue;
                    int o = 0;
                    if (POT)
                        for (int b = 0; b < QD; ++b) put_near(a, row, t0, ii[p], b, acc[p][o++]);
                    if (FLD)
                        for (int c = 0; c < 3; ++c) put_near(a, row, t0, ii[p], a.kf + c, acc[p][o++]);
                }
            }
        }
        if (broken) break;
    }
}

// ---------------------------------------------------------------- mixed precision
// The same decomposition in FP32: coordinates relative to the target leaf's
// centre (differences taken in FP64 when a tile is staged, then rounded, so
// the FP32 offsets keep the leaf's own scale; each coordinate is kept as
// hi + lo so separations of nearby points stay exact to FP32), 1/r from
// rsqrtf refined by one Newton-Raphson step, and blocked compensated sums:
// each source tile's terms (at most kChunk / slices per lane) are summed in
// plain FP32 and the tile partials are added into a two-sum (Knuth's TwoSum:
// value + running rounding error), converted to FP64 at the end.

struct Sum2 {
    float s, e;
};

__device__ __forceinline__ void two_sum_add(Sum2& a, float x)
{
    const float s = a.s + x;
    const float bb = s - a.s;
    a.e += (a.s - (s - bb)) + (x - bb);
    a.s = s;
}

// x = hi + lo with hi = float(x): differences of nearby points keep FP32
// relative precision in the separation itself (the hi parts subtract exactly)
struct F2 {
    float h, l;
};

__device__ __forceinline__ F2 split_f(double x)
{
    const float h = static_cast<float>(x);
    return F2{h, static_cast<float>(x - static_cast<double>(h))};
}

template<int QD>
struct P2PSmemF {
    static constexpr int per_warp = kChunk * (32 + (QD > 1 ? 8 : 0));
    static constexpr int total = kWarps * per_warp;
};

// 1/sqrt(r2): the hardware approximation (rsqrt.approx.ftz, relative error
// ~2^-22.9; a denormal r2 -- separations below 1e-19 of the leaf's scale --
// counts as 0) and one Newton-Raphson step.  r2 = 0 gives +inf, as 1/0 does
// in FP64: the step runs on min(y, 2^126) so that 0 x inf never forms.
__device__ __forceinline__ float rsqrt_newton(float r2)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(r2));
    const float yc = fminf(y, 8.507059e37f);
    const float e = fmaf(-0.5f * r2 * yc, yc, 0.5f);
    return fmaf(y, e, y);
}

// One staged tile against NP target passes of the lane: plain FP32 partial
// sums (the caller folds them into two-sums after the tile).  ks[p] is the
// tile slot of pass p's own target (-1 if it is not in this tile).
template<int NP, int QD, bool POT, bool FLD, int NO, int MP>
__device__ __forceinline__ void p2p_mixed_tile(const float4* __restrict__ sxq, const float4* __restrict__ sxl,
                                               const float2* __restrict__ sq12, int s, int slices, int fill,
                                               const F2 (&xi)[MP], const F2 (&yi)[MP], const F2 (&zi)[MP],
                                               const int (&ks)[MP], float (&part)[MP][NO > 0 ? NO : 1])
{
    for (int k = s; k < fill; k += slices) {
        const float4 xq = sxq[k], xl = sxl[k];
        float2 qq = make_float2(0.f, 0.f);
        if (QD > 1) qq = sq12[k];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const float dx = (xi[p].h - xq.x) + (xi[p].l - xl.x);
            const float dy = (yi[p].h - xq.y) + (yi[p].l - xl.y);
            const float dz = (zi[p].h - xq.z) + (zi[p].l - xl.z);
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const float ir = k == ks[p] ? 0.f : rsqrt_newton(r2);
            int o = 0;
            if (POT) {
                part[p][o] = fmaf(xq.w, ir, part[p][o]);
                ++o;
                if (QD > 1) { part[p][o] = fmaf(qq.x, ir, part[p][o]); ++o; }
                if (QD > 2) { part[p][o] = fmaf(qq.y, ir, part[p][o]); ++o; }
            }
            if (FLD) {
                const float ir3 = ir * ir * ir;
                if (QD == 1) {
                    const float cq = xq.w * ir3;
                    part[p][o] = fmaf(cq, dx, part[p][o]);
                    part[p][o + 1] = fmaf(cq, dy, part[p][o + 1]);
                    part[p][o + 2] = fmaf(cq, dz, part[p][o + 2]);
                } else {
                    const float qa = xq.w, qb = qq.x, qc = qq.y;
                    part[p][o] = fmaf(qb * dz - qc * dy, ir3, part[p][o]);
                    part[p][o + 1] = fmaf(qc * dx - qa * dz, ir3, part[p][o + 1]);
                    part[p][o + 2] = fmaf(qa * dy - qb * dx, ir3, part[p][o + 2]);
                }
            }
        }
    }
}


template<int QD, bool POT, bool FLD, int kMaxPass, int MINB>
__global__ void __launch_bounds__(kWarps * 32, MINB) k_p2p_mixed(EvalArgs a)
{
    constexpr int kTargetsPerBlock = 32 * kMaxPass;
    constexpr int NO = (POT ? QD : 0) + (FLD ? 3 : 0);
    extern __shared__ __align__(16) unsigned char sm[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* mine = sm + w * P2PSmemF<QD>::per_warp;
    float4* sxq = reinterpret_cast<float4*>(mine);                 // x y z q0, high parts (leaf-centred)
    float4* sxl = sxq + kChunk;                                     // x y z low parts
    float2* sq12 = reinterpret_cast<float2*>(mine + kChunk * 32);   // only for QD > 1
    const double* q0 = a.qs;
    const double* q1 = a.qs + (QD > 1 ? a.n : 0);
    const double* q2 = a.qs + (QD > 2 ? 2 * a.n : 0);

    for (int it = next_item(a.p2p_ctr, lane); it < a.p2p_items; it = next_item(a.p2p_ctr, lane)) {
        const int4 item = a.p2p_item[it];
        if (a.own_leaf && !a.own_leaf[item.x]) continue;        // another shard's leaf
        const int row = a.p2p_row[it];
        const int g = a.leaf_node[item.x];
        // origin: the leaf's first point (any point near the leaf keeps the
        // FP32 offsets at the leaf's scale)
        const int t0 = a.pbeg[g], t1 = a.pend[g];
        const double c[3] = {a.px[t0], a.py[t0], a.pz[t0]};
        const int r1 = a.nr_ptr[item.x + 1];
        for (int tb = t0; tb < t1; tb += kTargetsPerBlock) {
            const int nt = min(kTargetsPerBlock, t1 - tb);
            int tg = 1;
            while (tg < 32 && tg * kMaxPass < nt) tg <<= 1;
            const int slices = 32 / tg;
            const int passes = (nt + tg - 1) / tg;
            const int ti = lane / slices, s = lane - ti * slices;
            F2 xi[kMaxPass], yi[kMaxPass], zi[kMaxPass];
            int ii[kMaxPass];
            Sum2 acc[kMaxPass][NO > 0 ? NO : 1];
            float part[kMaxPass][NO > 0 ? NO : 1];       // this chunk's plain FP32 partial sums
#pragma unroll
            for (int p = 0; p < kMaxPass; ++p) {
                const int t = p * tg + ti;
                const bool on = p < passes && t < nt;
                ii[p] = on ? tb + t : -1;
                const int i = on ? tb + t : tb;
                xi[p] = split_f(a.px[i] - c[0]);
                yi[p] = split_f(a.py[i] - c[1]);
                zi[p] = split_f(a.pz[i] - c[2]);
#pragma unroll
                for (int o = 0; o < NO; ++o) acc[p][o] = Sum2{0.f, 0.f};
            }
            int ri = item.y, roff = item.z, rem = item.w;
            while (rem > 0 && ri < r1) {
                int fill = 0;
                int self_s0 = 0, self_j0 = 0, self_len = 0;   // the tile's segment of the target leaf's own points
                while (rem > 0 && ri < r1 && fill < kChunk) {
                    const int2 rg = a.nr[ri];
                    const int len = min(min(rg.y - rg.x - roff, kChunk - fill), rem);
                    const int j0 = rg.x + roff;
                    for (int k = lane; k < len; k += 32) {
                        const int j = j0 + k;
                        const F2 x = split_f(a.px[j] - c[0]), y = split_f(a.py[j] - c[1]), z = split_f(a.pz[j] - c[2]);
                        sxq[fill + k] = make_float4(x.h, y.h, z.h, static_cast<float>(q0[j]));
                        sxl[fill + k] = make_float4(x.l, y.l, z.l, 0.f);
                        if (QD > 1) sq12[fill + k] = make_float2(static_cast<float>(q1[j]), static_cast<float>(q2[j]));
                    }
                    if (j0 < t1 && j0 + len > t0) {
                        self_s0 = fill;
                        self_j0 = j0;
                        self_len = len;
                    }
                    fill += len;
                    roff += len;
                    rem -= len;
                    if (roff == rg.y - rg.x) {
                        ++ri;
                        roff = 0;
                    }
                }
                __syncwarp();
#pragma unroll
                for (int p = 0; p < kMaxPass; ++p)
#pragma unroll
                    for (int o = 0; o < NO; ++o) part[p][o] = 0.f;
                int ks[kMaxPass];
#pragma unroll
                for (int p = 0; p < kMaxPass; ++p) {
                    const unsigned d = static_cast<unsigned>(ii[p] - self_j0);
                    ks[p] = ii[p] >= 0 && d < static_cast<unsigned>(self_len) ? self_s0 + static_cast<int>(d) : -1;
                }
                static_assert(kMaxPass <= 3, "passes dispatched up to 3");
                if (passes == 1)
                    p2p_mixed_tile<1, QD, POT, FLD, NO>(sxq, sxl, sq12, s, slices, fill, xi, yi, zi, ks, part);
                else if (passes == 2)
                    p2p_mixed_tile<(kMaxPass >= 2 ? 2 : 1), QD, POT, FLD, NO>(sxq, sxl, sq12, s, slices, fill, xi, yi, zi, ks, part);
                else
                    p2p_mixed_tile<kMaxPass, QD, POT, FLD, NO>(sxq, sxl, sq12, s, slices, fill, xi, yi, zi, ks, part);
                // fold the chunk's partials (at most kChunk / slices terms each) into the two-sums
#pragma unroll
                for (int p = 0; p < kMaxPass; ++p)
#pragma unroll
                    for (int o = 0; o < NO; ++o) two_sum_add(acc[p][o], part[p][o]);
                __syncwarp();
            }
            // FP64 from here: each lane's (sum, error), then the slices of a target
#pragma unroll
            for (int p = 0; p < kMaxPass; ++p)
#pragma unroll
                for (int o = 0; o < NO; ++o) {
                    double v = static_cast<double>(acc[p][o].s) + static_cast<double>(acc[p][o].e);
                    for (int off = slices >> 1; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
                    if (s == 0 && ii[p] >= 0) {
                        const int comp = POT ? (o < QD ? o : a.kf + (o - QD)) : a.kf + o;
                        put_near(a, row, t0, ii[p], comp, v);
                    }
                }
        }
    }
}

// Blocks that are resident at once (the warps take items until none is left).
template<typename K>
unsigned resident_grid(K kernel, size_t smem, int sms, int64_t items)
{
    int nb = 0;
    SFMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, kWarps * 32, smem));
    const int64_t need = (items + kWarps - 1) / kWarps;
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(need, int64_t(std::max(nb, 1)) * sms)));
}

template<int QD, bool POT, bool FLD, int MP, int MINB>
void launch_mixed(const EvalArgs& a, int sms, cudaStream_t st)
{
    const size_t smem = P2PSmemF<QD>::total;
    allow_max_smem(k_p2p_mixed<QD, POT, FLD, MP, MINB>);
    const unsigned grid = resident_grid(k_p2p_mixed<QD, POT, FLD, MP, MINB>, smem, sms, a.p2p_items);
    k_p2p_mixed<QD, POT, FLD, MP, MINB><<<grid, kWarps * 32, smem, st>>>(a);
    SFMM_CHECK_LAUNCH();
}

template<int QD, bool POT, bool FLD, int MP, int MINB>
void launch_fp64(const EvalArgs& a, int sms, cudaStream_t st)
{
    const size_t smem = P2PSmem<QD>::total;
    allow_max_smem(k_p2p<QD, POT, FLD, MP, MINB>);
    const unsigned grid = resident_grid(k_p2p<QD, POT, FLD, MP, MINB>, smem, sms, a.p2p_items);
    k_p2p<QD, POT, FLD, MP, MINB><<<grid, kWarps * 32, smem, st>>>(a);
    SFMM_CHECK_LAUNCH();
}

// Measured (kChunk 128): FP64 on 4M Plummer points, p = 10: 4 passes and two
// blocks per SM (128 registers) 58.9 ms; 3 passes / 3 blocks 77.1 ms and
// 2 passes / 4 blocks 83.4 ms (both spill).  FP32, 4M Plummer / 16M uniform:
// 4 passes, one block per SM 45.2 / 74.5 ms; 3 passes, two blocks 52.5 / 48.9 ms;
// 2 passes, two blocks 52.7 / 51.1 ms; 2 passes, three blocks 69.7 / 46.2 ms.
template<int QD, bool POT, bool FLD>
void launch(const EvalArgs& a, int sms, cudaStream_t st)
{
    if (a.mixed) return launch_mixed<QD, POT, FLD, 3, 2>(a, sms, st);
    return launch_fp64<QD, POT, FLD, 4, 2>(a, sms, st);
}

}  // namespace

void launch_p2p(const EvalArgs& a, int sms, cudaStream_t st)
{
    if (a.p2p_items == 0) return;
    SFMM_CUDA(cudaMemsetAsync(a.p2p_ctr, 0, sizeof(int), st));
    const int mode = (a.want_pot ? 1 : 0) | (a.want_field ? 2 : 0);
#define SFMM_P2P(Q)                                   \
    if (a.qdim == Q) {                                \
        if (mode == 1)                                \
            launch<Q, true, false>(a, sms, st);       \
        else if (mode == 2)                           \
            launch<Q, false, true>(a, sms, st);       \
        else                                          \
            launch<Q, true, true>(a, sms, st);        \
    }
    SFMM_P2P(1)
    SFMM_P2P(2)
    SFMM_P2P(3)
#undef SFMM_P2P
    if (a.p2p_split) {
        k_p2p_reduce<<<blocks_for(a.n_leaves * 32, 256, int64_t(sms) * 16), 256, 0, st>>>(a);
        SFMM_CHECK_LAUNCH();
    }
}

void p2p_setup(Plan& pl)
{
    Tree& t = *pl.tree;
    cudaStream_t st = t.ctx->stream;
    const int64_t nl = t.n_leaves;
    pl.p2p_items = 0;
    pl.p2p_rows = 0;
    pl.p2p_ctr.alloc(1, st);
    if (nl == 0) return;
    pl.p2p_parts.alloc(nl, st);
    pl.p2p_rowoff.alloc(nl + 1, st);                    // exclusive scans write n + 1 entries
    DevBuf<int32_t> rows, psize, nsrc, ioff;
    rows.alloc(nl, st);
    psize.alloc(nl, st);
    nsrc.alloc(nl, st);
    ioff.alloc(nl + 1, st);
    const unsigned grid = blocks_for(nl * 32, 256, int64_t(t.ctx->sm_count) * 16);
    k_p2p_cost<<<grid, 256, 0, st>>>(t.nr_ptr.ptr, t.nr.ptr, t.pbeg.ptr, t.pend.ptr, t.leaf_node.ptr, nl,
                                     pl.p2p_parts.ptr, rows.ptr, psize.ptr, nsrc.ptr);
    SFMM_CHECK_LAUNCH();
    exclusive_scan_i32(pl.p2p_parts.ptr, ioff.ptr, nl, st);
    exclusive_scan_i32(rows.ptr, pl.p2p_rowoff.ptr, nl, st);
    int32_t h[2] = {0, 0};                              // items, rows of partial sums
    SFMM_CUDA(cudaMemcpyAsync(&h[0], ioff.ptr + nl, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SFMM_CUDA(cudaMemcpyAsync(&h[1], pl.p2p_rowoff.ptr + nl, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SFMM_CUDA(cudaStreamSynchronize(st));
    pl.p2p_items = h[0];
    pl.p2p_rows = h[1];
    pl.p2p_item.alloc(size_t(h[0]), st);
    pl.p2p_row.alloc(size_t(h[0]), st);
    if (h[1] > 0) pl.p2p_part.alloc(size_t(h[1]) * (pl.qdim + 3), st);
    k_p2p_items<<<grid, 256, 0, st>>>(t.nr_ptr.ptr, t.nr.ptr, t.pbeg.ptr, t.pend.ptr, t.leaf_node.ptr, nl,
                                      pl.p2p_parts.ptr, psize.ptr, nsrc.ptr, ioff.ptr, pl.p2p_rowoff.ptr,
                                      pl.p2p_item.ptr, pl.p2p_row.ptr);
    SFMM_CHECK_LAUNCH();
}

}  // namespace sfmm
