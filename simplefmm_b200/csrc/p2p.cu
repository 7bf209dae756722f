// P2P (fmm.hpp:773-809) for the FP64 path: the near field of every leaf over
// its neighbour-list point ranges, with the reference's self exclusion
// (is_self: i == j, fmm.hpp:786, 880).
//
// Warp per target leaf.  The leaf's source ranges are gathered into full
// shared tiles of kChunk sources (x y | z q packed as double2).  Lanes are
// (target group, source slice): tg targets per pass and 32/tg slices, with tg
// chosen per leaf so that at most kMaxPass passes cover its targets; every
// source read from shared memory is applied to the lane's target of every
// pass (register blocking over passes).  Slices of a target are summed with
// xor shuffles at the end.
#include "eval_util.cuh"

namespace sfmm {
namespace {

constexpr int kWarps = 8;
constexpr int kChunk = 128;

template<int QD>
struct P2PSmem {
    static constexpr int per_warp = kChunk * (16 + 16 + (QD > 1 ? 16 : 0) + 4);
    static constexpr int total = kWarps * per_warp;
};

template<int QD, bool POT, bool FLD, int kMaxPass, int MINB>
__global__ void __launch_bounds__(kWarps * 32, MINB) k_p2p(EvalArgs a)
{
    constexpr int kTargetsPerBlock = 32 * kMaxPass;
    constexpr int NO = (POT ? QD : 0) + (FLD ? 3 : 0);
    extern __shared__ __align__(16) unsigned char sm[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* mine = sm + w * P2PSmem<QD>::per_warp;
    double2* sxy = reinterpret_cast<double2*>(mine);
    double2* szq = sxy + kChunk;
    double2* sq12 = szq + kChunk;                       // only for QD > 1
    int* sj = reinterpret_cast<int*>(mine + kChunk * (32 + (QD > 1 ? 16 : 0)));
    const double* q0 = a.qs;
    const double* q1 = a.qs + (QD > 1 ? a.n : 0);
    const double* q2 = a.qs + (QD > 2 ? 2 * a.n : 0);

    for (int64_t f = blockIdx.x * int64_t(kWarps) + w; f < a.n_leaves; f += int64_t(gridDim.x) * kWarps) {
        const int g = a.leaf_node[f];
        const int t0 = a.pbeg[g], t1 = a.pend[g];
        const int r0 = a.nr_ptr[f], r1 = a.nr_ptr[f + 1];
        for (int tb = t0; tb < t1; tb += kTargetsPerBlock) {
            const int nt = min(kTargetsPerBlock, t1 - tb);
            int tg = 1;
            while (tg < 32 && tg * kMaxPass < nt) tg <<= 1;
            const int slices = 32 / tg;
            const int passes = (nt + tg - 1) / tg;
            const int ti = lane / slices, s = lane - ti * slices;
            double xi[kMaxPass], yi[kMaxPass], zi[kMaxPass];
            int ii[kMaxPass];
            double acc[kMaxPass][NO > 0 ? NO : 1];
#pragma unroll
            for (int p = 0; p < kMaxPass; ++p) {
                const int t = p * tg + ti;
                const bool on = p < passes && t < nt;
                ii[p] = on ? tb + t : -1;
                const int i = on ? tb + t : tb;
                xi[p] = a.px[i];
                yi[p] = a.py[i];
                zi[p] = a.pz[i];
#pragma unroll
                for (int o = 0; o < NO; ++o) acc[p][o] = 0;
            }
            // stream the leaf's near-field sources through full shared tiles
            int ri = r0, roff = 0;
            while (ri < r1) {
                int fill = 0;
                while (ri < r1 && fill < kChunk) {
                    const int2 rg = a.nr[ri];
                    const int len = min(rg.y - rg.x - roff, kChunk - fill);
                    for (int k = lane; k < len; k += 32) {
                        const int j = rg.x + roff + k;
                        sxy[fill + k] = make_double2(a.px[j], a.py[j]);
                        szq[fill + k] = make_double2(a.pz[j], q0[j]);
                        if (QD > 1) sq12[fill + k] = make_double2(q1[j], q2[j]);
                        sj[fill + k] = j;
                    }
                    fill += len;
                    roff += len;
                    if (roff == rg.y - rg.x) {
                        ++ri;
                        roff = 0;
                    }
                }
                __syncwarp();
#pragma unroll 2
                for (int k = s; k < fill; k += slices) {
                    const double2 xy = sxy[k], zq = szq[k];
                    double2 qq = make_double2(0, 0);
                    if (QD > 1) qq = sq12[k];
                    const int j = sj[k];
#pragma unroll
                    for (int p = 0; p < kMaxPass; ++p) {
                        if (p >= passes) break;
                        const double dx = xi[p] - xy.x, dy = yi[p] - xy.y, dz = zi[p] - zq.x;
                        const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
                        const double ir = j == ii[p] ? 0.0 : rsqrt(r2);
                        int o = 0;
                        if (POT) {
                            acc[p][o++] = fma(zq.y, ir, acc[p][0]);
                            if (QD > 1) acc[p][o++] = fma(qq.x, ir, acc[p][1]);
                            if (QD > 2) acc[p][o++] = fma(qq.y, ir, acc[p][2]);
                        }
                        if (FLD) {
                            const double ir3 = ir * ir * ir;
                            if (QD == 1) {
                                const double cq = zq.y * ir3;
                                acc[p][o] = fma(cq, dx, acc[p][o]);
                                acc[p][o + 1] = fma(cq, dy, acc[p][o + 1]);
                                acc[p][o + 2] = fma(cq, dz, acc[p][o + 2]);
                            } else {
                                const double qa = zq.y, qb = qq.x, qc = qq.y;
                                acc[p][o] = fma((qb * dz - qc * dy), ir3, acc[p][o]);
                                acc[p][o + 1] = fma((qc * dx - qa * dz), ir3, acc[p][o + 1]);
                                acc[p][o + 2] = fma((qa * dy - qb * dx), ir3, acc[p][o + 2]);
                            }
                        }
                    }
                }
                __syncwarp();
            }
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
                        for (int b = 0; b < QD; ++b) a.out2[int64_t(b) * a.n + ii[p]] = acc[p][o++];
                    if (FLD)
                        for (int c = 0; c < 3; ++c) a.out2[int64_t(a.kf + c) * a.n + ii[p]] = acc[p][o++];
                }
            }
        }
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

template<int QD>
struct P2PSmemF {
    static constexpr int per_warp = kChunk * (32 + (QD > 1 ? 8 : 0) + 4);
    static constexpr int total = kWarps * per_warp;
};

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
    int* sj = reinterpret_cast<int*>(mine + kChunk * (32 + (QD > 1 ? 8 : 0)));
    const double* q0 = a.qs;
    const double* q1 = a.qs + (QD > 1 ? a.n : 0);
    const double* q2 = a.qs + (QD > 2 ? 2 * a.n : 0);

    for (int64_t f = blockIdx.x * int64_t(kWarps) + w; f < a.n_leaves; f += int64_t(gridDim.x) * kWarps) {
        const int g = a.leaf_node[f];
        // origin: the leaf's first point (any point near the leaf keeps the
        // FP32 offsets at the leaf's scale)
        const int t0 = a.pbeg[g], t1 = a.pend[g];
        const double c[3] = {a.px[t0], a.py[t0], a.pz[t0]};
        const int r0 = a.nr_ptr[f], r1 = a.nr_ptr[f + 1];
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
            int ri = r0, roff = 0;
            while (ri < r1) {
                int fill = 0;
                while (ri < r1 && fill < kChunk) {
                    const int2 rg = a.nr[ri];
                    const int len = min(rg.y - rg.x - roff, kChunk - fill);
                    for (int k = lane; k < len; k += 32) {
                        const int j = rg.x + roff + k;
                        const F2 x = split_f(a.px[j] - c[0]), y = split_f(a.py[j] - c[1]), z = split_f(a.pz[j] - c[2]);
                        sxq[fill + k] = make_float4(x.h, y.h, z.h, static_cast<float>(q0[j]));
                        sxl[fill + k] = make_float4(x.l, y.l, z.l, 0.f);
                        if (QD > 1) sq12[fill + k] = make_float2(static_cast<float>(q1[j]), static_cast<float>(q2[j]));
                        sj[fill + k] = j;
                    }
                    fill += len;
                    roff += len;
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
                for (int k = s; k < fill; k += slices) {
                    const float4 xq = sxq[k], xl = sxl[k];
                    float2 qq = make_float2(0.f, 0.f);
                    if (QD > 1) qq = sq12[k];
                    const int j = sj[k];
#pragma unroll
                    for (int p = 0; p < kMaxPass; ++p) {
                        if (p >= passes) break;
                        const float dx = (xi[p].h - xq.x) + (xi[p].l - xl.x);
                        const float dy = (yi[p].h - xq.y) + (yi[p].l - xl.y);
                        const float dz = (zi[p].h - xq.z) + (zi[p].l - xl.z);
                        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        float ir = rsqrtf(r2);
                        ir = ir * fmaf(-0.5f * r2 * ir, ir, 1.5f);      // one Newton step
                        ir = j == ii[p] ? 0.f : (r2 > 0.f ? ir : __int_as_float(0x7f800000));
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
                        a.out2[int64_t(comp) * a.n + ii[p]] = v;
                    }
                }
        }
    }
}

template<int QD, bool POT, bool FLD, int MP, int MINB>
void launch_mixed(const EvalArgs& a, int sms, cudaStream_t st)
{
    const size_t smem = P2PSmemF<QD>::total;
    allow_max_smem(k_p2p_mixed<QD, POT, FLD, MP, MINB>);
    const int64_t grid = std::min<int64_t>((a.n_leaves + kWarps - 1) / kWarps, int64_t(sms) * 16);
    k_p2p_mixed<QD, POT, FLD, MP, MINB><<<static_cast<unsigned>(std::max<int64_t>(grid, 1)), kWarps * 32, smem, st>>>(a);
    SFMM_CHECK_LAUNCH();
}

template<int QD, bool POT, bool FLD, int MP, int MINB>
void launch_fp64(const EvalArgs& a, int sms, cudaStream_t st)
{
    const size_t smem = P2PSmem<QD>::total;
    allow_max_smem(k_p2p<QD, POT, FLD, MP, MINB>);
    const int64_t grid = std::min<int64_t>((a.n_leaves + kWarps - 1) / kWarps, int64_t(sms) * 16);
    k_p2p<QD, POT, FLD, MP, MINB><<<static_cast<unsigned>(std::max<int64_t>(grid, 1)), kWarps * 32, smem, st>>>(a);
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
    const int mode = (a.want_pot ? 1 : 0) | (a.want_field ? 2 : 0);
#define SFMM_P2P(Q)                                              \
    if (a.qdim == Q) {                                           \
        if (mode == 1) return launch<Q, true, false>(a, sms, st); \
        if (mode == 2) return launch<Q, false, true>(a, sms, st); \
        return launch<Q, true, true>(a, sms, st);                \
    }
    SFMM_P2P(1)
    SFMM_P2P(2)
    SFMM_P2P(3)
#undef SFMM_P2P
}

}  // namespace sfmm
