// M2L of the mixed-precision plans (orders 2..12): dense per-offset operators
// applied in 8-bit integer slices on the fifth-generation tensor cores
// (tcgen05.mma kind::i8, accumulators in tensor memory).
//
// Formulation.  The M2L of one pair (fmm.hpp:592-618, the direct form of
// m2l_direct.cu) is linear in the source's moments.  Real form: per order n,
// Re M_n^0, then Re and Im of M_n^m for m = 1..n, (p+1)^2 reals (index
// n^2 + 2m - 1 + im).  With the expansions of a level scaled by its box size w
// (M~_n = w^-n M_n, L_j = w^-(j+1) L~_j) the pair's M2L is one dense matrix
// T_d of the offset d = source - target in {-3..3}^3, the same at every level:
//   L~ = T_d M~,   rows: the potential local (orders j <= p), then the field
//   local (j <= p + 1, from source orders n <= p - 1).
//
// Exact integer sums.  Both factors are scaled into [-1, 1] and written as
// ND = 4 signed 8-bit digits, x ~ sum_i d_i 2^(8 (3 - i)) / (127 2^24)
// (32 bits): operator row r by a fixed beta_r (its largest entry over all
// offsets), the moments of level l by alpha_l (their largest coefficient)
// after a fixed per-order factor gamma_n = (sqrt(3)/2)^n, the bound of a
// scaled order-n moment, that evens out the orders.  The ten digit products
// of weight >= 2^-24 (digit indices i + j <= 3) are summed exactly in 32-bit
// integers over every source of a target, grouped by weight into S0..S3, and
// converted once:
//   L~_r = alpha_l beta_r (S0 + S1 2^-8 + S2 2^-16 + S3 2^-24) / 127^2.
// Fixed-point digits give every term an absolute error of about 2^-31 of the
// row's and the level's largest values; three digits (2^-23) left ~1e-6 of
// relative error in the potential, four leave ~1e-7.  Integer sums do not
// depend on their order, so the result is deterministic whatever the
// schedule.  They cannot overflow for p <= 12: a target has at most 189
// sources of (p+1)^2 <= 169 nonzero terms, four products of magnitude
// <= 2^14 each per term in S3 (189 x 169 x 2^16 < 2^31).
//
// Work decomposition.  Targets (every node of levels >= 2) are grouped by
// level and octant (position in the parent): the offsets of a target's
// interaction list are among the 189 fixed by its octant (children of the
// parent's 27 neighbours that are not adjacent; partition.hpp:283-297),
// 216 slots in a 6 x 6 x 6 box.  A row block is up to 128 target rows
// (target x charge component) of one group; its slot table lists each
// target's source per slot.  The blocks of a level are numbered with the 8
// octants of a region adjacent, so blocks that run together share sources.  A work item is a row block and 128 operator rows;
// it runs over the slots that occur in the block and over K in steps of 32
// bytes.  Per step, the operator slab (128 rows x 32 B x 4 digits, stored in
// the MMA's canonical layout: one bulk copy) and the 128 sources' moment
// digits (gathered rows) go to shared memory, and one thread issues ten
// tcgen05.mma (M = 128 operator rows, N = 128 target rows, K = 32) into four
// int32 accumulators: the 512 columns of tensor memory.  An MMA costs the
// same whatever N (measured: 152 cycles for M = 128, K = 32, N = 32..256), so
// N is the widest the accumulators allow.
//
// Roles (one block per SM, persistent over the items): warps 0-3 gather the
// moment rows (cp.async) and issue the operator bulk copies; warp 8 allocates
// tensor memory and issues the MMAs; warps 4-7, one per 32-lane quarter of
// tensor memory, convert the sums and write the locals.  Shared-memory stages
// and the accumulator pass between them through mbarriers; every wait is
// bounded: on expiry the block records an error, stops its roles, waits for
// its MMAs and copies and frees tensor memory (the host reports
// FMM_ERR_TIMEOUT).
#include "eval_util.cuh"
#include "i8_ops.h"

#include <cub/device/device_radix_sort.cuh>

#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

namespace sfmm {

constexpr int kI8Slots = 216;
constexpr int kI8M = 128;                 // operator rows per item (MMA M, tensor-memory lanes)
constexpr int kI8Stages = 6;
constexpr int kI8Lag = 4;                 // gather stages in flight per producer thread
constexpr int kI8Threads = 9 * 32;
constexpr long kI8Spin = 1L << 22;        // mbarrier polls before a wait gives up

// ND digits per value: N target rows per item (ND accumulators of N columns
// fit the 512 tensor-memory columns), slab bytes, the digit-number scale.
// The plans use ND = 4.
template<int ND>
struct I8Cfg {
    static constexpr int N = ND == 3 ? 160 : 128;
    static constexpr int OpSlab = ND * kI8M * 32;
    static constexpr int MdSlab = ND * N * 32;
    static constexpr size_t Smem = size_t(kI8Stages) * (OpSlab + MdSlab);
};

struct I8DevTables {
    DevBuf<int8_t> op;       // [343 offsets][chunks][K steps][digit][128 rows x 32 B, canonical]
    DevBuf<double> beta;     // per operator row
    int R = 0, RA = 0, NCH = 0, KS = 0, ND = 4;
};

struct I8PlanData {
    std::shared_ptr<I8DevTables> tab;
    int64_t nrb = 0;
    int ND = 4, N = 128;                      // digits per value; target rows per item
    int tpb = 0;                              // targets per row block (N / qdim)
    DevBuf<int32_t> slot_src;                 // [row block][216][tpb]: source node or -1
    DevBuf<int32_t> used, nused;              // [row block][216]: slots that occur; their count
    DevBuf<int32_t> rb_tgt, rb_info;          // [row block][tpb] target nodes; level | octant << 8 | ntgt << 12
    DevBuf<int8_t> md;                        // moment digits [node][qdim][K steps][ND digits][32 B]
    DevBuf<uint32_t> alpha;                   // per (member tree, level): float bits of alpha
};

namespace {

__host__ __device__ inline int rdiv_up(int a, int b) { return (a + b - 1) / b; }

// beta_r = max over offsets and k of |T_d[r][k]| gamma_k (as float bits, rounded up)
__global__ void k_i8_beta(DirectArgs t, int p, int RA, int R, int KP, uint32_t* __restrict__ beta_bits)
{
    const int r = blockIdx.x;
    if (r >= R) return;
    float mx = 0.f;
    for (int e = threadIdx.x; e < 343 * KP; e += blockDim.x) {
        const int c = e / KP, k = e % KP;
        if (!offset_valid(c)) continue;
        int n, m, pi;
        real_nm(k, n, m, pi);
        const double v = fabs(op_entry(t, p, RA, c, r, k)) * i8_gamma(n);
        mx = fmaxf(mx, __double2float_ru(v));
    }
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(beta_bits + r, __float_as_uint(mx));
}

template<int ND>
__global__ void k_i8_opdigits(DirectArgs t, int p, int RA, int R, int NCH, int KS, const uint32_t* __restrict__ beta_bits,
                              int8_t* __restrict__ op, double* __restrict__ beta)
{
    const int KP = 32 * KS;
    const int64_t total = int64_t(343) * NCH * kI8M * KP;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
        const int k = static_cast<int>(e % KP);
        const int rr = static_cast<int>((e / KP) % kI8M);
        const int ch = static_cast<int>((e / (int64_t(KP) * kI8M)) % NCH);
        const int c = static_cast<int>(e / (int64_t(KP) * kI8M * NCH));
        const int r = ch * kI8M + rr;
        int8_t d[ND] = {};
        if (r < R && offset_valid(c)) {
            const double b = double(__uint_as_float(beta_bits[r]));
            int n, m, pi;
            real_nm(k, n, m, pi);
            if (b > 0) split_digits<ND>(op_entry(t, p, RA, c, r, k) * i8_gamma(n) / b, d);
        }
        int8_t* slab = op + ((int64_t(c) * NCH + ch) * KS + k / 32) * I8Cfg<ND>::OpSlab;
        for (int i = 0; i < ND; ++i) slab[i * (kI8M * 32) + canon_off(rr, k % 32)] = d[i];
        if (c == 0 && k == 0 && r < R) beta[r] = double(__uint_as_float(beta_bits[r]));
    }
}

// ------------------------------------------------------------------ per-plan set-up
// Sort key of each target: its (level, octant) group, then the pattern of its
// parent's 27 neighbours that have children (which of the 189 slots can hold
// a source).  Blocks of targets with one pattern use the same slots: near the
// edge of a level's refined region, where interaction lists are partly empty,
// Morton order alone would give each block the union of many patterns.
__global__ void k_i8_keys(const uint64_t* __restrict__ key, int64_t g0, int64_t g1, const int64_t* __restrict__ lvl_off, int depth,
                          const int32_t* __restrict__ parent, const int32_t* __restrict__ col, const int32_t* __restrict__ nchild,
                          uint64_t* __restrict__ skey, int32_t* __restrict__ sval, int32_t* __restrict__ cnt)
{
    for (int64_t g = g0 + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < g1; g += int64_t(gridDim.x) * blockDim.x) {
        int l = 2;
        while (l < depth && g >= lvl_off[l + 1]) ++l;
        const uint64_t k = key[g];
        const int oct = int(compact3(k) & 1) | int(compact3(k >> 1) & 1) << 1 | int(compact3(k >> 2) & 1) << 2;
        const int grp = (l - 2) * 8 + oct;
        const int32_t* pc = col + 27 * int64_t(parent[g]);
        uint32_t mask = 0;
        for (int s = 0; s < 27; ++s) {
            const int P = pc[s];
            if (P >= 0 && nchild[P] > 0) mask |= 1u << s;
        }
        skey[g - g0] = uint64_t(grp) << 27 | mask;
        sval[g - g0] = static_cast<int32_t>(g);
        atomicAdd(cnt + grp, 1);
    }
}

// Position of each target in its group from the sorted order.
__global__ void k_i8_pos(int64_t n, int64_t g0, const uint64_t* __restrict__ skey, const int32_t* __restrict__ sval,
                         const int32_t* __restrict__ grp_start, int32_t* __restrict__ pos)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        pos[sval[i] - g0] = static_cast<int32_t>(i - grp_start[skey[i] >> 27]);
}

__global__ void k_i8_assign(const uint64_t* __restrict__ key, int64_t g0, int64_t g1, const int64_t* __restrict__ lvl_off, int depth,
                            const int32_t* __restrict__ pos, const int32_t* __restrict__ rb_off, int tpb,
                            int32_t* __restrict__ rb_tgt, int32_t* __restrict__ rb_info)
{
    for (int64_t g = g0 + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < g1; g += int64_t(gridDim.x) * blockDim.x) {
        int l = 2;
        while (l < depth && g >= lvl_off[l + 1]) ++l;
        const uint64_t k = key[g];
        const int oct = int(compact3(k) & 1) | int(compact3(k >> 1) & 1) << 1 | int(compact3(k >> 2) & 1) << 2;
        const int ps = pos[g - g0];
        const int64_t rb = rb_off[(l - 2) * 8 + oct] + int64_t(ps / tpb) * 8;
        const int t = ps % tpb;
        rb_tgt[rb * tpb + t] = static_cast<int32_t>(g);
        atomicMax(rb_info + rb, l | oct << 8 | (t + 1) << 12);
    }
}

// Slot table of one row block (a block per row block): each target's sources
// by slot, built in shared memory from the interaction lists and written out
// whole; then the slots that occur, in slot order.
constexpr int kI8FillThreads = 256;
__global__ void __launch_bounds__(kI8FillThreads) k_i8_fill(int64_t nrb, int tpb, const int32_t* __restrict__ rb_tgt,
                                                           const int32_t* __restrict__ rb_info, const int32_t* __restrict__ il_ptr,
                                                           const int32_t* __restrict__ il_src, const int32_t* __restrict__ il_code,
                                                           int32_t* __restrict__ slot_src, int32_t* __restrict__ used,
                                                           int32_t* __restrict__ nused)
{
    extern __shared__ int32_t tab[];                     // [216][tpb]
    __shared__ int slot_on[kI8Slots];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = kI8FillThreads / 32;
    for (int64_t rb = blockIdx.x; rb < nrb; rb += gridDim.x) {
        const int info = rb_info[rb];
        const int oct = (info >> 8) & 7, ntg = info >> 12;
        const int cx = oct & 1, cy = (oct >> 1) & 1, cz = oct >> 2;
        for (int e = threadIdx.x; e < kI8Slots * tpb; e += kI8FillThreads) tab[e] = -1;
        __syncthreads();
        for (int t = warp; t < ntg; t += nw) {
            const int g = rb_tgt[rb * tpb + t];
            for (int e = il_ptr[g] + lane; e < il_ptr[g + 1]; e += 32) {
                const int code = il_code[e];
                const int dx = (code & 7) - 3, dy = ((code >> 3) & 7) - 3, dz = ((code >> 6) & 7) - 3;
                tab[((dx + 2 + cx) + 6 * (dy + 2 + cy) + 36 * (dz + 2 + cz)) * tpb + t] = il_src[e];
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < kI8Slots * tpb; e += kI8FillThreads) slot_src[rb * kI8Slots * tpb + e] = tab[e];
        // the slots that occur: a flag per slot (warps over slots), then warp 0
        // lists them in slot order (ballot + prefix)
        for (int sl = warp; sl < kI8Slots; sl += nw) {
            bool any = false;
            for (int t = lane; t < ntg; t += 32) any |= tab[sl * tpb + t] >= 0;
            const bool occ = __any_sync(0xffffffffu, any);
            if (lane == 0) slot_on[sl] = occ;
        }
        __syncthreads();
        if (warp == 0) {
            int cnt = 0;
            for (int s0 = 0; s0 < kI8Slots; s0 += 32) {
                const int sl = s0 + lane;
                const bool occ = sl < kI8Slots && slot_on[sl];
                const unsigned m = __ballot_sync(0xffffffffu, occ);
                if (occ) used[rb * kI8Slots + cnt + __popc(m & ((1u << lane) - 1u))] = sl;
                cnt += __popc(m);
            }
            if (lane == 0) nused[rb] = cnt;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ per evaluation
// Per-block tables of the moment scales, s_l^n (s_l = 2^l / width) and
// gamma_n, each entry the same expression a per-element evaluation would use.
struct I8Scales {
    double pw[kKeyLevel + 1][kI8MaxOrder + 1];    // pow(s_l, n)
    double sa[kKeyLevel + 1][kI8MaxOrder + 1];    // pow(s_l, n) / gamma_n
    double gm[kI8MaxOrder + 1];                   // gamma_n
};

__device__ void fill_scales(const EvalArgs& a, I8Scales& t)
{
    const int np = a.p + 1;
    for (int i = threadIdx.x; i < (a.depth + 1) * np; i += blockDim.x) {
        const int l = i / np, n = i % np;
        const double s = double(1 << l) / a.box->width;
        t.pw[l][n] = pow(s, double(n));
        t.sa[l][n] = pow(s, double(n)) / i8_gamma(n);
        if (l == 0) t.gm[n] = i8_gamma(n);
    }
    __syncthreads();
}

// alpha_l = max |M~| / gamma_n over the level's nodes (warp per node and
// component).  A warp keeps the running maximum of its current (tree, level)
// and issues one atomic when that changes, not one per node.
__global__ void k_i8_alpha(EvalArgs a, uint32_t* __restrict__ alpha_bits)
{
    __shared__ I8Scales sc;
    fill_scales(a, sc);
    const int lane = threadIdx.x & 31, qd = a.qdim, T = a.T;
    const int64_t g0 = a.lvl_off[2], g1 = a.lvl_off[a.depth + 1];
    const int64_t rows = (g1 - g0) * qd;
    int key = -1;
    float run = 0.f;
    for (int64_t w = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; w < rows; w += (int64_t(gridDim.x) * blockDim.x) >> 5) {
        const int64_t g = g0 + w / qd;
        const int l = level_of(a, g);
        float mx = 0.f;
        for (int t = lane; t < T; t += 32) {
            int n, m;
            tri_nm(t, n, m);
            const cplx v = a.M[(g * qd + w % qd) * T + t];
            mx = fmaxf(mx, __double2float_ru(fmax(fabs(v.re), fabs(v.im)) * sc.sa[l][n]));
        }
        for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        const int tr = a.node_tree ? a.node_tree[g] : 0;
        const int k = tr * (kKeyLevel + 2) + l;
        if (k != key) {
            if (lane == 0 && key >= 0 && run > 0.f) atomicMax(alpha_bits + key, __float_as_uint(run));
            key = k;
            run = 0.f;
        }
        run = fmaxf(run, mx);
    }
    if (lane == 0 && key >= 0 && run > 0.f) atomicMax(alpha_bits + key, __float_as_uint(run));
}

// moment digits of every node of levels >= 2 (warp per node and component)
template<int ND>
__global__ void k_i8_mdigits(EvalArgs a, int KS, const uint32_t* __restrict__ alpha_bits, int8_t* __restrict__ md)
{
    __shared__ I8Scales sc;
    fill_scales(a, sc);
    const int lane = threadIdx.x & 31, qd = a.qdim, T = a.T, p = a.p, KP = 32 * KS;
    const int64_t g0 = a.lvl_off[2], g1 = a.lvl_off[a.depth + 1];
    const int64_t rows = (g1 - g0) * qd;
    for (int64_t w = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; w < rows; w += (int64_t(gridDim.x) * blockDim.x) >> 5) {
        const int64_t g = g0 + w / qd;
        const int c = static_cast<int>(w % qd);
        const int l = level_of(a, g);
        const int tr = a.node_tree ? a.node_tree[g] : 0;
        const double al = double(__uint_as_float(alpha_bits[tr * (kKeyLevel + 2) + l]));
        int8_t* dst = md + (g * qd + c) * int64_t(KS) * (32 * ND);
        for (int k = lane; k < KP; k += 32) {
            int8_t d[ND] = {};
            if (k < (p + 1) * (p + 1) && al > 0) {
                int n, m, im;
                real_nm(k, n, m, im);
                const cplx v = a.M[(g * qd + c) * T + n * (n + 1) / 2 + m];
                split_digits<ND>((im ? v.im : v.re) * sc.pw[l][n] / sc.gm[n] / al, d);
            }
            int8_t* o = dst + (k / 32) * (32 * ND) + (k % 32);
#pragma unroll
            for (int i = 0; i < ND; ++i) o[32 * i] = d[i];
        }
    }
}

// ------------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ uint32_t su32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ uint64_t sdesc(uint32_t saddr)
{
    // no swizzle; leading (K) byte offset 128, stride (M/N) byte offset 256; descriptor version 1
    return uint64_t((saddr >> 4) & 0x3FFF) | uint64_t(128 >> 4) << 16 | uint64_t(256 >> 4) << 32 | uint64_t(1) << 46;
}

// kind::i8 instruction descriptor: S32 accumulator, signed A and B, both K-major
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N)
{
    return (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

template<int N>
__device__ __forceinline__ void mma_i8(uint32_t d, uint64_t a, uint64_t b, uint32_t acc)
{
    asm volatile("{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                 "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
                 "l"(a), "l"(b), "r"(idesc_i8(kI8M, N)), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar)) : "memory");
}

__device__ __forceinline__ void bar_init(uint64_t* bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void bar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(bar)) : "memory");
}

__device__ __forceinline__ void bar_arrive_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool bar_try(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(su32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// Bounded wait: false when the wait expired or another role gave up (abort).
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity, volatile int* abort)
{
    for (long it = 0; it < kI8Spin; ++it) {
        if (bar_try(bar, parity)) return true;
        if ((it & 255) == 255 && *abort) return false;
    }
    *abort = 1;
    return false;
}

// Bounded wait that ignores the abort flag: an aborting role waits for its own
// copies or MMAs in flight before shared or tensor memory is released.
__device__ __forceinline__ void bar_drain(uint64_t* bar, uint32_t parity)
{
    for (long it = 0; it < kI8Spin && !bar_try(bar, parity); ++it) {
    }
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(su32(dst)),
                 "l"(src), "r"(bytes), "r"(su32(bar))
                 : "memory");
}

__device__ __forceinline__ void cp16(void* dst, const void* src, bool valid)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(su32(dst)), "l"(src), "r"(valid ? 16 : 0) : "memory");
}

__device__ __forceinline__ void tld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
                   "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
}

struct I8Args {
    const int8_t* op;
    const double* beta;
    const int8_t* md;
    const uint32_t* alpha;
    const int32_t *slot_src, *used, *nused, *rb_tgt, *rb_info;
    int64_t nrb;
    int tpb, NCH, KS, RA, R;
    int* err;
};

struct I8Smem {
    uint64_t full[kI8Stages], empty[kI8Stages];
    uint64_t tfull, tempty;
    uint32_t tbase;
    int abort;
    long long nfilled;                    // stages the producers filled
};

template<int ND>
__global__ void __launch_bounds__(kI8Threads, 1) k_m2l_i8(EvalArgs a, I8Args g)
{
    using C = I8Cfg<ND>;
    constexpr int kN = C::N, kOpSlab = C::OpSlab, kMdSlab = C::MdSlab;
    extern __shared__ __align__(1024) uint8_t sm_raw[];
    __shared__ I8Smem ctl;
    uint8_t* opS = sm_raw;                                   // [stage][kOpSlab]
    uint8_t* mdS = sm_raw + kI8Stages * kOpSlab;             // [stage][kMdSlab]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qd = a.qdim, KS = g.KS, NCH = g.NCH, tpb = g.tpb;
    const int64_t items = g.nrb * NCH;
    volatile int* abort = &ctl.abort;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kI8Stages; ++s) {
            bar_init(&ctl.full[s], 128 + 1);
            bar_init(&ctl.empty[s], 1);
        }
        bar_init(&ctl.tfull, 1);
        bar_init(&ctl.tempty, 128);
        ctl.abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 8) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(su32(&ctl.tbase)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = ctl.tbase;

    if (warp < 4) {
        // ---------------- producers: operator slab (bulk copy) + gathered moment rows
        const int tp = threadIdx.x;
        int64_t n = 0;                                        // stages filled by this block
        bool ok = true;
        for (int64_t it = blockIdx.x; it < items && ok; it += gridDim.x) {
            const int64_t rb = it / NCH;
            const int ch = static_cast<int>(it % NCH);
            const int info = g.rb_info[rb];
            const int oct = (info >> 8) & 7, ntg = info >> 12;
            const int cx = oct & 1, cy = (oct >> 1) & 1, cz = oct >> 2;
            const int nst = g.nused[rb] * KS;
            for (int st = 0; st < nst; ++st, ++n) {
                const int s = static_cast<int>(n % kI8Stages);
                const uint32_t ph = static_cast<uint32_t>(n / kI8Stages) & 1;
                if (!bar_wait(&ctl.empty[s], ph ^ 1, abort)) {
                    ok = false;
                    break;
                }
                const int slot = g.used[rb * kI8Slots + st / KS], ks = st % KS;
                const int dx = slot % 6 - 2 - cx, dy = (slot / 6) % 6 - 2 - cy, dz = slot / 36 - 2 - cz;
                const int c = (dx + 3) + 7 * (dy + 3) + 49 * (dz + 3);
                if (tp == 0) {
                    bar_arrive_tx(&ctl.full[s], kOpSlab);
                    bulk_g2s(opS + s * kOpSlab, g.op + ((int64_t(c) * NCH + ch) * KS + ks) * kOpSlab, kOpSlab, &ctl.full[s]);
                }
                uint8_t* dst = mdS + s * kMdSlab;
                for (int row = tp; row < kN; row += 128) {
                    const int t = row / qd, comp = row % qd;
                    const int src = t < ntg ? g.slot_src[(rb * kI8Slots + slot) * tpb + t] : -1;
                    const int8_t* sp = g.md + ((int64_t(src < 0 ? 0 : src) * qd + comp) * KS + ks) * (32 * ND);
                    const int ro = (row >> 3) * 256 + (row & 7) * 16;
#pragma unroll
                    for (int i = 0; i < ND; ++i) {
                        cp16(dst + i * (kN * 32) + ro, sp + i * 32, src >= 0);
                        cp16(dst + i * (kN * 32) + ro + 128, sp + i * 32 + 16, src >= 0);
                    }
                }
                asm volatile("cp.async.commit_group;" ::: "memory");
                // the stage issued kI8Lag steps ago has landed: publish it to the MMA (async proxy)
                asm volatile("cp.async.wait_group %0;" ::"n"(kI8Lag) : "memory");
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                if (n >= kI8Lag) bar_arrive(&ctl.full[(n - kI8Lag) % kI8Stages]);
            }
        }
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        for (int64_t m = n - kI8Lag < 0 ? 0 : n - kI8Lag; m < n; ++m) bar_arrive(&ctl.full[m % kI8Stages]);
        if (tp == 0) ctl.nfilled = n;
    } else if (warp == 8) {
        // ---------------- MMA issue (one thread)
        if (lane == 0) {
            int64_t n = 0, nb = 0;
            bool ok = true;
            for (int64_t it = blockIdx.x; it < items && ok; it += gridDim.x) {
                const int64_t rb = it / NCH;
                const int nst = g.nused[rb] * KS;
                if (nst == 0) continue;
                if (!bar_wait(&ctl.tempty, (static_cast<uint32_t>(nb) & 1) ^ 1, abort)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                for (int st = 0; st < nst; ++st, ++n) {
                    const int s = static_cast<int>(n % kI8Stages);
                    const uint32_t ph = static_cast<uint32_t>(n / kI8Stages) & 1;
                    if (!bar_wait(&ctl.full[s], ph, abort)) {
                        ok = false;
                        break;
                    }
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t ao = su32(opS + s * kOpSlab), bo = su32(mdS + s * kMdSlab);
                    // products of operator digit i and moment digit j of weight 2^-8(i+j) >= 2^-8(ND-1),
                    // summed into accumulator i + j; the first of each accumulator in an item overwrites it
#pragma unroll
                    for (int gsum = 0; gsum < ND; ++gsum)
#pragma unroll
                        for (int i = 0; i <= gsum; ++i)
                            mma_i8<kN>(tbase + gsum * kN, sdesc(ao + i * (kI8M * 32)), sdesc(bo + (gsum - i) * (kN * 32)),
                                       (st > 0 || i > 0) ? 1u : 0u);
                    mma_commit(&ctl.empty[s]);
                }
                if (!ok) break;
                mma_commit(&ctl.tfull);
                ++nb;
            }
            if (!ok || *abort) {
                // let the MMAs already issued finish before tensor memory is freed
                mma_commit(&ctl.tfull);
                bar_drain(&ctl.tfull, static_cast<uint32_t>(nb) & 1);
            }
        }
        __syncwarp();
    } else {
        // ---------------- epilogue: lanes of quarter q = warp - 4 are operator rows
        const int q = warp - 4;
        const int rl = q * 32 + lane;                         // tensor-memory lane = row in the item
        const int T = a.T, T1 = a.T1;
        int64_t nb = 0;
        bool ok = true;
        for (int64_t it = blockIdx.x; it < items && ok; it += gridDim.x) {
            const int64_t rb = it / NCH;
            const int ch = static_cast<int>(it % NCH);
            const int info = g.rb_info[rb];
            const int l = info & 255, ntg = info >> 12;
            const int nst = g.nused[rb] * KS;
            const int r = ch * kI8M + rl;
            // this lane's output coefficient
            bool on = r < g.R;
            int j = 0, kk = 0, po = 0, isA = 1;
            if (on) {
                if (r < g.RA) {
                    real_nm(r, j, kk, po);
                } else {
                    real_nm(r - g.RA, j, kk, po);
                    isA = 0;
                }
                on = isA ? a.want_pot : a.want_field;
            }
            // alpha of the column's tree (a forest's members keep their own moment scales)
            double scale = 0.0;
            if (on && nst > 0) scale = g.beta[r] / (127.0 * 127.0) * pow(double(1 << l) / a.box->width, double(j + 1));
            if (nst > 0) {
                const bool got = bar_wait(&ctl.tfull, static_cast<uint32_t>(nb) & 1, abort);
                if (!__all_sync(0xffffffffu, got)) {          // warp-uniform: the loads below are .aligned
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            }
            const int tri_i = j * (j + 1) / 2 + kk;
            double* base = on ? (isA ? &a.LA[0].re : &a.LB[0].re) : nullptr;
            const int stride = isA ? T : T1;
            for (int c0 = 0; c0 < kN; c0 += 16) {
                uint32_t sg[ND][16];
                if (nst > 0) {
                    const uint32_t ta = tbase + (uint32_t(q * 32) << 16) + c0;
#pragma unroll
                    for (int gsum = 0; gsum < ND; ++gsum) tld16(ta + gsum * kN, sg[gsum]);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                }
                if (!on) continue;
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const int col = c0 + e;
                    const int t = col / qd, comp = col % qd;
                    if (t >= ntg || t >= tpb) continue;
                    const int64_t node = g.rb_tgt[rb * tpb + t];
                    double v = 0.0;
                    if (nst > 0) {
#pragma unroll
                        for (int gsum = ND - 1; gsum >= 0; --gsum) v = v * (1.0 / 256) + double(int(sg[gsum][e]));
                        const int tr = a.node_tree ? a.node_tree[node] : 0;
                        v *= scale * double(__uint_as_float(g.alpha[tr * (kKeyLevel + 2) + l]));
                    }
                    double* dst = base + 2 * ((node * qd + comp) * stride + tri_i);
                    dst[po] = v;
                    if (kk == 0) dst[1] = 0.0;               // Im of an m = 0 coefficient
                }
            }
            if (nst > 0) {
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                bar_arrive(&ctl.tempty);
                ++nb;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (ctl.abort && threadIdx.x == 0) {
        atomicExch(g.err, 1);
        // operator copies into stages the MMA may not have consumed land before shared memory is released
        const long long n = ctl.nfilled;
        for (long long m = n - kI8Stages < 0 ? 0 : n - kI8Stages; m < n; ++m)
            bar_drain(&ctl.full[m % kI8Stages], static_cast<uint32_t>(m / kI8Stages) & 1);
    }
    __syncthreads();
    if (warp == 8) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tbase));
}

}  // namespace

// ------------------------------------------------------------------ host
static std::shared_ptr<I8DevTables> i8_tables_on_device(int device, int p, int ND, cudaStream_t st)
{
    static std::mutex mu;
    static auto* cache = new std::map<std::tuple<int, int, int>, std::shared_ptr<I8DevTables>>();   // kept until exit
    std::lock_guard<std::mutex> lk(mu);
    auto& slot = (*cache)[std::make_tuple(device, p, ND)];
    if (slot) return slot;
    auto dt = direct_tables_on_device(device, p, st);
    auto t = std::make_shared<I8DevTables>();
    t->RA = (p + 1) * (p + 1);
    t->R = t->RA + (p + 2) * (p + 2);
    t->NCH = rdiv_up(t->R, kI8M);
    t->KS = rdiv_up((p + 1) * (p + 1), 32);
    const int KP = 32 * t->KS;
    DirectArgs da{dt->coef.ptr, dt->ncoef, dt->zil.ptr, dt->nz, reinterpret_cast<const cplx*>(dt->eil2.ptr), dt->ne};
    DevBuf<uint32_t> bb;
    bb.alloc(t->R, st);
    SFMM_CUDA(cudaMemsetAsync(bb.ptr, 0, bb.bytes(), st));
    k_i8_beta<<<t->R, 256, 0, st>>>(da, p, t->RA, t->R, KP, bb.ptr);
    SFMM_CHECK_LAUNCH();
    t->ND = ND;
    t->op.alloc(size_t(343) * t->NCH * t->KS * ND * kI8M * 32, st);
    t->beta.alloc(t->R, st);
    k_i8_opdigits<4><<<2048, 256, 0, st>>>(da, p, t->RA, t->R, t->NCH, t->KS, bb.ptr, t->op.ptr, t->beta.ptr);
    SFMM_CHECK_LAUNCH();
    SFMM_CUDA(cudaStreamSynchronize(st));
    slot = t;
    return t;
}

bool m2l_i8_supported(const Plan& pl)
{
    return pl.precision == FMM_PRECISION_MIXED && pl.p >= 2 && pl.p <= kI8MaxOrder && pl.tree->depth >= 2 &&
           pl.shard_count == 1 && !pl.m2l_force_rows && !pl.m2l_rotation_only;
}

void m2l_i8_setup(Plan& pl)
{
    pl.i8.reset();
    if (!m2l_i8_supported(pl)) return;
    Tree& t = *pl.tree;
    cudaStream_t st = t.ctx->stream;
    auto d = std::make_shared<I8PlanData>();
    d->ND = 4;
    d->N = I8Cfg<4>::N;
    d->tab = i8_tables_on_device(t.ctx->device, pl.p, d->ND, st);
    d->tpb = d->N / pl.qdim;
    const int64_t g0 = t.lvl_off[2], g1 = t.lvl_off[t.depth + 1];
    const int ngrp = (t.depth - 1) * 8;
    DevBuf<int64_t> loff;
    loff.alloc(t.depth + 2, st);
    SFMM_CUDA(cudaMemcpyAsync(loff.ptr, t.lvl_off.data(), (t.depth + 2) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    const int64_t nt = g1 - g0;
    DevBuf<int32_t> cnt, pos, rb_off, gstart, v0, v1;
    DevBuf<uint64_t> k0, k1;
    cnt.alloc(ngrp, st);
    pos.alloc(std::max<int64_t>(nt, 1), st);
    k0.alloc(std::max<int64_t>(nt, 1), st);
    k1.alloc(std::max<int64_t>(nt, 1), st);
    v0.alloc(std::max<int64_t>(nt, 1), st);
    v1.alloc(std::max<int64_t>(nt, 1), st);
    SFMM_CUDA(cudaMemsetAsync(cnt.ptr, 0, cnt.bytes(), st));
    const int sms = t.ctx->sm_count;
    const unsigned grid = static_cast<unsigned>(std::min<int64_t>(nt / 256 + 1, int64_t(sms) * 8));
    k_i8_keys<<<grid, 256, 0, st>>>(t.key.ptr, g0, g1, loff.ptr, t.depth, t.parent.ptr, t.colleague.ptr, t.nchild.ptr, k0.ptr,
                                    v0.ptr, cnt.ptr);
    SFMM_CHECK_LAUNCH();
    // stable radix sort of (group, pattern) keys; Morton order within a key
    int end_bit = 27;
    while ((int64_t(1) << (end_bit - 27)) < ngrp) ++end_bit;
    cub::DoubleBuffer<uint64_t> kb(k0.ptr, k1.ptr);
    cub::DoubleBuffer<int32_t> vb(v0.ptr, v1.ptr);
    size_t tmp_bytes = 0;
    SFMM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, kb, vb, static_cast<int>(nt), 0, end_bit, st));
    DevBuf<uint8_t> tmp;
    tmp.alloc(std::max<size_t>(tmp_bytes, 1), st);
    SFMM_CUDA(cub::DeviceRadixSort::SortPairs(tmp.ptr, tmp_bytes, kb, vb, static_cast<int>(nt), 0, end_bit, st));
    std::vector<int32_t> hc(ngrp), ho(ngrp), hs(ngrp);
    SFMM_CUDA(cudaMemcpyAsync(hc.data(), cnt.ptr, ngrp * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SFMM_CUDA(cudaStreamSynchronize(st));
    for (int i = 0, acc = 0; i < ngrp; ++i) {
        hs[i] = acc;
        acc += hc[i];
    }
    gstart.alloc(ngrp, st);
    SFMM_CUDA(cudaMemcpyAsync(gstart.ptr, hs.data(), ngrp * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    k_i8_pos<<<grid, 256, 0, st>>>(nt, g0, kb.Current(), vb.Current(), gstart.ptr, pos.ptr);
    SFMM_CHECK_LAUNCH();
    // row blocks of a level interleaved by octant: block b of the 8 octant
    // groups (targets that share most sources) are adjacent, so the items that
    // run together gather the same source moments; an octant with fewer
    // blocks leaves empty ones (no targets, no work)
    int64_t nrb = 0;
    for (int l = 0; l < t.depth - 1; ++l) {
        int nb = 0;
        for (int o = 0; o < 8; ++o) nb = std::max(nb, rdiv_up(hc[l * 8 + o], d->tpb));
        for (int o = 0; o < 8; ++o) ho[l * 8 + o] = static_cast<int32_t>(nrb + o);
        nrb += int64_t(nb) * 8;
    }
    d->nrb = nrb;
    rb_off.alloc(ngrp, st);
    SFMM_CUDA(cudaMemcpyAsync(rb_off.ptr, ho.data(), ngrp * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    d->slot_src.alloc(size_t(nrb) * kI8Slots * d->tpb, st);
    d->used.alloc(size_t(nrb) * kI8Slots, st);
    d->nused.alloc(nrb, st);
    d->rb_tgt.alloc(size_t(nrb) * d->tpb, st);
    d->rb_info.alloc(nrb, st);
    SFMM_CUDA(cudaMemsetAsync(d->rb_info.ptr, 0, d->rb_info.bytes(), st));
    k_i8_assign<<<grid, 256, 0, st>>>(t.key.ptr, g0, g1, loff.ptr, t.depth, pos.ptr, rb_off.ptr, d->tpb, d->rb_tgt.ptr,
                                      d->rb_info.ptr);
    SFMM_CHECK_LAUNCH();
    const size_t fill_smem = size_t(kI8Slots) * d->tpb * sizeof(int32_t);
    static std::once_flag fill_attr;
    std::call_once(fill_attr, [] {
        SFMM_CUDA(cudaFuncSetAttribute(k_i8_fill, cudaFuncAttributeMaxDynamicSharedMemorySize, kI8Slots * 128 * 4));
    });
    const unsigned fill_grid = static_cast<unsigned>(std::max<int64_t>(std::min<int64_t>(nrb, int64_t(sms) * 2), 1));
    k_i8_fill<<<fill_grid, kI8FillThreads, fill_smem, st>>>(nrb, d->tpb, d->rb_tgt.ptr, d->rb_info.ptr, t.il_ptr.ptr,
                                                           t.il_src.ptr, t.il_code.ptr, d->slot_src.ptr, d->used.ptr,
                                                           d->nused.ptr);
    SFMM_CHECK_LAUNCH();
    d->md.alloc(size_t(t.n_nodes) * pl.qdim * d->tab->KS * 32 * d->ND, st);
    d->alpha.alloc(size_t(kKeyLevel + 2) * t.n_trees, st);
    SFMM_CUDA(cudaStreamSynchronize(st));       // the set-up's temporaries are freed on return
    pl.i8 = d;
}

void launch_m2l_i8(Plan& pl, const EvalArgs& a, cudaStream_t st)
{
    I8PlanData& d = *pl.i8;
    const I8DevTables& tb = *d.tab;
    const int sms = pl.tree->ctx->sm_count;
    SFMM_CUDA(cudaMemsetAsync(d.alpha.ptr, 0, d.alpha.bytes(), st));
    const int64_t rows = (a.lvl_off[a.depth + 1] - a.lvl_off[2]) * a.qdim;
    const unsigned gw = static_cast<unsigned>(std::min<int64_t>(rows / 8 + 1, int64_t(sms) * 16));
    k_i8_alpha<<<gw, 256, 0, st>>>(a, d.alpha.ptr);
    SFMM_CHECK_LAUNCH();
    k_i8_mdigits<4><<<gw, 256, 0, st>>>(a, tb.KS, d.alpha.ptr, d.md.ptr);
    SFMM_CHECK_LAUNCH();
    I8Args g{tb.op.ptr, tb.beta.ptr, d.md.ptr, d.alpha.ptr, d.slot_src.ptr, d.used.ptr, d.nused.ptr, d.rb_tgt.ptr,
             d.rb_info.ptr, d.nrb, d.tpb, tb.NCH, tb.KS, tb.RA, tb.R, a.wait_err};
    static std::once_flag attr;
    std::call_once(attr, [] {
        SFMM_CUDA(cudaFuncSetAttribute(k_m2l_i8<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(I8Cfg<4>::Smem)));
    });
    const int64_t items = d.nrb * tb.NCH;
    const unsigned grid = static_cast<unsigned>(std::max<int64_t>(std::min<int64_t>(items, sms), 1));
    k_m2l_i8<4><<<grid, kI8Threads, I8Cfg<4>::Smem, st>>>(a, g);
    SFMM_CHECK_LAUNCH();
}

void m2l_i8_check(Plan& pl)
{
    if (!pl.wait_err.ptr) return;
    cudaStream_t st = pl.tree->ctx->stream;
    int v = 0;
    SFMM_CUDA(cudaMemcpyAsync(&v, pl.wait_err.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    SFMM_CUDA(cudaStreamSynchronize(st));
    if (v) {
        SFMM_CUDA(cudaMemsetAsync(pl.wait_err.ptr, 0, sizeof(int), st));
        throw Error(FMM_ERR_TIMEOUT, "a pipeline wait of the evaluation expired (tensor-core M2L or near-field copies)");
    }
}

}  // namespace sfmm
