// M2M and L2L (fmm.hpp:558-590, 714-745) as FP64 tensor-core products, one
// fused kernel per level.
//
// A shift between a box and one of its children is a fixed real-linear map
// on the box's coefficient row (the m >= 0 triangle stored as re, im pairs:
// R = 2T doubles) that depends only on the child's octant and on the level
// (through rho = sqrt(3/4) w / 2^l).  Per children level the maps are built
// once per plan by applying the direct term sums of fmm_ops.cuh
// (shift_output, the code of the warp-per-node kernels k_m2m / k_l2l) to
// unit vectors, and stored in MMA fragment order:
//   M2M  OpM (R x 8R): a parent's row is OpM times its eight children's rows
//        stacked in octant order (absent children are zero);
//   L2L  OpL (8R x R): rows oct * R + i, one product gives all eight
//        children's shifts of a parent's local.
// Only parents with children take part (compact slots from a scan at
// set-up).  A block takes 32 (M2M) or 64 (L2L) columns (parent slot x charge
// component); K chunks that hold only zero operator entries (the maps are
// triangular in the expansion order) are skipped:
//   k_m2m_mma  for each octant, stages the 32 children's moments in shared
//              memory (the B operand) and accumulates OpM's octant block on the
//              FP64 tensor cores (mma.sync m8n8k4, operator fragments read
//              from L2 once per 4 column tiles); then writes the parents.
//   k_l2l_mma  stages the 64 parents' locals, and for each 8-row tile of OpL
//              adds the product into the child of that row's octant (each
//              child coefficient has one writer: no atomics, deterministic).
// The sums differ from the direct ones in rounding order only (FP64, about
// 1e-16 relative per term).  Evaluations allocate nothing here, so they can
// be captured as CUDA graphs.
#include "eval_util.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace sfmm {
namespace {

constexpr int kShiftCols = 32;            // M2M columns per block: four 8-column MMA tiles
constexpr int kL2LTiles = 8;              // L2L: eight 8-column MMA tiles (64 columns) per block
constexpr int kL2LRowGroups = 4;          // L2L: the 8R output rows split over at least 4 blocks
constexpr int kM2MRowGroups = 2;          // M2M: the R output rows split over 2 blocks
constexpr int kShiftWarps = 8;

__host__ __device__ constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }

// padded leading dimension of a [col][k] operand buffer (>= k + 4, = 4 or
// 12 mod 16 doubles: the B-fragment loads are bank-conflict free)
__host__ __device__ constexpr int shift_ld(int k)
{
    int ld = k + 4;
    while (ld % 16 != 4 && ld % 16 != 12) ++ld;
    return ld;
}

__device__ __forceinline__ void mma884(double& d0, double& d1, double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Column k (input re / im part of coefficient k / 2) of the octant maps of
// one level, written in fragment order (lane l of fragment (rt, kc) holds
// A[8 rt + l / 4][4 kc + l % 4]):
//   M2M  fragment ((oct * RT + rt) * KC + kc), RT = ceil(R / 8), KC = ceil(R / 4)
//   L2L  fragment (rt * KC + kc), rt over the 8R rows oct * R + i
template<bool kM2M>
__global__ void k_shift_ops(const int* __restrict__ ptr, const int* __restrict__ code, const double* __restrict__ g,
                            const cplx* __restrict__ phase, int pp, double rho, double* __restrict__ op)
{
    const int Tn = (pp + 1) * (pp + 2) / 2, R = 2 * Tn, RT = cdiv(R, 8), KC = cdiv(R, 4);
    const int oct = blockIdx.x / R, k = blockIdx.x - oct * R, in = k >> 1, part = k & 1;
    extern __shared__ double sm[];
    double* rpow = sm;                                      // pp + 1 <= 32
    cplx* X = reinterpret_cast<cplx*>(sm + 32);
    for (int t = threadIdx.x; t < Tn; t += blockDim.x) X[t] = cplx{t == in && !part ? 1.0 : 0.0, t == in && part ? 1.0 : 0.0};
    if (threadIdx.x == 0) {
        rpow[0] = 1;
        for (int q = 1; q <= pp; ++q) rpow[q] = rpow[q - 1] * rho;
    }
    __syncthreads();
    const int kc = k >> 2, lc = k & 3;
    for (int o = threadIdx.x; o < Tn; o += blockDim.x) {
        const cplx v = shift_output<kM2M>(o, ptr, code, g, X, oct, rpow, phase + (oct & 3) * (2 * pp + 1), pp);
        for (int h = 0; h < 2; ++h) {
            const int row = kM2M ? 2 * o + h : oct * R + 2 * o + h;
            const int rt = row >> 3, lr = row & 7;
            const int64_t f = kM2M ? (int64_t(oct) * RT + rt) * KC + kc : int64_t(rt) * KC + kc;
            op[f * 32 + lr * 4 + lc] = h ? v.im : v.re;
        }
    }
}

__global__ void k_has_children(const int32_t* __restrict__ nchild, int64_t base, int64_t n, int32_t* __restrict__ flag)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        flag[i] = nchild[base + i] > 0 ? 1 : 0;
}

// slot -> node, and the slot of each level's first parent (S[q], q = 2..depth; S[depth] = total)
__global__ void k_slots(const int32_t* __restrict__ flag, const int32_t* __restrict__ slot, int64_t base, int64_t n,
                        int32_t* __restrict__ list, const int64_t* __restrict__ lvl, int depth, int32_t* __restrict__ S)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        if (flag[i]) list[slot[i]] = static_cast<int32_t>(base + i);
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (int q = 2; q <= depth; ++q) {
            const int64_t i = lvl[q] - base;
            S[q] = i < n ? slot[i] : (n ? slot[n - 1] + flag[n - 1] : 0);
        }
}

// Order of coefficient index t of the m >= 0 triangle, and the number of
// coefficients of orders < j.
__device__ __forceinline__ int tri_order(int t)
{
    int n, m;
    tri_nm(t, n, m);
    return n;
}
__host__ __device__ constexpr int tri_count(int j) { return j * (j + 1) / 2; }

// The shift maps are triangular in the expansion order: an M2M output of
// order j takes inputs of orders <= j, an L2L output of order j inputs of
// orders >= j.  K chunks that hold only zero operator entries are skipped
// (a zero product adds nothing, so the sums are unchanged).
__device__ __forceinline__ int m2m_kc_end(int rt, int R)
{
    const int r = min(8 * rt + 7, R - 1);                  // the tile's last (highest-order) row
    return min(cdiv(2 * tri_count(tri_order(r >> 1) + 1), 4), cdiv(R, 4));
}
__device__ __forceinline__ int l2l_kc_begin(int rt, int R)
{
    int jmin = 1 << 20;
    for (int q = 0; q < 8; ++q) {
        const int i = (8 * rt + q) % R;                    // coefficient row within its octant block
        jmin = min(jmin, tri_order(i >> 1));
    }
    return (2 * tri_count(jmin)) / 4;
}

// The block's columns (slot x component) and each slot's child per octant.
struct ShiftTile {
    int node[kShiftCols];                 // parent node of column c (-1 past the end)
    int b[kShiftCols];                    // charge component of column c
    int kid[kShiftCols][8];               // child node of column c's parent per octant (-1 absent)
};

// Columns [(blockIdx.x * per + h) * 32, + 32): part h of the block's per x 32 columns.
__device__ void shift_tile(ShiftTile& t, const int32_t* __restrict__ list, int32_t slot0, int64_t ncols, int qd,
                           const int32_t* __restrict__ child_beg, const int32_t* __restrict__ nchild,
                           const uint64_t* __restrict__ key, int per = 1, int h = 0)
{
    const int64_t c0 = (int64_t(blockIdx.x) * per + h) * kShiftCols;
    for (int c = threadIdx.x; c < kShiftCols; c += blockDim.x) {
        const int64_t col = c0 + c;
        for (int o = 0; o < 8; ++o) t.kid[c][o] = -1;
        if (col < ncols) {
            const int64_t s = col / qd;
            const int g = list[slot0 + s];
            t.node[c] = g;
            t.b[c] = static_cast<int>(col - s * qd);
            const int cb = child_beg[g], nc = nchild[g];
            for (int k = cb; k < cb + nc; ++k) t.kid[c][key[k] & 7] = k;
        } else {
            t.node[c] = -1;
            t.b[c] = 0;
        }
    }
}

// M2M into the parents of one level: columns [blockIdx.x * 32, + 32) of the
// ncols = slots x qd columns; op = that level's OpM fragments.
__global__ void __launch_bounds__(32 * kShiftWarps) k_m2m_mma(const double* __restrict__ op, int R,
                                                              const int32_t* __restrict__ list, int32_t slot0,
                                                              int64_t ncols, int qd, const int32_t* __restrict__ child_beg,
                                                              const int32_t* __restrict__ nchild,
                                                              const uint64_t* __restrict__ key, double* __restrict__ M)
{
    constexpr int kMaxRowTiles = 5;       // R / 8 / warps: R <= 306 (p <= 16)
    __shared__ ShiftTile tile;
    extern __shared__ double Bs[];        // [32 cols][LD]
    const int RT = cdiv(R, 8), KC = cdiv(R, 4), LD = shift_ld(4 * KC);
    // this block's share of the R output rows: row tiles [rt0, rt1)
    const int per = cdiv(RT, gridDim.y), rt0 = blockIdx.y * per, rt1 = min(RT, rt0 + per);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, lr = lane >> 2, lc = lane & 3;
    shift_tile(tile, list, slot0, ncols, qd, child_beg, nchild, key);
    double acc[kMaxRowTiles][4][2];
#pragma unroll
    for (int j = 0; j < kMaxRowTiles; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[j][q][0] = acc[j][q][1] = 0.0;
    for (int oct = 0; oct < 8; ++oct) {
        __syncthreads();                  // the tile is set / the previous octant's operands are consumed
        for (int e = threadIdx.x; e < kShiftCols * LD; e += blockDim.x) {
            const int c = e / LD, k = e - c * LD;
            const int kid = tile.kid[c][oct];
            Bs[e] = (k < R && kid >= 0) ? M[(int64_t(kid) * qd + tile.b[c]) * R + k] : 0.0;
        }
        __syncthreads();
        const double* fo = op + int64_t(oct) * RT * KC * 32 + lane;
#pragma unroll
        for (int j = 0; j < kMaxRowTiles; ++j) {
            const int rt = rt0 + warp + kShiftWarps * j;
            if (rt >= rt1) break;
            const double* fr = fo + int64_t(rt) * KC * 32;
            const int kce = m2m_kc_end(rt, R);
            // operator fragments four K chunks ahead of their products
            double a4[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) a4[u] = u < kce ? __ldg(fr + u * 32) : 0.0;
            for (int kc = 0; kc < kce; kc += 4) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const double a = a4[u];
                    a4[u] = kc + 4 + u < kce ? __ldg(fr + (kc + 4 + u) * 32) : 0.0;
                    if (kc + u < kce) {
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            mma884(acc[j][q][0], acc[j][q][1], a, Bs[(q * 8 + lr) * LD + 4 * (kc + u) + lc]);
                    }
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < kMaxRowTiles; ++j) {
        const int rt = rt0 + warp + kShiftWarps * j;
        if (rt >= rt1) break;
        const int r = 8 * rt + lr;
        if (r >= R) continue;
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = q * 8 + 2 * lc + h;
                if (tile.node[c] >= 0) M[(int64_t(tile.node[c]) * qd + tile.b[c]) * R + r] = acc[j][q][h];
            }
    }
}

// L2L into the children of one level; blockIdx.y = 0: potential local
// (LA, R = 2T), 1: field local (LB, R = 2 T1).
struct L2LSide {
    const double* op;
    int R;
    double* L;
};

template<int NQ>                          // NQ 8-column MMA tiles: 8 NQ columns per block
__global__ void __launch_bounds__(32 * kShiftWarps) k_l2l_mma(L2LSide sa, L2LSide sb, const int32_t* __restrict__ list,
                                                              int32_t slot0, int64_t ncols, int qd,
                                                              const int32_t* __restrict__ child_beg,
                                                              const int32_t* __restrict__ nchild,
                                                              const uint64_t* __restrict__ key)
{
    constexpr int NC = 8 * NQ;
    const L2LSide sd = blockIdx.y ? sb : sa;
    if (!sd.L) return;
    __shared__ ShiftTile tile[NQ / 4];
    extern __shared__ double Bs[];        // [NC cols][LD]
    const int R = sd.R, RT8 = R, KC = cdiv(R, 4), LD = shift_ld(4 * KC);   // 8R rows: R row tiles
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, lr = lane >> 2, lc = lane & 3;
    for (int h = 0; h < NQ / 4; ++h) shift_tile(tile[h], list, slot0, ncols, qd, child_beg, nchild, key, NQ / 4, h);
    __syncthreads();
    for (int e = threadIdx.x; e < NC * LD; e += blockDim.x) {
        const int c = e / LD, k = e - c * LD;
        const int g = tile[c / kShiftCols].node[c % kShiftCols];
        Bs[e] = (k < R && g >= 0) ? sd.L[(int64_t(g) * qd + tile[c / kShiftCols].b[c % kShiftCols]) * R + k] : 0.0;
    }
    __syncthreads();
    // this block's share of the 8R output rows: row tiles [rt0, rt1)
    const int per = cdiv(RT8, gridDim.z), rt0 = blockIdx.z * per, rt1 = min(RT8, rt0 + per);
    for (int rt = rt0 + warp; rt < rt1; rt += kShiftWarps) {
        double acc[NQ][2] = {};
        const double* fr = sd.op + int64_t(rt) * KC * 32 + lane;
        const int kcb = l2l_kc_begin(rt, R);
        // operator fragments four K chunks ahead of their products
        double a4[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) a4[u] = kcb + u < KC ? __ldg(fr + (kcb + u) * 32) : 0.0;
        for (int kc = kcb; kc < KC; kc += 4) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const double a = a4[u];
                a4[u] = kc + 4 + u < KC ? __ldg(fr + (kc + 4 + u) * 32) : 0.0;
                if (kc + u < KC) {
#pragma unroll
                    for (int q = 0; q < NQ; ++q)
                        mma884(acc[q][0], acc[q][1], a, Bs[(q * 8 + lr) * LD + 4 * (kc + u) + lc]);
                }
            }
        }
        const int row = 8 * rt + lr, oct = row / R, i = row - oct * R;
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = q * 8 + 2 * lc + h;
                const ShiftTile& t = tile[c / kShiftCols];
                const int cc = c % kShiftCols;
                const int kid = t.node[cc] >= 0 ? t.kid[cc][oct] : -1;
                if (kid >= 0) sd.L[(int64_t(kid) * qd + t.b[cc]) * R + i] += acc[q][h];
            }
    }
}

unsigned grid_for(int64_t n, int sms) { return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, int64_t(sms) * 16))); }

// fragment counts of one level's maps
__host__ __device__ int64_t m2m_frags(int R) { return int64_t(8) * cdiv(R, 8) * cdiv(R, 4); }
__host__ __device__ int64_t l2l_frags(int R) { return int64_t(R) * cdiv(R, 4); }

// rho of each children level 3 .. depth (index l - 3)
struct LevelRho {
    double rho[kKeyLevel];
};

// A level's maps from the maps at rho = 1: every M2M / L2L term of output
// order n(out) and input order n(in) carries rho^|n(out) - n(in)|, so entry
// (out, in) is the unit entry times that power (the power taken as the same
// running product the term sums use).  Zero and padding entries stay zero.
__global__ void k_shift_scale(const double* __restrict__ unit, int64_t per_level, int nlev, LevelRho r, int RA, int RB,
                              double* __restrict__ out)
{
    const int64_t fm = m2m_frags(RA), fla = l2l_frags(RA);
    const int64_t total = per_level * nlev;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const int lv = static_cast<int>(i / per_level);
        const int64_t e = i - int64_t(lv) * per_level;
        double v = unit[e];
        if (v != 0.0) {
            int64_t f = e >> 5;
            const int lr = static_cast<int>(e & 31) >> 2, lc = static_cast<int>(e & 3);
            int row, col;
            if (f < fm) {                                   // OpM: ((oct * RT + rt) * KC + kc)
                const int KC = cdiv(RA, 4), RT = cdiv(RA, 8);
                const int kc = static_cast<int>(f % KC), rt = static_cast<int>((f / KC) % RT);
                row = 8 * rt + lr;
                col = 4 * kc + lc;
            } else {                                        // OpL: (rt * KC + kc), rows oct * R + i
                const bool la = f < fm + fla;
                const int R = la ? RA : RB, KC = cdiv(R, 4);
                f -= la ? fm : fm + fla;
                row = (8 * static_cast<int>(f / KC) + lr) % R;
                col = 4 * static_cast<int>(f % KC) + lc;
            }
            const int pw = abs(tri_order(row >> 1) - tri_order(col >> 1));
            double s = 1.0;
            for (int q = 0; q < pw; ++q) s *= r.rho[lv];
            v *= s;
        }
        out[i] = v;
    }
}

}  // namespace

// The shift maps at rho = 1 for order p (OpM, OpLA, OpLB in the fragment
// order of one level), built once per (device, p) with the term sums.
void build_unit_shift_ops(PlanTables& tab, int p, cudaStream_t st)
{
    const int T = (p + 1) * (p + 2) / 2, T1 = (p + 2) * (p + 3) / 2, RA = 2 * T, RB = 2 * T1;
    const int64_t per_level = (m2m_frags(RA) + l2l_frags(RA) + l2l_frags(RB)) * 32;
    tab.sh_unit.alloc(per_level, st);
    SFMM_CUDA(cudaMemsetAsync(tab.sh_unit.ptr, 0, size_t(per_level) * sizeof(double), st));
    double* op = tab.sh_unit.ptr;
    const size_t shm = (32 + 2 * (T1 + 1)) * sizeof(double);
    k_shift_ops<true><<<8 * RA, 128, shm, st>>>(tab.m2m_ptr.ptr, tab.m2m_code.ptr, tab.m2m_g.ptr,
                                                reinterpret_cast<const cplx*>(tab.echild.ptr), p, 1.0, op);
    SFMM_CHECK_LAUNCH();
    k_shift_ops<false><<<8 * RA, 128, shm, st>>>(tab.l2l_ptr.ptr, tab.l2l_code.ptr, tab.l2l_g.ptr,
                                                 reinterpret_cast<const cplx*>(tab.eparent.ptr), p, 1.0,
                                                 op + m2m_frags(RA) * 32);
    SFMM_CHECK_LAUNCH();
    k_shift_ops<false><<<8 * RB, 128, shm, st>>>(tab.l2l1_ptr.ptr, tab.l2l1_code.ptr, tab.l2l1_g.ptr,
                                                 reinterpret_cast<const cplx*>(tab.eparent1.ptr), p + 1, 1.0,
                                                 op + (m2m_frags(RA) + l2l_frags(RA)) * 32);
    SFMM_CHECK_LAUNCH();
}

void shift_setup(Plan& pl)
{
    Tree& t = *pl.tree;
    pl.shift_on = false;
    if (t.depth < 3) return;
    Context& c = *t.ctx;
    cudaStream_t st = c.stream;
    const int RA = 2 * pl.T, RB = 2 * pl.T1;
    // parents of levels 2 .. depth - 1 with children: compact slots
    const int64_t base = t.lvl_off[2], n = t.lvl_off[t.depth] - base;
    DevBuf<int32_t> flag;
    flag.alloc(n, st);
    pl.sh_slot.alloc(n + 1, st);                        // exclusive scans write n + 1 entries
    pl.sh_list.alloc(std::max<int64_t>(n, 1), st);
    k_has_children<<<grid_for(n, c.sm_count), 256, 0, st>>>(t.nchild.ptr, base, n, flag.ptr);
    SFMM_CHECK_LAUNCH();
    exclusive_scan_i32(flag.ptr, pl.sh_slot.ptr, n, st);
    DevBuf<int64_t> lvl;
    lvl.alloc(t.lvl_off.size(), st);
    SFMM_CUDA(cudaMemcpyAsync(lvl.ptr, t.lvl_off.data(), t.lvl_off.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    DevBuf<int32_t> S;
    S.alloc(t.depth + 1, st);
    k_slots<<<grid_for(n, c.sm_count), 256, 0, st>>>(flag.ptr, pl.sh_slot.ptr, base, n, pl.sh_list.ptr, lvl.ptr, t.depth, S.ptr);
    SFMM_CHECK_LAUNCH();
    pl.sh_S.assign(t.depth + 1, 0);
    SFMM_CUDA(cudaMemcpyAsync(pl.sh_S.data(), S.ptr, (t.depth + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SFMM_CUDA(cudaStreamSynchronize(st));
    // maps per children level 3 .. depth, fragment order: OpM (RA x 8RA),
    // OpLA (8RA x RA), OpLB (8RB x RB); zero padding rows / columns; each
    // the order's maps at rho = 1 scaled to the level's rho
    const int64_t per_level = (m2m_frags(RA) + l2l_frags(RA) + l2l_frags(RB)) * 32;
    const int nlev = t.depth - 2;
    pl.sh_ops.alloc(size_t(per_level) * nlev, st);
    LevelRho r{};
    for (int l = 3; l <= t.depth; ++l) r.rho[l - 3] = std::sqrt(0.75) * t.box.width / double(1 << l);
    k_shift_scale<<<grid_for(per_level * nlev, c.sm_count), 256, 0, st>>>(pl.tab->sh_unit.ptr, per_level, nlev, r, RA,
                                                                          RB, pl.sh_ops.ptr);
    SFMM_CHECK_LAUNCH();
    const size_t smem = size_t(8 * kL2LTiles) * shift_ld(4 * cdiv(RB, 4)) * sizeof(double);
    SFMM_REQUIRE(smem + 2 * sizeof(ShiftTile) <= 227 * 1024, FMM_ERR_UNSUPPORTED, "shift operands exceed shared memory");
    allow_max_smem(k_m2m_mma);
    allow_max_smem(k_l2l_mma<kL2LTiles>);
    pl.shift_on = true;
}

void shift_m2m(Plan& pl, const EvalArgs& a, int lp, cudaStream_t st)
{
    Tree& t = *pl.tree;
    const int qd = pl.qdim, R = 2 * pl.T;
    const int32_t slot0 = pl.sh_S[lp];
    const int64_t n = pl.sh_S[lp + 1] - slot0;
    if (n <= 0) return;
    const int lc = lp + 1;
    const int64_t per_level = (m2m_frags(R) + l2l_frags(R) + l2l_frags(2 * pl.T1)) * 32;
    const double* op = pl.sh_ops.ptr + per_level * (lc - 3);
    const int64_t ncols = n * qd;
    const size_t smem = size_t(kShiftCols) * shift_ld(4 * cdiv(R, 4)) * sizeof(double);
    k_m2m_mma<<<dim3(static_cast<unsigned>((ncols + kShiftCols - 1) / kShiftCols), kM2MRowGroups), 32 * kShiftWarps, smem,
                st>>>(
        op, R, pl.sh_list.ptr, slot0, ncols, qd, t.child_beg.ptr, t.nchild.ptr, t.key.ptr, reinterpret_cast<double*>(a.M));
    SFMM_CHECK_LAUNCH();
}

void shift_l2l(Plan& pl, const EvalArgs& a, int lc, cudaStream_t st)
{
    Tree& t = *pl.tree;
    const int qd = pl.qdim, RA = 2 * pl.T, RB = 2 * pl.T1;
    const int32_t slot0 = pl.sh_S[lc - 1];
    const int64_t n = pl.sh_S[lc] - slot0;
    if (n <= 0) return;
    const int64_t per_level = (m2m_frags(RA) + l2l_frags(RA) + l2l_frags(RB)) * 32;
    const double* op = pl.sh_ops.ptr + per_level * (lc - 3);
    const L2LSide sa{op + m2m_frags(RA) * 32, RA, a.want_pot ? reinterpret_cast<double*>(a.LA) : nullptr};
    const L2LSide sb{op + (m2m_frags(RA) + l2l_frags(RA)) * 32, RB, a.want_field ? reinterpret_cast<double*>(a.LB) : nullptr};
    const int64_t ncols = n * qd;
    constexpr int NC = 8 * kL2LTiles;
    const size_t smem = size_t(NC) * shift_ld(4 * cdiv(RB, 4)) * sizeof(double);
    // small levels (few column tiles) split their rows over more blocks so
    // the level still spreads over the SMs (each block keeps >= 8 row tiles)
    const int64_t ctiles = (ncols + NC - 1) / NC;
    const int rg = static_cast<int>(std::min<int64_t>(std::max<int64_t>(kL2LRowGroups, int64_t(t.ctx->sm_count) / ctiles),
                                                      std::max(1, RA / kShiftWarps)));
    k_l2l_mma<kL2LTiles><<<dim3(static_cast<unsigned>(ctiles), 2, static_cast<unsigned>(rg)), 32 * kShiftWarps, smem, st>>>(
        sa, sb, pl.sh_list.ptr, slot0, ncols, qd, t.child_beg.ptr, t.nchild.ptr, t.key.ptr);
    SFMM_CHECK_LAUNCH();
}

}  // namespace sfmm
