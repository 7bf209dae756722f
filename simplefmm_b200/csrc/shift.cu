// M2M and L2L (fmm.hpp:558-590, 714-745) as FP64 matrix products on the
// tensor cores.
//
// A shift between a box and one of its children is a fixed real-linear map
// on the box's coefficient row (the m >= 0 triangle stored as re, im pairs:
// R = 2T doubles) that depends only on the child's octant and on the level
// (through rho = sqrt(3/4) w / 2^l).  Per children level the maps are built
// once per plan by applying the direct term sums of fmm_ops.cuh
// (shift_output, the same code as k_m2m / k_l2l) to unit vectors:
//   L2L  OpL (8R x R): rows oct * R + i, so one product gives all eight
//        children's shifts of a parent's local;
//   M2M  OpM (R x 8R): columns oct * R + i, applied to a parent's eight
//        children stacked (absent children are zero columns).
// Only parents with children take part: their compact slots come from a
// scan at set-up.  Per level, a gather kernel stacks the rows, one cuBLAS
// DGEMM (FP64 tensor cores) applies the map to every slot, and a scatter
// kernel adds the result to the children (L2L) or writes the parents (M2M).
// The sums differ from the direct ones in rounding order only (FP64, about
// 1e-16 relative per term).
#include "eval_util.cuh"

#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <vector>

namespace sfmm {
namespace {

#define SFMM_BLAS(call)                                                                              \
    do {                                                                                             \
        const cublasStatus_t s_ = (call);                                                            \
        if (s_ != CUBLAS_STATUS_SUCCESS)                                                             \
            throw Error(FMM_ERR_CUDA, std::string("cuBLAS error ") + std::to_string(int(s_)) + " in " #call); \
    } while (0)

constexpr size_t kBlasWorkspace = size_t(32) << 20;

// Column k (input re / im part of coefficient k / 2) of the octant maps of one level.
template<bool kM2M>
__global__ void k_shift_ops(const int* __restrict__ ptr, const int* __restrict__ code, const double* __restrict__ g,
                            const cplx* __restrict__ phase, int pp, double rho, double* __restrict__ op)
{
    const int Tn = (pp + 1) * (pp + 2) / 2, R = 2 * Tn;
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
    for (int o = threadIdx.x; o < Tn; o += blockDim.x) {
        const cplx v = shift_output<kM2M>(o, ptr, code, g, X, oct, rpow, phase + (oct & 3) * (2 * pp + 1), pp);
        const int64_t idx = kM2M ? int64_t(oct * R + k) * R + 2 * o : int64_t(k) * 8 * R + oct * R + 2 * o;
        op[idx] = v.re;
        op[idx + 1] = v.im;
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

// M2M: children of level lc stacked under their parent's slot
__global__ void k_m2m_gather(const double* __restrict__ M, const uint64_t* __restrict__ key, const int32_t* __restrict__ parent,
                             const int32_t* __restrict__ slot, int64_t base, int32_t slot0, int64_t c0, int64_t nc, int qd,
                             int R, double* __restrict__ X)
{
    const int64_t per = int64_t(qd) * R, total = nc * per;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t c = c0 + i / per;
        const int e = static_cast<int>(i % per), b = e / R, r = e - b * R;
        const int s = slot[parent[c] - base] - slot0, oct = static_cast<int>(key[c] & 7);
        X[(int64_t(s) * qd + b) * 8 * R + oct * R + r] = M[c * per + e];
    }
}

// rows of the n slots -> nodes list[slot0 + s] (add = false) or from them (gather)
__global__ void k_slot_rows(double* __restrict__ node_rows, const int32_t* __restrict__ list, int32_t slot0, int64_t n, int qd,
                            int R, double* __restrict__ slot_rows, bool to_nodes)
{
    const int64_t per = int64_t(qd) * R, total = n * per;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t s = i / per, e = i - s * per;
        const int64_t g = list[slot0 + s];
        if (to_nodes) node_rows[g * per + e] = slot_rows[i];
        else slot_rows[i] = node_rows[g * per + e];
    }
}

// L2L: each child of level lc adds its octant's block of its parent's product
__global__ void k_l2l_scatter(double* __restrict__ L, const uint64_t* __restrict__ key, const int32_t* __restrict__ parent,
                              const int32_t* __restrict__ slot, int64_t base, int32_t slot0, int64_t c0, int64_t nc, int qd,
                              int R, const double* __restrict__ Y)
{
    const int64_t per = int64_t(qd) * R, total = nc * per;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t c = c0 + i / per;
        const int e = static_cast<int>(i % per), b = e / R, r = e - b * R;
        const int s = slot[parent[c] - base] - slot0, oct = static_cast<int>(key[c] & 7);
        L[c * per + e] += Y[(int64_t(s) * qd + b) * 8 * R + oct * R + r];
    }
}

unsigned grid_for(int64_t n, int sms) { return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, int64_t(sms) * 16))); }

cublasHandle_t blas(Context& c)
{
    if (!c.blas) {
        cublasHandle_t h = nullptr;
        SFMM_BLAS(cublasCreate(&h));
        c.blas = h;
        c.blas_ws = device_alloc(kBlasWorkspace, c.device, c.stream);
        SFMM_BLAS(cublasSetWorkspace(h, c.blas_ws, kBlasWorkspace));
    }
    return static_cast<cublasHandle_t>(c.blas);
}

}  // namespace

void release_blas(Context& c) noexcept
{
    if (c.blas) cublasDestroy(static_cast<cublasHandle_t>(c.blas));
    if (c.blas_ws) device_free(c.blas_ws, kBlasWorkspace, c.device, c.stream);
    c.blas = nullptr;
    c.blas_ws = nullptr;
}

void shift_setup(Plan& pl)
{
    Tree& t = *pl.tree;
    pl.shift_on = false;
    if (t.depth < 3) return;
    Context& c = *t.ctx;
    cudaStream_t st = c.stream;
    blas(c);
    const int p = pl.p, qd = pl.qdim, RA = 2 * pl.T, RB = 2 * pl.T1;
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
    // operators per children level 3 .. depth: OpM (RA x 8RA), OpLA (8RA x RA), OpLB (8RB x RB)
    const int64_t per_level = 8LL * RA * RA * 2 + 8LL * RB * RB;
    pl.sh_ops.alloc(size_t(per_level) * (t.depth - 2), st);
    int64_t max_slots = 0;
    for (int l = 3; l <= t.depth; ++l) {
        double* op = pl.sh_ops.ptr + per_level * (l - 3);
        const double rho = std::sqrt(0.75) * t.box.width / double(1 << l);
        const size_t shm = (32 + 2 * (pl.T1 + 1)) * sizeof(double);
        k_shift_ops<true><<<8 * RA, 128, shm, st>>>(pl.tab->m2m_ptr.ptr, pl.tab->m2m_code.ptr, pl.tab->m2m_g.ptr,
                                                    reinterpret_cast<const cplx*>(pl.tab->echild.ptr), p, rho, op);
        SFMM_CHECK_LAUNCH();
        k_shift_ops<false><<<8 * RA, 128, shm, st>>>(pl.tab->l2l_ptr.ptr, pl.tab->l2l_code.ptr, pl.tab->l2l_g.ptr,
                                                     reinterpret_cast<const cplx*>(pl.tab->eparent.ptr), p, rho,
                                                     op + 8LL * RA * RA);
        SFMM_CHECK_LAUNCH();
        k_shift_ops<false><<<8 * RB, 128, shm, st>>>(pl.tab->l2l1_ptr.ptr, pl.tab->l2l1_code.ptr, pl.tab->l2l1_g.ptr,
                                                     reinterpret_cast<const cplx*>(pl.tab->eparent1.ptr), p + 1, rho,
                                                     op + 16LL * RA * RA);
        SFMM_CHECK_LAUNCH();
        max_slots = std::max<int64_t>(max_slots, pl.sh_S[l] - pl.sh_S[l - 1]);
    }
    pl.sh_x.alloc(size_t(std::max<int64_t>(max_slots, 1)) * qd * 8 * RB, st);
    pl.sh_y.alloc(size_t(std::max<int64_t>(max_slots, 1)) * qd * 8 * RB, st);
    pl.shift_on = true;
}

void shift_m2m(Plan& pl, const EvalArgs& a, int lp, cudaStream_t st)
{
    Tree& t = *pl.tree;
    const int qd = pl.qdim, R = 2 * pl.T, sms = t.ctx->sm_count;
    const int32_t slot0 = pl.sh_S[lp];
    const int64_t n = pl.sh_S[lp + 1] - slot0;
    if (n <= 0) return;
    const int lc = lp + 1;
    const int64_t c0 = t.lvl_off[lc], nc = t.lvl_off[lc + 1] - c0, base = t.lvl_off[2];
    const double* op = pl.sh_ops.ptr + (8LL * R * R * 2 + 8LL * (2 * pl.T1) * (2 * pl.T1)) * (lc - 3);
    SFMM_CUDA(cudaMemsetAsync(pl.sh_x.ptr, 0, size_t(n) * qd * 8 * R * sizeof(double), st));
    k_m2m_gather<<<grid_for(nc * qd * R, sms), 256, 0, st>>>(reinterpret_cast<const double*>(a.M), a.key, a.parent,
                                                            pl.sh_slot.ptr, base, slot0, c0, nc, qd, R, pl.sh_x.ptr);
    SFMM_CHECK_LAUNCH();
    cublasHandle_t h = blas(*t.ctx);
    SFMM_BLAS(cublasSetStream(h, st));
    const double one = 1.0, zero = 0.0;
    SFMM_BLAS(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, R, static_cast<int>(n * qd), 8 * R, &one, op, R, pl.sh_x.ptr, 8 * R,
                          &zero, pl.sh_y.ptr, R));
    k_slot_rows<<<grid_for(n * qd * R, sms), 256, 0, st>>>(reinterpret_cast<double*>(a.M), pl.sh_list.ptr, slot0, n, qd, R,
                                                          pl.sh_y.ptr, true);
    SFMM_CHECK_LAUNCH();
}

void shift_l2l(Plan& pl, const EvalArgs& a, int lc, cudaStream_t st)
{
    Tree& t = *pl.tree;
    const int qd = pl.qdim, RA = 2 * pl.T, RB = 2 * pl.T1, sms = t.ctx->sm_count;
    const int32_t slot0 = pl.sh_S[lc - 1];
    const int64_t n = pl.sh_S[lc] - slot0;
    if (n <= 0) return;
    const int64_t c0 = t.lvl_off[lc], nc = t.lvl_off[lc + 1] - c0, base = t.lvl_off[2];
    const double* op = pl.sh_ops.ptr + (8LL * RA * RA * 2 + 8LL * RB * RB) * (lc - 3);
    cublasHandle_t h = blas(*t.ctx);
    SFMM_BLAS(cublasSetStream(h, st));
    const double one = 1.0, zero = 0.0;
    for (int which = 0; which < 2; ++which) {
        if (which == 0 && !a.want_pot) continue;
        if (which == 1 && !a.want_field) continue;
        const int R = which ? RB : RA;
        double* L = reinterpret_cast<double*>(which ? a.LB : a.LA);
        const double* opl = which ? op + 16LL * RA * RA : op + 8LL * RA * RA;
        k_slot_rows<<<grid_for(n * qd * R, sms), 256, 0, st>>>(L, pl.sh_list.ptr, slot0, n, qd, R, pl.sh_x.ptr, false);
        SFMM_CHECK_LAUNCH();
        SFMM_BLAS(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, 8 * R, static_cast<int>(n * qd), R, &one, opl, 8 * R, pl.sh_x.ptr, R,
                              &zero, pl.sh_y.ptr, 8 * R));
        k_l2l_scatter<<<grid_for(nc * qd * R, sms), 256, 0, st>>>(L, a.key, a.parent, pl.sh_slot.ptr, base, slot0, c0, nc, qd, R,
                                                                 pl.sh_y.ptr);
        SFMM_CHECK_LAUNCH();
    }
}

}  // namespace sfmm
