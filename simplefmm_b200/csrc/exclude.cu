// Excluded interactions: the reference's self_generator / is_self hook
// (fmm.hpp:204, 398-408, 773-807).  For target i and each listed source
// j != i the evaluation has included the pair (exactly in the near field,
// through the expansions otherwise); this pass subtracts the exact pair term
// Q_j / |x_i - x_j| (and its field) again:
//   near_too = 0: only for j outside i's near field -- the reference's slist,
//                 which rinv(Q, U) always removes (the default is_self only
//                 skips i == j inside the near field);
//   near_too = 1: for every listed j -- rinv(Q, U, is_self) with an is_self
//                 that names the same pairs.
// A near-field pair is removed by subtracting the same FP64 term P2P added.
// One thread per target walks its list in order (deterministic).
#include "fmm_eval.cuh"

namespace sfmm {
namespace {

__global__ void k_inverse_order(const int32_t* __restrict__ order, int64_t n, int32_t* __restrict__ inv)
{
    for (int64_t s = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; s < n; s += int64_t(gridDim.x) * blockDim.x)
        inv[order[s]] = static_cast<int32_t>(s);
}

__global__ void k_point_leaf(const int32_t* __restrict__ leaf_node, const int32_t* __restrict__ pbeg,
                             const int32_t* __restrict__ pend, int64_t n_leaves, int32_t* __restrict__ leaf_of)
{
    for (int64_t f = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; f < n_leaves; f += int64_t(gridDim.x) * blockDim.x) {
        const int g = leaf_node[f];
        for (int s = pbeg[g]; s < pend[g]; ++s) leaf_of[s] = static_cast<int32_t>(f);
    }
}

__global__ void k_exclude(int64_t n, int qdim, int near_too, const int64_t* __restrict__ ptr,
                          const int32_t* __restrict__ col, const int32_t* __restrict__ inv,
                          const int32_t* __restrict__ leaf_of, const int32_t* __restrict__ nr_ptr,
                          const int2* __restrict__ nr, const double* __restrict__ px, const double* __restrict__ py,
                          const double* __restrict__ pz, const double* __restrict__ Q, double* __restrict__ pot,
                          double* __restrict__ field)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t e0 = ptr[i], e1 = ptr[i + 1];
        if (e0 >= e1) continue;
        const int si = inv[i];
        const int f = leaf_of[si];
        const int r0 = nr_ptr[f], r1 = nr_ptr[f + 1];
        double dp[3] = {0, 0, 0}, df[3] = {0, 0, 0};
        for (int64_t e = e0; e < e1; ++e) {
            const int j = col[e];
            if (j == i || j < 0 || j >= n) continue;           // self is always excluded; bad ids ignored
            const int sj = inv[j];
            if (!near_too) {
                bool near = false;
                for (int r = r0; r < r1 && !near; ++r) near = sj >= nr[r].x && sj < nr[r].y;
                if (near) continue;
            }
            const double R[3] = {px[si] - px[sj], py[si] - py[sj], pz[si] - pz[sj]};
            const double r = sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]);
            for (int b = 0; b < qdim; ++b) dp[b] += Q[int64_t(j) * qdim + b] / r;
            const double r3 = r * r * r;
            if (qdim == 1) {
                for (int c = 0; c < 3; ++c) df[c] += Q[j] * R[c] / r3;
            } else if (qdim == 3) {
                const double* q = Q + int64_t(j) * 3;
                df[0] += (q[1] * R[2] - q[2] * R[1]) / r3;
                df[1] += (q[2] * R[0] - q[0] * R[2]) / r3;
                df[2] += (q[0] * R[1] - q[1] * R[0]) / r3;
            }
        }
        if (pot)
            for (int b = 0; b < qdim; ++b) pot[i * qdim + b] -= dp[b];
        if (field)
            for (int c = 0; c < 3; ++c) field[i * 3 + c] -= df[c];
    }
}

}  // namespace

void plan_set_exclusions(Plan& pl, const int64_t* ptr, const int32_t* cols, int near_too)
{
    Tree& t = *pl.tree;
    cudaStream_t st = t.ctx->stream;
    const int64_t n = t.n;
    int64_t nnz = 0;
    SFMM_CUDA(cudaMemcpyAsync(&nnz, ptr + n, sizeof(nnz), cudaMemcpyDeviceToHost, st));
    SFMM_CUDA(cudaStreamSynchronize(st));
    SFMM_REQUIRE(nnz >= 0, FMM_ERR_INVALID_ARGUMENT, "exclusion row pointers must end with a count >= 0");
    pl.ex_ptr.alloc(n + 1, st);
    SFMM_CUDA(cudaMemcpyAsync(pl.ex_ptr.ptr, ptr, size_t(n + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, st));
    pl.ex_col.alloc(std::max<int64_t>(nnz, 1), st);
    if (nnz) SFMM_CUDA(cudaMemcpyAsync(pl.ex_col.ptr, cols, size_t(nnz) * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    pl.ex_inv.alloc(n, st);
    pl.ex_leaf.alloc(n, st);
    k_inverse_order<<<blocks_for(n, 256, 8192), 256, 0, st>>>(t.order.ptr, n, pl.ex_inv.ptr);
    SFMM_CHECK_LAUNCH();
    k_point_leaf<<<blocks_for(t.n_leaves, 256, 8192), 256, 0, st>>>(t.leaf_node.ptr, t.pbeg.ptr, t.pend.ptr,
                                                                      t.n_leaves, pl.ex_leaf.ptr);
    SFMM_CHECK_LAUNCH();
    pl.ex_near_too = near_too ? 1 : 0;
    pl.ex_on = true;
}

void plan_clear_exclusions(Plan& pl)
{
    pl.ex_on = false;
    pl.ex_ptr.release();
    pl.ex_col.release();
    pl.ex_inv.release();
    pl.ex_leaf.release();
}

void apply_exclusions(const Plan& pl, const double* Q, double* pot, double* field)
{
    const Tree& t = *pl.tree;
    cudaStream_t st = t.ctx->stream;
    k_exclude<<<blocks_for(t.n, 128, 8192), 128, 0, st>>>(
        t.n, pl.qdim, pl.ex_near_too, pl.ex_ptr.ptr, pl.ex_col.ptr, pl.ex_inv.ptr, pl.ex_leaf.ptr, t.nr_ptr.ptr,
        t.nr.ptr, t.pts.ptr, t.pts.ptr + t.n, t.pts.ptr + 2 * t.n, Q, pot, field);
    SFMM_CHECK_LAUNCH();
}

}  // namespace sfmm
