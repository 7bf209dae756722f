// Batched solves: several independent point sets evaluated by one plan.
//
// Each set's tree is built on its own, exactly as a single solve builds it
// (its own fitted root cube, keys, lists).  The trees are then merged into
// a forest: one Tree whose nodes are the members' nodes level by level
// (level l holds member 0's level-l nodes, then member 1's, ...), whose
// leaves are ordered the same way, and whose points are the members' points
// one member after another, each scaled into the unit cube by its own box,
// x' = (x - corner) / width.  The keys are unchanged: a key is
// trunc((x - corner) / width 2^20), the same number for x and x' in the unit
// cube.  All members so share one geometry -- the unit cube -- and every
// per-level table of a plan (shift operators, translation powers) serves all
// of them, while no list connects two members: the evaluation kernels run
// over all members at once and each member's results are those of its solve
// alone, in scaled units (potential x width, field x width^2), which the
// batch undoes.  The one per-level quantity of the evaluation that depends on
// the data, the moment scale of the tensor-core M2L, is kept per member
// (node_tree).
//
// fmm_solve_batch: upload, per-member builds, merge, plan, evaluation through
// a CUDA graph that the context keeps and updates in place for the next batch
// of the same launch shape (cudaGraphExecUpdate), download, rescale.
#include "eval_util.cuh"

#include <algorithm>
#include <vector>

namespace sfmm {
namespace {

constexpr int kLv = kKeyLevel + 2;

// Device view of one member tree and its place in the forest.
struct MemberView {
    int64_t n, pbase;                    // points; first forest point
    int depth;
    int64_t lvl_off[kLv], leaf_off[kLv]; // the member's own offsets
    int64_t nbase[kLv], lbase[kLv];      // forest index of its first node / leaf of each level
    double corner[3], width;
    const uint64_t* key;
    const int32_t *pbeg, *pend, *parent, *child_beg, *nchild, *leaf_id, *leaf_node, *colleague;
    const int32_t *il_ptr, *il_src, *il_code, *nr_ptr, *order;
    const int2* nr;
    const double* pts;
};

struct ForestArgs {
    const MemberView* m;
    int count, depth;
    int64_t lvl_off[kLv], leaf_off[kLv];
};

__device__ inline int find_level(const int64_t* off, int depth, int64_t x)
{
    int l = 0;
    while (l < depth && x >= off[l + 1]) ++l;
    return l;
}

// member holding forest index x of level l (bases ascend with the member)
__device__ inline int find_member(const ForestArgs& f, bool leaves, int l, int64_t x)
{
    int r = 0;
    while (r + 1 < f.count && x >= (leaves ? f.m[r + 1].lbase[l] : f.m[r + 1].nbase[l])) ++r;
    return r;
}

__device__ inline int32_t map_node(const MemberView& m, int l, int32_t g)
{
    return g < 0 ? -1 : static_cast<int32_t>(m.nbase[l] + (g - m.lvl_off[l]));
}

__global__ void k_forest_nodes(ForestArgs f, int64_t n_nodes, uint64_t* __restrict__ key, int32_t* __restrict__ pbeg,
                               int32_t* __restrict__ pend, int32_t* __restrict__ parent, int32_t* __restrict__ child_beg,
                               int32_t* __restrict__ nchild, int32_t* __restrict__ leaf_id, int32_t* __restrict__ colleague,
                               int32_t* __restrict__ node_tree, int32_t* __restrict__ ilcnt)
{
    for (int64_t x = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; x < n_nodes; x += int64_t(gridDim.x) * blockDim.x) {
        const int l = find_level(f.lvl_off, f.depth, x);
        const int r = find_member(f, false, l, x);
        const MemberView& m = f.m[r];
        const int64_t g = x - m.nbase[l] + m.lvl_off[l];
        node_tree[x] = r;
        key[x] = m.key[g];
        pbeg[x] = static_cast<int32_t>(m.pbeg[g] + m.pbase);
        pend[x] = static_cast<int32_t>(m.pend[g] + m.pbase);
        parent[x] = l == 0 ? -1 : map_node(m, l - 1, m.parent[g]);
        const int nc = m.nchild[g];
        nchild[x] = nc;
        child_beg[x] = nc > 0 ? map_node(m, l + 1, m.child_beg[g]) : 0;
        const int32_t lf = m.leaf_id[g];
        leaf_id[x] = lf < 0 ? -1 : static_cast<int32_t>(m.lbase[l] + (lf - m.leaf_off[l]));
        for (int s = 0; s < 27; ++s) colleague[27 * x + s] = map_node(m, l, m.colleague[27 * g + s]);
        ilcnt[x] = m.il_ptr[g + 1] - m.il_ptr[g];
    }
}

__global__ void k_forest_leaves(ForestArgs f, int64_t n_leaves, int32_t* __restrict__ leaf_node, int32_t* __restrict__ nrcnt)
{
    for (int64_t x = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; x < n_leaves; x += int64_t(gridDim.x) * blockDim.x) {
        const int l = find_level(f.leaf_off, f.depth, x);
        const int r = find_member(f, true, l, x);
        const MemberView& m = f.m[r];
        const int64_t lf = x - m.lbase[l] + m.leaf_off[l];
        leaf_node[x] = map_node(m, l, m.leaf_node[lf]);
        nrcnt[x] = m.nr_ptr[lf + 1] - m.nr_ptr[lf];
    }
}

__global__ void k_forest_lists(ForestArgs f, int64_t n_nodes, int64_t n_leaves, const int32_t* __restrict__ il_ptr,
                               int32_t* __restrict__ il_src, int32_t* __restrict__ il_code, const int32_t* __restrict__ nr_ptr,
                               int2* __restrict__ nr)
{
    for (int64_t x = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; x < n_nodes + n_leaves; x += int64_t(gridDim.x) * blockDim.x) {
        if (x < n_nodes) {
            const int l = find_level(f.lvl_off, f.depth, x);
            const MemberView& m = f.m[find_member(f, false, l, x)];
            const int64_t g = x - m.nbase[l] + m.lvl_off[l];
            int32_t o = il_ptr[x];
            for (int32_t e = m.il_ptr[g]; e < m.il_ptr[g + 1]; ++e, ++o) {
                il_src[o] = map_node(m, l, m.il_src[e]);
                il_code[o] = m.il_code[e];
            }
        } else {
            const int64_t y = x - n_nodes;
            const int l = find_level(f.leaf_off, f.depth, y);
            const MemberView& m = f.m[find_member(f, true, l, y)];
            const int64_t lf = y - m.lbase[l] + m.leaf_off[l];
            int32_t o = nr_ptr[y];
            for (int32_t e = m.nr_ptr[lf]; e < m.nr_ptr[lf + 1]; ++e, ++o) {
                const int2 v = m.nr[e];
                nr[o] = make_int2(static_cast<int>(v.x + m.pbase), static_cast<int>(v.y + m.pbase));
            }
        }
    }
}

// points in the members' leaf orders, one member after another, scaled into
// the unit cube; order maps to the concatenated input of the batch
__global__ void k_forest_points(ForestArgs f, int64_t n, double* __restrict__ pts, int32_t* __restrict__ order)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        int r = 0;
        while (r + 1 < f.count && i >= f.m[r + 1].pbase) ++r;
        const MemberView& m = f.m[r];
        const int64_t j = i - m.pbase;
        for (int a = 0; a < 3; ++a) pts[a * n + i] = (m.pts[a * m.n + j] - m.corner[a]) / m.width;
        order[i] = static_cast<int32_t>(m.order[j] + m.pbase);
    }
}

}  // namespace

void build_forest(Tree& F, const std::vector<const Tree*>& members)
{
    SFMM_REQUIRE(!members.empty() && members.size() <= 4096, FMM_ERR_INVALID_ARGUMENT, "a forest takes 1..4096 trees");
    const Tree& t0 = *members[0];
    cudaStream_t st = t0.ctx->stream;
    const int B = static_cast<int>(members.size());
    F.ctx = t0.ctx;
    F.max_level = t0.max_level;
    F.max_ppn = t0.max_ppn;
    F.vertical_axis = 2;
    F.phideg = 0;
    F.n = 0;
    F.depth = 0;
    for (const Tree* t : members) {
        SFMM_REQUIRE(t->ctx == t0.ctx, FMM_ERR_INVALID_ARGUMENT, "the trees of a forest share one context");
        SFMM_REQUIRE(!t->box.rotated && t->box.X == 0 && t->box.Y == 1 && t->box.Z == 2, FMM_ERR_UNSUPPORTED,
                     "forest members need the z axis vertical and no azimuthal rotation");
        F.n += t->n;
        F.depth = std::max(F.depth, t->depth);
    }
    SFMM_REQUIRE(F.n < (int64_t(1) << 31), FMM_ERR_UNSUPPORTED, "a forest holds fewer than 2^31 points");
    // per-member views and forest offsets
    std::vector<MemberView> mv(B);
    F.lvl_off.assign(F.depth + 2, 0);
    F.leaf_off.assign(F.depth + 2, 0);
    int64_t pbase = 0;
    for (int l = 0; l <= F.depth; ++l) {
        int64_t nb = F.lvl_off[l], lb = F.leaf_off[l];
        for (int r = 0; r < B; ++r) {
            const Tree& t = *members[r];
            mv[r].nbase[l] = nb;
            mv[r].lbase[l] = lb;
            if (l <= t.depth) {
                nb += t.lvl_off[l + 1] - t.lvl_off[l];
                lb += t.leaf_off[l + 1] - t.leaf_off[l];
            }
        }
        F.lvl_off[l + 1] = nb;
        F.leaf_off[l + 1] = lb;
    }
    for (int r = 0; r < B; ++r) {
        const Tree& t = *members[r];
        MemberView& m = mv[r];
        m.n = t.n;
        m.pbase = pbase;
        pbase += t.n;
        m.depth = t.depth;
        for (int l = 0; l < kLv; ++l) {
            m.lvl_off[l] = l <= t.depth + 1 ? t.lvl_off[l] : t.lvl_off[t.depth + 1];
            m.leaf_off[l] = l <= t.depth + 1 ? t.leaf_off[l] : t.leaf_off[t.depth + 1];
        }
        for (int l = F.depth + 1; l < kLv; ++l) m.nbase[l] = m.lbase[l] = 0;
        for (int a = 0; a < 3; ++a) m.corner[a] = t.box.corner[a];
        // a box of zero width (all points coincide: one key) is taken as width 1
        m.width = t.box.width > 0 ? t.box.width : 1.0;
        m.key = t.key.ptr;
        m.pbeg = t.pbeg.ptr;
        m.pend = t.pend.ptr;
        m.parent = t.parent.ptr;
        m.child_beg = t.child_beg.ptr;
        m.nchild = t.nchild.ptr;
        m.leaf_id = t.leaf_id.ptr;
        m.leaf_node = t.leaf_node.ptr;
        m.colleague = t.colleague.ptr;
        m.il_ptr = t.il_ptr.ptr;
        m.il_src = t.il_src.ptr;
        m.il_code = t.il_code.ptr;
        m.nr_ptr = t.nr_ptr.ptr;
        m.nr = t.nr.ptr;
        m.order = t.order.ptr;
        m.pts = t.pts.ptr;
    }
    F.n_nodes = F.lvl_off[F.depth + 1];
    F.n_leaves = F.leaf_off[F.depth + 1];
    DevBuf<MemberView> dmv;
    dmv.alloc(B, st);
    SFMM_CUDA(cudaMemcpyAsync(dmv.ptr, mv.data(), B * sizeof(MemberView), cudaMemcpyHostToDevice, st));
    ForestArgs fa{};
    fa.m = dmv.ptr;
    fa.count = B;
    fa.depth = F.depth;
    for (int l = 0; l <= F.depth + 1; ++l) {
        fa.lvl_off[l] = F.lvl_off[l];
        fa.leaf_off[l] = F.leaf_off[l];
    }
    // the unit cube (keys, node centres and level tables of every member)
    BoxDev box = t0.box;
    box.width = 1.0;
    box.corner[0] = box.corner[1] = box.corner[2] = 0.0;
    F.box = box;
    F.d_box.alloc(1, st);
    SFMM_CUDA(cudaMemcpyAsync(F.d_box.ptr, &F.box, sizeof(BoxDev), cudaMemcpyHostToDevice, st));
    // nodes and leaves
    const int64_t nn = F.n_nodes, nl = F.n_leaves;
    F.key.alloc(nn, st);
    F.pbeg.alloc(nn, st);
    F.pend.alloc(nn, st);
    F.parent.alloc(nn, st);
    F.child_beg.alloc(nn, st);
    F.nchild.alloc(nn, st);
    F.leaf_id.alloc(nn, st);
    F.colleague.alloc(size_t(27) * nn, st);
    F.node_tree.alloc(nn, st);
    F.n_trees = B;
    F.member_width.resize(B);
    for (int r = 0; r < B; ++r) F.member_width[r] = mv[r].width;
    F.leaf_node.alloc(nl, st);
    DevBuf<int32_t> ilcnt, nrcnt;
    ilcnt.alloc(nn + 1, st);
    nrcnt.alloc(nl + 1, st);
    const int sms = t0.ctx->sm_count;
    k_forest_nodes<<<blocks_for(nn, 256, int64_t(sms) * 16), 256, 0, st>>>(fa, nn, F.key.ptr, F.pbeg.ptr, F.pend.ptr, F.parent.ptr,
                                                                            F.child_beg.ptr, F.nchild.ptr, F.leaf_id.ptr,
                                                                            F.colleague.ptr, F.node_tree.ptr, ilcnt.ptr);
    SFMM_CHECK_LAUNCH();
    k_forest_leaves<<<blocks_for(nl, 256, int64_t(sms) * 16), 256, 0, st>>>(fa, nl, F.leaf_node.ptr, nrcnt.ptr);
    SFMM_CHECK_LAUNCH();
    // list offsets, then the entries
    F.il_nnz = 0;
    F.nr_nnz = 0;
    F.near_pairs = 0;
    for (const Tree* t : members) {
        F.il_nnz += t->il_nnz;
        F.nr_nnz += t->nr_nnz;
        F.near_pairs += t->near_pairs;
    }
    require_i32_total(F.il_nnz, "forest interaction list");
    require_i32_total(F.nr_nnz, "forest near-field list");
    F.il_ptr.alloc(nn + 1, st);
    F.nr_ptr.alloc(nl + 1, st);
    exclusive_scan_i32(ilcnt.ptr, F.il_ptr.ptr, nn, st);
    exclusive_scan_i32(nrcnt.ptr, F.nr_ptr.ptr, nl, st);
    F.il_src.alloc(std::max<int64_t>(F.il_nnz, 1), st);
    F.il_code.alloc(std::max<int64_t>(F.il_nnz, 1), st);
    F.nr.alloc(std::max<int64_t>(F.nr_nnz, 1), st);
    k_forest_lists<<<blocks_for(nn + nl, 256, int64_t(sms) * 16), 256, 0, st>>>(fa, nn, nl, F.il_ptr.ptr, F.il_src.ptr,
                                                                                  F.il_code.ptr, F.nr_ptr.ptr, F.nr.ptr);
    SFMM_CHECK_LAUNCH();
    // points
    F.pts.alloc(size_t(3) * F.n, st);
    F.order.alloc(F.n, st);
    k_forest_points<<<blocks_for(F.n, 256, int64_t(sms) * 16), 256, 0, st>>>(fa, F.n, F.pts.ptr, F.order.ptr);
    SFMM_CHECK_LAUNCH();
    F.far_x = F.pts.ptr;
    F.far_y = F.pts.ptr + F.n;
    F.far_z = F.pts.ptr + 2 * F.n;
    SFMM_CUDA(cudaStreamSynchronize(st));      // the views and counts are freed on return
    check_scan_error();
}

}  // namespace sfmm
