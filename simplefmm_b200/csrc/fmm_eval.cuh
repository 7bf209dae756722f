// Evaluation plan (the FMM3D object of the reference, fmm.hpp:134-427).
#pragma once

#include "fmm_internal.cuh"
#include "i8_ops.h"

#include <memory>

namespace sfmm {

// Everything a kernel of one evaluation reads, passed by value.
//
// Far-field expansions per node and charge component b:
//   M   plain multipoles of order p (P2M/M2M)
//   LA  potential local of order p  (M2L of M, orders <= p)
//   LB  field local of order p + 1  (M2L of M restricted to orders <= p - 1);
//       the field at a target is minus its gradient (fmm_ops.cuh grad_local),
//       which equals the reference's source-gradient moments term by term.
struct EvalArgs {
    int64_t n;
    int depth;
    int64_t lvl_off[kKeyLevel + 2];
    int64_t n_leaves, far_leaf0;         // leaves of level >= 2 are [far_leaf0, n_leaves)
    const BoxDev* box;
    const uint64_t* key;
    const int32_t *pbeg, *pend, *parent, *child_beg, *nchild, *leaf_node, *order;
    const double *px, *py, *pz;          // original frame (near field)
    const double *fx, *fy, *fz;          // rotated frame (expansions)
    const int32_t *il_ptr, *il_src, *il_code;
    const int32_t* nr_ptr;
    const int2* nr;
    int p, T, T1, qdim;
    int want_pot, want_field;
    int mixed;                            // FMM_PRECISION_MIXED: FP32 near field, tensor-core M2L
    int K;                                // output components: qdim (if pot) + 3 (if field)
    int kf;                               // first field output component
    const double* rot;                    // rotation classes up to order p + 1
    const int* rot_off;
    int rot_len;
    const double* tzx;                    // z-translation, target orders <= p+1, source orders <= p
    const int* tzx_off;
    int tzx_len;
    const cplx* eil;                      // 49 x (p + 2)
    const cplx* echild;                   // 4 x (2p + 1)
    const cplx* eparent;                  // 4 x (2p + 1)
    const cplx* eparent1;                 // 4 x (2p + 3)
    const int *m2m_ptr, *m2m_code;
    const double* m2m_g;
    const int *l2l_ptr, *l2l_code;        // order p
    const double* l2l_g;
    const int *l2l1_ptr, *l2l1_code;      // order p + 1
    const double* l2l1_g;
    const double* ipow;                   // rho^{-(k+1)} per (level, |d|^2), k = 0..2p+2
    int ipow_w;
    // M2L operators in tensor-core fragment order (m2l.cu): rotation /
    // inverse rotation per class, z-translation, and the order-p translation
    // column that the potential local adds to the field local's sources
    const double* rfrag;
    int rfrag_nf;                         // fragments per class and matrix
    const double* tzfrag;
    const double* tzl;
    // mixed precision: FP32 operators in TF32 fragment order (per class, the
    // z-translation pre-scaled by the class's distance)
    const float* rf32;
    int rf32_nf;
    const float* tz32;
    int tz32_nf;
    const float* tzl32;
    float2* m32;                          // mixed: s^-n M (FP32) per node, written before the M2L
    cplx* M;
    cplx* LA;
    cplx* LB;
    const double* qs;
    const double4* src4;                  // FP64 near field: x y z q0 per point, leaf order
    const double2* src2;                  // q1 q2 per point (qdim > 1)
    // near-field work items (p2p.cu): (leaf, first range, offset in it,
    // sources) and the item's first row of partial sums (-1: the leaf is
    // one item and writes out2 directly); per leaf the number of parts and
    // the first row; a counter the warps take items from
    const int4* p2p_item;
    const int32_t* p2p_row;
    int64_t p2p_items;
    const int32_t *p2p_parts, *p2p_rowoff;
    double* p2p_part;
    int* p2p_ctr;
    int* m2l_ctr;                         // FP64 M2L: the counter blocks take sibling groups from
    int m2l_force_rows;                   // run the row-owner M2L kernel (plan made with SFMM_M2L_KERNEL=rows)
    const uint8_t* own_leaf;              // sharded plan: 1 for this shard's leaves (global leaf id); NULL = all
    const int32_t* node_tree;             // forest: member tree of each node; NULL = one tree
    int* wait_err;                        // set by a kernel whose bounded pipeline wait expired
    // direct M2L (m2l_direct.cu, FMM_M2L_METHOD_DIRECT): dense coefficient table,
    // Z of the interaction-list angles, phases; row lengths
    int m2l_direct;
    const double* dcoef;
    int dncoef;
    const double* dzil;
    int dnz;
    const cplx* deil2;
    int dne;
    int p2p_split;                        // some leaf has more than one part
    double* out;                         // far field per component, sorted order
    double* out2;                        // near field per component, sorted order
};

// Operator tables of one expansion order on one device: immutable once built,
// shared by every plan of that (device, p, precision) (built once, on the
// first plan's stream, then kept until the process exits).
struct PlanTables {
    int rot_len = 0, tzx_len = 0;
    DevBuf<double> rot, tzx, eil, echild, eparent, eparent1, m2m_g, l2l_g, l2l1_g;
    DevBuf<int> rot_off, tzx_off, m2m_ptr, m2m_code, l2l_ptr, l2l_code, l2l1_ptr, l2l1_code;
    DevBuf<double> rfrag, tzfrag, tzl;
    int rfrag_nf = 0;
    DevBuf<float> rf32, tz32, tzl32;
    int rf32_nf = 0, tz32_nf = 0;
    DevBuf<double> sh_unit;                 // M2M / L2L maps at rho = 1 (shift.cu)
};

// Direct-M2L tables of one order on one device (shared like PlanTables).
struct DirectDevTables {
    DevBuf<double> coef, zil, eil2;
    int ncoef = 0, nz = 0, ne = 0;
};

// Dense int8-slice M2L of mixed plans (m2l_i8.cu): per-plan target blocks,
// slot tables and moment digits.
struct I8PlanData;

struct Plan {
    Tree* tree = nullptr;
    int p = 0, T = 0, T1 = 0, qdim = 1, precision = FMM_PRECISION_FP64;
    int ipow_w = 0;
    std::shared_ptr<PlanTables> tab;
    DevBuf<double> ipow;
    // excluded source lists (self_generator / is_self): CSR over original target
    // indices, original -> sorted index, sorted point -> leaf
    DevBuf<int64_t> ex_ptr;
    DevBuf<int32_t> ex_col, ex_inv, ex_leaf;
    int ex_near_too = 0;
    bool ex_on = false;
    DevBuf<double2> M, LA, LB;
    DevBuf<double> qs, out, out2;
    DevBuf<double4> src4;                     // FP64 near-field source records (p2p.cu)
    DevBuf<double2> src2;
    // near-field work items (p2p.cu, p2p_setup)
    DevBuf<int4> p2p_item;
    DevBuf<int32_t> p2p_row, p2p_parts, p2p_rowoff, p2p_ctr;
    DevBuf<int32_t> m2l_ctr;                  // M2L group counter (m2l.cu)
    bool m2l_force_rows = false;              // SFMM_M2L_KERNEL=rows at plan creation
    int m2l_method = FMM_M2L_METHOD_ROTATION;        // fmm_plan_set_m2l
    // sharded evaluation (fmm_plan_set_shard): this plan's share of one solve
    int shard_index = 0, shard_count = 1;
    DevBuf<uint8_t> own_leaf;                 // per global leaf id
    std::vector<int64_t> own_parent_b, own_parent_e;   // per parent level q: node range [b, e)
    std::shared_ptr<DirectDevTables> dtab;    // FMM_M2L_METHOD_DIRECT
    std::shared_ptr<I8PlanData> i8;           // mixed plans: the tensor-core (tcgen05, int8 slices) M2L
    DevBuf<int32_t> wait_err;                 // a kernel's bounded wait expired (EvalArgs::wait_err)
    bool m2l_rotation_only = false;           // SFMM_M2L_KERNEL=rotation: mixed plans keep the TF32 rotation M2L
    DevBuf<double> p2p_part;
    int64_t p2p_items = 0, p2p_rows = 0;
    DevBuf<double> qin, uio_pot, uio_field;   // staging for host pointers
    // M2M / L2L as matrix products (shift.cu): per children level the octant
    // maps, compact slots of the parents that have children, scratch rows
    bool shift_on = false;
    DevBuf<double> sh_ops;
    DevBuf<int32_t> sh_slot, sh_list;
    std::vector<int32_t> sh_S;
    DevBuf<float2> m32;                       // mixed precision: scaled FP32 source moments
    // timing: evaluation start, far field (upward, M2L, downward) ends, end;
    // ev[6] / ev[7] bracket the near field on the side stream
    cudaEvent_t ev[8] = {};
    cudaEvent_t fork = nullptr, join = nullptr;   // side stream: start after the charges, join before the sums
    cudaEvent_t io_start = nullptr, io_done = nullptr;   // host-array evaluations: output copies on the copy stream
    // one captured evaluation (fmm_plan_capture / fmm_plan_replay)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
};

void plan_init(Plan& pl);
// shift.cu: set-up at plan creation, M2M into parent level lp, L2L into
// children level lc, and the context's cuBLAS handle at context teardown
void build_unit_shift_ops(PlanTables& tab, int p, cudaStream_t st);
void shift_setup(Plan& pl);
void shift_m2m(Plan& pl, const EvalArgs& a, int lp, cudaStream_t st);
void shift_l2l(Plan& pl, const EvalArgs& a, int lc, cudaStream_t st);
// p2p.cu: near-field work items of the plan's tree (leaves with a large near
// field split into parts), built at plan creation
void p2p_setup(Plan& pl);
// Fills the fragment-order operators of tb (rfrag / tzfrag / tzl, and the
// FP32 ones when mixed) from its rotation and translation tables (m2l.cu).
void build_m2l_fragments(PlanTables& tb, int p, bool mixed, cudaStream_t st);
// before_sums (may be NULL): an event the stream waits for before the final
// sums into pot / field (their host-to-device copies on another stream).
void plan_evaluate(Plan& pl, const double* Q_dev, double* pot_dev, double* field_dev,
                   cudaEvent_t before_sums = nullptr);
// Selects the M2L formulation (FMM_M2L_METHOD_ROTATION / FMM_M2L_METHOD_DIRECT); the
// direct one's tables are built on first use per (device, p).
void plan_set_m2l(Plan& pl, int method);
// Sharded evaluation of one solve (shard_ranges.h): set_shard fixes the
// plan's share; evaluate_stage runs stage 0 (charges, near field and
// moments of own leaves), 1 (M2M, M2L into own targets) or 2 (L2L, L2P of
// own leaves, sums); the caller sums the shards' moments (after stage 0) and
// locals (after stage 1) across shards, and finally their outputs.
void plan_set_shard(Plan& pl, int index, int count);
void plan_evaluate_stage(Plan& pl, const double* Q_dev, double* pot_dev, double* field_dev, int stage);
void plan_read_timings(Plan& pl, double* ms6);
// Direct-M2L tables of order p on a device, built on first use and kept (eval.cu).
std::shared_ptr<DirectDevTables> direct_tables_on_device(int device, int p, cudaStream_t st);
// m2l_i8.cu: whether a plan takes the tensor-core M2L; its set-up at plan
// creation (fills pl.i8); the launch (moment digits, then the M2L of every
// level); the report of an expired pipeline wait of the plan's kernels (the
// tensor-core M2L, the near field's bulk copies): throws FMM_ERR_TIMEOUT.
bool m2l_i8_supported(const Plan& pl);
void m2l_i8_setup(Plan& pl);
void launch_m2l_i8(Plan& pl, const EvalArgs& a, cudaStream_t st);
void m2l_i8_check(Plan& pl);
// Exclusions (exclude.cu): ptr / cols are device arrays (n + 1, ptr[n]).
void plan_set_exclusions(Plan& pl, const int64_t* ptr, const int32_t* cols, int near_too);
void plan_clear_exclusions(Plan& pl);
void apply_exclusions(const Plan& pl, const double* Q, double* pot, double* field);

}  // namespace sfmm
