// Evaluation plan (the FMM3D object of the reference, fmm.hpp:134-427).
#pragma once

#include "fmm_internal.cuh"

namespace sfmm {

// Everything a kernel of one evaluation reads, passed by value.
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
    int p, T, qdim;
    CompSpec cs;
    const double* rot;
    const int* rot_off;
    int rot_len;
    const double* tz;
    const int* tz_off;
    int tz_len;
    const cplx *eil, *echild, *eparent;
    const int *m2m_ptr, *m2m_code;
    const double* m2m_g;
    const int *l2l_ptr, *l2l_code;
    const double* l2l_g;
    const double* ipow;
    cplx* M;
    cplx* L;
    const double* qs;
    double* out;                         // far field per component, sorted order
    double* out2;                        // near field per component, sorted order
};

struct Plan {
    Tree* tree = nullptr;
    int p = 0, T = 0, qdim = 1, precision = FMM_PRECISION_FP64;
    int rot_len = 0, tz_len = 0;
    DevBuf<double> rot, tz, eil, echild, eparent, m2m_g, l2l_g, ipow;
    DevBuf<int> rot_off, tz_off, m2m_ptr, m2m_code, l2l_ptr, l2l_code;
    DevBuf<double2> M, L;
    DevBuf<double> qs, out, out2;
    DevBuf<double> qin, uio_pot, uio_field;   // staging for host pointers
    cudaEvent_t ev[6] = {};
};

void plan_init(Plan& pl);
void plan_evaluate(Plan& pl, const double* Q_dev, double* pot_dev, double* field_dev);
void plan_read_timings(Plan& pl, double* ms6);

}  // namespace sfmm
