// FP64 evaluation kernels: P2M, M2M, M2L, L2L, L2P, P2P and the plan.
//
// Phase structure of FMM3D::rinv (fmm.hpp:811-881): far field only when the
// tree is at least 2 levels deep; multipoles at every leaf of level >= 2;
// M2M up to level 2; M2L on levels 2..depth; L2L down; L2P at every leaf of
// level >= 2; near field over the neighbour lists.  Per-coefficient math is
// in fmm_ops.cuh; expansions keep only m >= 0.
//
// Potential and field share one M2L: for every (target, source) pair the
// source multipole is rotated once, z-translated into both the order-p
// potential local LA and the order-(p+1) field local LB (source orders
// <= p-1), and the two are rotated back.  The field is minus the gradient of
// LB at the target, identical term by term to the reference's
// source-gradient moments (fmm.hpp:234-253, 549-551).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>

#include "eval_util.cuh"
#include "fmm_tables.h"
#include "shard_ranges.h"

namespace sfmm {

__constant__ HarmCoef c_harm;

namespace {

constexpr int kMaxWarps = 8;

// Charges into leaf order (qs, one array per component) and, for the FP64
// near field, the packed source records (x y z q0 | q1 q2).
__global__ void k_gather_q(const double* __restrict__ Q, const int32_t* __restrict__ order, int64_t n, int qdim,
                           double* __restrict__ qs, const double* __restrict__ pts, double4* __restrict__ src4,
                           double2* __restrict__ src2)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t o = order[i];
        double q[3] = {0, 0, 0};
        for (int b = 0; b < qdim; ++b) {
            q[b] = Q[o * qdim + b];
            qs[b * n + i] = q[b];
        }
        if (src4) src4[i] = make_double4(pts[i], pts[n + i], pts[2 * n + i], q[0]);
        if (src2) src2[i] = make_double2(q[1], q[2]);
    }
}

// P2M (fmm.hpp:524-556): warp per leaf of level >= 2, lanes over points.
// The lanes' terms q_b S_n^m go through a per-warp staging block of
// kP2MStage values: each lane writes its terms, then two lanes per value add
// the 32 lanes' entries (16 each and one shuffle) into the coefficient.  That
// is about four instructions per term and lane, against a five-step warp sum.
constexpr int kP2MStage = 16;                   // values staged per reduction
constexpr int kP2MLd = 33;                      // doubles per staged value (32 lanes + pad)
constexpr size_t kP2MStageBytes = size_t(kP2MStage) * kP2MLd * sizeof(double) + kP2MStage * sizeof(int);

template<int QD>
__global__ void __launch_bounds__(kMaxWarps * 32) k_p2m(EvalArgs a)
{
    extern __shared__ double smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const size_t per_warp = size_t(a.qdim) * a.T * sizeof(cplx) + kP2MStageBytes;
    char* wbase = reinterpret_cast<char*>(smem) + w * per_warp;
    cplx* acc = reinterpret_cast<cplx*>(wbase);
    double* accd = reinterpret_cast<double*>(wbase);
    double* stage = reinterpret_cast<double*>(wbase + size_t(a.qdim) * a.T * sizeof(cplx));
    int* sidx = reinterpret_cast<int*>(stage + kP2MStage * kP2MLd);
    const int j = lane & 15, h = lane >> 4;
    const int64_t nfar = a.n_leaves - a.far_leaf0;
    for (int64_t f = blockIdx.x * int64_t(nw) + w; f < nfar; f += int64_t(gridDim.x) * nw) {
        const int g = a.leaf_node[a.far_leaf0 + f];
        if (a.own_leaf && !a.own_leaf[a.far_leaf0 + f]) {      // another shard's leaf: zero moments
            for (int t = lane; t < a.qdim * a.T; t += 32) a.M[int64_t(g) * a.qdim * a.T + t] = cplx{0, 0};
            continue;
        }
        const int l = level_of(a, g);
        double c[3];
        node_center(*a.box, a.key[g], l, c);
        for (int t = lane; t < a.qdim * a.T; t += 32) acc[t] = cplx{0, 0};
        __syncwarp();
        const int b0 = a.pbeg[g], b1 = a.pend[g];
        for (int base = b0; base < b1; base += 32) {
            const int i = base + lane;
            const bool on = i < b1;
            const double x = on ? a.fx[i] - c[0] : 0, y = on ? a.fy[i] - c[1] : 0, z = on ? a.fz[i] - c[2] : 0;
            double q[QD];                                 // QD = qdim: the charges stay in registers
#pragma unroll
            for (int b = 0; b < QD; ++b) q[b] = on ? a.qs[b * a.n + i] : 0.0;
            int cnt = 0;                                  // staged values (the same in every lane)
            auto flush = [&](int nv) {
                __syncwarp();
                double sum = 0.0;
                if (j < nv) {
                    const double* col = stage + j * kP2MLd + h * 16;
#pragma unroll
                    for (int u = 0; u < 16; ++u) sum += col[u];
                }
                sum += __shfl_xor_sync(0xffffffffu, sum, 16);
                if (h == 0 && j < nv) accd[sidx[j]] += sum;
                __syncwarp();
            };
            for_each_harmonic(a.p, x, y, z, c_harm, [&](int n, int m, cplx s) {
                const int t = tri(n, m);
#pragma unroll
                for (int b = 0; b < QD; ++b) {
                    stage[cnt * kP2MLd + lane] = q[b] * s.re;
                    stage[(cnt + 1) * kP2MLd + lane] = q[b] * s.im;
                    if (lane == 0) {
                        sidx[cnt] = 2 * (b * a.T + t);
                        sidx[cnt + 1] = 2 * (b * a.T + t) + 1;
                    }
                    cnt += 2;
                    if (cnt == kP2MStage) {
                        flush(kP2MStage);
                        cnt = 0;
                    }
                }
            });
            if (cnt) flush(cnt);
        }
        __syncwarp();
        cplx* M = a.M + int64_t(g) * a.qdim * a.T;
        for (int t = lane; t < a.qdim * a.T; t += 32) M[t] = acc[t];
        __syncwarp();
    }
}

// M2M (fmm.hpp:558-590): warp per parent at level lp.
__global__ void __launch_bounds__(kMaxWarps * 32) k_m2m(EvalArgs a, int lp, int64_t off, int64_t cnt)
{
    extern __shared__ double smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int p = a.p, T = a.T;
    double* rpow = smem;                                         // p + 1
    cplx* phase = reinterpret_cast<cplx*>(smem + 32);            // 4 x (2p+1)
    cplx* child = reinterpret_cast<cplx*>(smem + 32) + 4 * (2 * kMaxOrder + 1) + w * 2 * a.qdim * T;
    cplx* accs = child + a.qdim * T;
    if (threadIdx.x == 0) {
        const double rho = sqrt(0.75) * a.box->width / (1 << (lp + 1));
        rpow[0] = 1;
        for (int k = 1; k <= p; ++k) rpow[k] = rpow[k - 1] * rho;
    }
    for (int t = threadIdx.x; t < 4 * (2 * p + 1); t += blockDim.x) phase[t] = a.echild[t];
    __syncthreads();
    for (int64_t i = blockIdx.x * int64_t(nw) + w; i < cnt; i += int64_t(gridDim.x) * nw) {
        const int64_t g = off + i;
        const int nc = a.nchild[g];
        if (nc == 0) continue;
        const int cb = a.child_beg[g];
        cplx* M = a.M + g * a.qdim * T;
        for (int o = lane; o < a.qdim * T; o += 32) accs[o] = cplx{0, 0};
        for (int c = cb; c < cb + nc; ++c) {
            const cplx* Mc = a.M + int64_t(c) * a.qdim * T;
            for (int t = lane; t < a.qdim * T; t += 32) child[t] = Mc[t];
            __syncwarp();
            const int oct = static_cast<int>(a.key[c] & 7);
            for (int o = lane; o < a.qdim * T; o += 32) {
                const int b = o / T, t = o - b * T;
                const cplx v = shift_output<true>(t, a.m2m_ptr, a.m2m_code, a.m2m_g, child + b * T, oct, rpow,
                                                  phase + (oct & 3) * (2 * p + 1), p);
                accs[o].re += v.re;
                accs[o].im += v.im;
            }
            __syncwarp();
        }
        for (int o = lane; o < a.qdim * T; o += 32) M[o] = accs[o];
        __syncwarp();
    }
}

// L2L (fmm.hpp:714-745): warp per child node at level lc; LA at order p,
// LB at order p + 1 (exact: a polynomial of degree p + 1 re-expanded).
__global__ void __launch_bounds__(kMaxWarps * 32) k_l2l(EvalArgs a, int lc, int64_t off, int64_t cnt)
{
    extern __shared__ double smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int p = a.p, T = a.T, T1 = a.T1, qd = a.qdim;
    double* rpow = smem;                                                   // p + 2
    cplx* ph = reinterpret_cast<cplx*>(smem + 32);                         // 4 x (2p+1)
    cplx* ph1 = ph + 4 * (2 * kMaxOrder + 1);                              // 4 x (2p+3)
    cplx* parA = ph1 + 4 * (2 * kMaxOrder + 3) + w * qd * (T + T1);
    cplx* parB = parA + qd * T;
    if (threadIdx.x == 0) {
        const double rho = sqrt(0.75) * a.box->width / (1 << lc);
        rpow[0] = 1;
        for (int k = 1; k <= p + 1; ++k) rpow[k] = rpow[k - 1] * rho;
    }
    for (int t = threadIdx.x; t < 4 * (2 * p + 1); t += blockDim.x) ph[t] = a.eparent[t];
    for (int t = threadIdx.x; t < 4 * (2 * p + 3); t += blockDim.x) ph1[t] = a.eparent1[t];
    __syncthreads();
    for (int64_t i = blockIdx.x * int64_t(nw) + w; i < cnt; i += int64_t(gridDim.x) * nw) {
        const int64_t g = off + i;
        const int64_t pg = a.parent[g];
        if (a.want_pot)
            for (int t = lane; t < qd * T; t += 32) parA[t] = a.LA[pg * qd * T + t];
        if (a.want_field)
            for (int t = lane; t < qd * T1; t += 32) parB[t] = a.LB[pg * qd * T1 + t];
        __syncwarp();
        const int oct = static_cast<int>(a.key[g] & 7);
        if (a.want_pot)
            for (int o = lane; o < qd * T; o += 32) {
                const int b = o / T, t = o - b * T;
                const cplx v = shift_output<false>(t, a.l2l_ptr, a.l2l_code, a.l2l_g, parA + b * T, oct, rpow,
                                                   ph + (oct & 3) * (2 * p + 1), p);
                cplx& d = a.LA[g * qd * T + o];
                d.re += v.re;
                d.im += v.im;
            }
        if (a.want_field)
            for (int o = lane; o < qd * T1; o += 32) {
                const int b = o / T1, t = o - b * T1;
                const cplx v = shift_output<false>(t, a.l2l1_ptr, a.l2l1_code, a.l2l1_g, parB + b * T1, oct, rpow,
                                                   ph1 + (oct & 3) * (2 * p + 3), p + 1);
                cplx& d = a.LB[g * qd * T1 + o];
                d.re += v.re;
                d.im += v.im;
            }
        __syncwarp();
    }
}

// L2P (fmm.hpp:747-771): warp per leaf of level >= 2.  The leaf's output
// locals (potential: LA; field: minus grad of LB for scalar charges, curl
// of LB for vector charges) are formed in shared memory, then lanes
// evaluate them at the leaf's points.
template<int KM>
__global__ void __launch_bounds__(kMaxWarps * 32) k_l2p(EvalArgs a)
{
    extern __shared__ double smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int T = a.T, T1 = a.T1, qd = a.qdim, K = a.K;
    cplx* loc = reinterpret_cast<cplx*>(smem) + w * K * T;
    const int64_t nfar = a.n_leaves - a.far_leaf0;
    for (int64_t f = blockIdx.x * int64_t(nw) + w; f < nfar; f += int64_t(gridDim.x) * nw) {
        if (a.own_leaf && !a.own_leaf[a.far_leaf0 + f]) continue;   // another shard's leaf
        const int64_t g = a.leaf_node[a.far_leaf0 + f];
        const int l = level_of(a, g);
        double c[3];
        node_center(*a.box, a.key[g], l, c);
        if (a.want_pot)
            for (int t = lane; t < qd * T; t += 32) loc[t] = a.LA[g * qd * T + t];
        if (a.want_field)
            for (int t = lane; t < T; t += 32) {
                int n, m;
                tri_nm(t, n, m);
                cplx G[3][3];
                for (int b = 0; b < qd; ++b) grad_local(a.LB + (g * qd + b) * T1, n, m, &G[b][0], &G[b][1], &G[b][2]);
                for (int ax = 0; ax < 3; ++ax) {
                    cplx v;
                    if (qd == 1) {
                        v = cplx{-G[0][ax].re, -G[0][ax].im};
                    } else {
                        const int b1 = (ax + 1) % 3, c1 = (ax + 2) % 3;
                        v = cplx{G[c1][b1].re - G[b1][c1].re, G[c1][b1].im - G[b1][c1].im};
                    }
                    loc[(a.kf + ax) * T + t] = v;
                }
            }
        __syncwarp();
        const int b0 = a.pbeg[g], b1 = a.pend[g];
        for (int i = b0 + lane; i < b1; i += 32) {
            // KM = K, a compile-time bound: the sums stay in registers
            double u[KM];
#pragma unroll
            for (int k = 0; k < KM; ++k) u[k] = 0.0;
            for_each_harmonic(a.p, a.fx[i] - c[0], a.fy[i] - c[1], a.fz[i] - c[2], c_harm, [&](int n, int m, cplx s) {
                const int t = tri(n, m);
                const double wt = m == 0 ? 1.0 : 2.0;
#pragma unroll
                for (int k = 0; k < KM; ++k) u[k] += wt * (loc[k * T + t].re * s.re + loc[k * T + t].im * s.im);
            });
#pragma unroll
            for (int k = 0; k < KM; ++k) a.out[int64_t(k) * a.n + i] += u[k];
        }
        __syncwarp();
    }
}

// U += far + near, back in the caller's point order.
__global__ void k_finalize(EvalArgs a, double* __restrict__ pot, double* __restrict__ field)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < a.n; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t o = a.order[i];
        if (pot)
            for (int b = 0; b < a.qdim; ++b) pot[o * a.qdim + b] += a.out[b * a.n + i] + a.out2[b * a.n + i];
        if (field)
            for (int c = 0; c < 3; ++c)
                field[o * 3 + c] += a.out[(a.kf + c) * a.n + i] + a.out2[(a.kf + c) * a.n + i];
    }
}

size_t g_smem_optin = 227 * 1024;

// Warps per block such that head + warps * per_warp shared bytes fits.
int warps_for(size_t head, size_t per_warp, int maxw = 4)
{
    int w = maxw;
    while (w > 1 && head + per_warp * w > g_smem_optin) --w;
    return w;
}

template<typename KernelT>
void allow_smem(KernelT k, size_t smem)
{
    SFMM_REQUIRE(smem <= g_smem_optin, FMM_ERR_UNSUPPORTED, "kernel working set exceeds shared memory");
    allow_max_smem(k);
}

// P2M for one, two or three charge components
void launch_p2m(const EvalArgs& a, int64_t nfar, int w, size_t smem, cudaStream_t st)
{
    switch (a.qdim) {
    case 1:
        allow_smem(k_p2m<1>, smem);
        k_p2m<1><<<blocks_for(nfar, w, 65535), w * 32, smem, st>>>(a);
        break;
    case 2:
        allow_smem(k_p2m<2>, smem);
        k_p2m<2><<<blocks_for(nfar, w, 65535), w * 32, smem, st>>>(a);
        break;
    case 3:
        allow_smem(k_p2m<3>, smem);
        k_p2m<3><<<blocks_for(nfar, w, 65535), w * 32, smem, st>>>(a);
        break;
    default: SFMM_REQUIRE(false, FMM_ERR_UNSUPPORTED, "P2M: charges have 1, 2 or 3 components");
    }
    SFMM_CHECK_LAUNCH();
}

template<int KM>
void launch_l2p_k(const EvalArgs& a, int64_t nfar, int w, size_t smem, cudaStream_t st)
{
    allow_smem(k_l2p<KM>, smem);
    k_l2p<KM><<<blocks_for(nfar, w, 65535), w * 32, smem, st>>>(a);
}

// L2P for K output components: qdim (potential) + 3 (field, qdim 1 or 3),
// so 1, 2, 3, 4 or 6
void launch_l2p(const EvalArgs& a, int K, int64_t nfar, int w, size_t smem, cudaStream_t st)
{
    switch (K) {
    case 1: launch_l2p_k<1>(a, nfar, w, smem, st); break;
    case 2: launch_l2p_k<2>(a, nfar, w, smem, st); break;
    case 3: launch_l2p_k<3>(a, nfar, w, smem, st); break;
    case 4: launch_l2p_k<4>(a, nfar, w, smem, st); break;
    case 6: launch_l2p_k<6>(a, nfar, w, smem, st); break;
    default: SFMM_REQUIRE(false, FMM_ERR_UNSUPPORTED, "L2P: unexpected number of output components");
    }
    SFMM_CHECK_LAUNCH();
}

}  // namespace

// ------------------------------------------------------------------ plan
void upload_harm_coef(int device)
{
    static std::mutex mu;
    static bool done[64] = {false};
    std::lock_guard<std::mutex> lk(mu);
    if (device >= 0 && device < 64 && done[device]) return;
    HarmCoef h;
    fill_harm_coef(h);
    SFMM_CUDA(cudaMemcpyToSymbol(c_harm, &h, sizeof(h)));
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) == cudaSuccess && v > 0)
        g_smem_optin = static_cast<size_t>(v);
    if (device >= 0 && device < 64) done[device] = true;
}

// Host tables depend on p only; built once per order and shared.
static std::shared_ptr<const HostTables> tables_for(int p)
{
    static std::mutex mu;
    static std::map<int, std::shared_ptr<const HostTables>> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(p);
    if (it != cache.end()) return it->second;
    auto t = std::make_shared<const HostTables>(make_tables(p));
    cache[p] = t;
    return t;
}

template<typename T>
static void upload(DevBuf<T>& d, const std::vector<T>& h, cudaStream_t s)
{
    d.alloc(std::max<size_t>(h.size(), 1), s);
    if (!h.empty()) SFMM_CUDA(cudaMemcpyAsync(d.ptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

// Device operator tables per (device, p, precision), shared by all plans.
static std::shared_ptr<PlanTables> tables_on_device(int device, int p, bool mixed, cudaStream_t st)
{
    static std::mutex mu;
    static auto* cache = new std::map<std::tuple<int, int, bool>, std::shared_ptr<PlanTables>>();   // kept until exit
    std::lock_guard<std::mutex> lk(mu);
    auto& slot = (*cache)[std::make_tuple(device, p, mixed)];
    if (slot) return slot;
    const auto tb = tables_for(p);
    const auto tb1 = tables_for(p + 1);
    auto t = std::make_shared<PlanTables>();
    t->rot_len = tb1->rot_len;
    t->tzx_len = static_cast<int>(tb->tzx.size());
    upload(t->rot, tb1->rot, st);
    upload(t->rot_off, tb1->rot_off, st);
    upload(t->tzx, tb->tzx, st);
    upload(t->tzx_off, tb->tzx_off, st);
    upload(t->eil, tb1->eil, st);
    upload(t->echild, tb->echild, st);
    upload(t->eparent, tb->eparent, st);
    upload(t->eparent1, tb1->eparent, st);
    upload(t->m2m_ptr, tb->m2m_ptr, st);
    upload(t->m2m_code, tb->m2m_code, st);
    upload(t->m2m_g, tb->m2m_g, st);
    upload(t->l2l_ptr, tb->l2l_ptr, st);
    upload(t->l2l_code, tb->l2l_code, st);
    upload(t->l2l_g, tb->l2l_g, st);
    upload(t->l2l1_ptr, tb1->l2l_ptr, st);
    upload(t->l2l1_code, tb1->l2l_code, st);
    upload(t->l2l1_g, tb1->l2l_g, st);
    build_m2l_fragments(*t, p, mixed, st);
    build_unit_shift_ops(*t, p, st);
    SFMM_CUDA(cudaStreamSynchronize(st));         // other streams read it from now on
    slot = t;
    return t;
}

std::shared_ptr<DirectDevTables> direct_tables_on_device(int device, int p, cudaStream_t st)
{
    static std::mutex mu;
    static auto* cache = new std::map<std::pair<int, int>, std::shared_ptr<DirectDevTables>>();   // kept until exit
    std::lock_guard<std::mutex> lk(mu);
    auto& slot = (*cache)[std::make_pair(device, p)];
    if (slot) return slot;
    const DirectTables h = make_direct_tables(p);
    auto t = std::make_shared<DirectDevTables>();
    upload(t->coef, h.coef, st);
    upload(t->zil, h.zil, st);
    upload(t->eil2, h.eil2, st);
    t->ncoef = h.ncoef;
    t->nz = h.nz;
    t->ne = h.ne;
    SFMM_CUDA(cudaStreamSynchronize(st));
    slot = t;
    return t;
}

void plan_set_m2l(Plan& pl, int method)
{
    SFMM_REQUIRE(method == FMM_M2L_METHOD_ROTATION || method == FMM_M2L_METHOD_DIRECT, FMM_ERR_INVALID_ARGUMENT,
                 "method must be FMM_M2L_METHOD_ROTATION or FMM_M2L_METHOD_DIRECT");
    if (method == FMM_M2L_METHOD_DIRECT) {
        SFMM_REQUIRE(pl.precision == FMM_PRECISION_FP64, FMM_ERR_UNSUPPORTED, "the direct M2L is FP64 only");
        SFMM_REQUIRE(pl.T + pl.T1 <= 512, FMM_ERR_UNSUPPORTED, "the direct M2L takes p <= 20");
        if (!pl.dtab) pl.dtab = direct_tables_on_device(pl.tree->ctx->device, pl.p, pl.tree->ctx->stream);
    }
    pl.m2l_method = method;
}

void plan_init(Plan& pl)
{
    Tree& t = *pl.tree;
    cudaStream_t st = t.ctx->stream;
    upload_harm_coef(t.ctx->device);
    pl.T = (pl.p + 1) * (pl.p + 2) / 2;
    pl.T1 = (pl.p + 2) * (pl.p + 3) / 2;
    pl.tab = tables_on_device(t.ctx->device, pl.p, pl.precision == FMM_PRECISION_MIXED, st);
    // rho^{-(k+1)} per (level, |d|^2), k = 0..2p+2, formed as fmm.hpp:629-633 does
    pl.ipow_w = 2 * pl.p + 3;
    std::vector<double> ipw(size_t(t.depth + 1) * 28 * pl.ipow_w, 0.0);
    for (int l = 0; l <= t.depth; ++l)
        for (int d2 = 1; d2 < 28; ++d2) {
            const double rho = t.box.width / (1 << l) * std::sqrt(double(d2));
            double* r = &ipw[(size_t(l) * 28 + d2) * pl.ipow_w];
            r[0] = 1 / rho;
            for (int k = 0; k + 1 < pl.ipow_w; ++k) r[k + 1] = r[k] / rho;
        }
    upload(pl.ipow, ipw, st);
    pl.M.alloc(size_t(t.n_nodes) * pl.qdim * pl.T, st);
    pl.LA.alloc(size_t(t.n_nodes) * pl.qdim * pl.T, st);
    pl.LB.alloc(size_t(t.n_nodes) * pl.qdim * pl.T1, st);
    if (pl.precision == FMM_PRECISION_MIXED) pl.m32.alloc(size_t(t.n_nodes) * pl.qdim * pl.T, st);
    shift_setup(pl);
    p2p_setup(pl);
    pl.m2l_ctr.alloc(1, st);
    pl.wait_err.alloc(1, st);
    SFMM_CUDA(cudaMemsetAsync(pl.wait_err.ptr, 0, sizeof(int32_t), st));
    // test switch: the row-owner M2L kernel instead of the tensor-core ones
    const char* mk = std::getenv("SFMM_M2L_KERNEL");
    pl.m2l_force_rows = mk && std::strcmp(mk, "rows") == 0;
    pl.m2l_rotation_only = mk && std::strcmp(mk, "rotation") == 0;
    const int kmax = pl.qdim + 3;
    pl.qs.alloc(size_t(t.n) * pl.qdim, st);
    if (pl.precision == FMM_PRECISION_FP64) {
        pl.src4.alloc(size_t(t.n), st);
        if (pl.qdim > 1) pl.src2.alloc(size_t(t.n), st);
    }
    pl.out.alloc(size_t(t.n) * kmax, st);
    pl.out2.alloc(size_t(t.n) * kmax, st);
    m2l_i8_setup(pl);
}

static EvalArgs make_args(Plan& pl, double* pot, double* field)
{
    Tree& t = *pl.tree;
    EvalArgs a{};
    a.n = t.n;
    a.depth = t.depth;
    for (int l = 0; l <= t.depth + 1; ++l) a.lvl_off[l] = t.lvl_off[l];
    a.n_leaves = t.n_leaves;
    a.far_leaf0 = t.depth >= 2 ? t.leaf_off[2] : t.n_leaves;
    a.box = t.d_box.ptr;
    a.node_tree = t.n_trees > 1 ? t.node_tree.ptr : nullptr;
    a.wait_err = pl.wait_err.ptr;
    a.key = t.key.ptr;
    a.pbeg = t.pbeg.ptr;
    a.pend = t.pend.ptr;
    a.parent = t.parent.ptr;
    a.child_beg = t.child_beg.ptr;
    a.nchild = t.nchild.ptr;
    a.leaf_node = t.leaf_node.ptr;
    a.order = t.order.ptr;
    a.px = t.pts.ptr;
    a.py = t.pts.ptr + t.n;
    a.pz = t.pts.ptr + 2 * t.n;
    a.fx = t.far_x;
    a.fy = t.far_y;
    a.fz = t.far_z;
    a.il_ptr = t.il_ptr.ptr;
    a.il_src = t.il_src.ptr;
    a.il_code = t.il_code.ptr;
    a.nr_ptr = t.nr_ptr.ptr;
    a.nr = t.nr.ptr;
    a.p = pl.p;
    a.T = pl.T;
    a.T1 = pl.T1;
    a.qdim = pl.qdim;
    a.want_pot = pot != nullptr;
    a.want_field = field != nullptr;
    a.mixed = pl.precision == FMM_PRECISION_MIXED;
    a.kf = a.want_pot ? pl.qdim : 0;
    a.K = a.kf + (a.want_field ? 3 : 0);
    a.rot = pl.tab->rot.ptr;
    a.rot_off = pl.tab->rot_off.ptr;
    a.rot_len = pl.tab->rot_len;
    a.tzx = pl.tab->tzx.ptr;
    a.tzx_off = pl.tab->tzx_off.ptr;
    a.tzx_len = pl.tab->tzx_len;
    a.eil = reinterpret_cast<const cplx*>(pl.tab->eil.ptr);
    a.echild = reinterpret_cast<const cplx*>(pl.tab->echild.ptr);
    a.eparent = reinterpret_cast<const cplx*>(pl.tab->eparent.ptr);
    a.eparent1 = reinterpret_cast<const cplx*>(pl.tab->eparent1.ptr);
    a.m2m_ptr = pl.tab->m2m_ptr.ptr;
    a.m2m_code = pl.tab->m2m_code.ptr;
    a.m2m_g = pl.tab->m2m_g.ptr;
    a.l2l_ptr = pl.tab->l2l_ptr.ptr;
    a.l2l_code = pl.tab->l2l_code.ptr;
    a.l2l_g = pl.tab->l2l_g.ptr;
    a.l2l1_ptr = pl.tab->l2l1_ptr.ptr;
    a.l2l1_code = pl.tab->l2l1_code.ptr;
    a.l2l1_g = pl.tab->l2l1_g.ptr;
    a.ipow = pl.ipow.ptr;
    a.ipow_w = pl.ipow_w;
    a.rfrag = pl.tab->rfrag.ptr;
    a.rfrag_nf = pl.tab->rfrag_nf;
    a.tzfrag = pl.tab->tzfrag.ptr;
    a.tzl = pl.tab->tzl.ptr;
    a.rf32 = pl.tab->rf32.ptr;
    a.rf32_nf = pl.tab->rf32_nf;
    a.tz32 = pl.tab->tz32.ptr;
    a.tz32_nf = pl.tab->tz32_nf;
    a.tzl32 = pl.tab->tzl32.ptr;
    a.m32 = pl.m32.ptr;
    a.M = reinterpret_cast<cplx*>(pl.M.ptr);
    a.LA = reinterpret_cast<cplx*>(pl.LA.ptr);
    a.LB = reinterpret_cast<cplx*>(pl.LB.ptr);
    a.qs = pl.qs.ptr;
    a.src4 = pl.src4.ptr;
    a.src2 = pl.src2.ptr;
    a.p2p_item = pl.p2p_item.ptr;
    a.p2p_row = pl.p2p_row.ptr;
    a.p2p_items = pl.p2p_items;
    a.p2p_parts = pl.p2p_parts.ptr;
    a.p2p_rowoff = pl.p2p_rowoff.ptr;
    a.p2p_part = pl.p2p_part.ptr;
    a.p2p_ctr = pl.p2p_ctr.ptr;
    a.m2l_ctr = pl.m2l_ctr.ptr;
    a.m2l_force_rows = pl.m2l_force_rows;
    a.m2l_direct = pl.m2l_method == FMM_M2L_METHOD_DIRECT;
    if (a.m2l_direct) {
        a.dcoef = pl.dtab->coef.ptr;
        a.dncoef = pl.dtab->ncoef;
        a.dzil = pl.dtab->zil.ptr;
        a.dnz = pl.dtab->nz;
        a.deil2 = reinterpret_cast<const cplx*>(pl.dtab->eil2.ptr);
        a.dne = pl.dtab->ne;
    }
    a.p2p_split = pl.p2p_rows > 0;
    a.out = pl.out.ptr;
    a.out2 = pl.out2.ptr;
    a.own_leaf = pl.shard_count > 1 ? pl.own_leaf.ptr : nullptr;
    return a;
}

void plan_evaluate(Plan& pl, const double* Q, double* pot, double* field, cudaEvent_t before_sums)
{
    Tree& t = *pl.tree;
    cudaStream_t st = t.ctx->stream;
    SFMM_REQUIRE(pl.shard_count == 1, FMM_ERR_INVALID_ARGUMENT, "a sharded plan evaluates by stages (fmm_evaluate_stage)");
    EvalArgs a = make_args(pl, pot, field);
    if (a.K == 0) return;
    SFMM_REQUIRE(!(a.want_field && pl.qdim == 2), FMM_ERR_UNSUPPORTED,
                 "the field needs scalar (qdim 1) or vector (qdim 3) charges");
    const int K = a.K, T = pl.T, T1 = pl.T1, qd = pl.qdim;
    const int sms = t.ctx->sm_count;

    SFMM_CUDA(cudaEventRecord(pl.ev[0], st));
    k_gather_q<<<blocks_for(t.n, 256, 8192), 256, 0, st>>>(Q, t.order.ptr, t.n, qd, pl.qs.ptr, t.pts.ptr,
                                                               pl.src4.ptr, pl.src2.ptr);
    SFMM_CHECK_LAUNCH();
    SFMM_CUDA(cudaMemsetAsync(pl.out.ptr, 0, size_t(t.n) * K * sizeof(double), st));
    // The near field (P2P) depends only on the points and the gathered charges:
    // it runs on the context's side stream, issued after the M2L so that the
    // M2L's blocks are dispatched first and the near field fills the M2L's
    // tail and the downward pass; the stream joins back before the sums.
    SFMM_CUDA(cudaEventRecord(pl.fork, st));
    cudaStream_t side = t.ctx->side ? t.ctx->side : st;
    auto near_field = [&] {
        SFMM_CUDA(cudaStreamWaitEvent(side, pl.fork, 0));
        SFMM_CUDA(cudaEventRecord(pl.ev[6], side));
        launch_p2p(a, sms, side);
        SFMM_CUDA(cudaEventRecord(pl.ev[7], side));
        SFMM_CUDA(cudaEventRecord(pl.join, side));
    };
    const bool far = t.depth >= 2;
    if (far) {
        const int64_t nfar = t.n_leaves - a.far_leaf0;
        const size_t sm_p2m_w = size_t(qd) * T * sizeof(cplx) + kP2MStageBytes;
        const int w_p2m = warps_for(0, sm_p2m_w);
        launch_p2m(a, nfar, w_p2m, sm_p2m_w * w_p2m, st);
        const size_t head = (32 + 2 * 4 * (2 * kMaxOrder + 1)) * sizeof(double);
        const size_t sm_m2m_w = 2 * size_t(qd) * T * sizeof(cplx);
        const int w_m2m = warps_for(head, sm_m2m_w);
        allow_smem(k_m2m, head + sm_m2m_w * w_m2m);
        for (int l = t.depth - 1; l >= 2; --l) {
            if (pl.shift_on) {
                shift_m2m(pl, a, l, st);
                continue;
            }
            const int64_t c = t.lvl_off[l + 1] - t.lvl_off[l];
            k_m2m<<<blocks_for(c, w_m2m, 65535), w_m2m * 32, head + sm_m2m_w * w_m2m, st>>>(a, l, t.lvl_off[l], c);
            SFMM_CHECK_LAUNCH();
        }
        SFMM_CUDA(cudaEventRecord(pl.ev[1], st));
        if (a.m2l_direct) launch_m2l_direct(a, t.lvl_off[1], t.lvl_off[t.depth], sms, st);
        else if (pl.i8) launch_m2l_i8(pl, a, st);
        else launch_m2l(a, t.lvl_off[1], t.lvl_off[t.depth], sms, st);
        near_field();
        SFMM_CUDA(cudaEventRecord(pl.ev[2], st));
        const size_t head2 = (32 + 2 * 4 * (2 * kMaxOrder + 1) + 2 * 4 * (2 * kMaxOrder + 3)) * sizeof(double);
        const size_t sm_l2l_w = size_t(qd) * (T + T1) * sizeof(cplx);
        const int w_l2l = warps_for(head2, sm_l2l_w);
        allow_smem(k_l2l, head2 + sm_l2l_w * w_l2l);
        for (int l = 3; l <= t.depth; ++l) {
            if (pl.shift_on) {
                shift_l2l(pl, a, l, st);
                continue;
            }
            const int64_t c = t.lvl_off[l + 1] - t.lvl_off[l];
            k_l2l<<<blocks_for(c, w_l2l, 65535), w_l2l * 32, head2 + sm_l2l_w * w_l2l, st>>>(a, l, t.lvl_off[l], c);
            SFMM_CHECK_LAUNCH();
        }
        const size_t sm_l2p_w = size_t(K) * T * sizeof(cplx);
        const int w_l2p = warps_for(0, sm_l2p_w);
        launch_l2p(a, K, nfar, w_l2p, sm_l2p_w * w_l2p, st);
    } else {
        SFMM_CUDA(cudaEventRecord(pl.ev[1], st));
        near_field();
        SFMM_CUDA(cudaEventRecord(pl.ev[2], st));
    }
    SFMM_CUDA(cudaEventRecord(pl.ev[3], st));
    SFMM_CUDA(cudaStreamWaitEvent(st, pl.join, 0));
    if (before_sums) SFMM_CUDA(cudaStreamWaitEvent(st, before_sums, 0));
    SFMM_CUDA(cudaEventRecord(pl.ev[4], st));
    k_finalize<<<blocks_for(t.n, 256, 8192), 256, 0, st>>>(a, pot, field);
    SFMM_CHECK_LAUNCH();
    if (pl.ex_on) apply_exclusions(pl, Q, pot, field);
    SFMM_CUDA(cudaEventRecord(pl.ev[5], st));
}

// ------------------------------------------------------------------ sharded evaluation
void plan_set_shard(Plan& pl, int index, int count)
{
    SFMM_REQUIRE(count >= 1 && count <= 4096 && index >= 0 && index < count, FMM_ERR_INVALID_ARGUMENT,
                 "shard index must be in [0, count), 1 <= count <= 4096");
    Tree& t = *pl.tree;
    cudaStream_t st = t.ctx->stream;
    pl.shard_index = index;
    pl.shard_count = count;
    if (count > 1) pl.i8.reset();                 // sharded mixed plans take the rotation M2L
    pl.own_parent_b.clear();
    pl.own_parent_e.clear();
    if (count == 1) {
        pl.own_leaf.release();
        return;
    }
    // this shard's leaves, level by level, balanced by points (shard_ranges.h)
    std::vector<int32_t> ln(t.n_leaves), pb(t.n_nodes), pe(t.n_nodes);
    SFMM_CUDA(cudaMemcpyAsync(ln.data(), t.leaf_node.ptr, ln.size() * 4, cudaMemcpyDeviceToHost, st));
    SFMM_CUDA(cudaMemcpyAsync(pb.data(), t.pbeg.ptr, pb.size() * 4, cudaMemcpyDeviceToHost, st));
    SFMM_CUDA(cudaMemcpyAsync(pe.data(), t.pend.ptr, pe.size() * 4, cudaMemcpyDeviceToHost, st));
    SFMM_CUDA(cudaStreamSynchronize(st));
    std::vector<uint8_t> own(std::max<int64_t>(t.n_leaves, 1), 0);
    for (int l = 0; l <= t.depth; ++l) {
        const int64_t f0 = t.leaf_off[l], nl = t.leaf_off[l + 1] - f0;
        std::vector<int64_t> prefix(nl + 1, 0);
        for (int64_t i = 0; i < nl; ++i) prefix[i + 1] = prefix[i] + (pe[ln[f0 + i]] - pb[ln[f0 + i]]);
        const auto r = balanced_leaf_range(prefix.data(), nl, count, index);
        for (int64_t i = r.first; i < r.second; ++i) own[f0 + i] = 1;
    }
    pl.own_leaf.alloc(own.size(), st);
    SFMM_CUDA(cudaMemcpyAsync(pl.own_leaf.ptr, own.data(), own.size(), cudaMemcpyHostToDevice, st));
    SFMM_CUDA(cudaStreamSynchronize(st));
    // this shard's parents of M2L targets, level by level (contiguous ranges)
    for (int q = 0; q <= t.depth; ++q) {
        const int64_t b = t.lvl_off[q], nq = t.lvl_off[q + 1] - b;
        pl.own_parent_b.push_back(b + shard_begin(nq, count, index));
        pl.own_parent_e.push_back(b + shard_end(nq, count, index));
    }
}

void plan_evaluate_stage(Plan& pl, const double* Q, double* pot, double* field, int stage)
{
    Tree& t = *pl.tree;
    cudaStream_t st = t.ctx->stream;
    SFMM_REQUIRE(stage >= 0 && stage <= 2, FMM_ERR_INVALID_ARGUMENT, "stage must be 0, 1 or 2");
    EvalArgs a = make_args(pl, pot, field);
    if (a.K == 0) return;
    SFMM_REQUIRE(!(a.want_field && pl.qdim == 2), FMM_ERR_UNSUPPORTED,
                 "the field needs scalar (qdim 1) or vector (qdim 3) charges");
    const int K = a.K, T = pl.T, T1 = pl.T1, qd = pl.qdim;
    const int sms = t.ctx->sm_count;
    const bool far = t.depth >= 2;
    const int64_t nfar = t.n_leaves - a.far_leaf0;
    cudaStream_t side = t.ctx->side ? t.ctx->side : st;
    if (stage == 0) {
        // charges; the near field of this shard's leaves on the side stream
        // (others' targets stay zero); moments of this shard's leaves
        k_gather_q<<<blocks_for(t.n, 256, 8192), 256, 0, st>>>(Q, t.order.ptr, t.n, qd, pl.qs.ptr, t.pts.ptr,
                                                                   pl.src4.ptr, pl.src2.ptr);
        SFMM_CHECK_LAUNCH();
        SFMM_CUDA(cudaMemsetAsync(pl.out.ptr, 0, size_t(t.n) * K * sizeof(double), st));
        SFMM_CUDA(cudaMemsetAsync(pl.out2.ptr, 0, size_t(t.n) * K * sizeof(double), st));
        SFMM_CUDA(cudaEventRecord(pl.fork, st));
        SFMM_CUDA(cudaStreamWaitEvent(side, pl.fork, 0));
        launch_p2p(a, sms, side);
        SFMM_CUDA(cudaEventRecord(pl.join, side));
        if (far) {
            const size_t sm_p2m_w = size_t(qd) * T * sizeof(cplx) + kP2MStageBytes;
            const int w_p2m = warps_for(0, sm_p2m_w);
            launch_p2m(a, nfar, w_p2m, sm_p2m_w * w_p2m, st);
        }
        return;
    }
    if (stage == 1) {
        // moments summed over the shards by the caller: M2M in full, then
        // M2L into the children of this shard's parents
        if (!far) return;
        const size_t head = (32 + 2 * 4 * (2 * kMaxOrder + 1)) * sizeof(double);
        const size_t sm_m2m_w = 2 * size_t(qd) * T * sizeof(cplx);
        const int w_m2m = warps_for(head, sm_m2m_w);
        allow_smem(k_m2m, head + sm_m2m_w * w_m2m);
        for (int l = t.depth - 1; l >= 2; --l) {
            if (pl.shift_on) {
                shift_m2m(pl, a, l, st);
                continue;
            }
            const int64_t c = t.lvl_off[l + 1] - t.lvl_off[l];
            k_m2m<<<blocks_for(c, w_m2m, 65535), w_m2m * 32, head + sm_m2m_w * w_m2m, st>>>(a, l, t.lvl_off[l], c);
            SFMM_CHECK_LAUNCH();
        }
        SFMM_CUDA(cudaMemsetAsync(pl.LA.ptr, 0, pl.LA.bytes(), st));
        SFMM_CUDA(cudaMemsetAsync(pl.LB.ptr, 0, pl.LB.bytes(), st));
        for (int q = 1; q < t.depth; ++q) {
            if (a.m2l_direct) launch_m2l_direct(a, pl.own_parent_b[q], pl.own_parent_e[q], sms, st);
            else launch_m2l(a, pl.own_parent_b[q], pl.own_parent_e[q], sms, st);
        }
        return;
    }
    // locals summed over the shards by the caller: L2L in full, L2P of this
    // shard's leaves, then the sums (zero at other shards' points)
    if (far) {
        const size_t head2 = (32 + 2 * 4 * (2 * kMaxOrder + 1) + 2 * 4 * (2 * kMaxOrder + 3)) * sizeof(double);
        const size_t sm_l2l_w = size_t(qd) * (T + T1) * sizeof(cplx);
        const int w_l2l = warps_for(head2, sm_l2l_w);
        allow_smem(k_l2l, head2 + sm_l2l_w * w_l2l);
        for (int l = 3; l <= t.depth; ++l) {
            if (pl.shift_on) {
                shift_l2l(pl, a, l, st);
                continue;
            }
            const int64_t c = t.lvl_off[l + 1] - t.lvl_off[l];
            k_l2l<<<blocks_for(c, w_l2l, 65535), w_l2l * 32, head2 + sm_l2l_w * w_l2l, st>>>(a, l, t.lvl_off[l], c);
            SFMM_CHECK_LAUNCH();
        }
        const size_t sm_l2p_w = size_t(K) * T * sizeof(cplx);
        const int w_l2p = warps_for(0, sm_l2p_w);
        launch_l2p(a, K, nfar, w_l2p, sm_l2p_w * w_l2p, st);
    }
    SFMM_CUDA(cudaStreamWaitEvent(st, pl.join, 0));
    k_finalize<<<blocks_for(t.n, 256, 8192), 256, 0, st>>>(a, pot, field);
    SFMM_CHECK_LAUNCH();
    // excluded interactions are removed once, by shard 0, for every target
    if (pl.ex_on && pl.shard_index == 0) apply_exclusions(pl, Q, pot, field);
}

void plan_read_timings(Plan& pl, double* ms6)
{
    SFMM_CUDA(cudaEventSynchronize(pl.ev[5]));
    float v;
    SFMM_CUDA(cudaEventElapsedTime(&v, pl.ev[0], pl.ev[1]));
    ms6[0] = v;
    SFMM_CUDA(cudaEventElapsedTime(&v, pl.ev[1], pl.ev[2]));
    ms6[1] = v;
    SFMM_CUDA(cudaEventElapsedTime(&v, pl.ev[2], pl.ev[3]));
    ms6[2] = v;
    SFMM_CUDA(cudaEventElapsedTime(&v, pl.ev[6], pl.ev[7]));      // near field, on the side stream
    ms6[3] = v;
    SFMM_CUDA(cudaEventElapsedTime(&v, pl.ev[0], pl.ev[5]));
    ms6[4] = v;
    ms6[5] = pl.tree->build_ms;
}

}  // namespace sfmm
