// FP64 evaluation kernels: P2M, M2M, M2L, L2L, L2P, P2P and the plan.
//
// Phase structure of FMM3D::rinv (fmm.hpp:811-881): far field only when the
// tree is at least 2 levels deep; multipoles at every leaf of level >= 2;
// M2M up to level 2; M2L on levels 2..depth; L2L down; L2P at every leaf of
// level >= 2; near field over the neighbour lists.  All per-coefficient
// math is in fmm_ops.cuh; expansions keep only m >= 0.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "fmm_eval.cuh"
#include "fmm_tables.h"

namespace sfmm {

__constant__ HarmCoef c_harm;

namespace {

constexpr int kMaxWarps = 4;              // warps per block in the per-box kernels (fewer when shared memory is short)

__device__ __forceinline__ int level_of(const EvalArgs& a, int64_t g)
{
    int l = 0;
    while (l < a.depth && g >= a.lvl_off[l + 1]) ++l;
    return l;
}

// box.hpp:147-150
__device__ __forceinline__ void node_center(const BoxDev& b, uint64_t key, int l, double* c)
{
    const uint32_t ix = compact3(key), iy = compact3(key >> 1), iz = compact3(key >> 2);
    const double s = double(1 << l);
    c[0] = b.corner[0] + b.width * ((ix + 0.5) / s);
    c[1] = b.corner[1] + b.width * ((iy + 0.5) / s);
    c[2] = b.corner[2] + b.width * ((iz + 0.5) / s);
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void tri_nm(int t, int& n, int& m)
{
    n = static_cast<int>((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
    if ((n + 1) * (n + 2) / 2 <= t) ++n;
    if (n * (n + 1) / 2 > t) --n;
    m = t - n * (n + 1) / 2;
}

__global__ void k_gather_q(const double* __restrict__ Q, const int32_t* __restrict__ order, int64_t n, int qdim,
                           double* __restrict__ qs)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t o = order[i];
        for (int b = 0; b < qdim; ++b) qs[b * n + i] = Q[o * qdim + b];
    }
}

// P2M (fmm.hpp:524-556): warp per leaf of level >= 2, lanes over points,
// one warp-sum per coefficient.
__global__ void __launch_bounds__(kMaxWarps * 32) k_p2m(EvalArgs a)
{
    extern __shared__ double smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    cplx* acc = reinterpret_cast<cplx*>(smem) + w * a.qdim * a.T;
    const int64_t nfar = a.n_leaves - a.far_leaf0;
    for (int64_t f = blockIdx.x * int64_t(nw) + w; f < nfar; f += int64_t(gridDim.x) * nw) {
        const int g = a.leaf_node[a.far_leaf0 + f];
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
            double q[3] = {0, 0, 0};
            if (on)
                for (int b = 0; b < a.qdim; ++b) q[b] = a.qs[b * a.n + i];
            for_each_harmonic(a.p, x, y, z, c_harm, [&](int n, int m, cplx s) {
                const int t = tri(n, m);
                for (int b = 0; b < a.qdim; ++b) {
                    const double re = warp_sum(q[b] * s.re), im = warp_sum(q[b] * s.im);
                    if (lane == 0) {
                        acc[b * a.T + t].re += re;
                        acc[b * a.T + t].im += im;
                    }
                }
            });
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

// M2L (fmm.hpp:620-712) first version: warp per target node, pairs in
// ilist order; rotate -> z-translate -> rotate back in warp-private shared
// buffers, accumulation in shared memory, one store per target.
__global__ void __launch_bounds__(kMaxWarps * 32) k_m2l(EvalArgs a, int64_t off, int64_t cnt)
{
    extern __shared__ double smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int p = a.p, T = a.T, K = a.cs.K, KT = K * T;
    double* tz = smem;                                           // tz_len
    cplx* eil = reinterpret_cast<cplx*>(smem + a.tz_len);        // 49 x (p+1)
    cplx* wbase = eil + 49 * (p + 1) + w * (3 * KT + a.qdim * T);
    cplx* A = wbase;
    cplx* B = A + KT;
    cplx* acc = B + KT;
    cplx* src = acc + KT;
    for (int t = threadIdx.x; t < a.tz_len; t += blockDim.x) tz[t] = a.tz[t];
    for (int t = threadIdx.x; t < 49 * (p + 1); t += blockDim.x) eil[t] = a.eil[t];
    __syncthreads();
    for (int64_t i = blockIdx.x * int64_t(nw) + w; i < cnt; i += int64_t(gridDim.x) * nw) {
        const int64_t g = off + i;
        const int e0 = a.il_ptr[g], e1 = a.il_ptr[g + 1];
        const int l = level_of(a, g);
        for (int t = lane; t < KT; t += 32) acc[t] = cplx{0, 0};
        for (int e = e0; e < e1; ++e) {
            const int s = a.il_src[e];
            const int code = a.il_code[e];
            const int di = (code & 7) - 3, dj = ((code >> 3) & 7) - 3, dk = ((code >> 6) & 7) - 3;
            const double* R = a.rot + int64_t(rot_class(di, dj, dk)) * a.rot_len;
            const cplx* ph = eil + (7 * (dj + 3) + (di + 3)) * (p + 1);
            const double* ipw = a.ipow + (int64_t(l) * 28 + (di * di + dj * dj + dk * dk)) * (2 * p + 2);
            const cplx* Ms = a.M + int64_t(s) * a.qdim * T;
            for (int t = lane; t < a.qdim * T; t += 32) src[t] = Ms[t];
            __syncwarp();
            // derive + phase: Mt = e^{i m phi} X
            for (int o = lane; o < KT; o += 32) {
                const int k = o / T, t = o - k * T;
                int n, m;
                tri_nm(t, n, m);
                A[o] = cmul(ph[m], derive_component(a.cs, src, T, k, n, m));
            }
            __syncwarp();
            // rotation: W_n = (P Re Mt_n, Q Im Mt_n) rho^{-n}
            for (int o = lane; o < KT; o += 32) {
                const int k = o / T, t = o - k * T;
                int n, aa;
                tri_nm(t, n, aa);
                const double* P = R + a.rot_off[n] + aa * (n + 1);
                const double* Qm = P + (n + 1) * (n + 1);
                const cplx* x = A + k * T + n * (n + 1) / 2;
                double re = 0, im = 0;
                for (int b = 0; b <= n; ++b) {
                    re += __ldg(P + b) * x[b].re;
                    im += __ldg(Qm + b) * x[b].im;
                }
                const double sc = n ? ipw[n - 1] : 1.0;
                B[o] = cplx{re * sc, im * sc};
            }
            __syncwarp();
            // z-translation: Lz_j^k = rho^{-(j+1)} sum_n tz[k][j][n] W_n^k
            for (int o = lane; o < KT; o += 32) {
                const int k = o / T, t = o - k * T;
                int j, kk;
                tri_nm(t, j, kk);
                const int wd = p + 1 - kk;
                const double* row = tz + a.tz_off[kk] + (j - kk) * wd;
                const cplx* x = B + k * T;
                double re = 0, im = 0;
                for (int n = kk; n <= p; ++n) {
                    const cplx v = x[n * (n + 1) / 2 + kk];
                    re += row[n - kk] * v.re;
                    im += row[n - kk] * v.im;
                }
                const double sc = ipw[j];
                A[o] = cplx{re * sc, im * sc};
            }
            __syncwarp();
            // rotate back + phase, accumulate
            for (int o = lane; o < KT; o += 32) {
                const int k = o / T, t = o - k * T;
                int j, aa;
                tri_nm(t, j, aa);
                const int wd = (j + 1) * (j + 1);
                const double* PB = R + a.rot_off[j] + 2 * wd + aa * (j + 1);
                const double* QB = PB + wd;
                const cplx* x = A + k * T + j * (j + 1) / 2;
                double re = 0, im = 0;
                for (int b = 0; b <= j; ++b) {
                    re += __ldg(PB + b) * x[b].re;
                    im += __ldg(QB + b) * x[b].im;
                }
                const cplx v = cmul(cconj(ph[aa]), cplx{re, im});
                acc[o].re += v.re;
                acc[o].im += v.im;
            }
            __syncwarp();
        }
        cplx* Lt = a.L + g * KT;
        for (int t = lane; t < KT; t += 32) Lt[t] = acc[t];
        __syncwarp();
    }
}

// L2L (fmm.hpp:714-745): warp per child node at level lc.
__global__ void __launch_bounds__(kMaxWarps * 32) k_l2l(EvalArgs a, int lc, int64_t off, int64_t cnt)
{
    extern __shared__ double smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int p = a.p, T = a.T, K = a.cs.K, KT = K * T;
    double* rpow = smem;
    cplx* phase = reinterpret_cast<cplx*>(smem + 32);
    cplx* par = reinterpret_cast<cplx*>(smem + 32) + 4 * (2 * kMaxOrder + 1) + w * KT;
    if (threadIdx.x == 0) {
        const double rho = sqrt(0.75) * a.box->width / (1 << lc);
        rpow[0] = 1;
        for (int k = 1; k <= p; ++k) rpow[k] = rpow[k - 1] * rho;
    }
    for (int t = threadIdx.x; t < 4 * (2 * p + 1); t += blockDim.x) phase[t] = a.eparent[t];
    __syncthreads();
    for (int64_t i = blockIdx.x * int64_t(nw) + w; i < cnt; i += int64_t(gridDim.x) * nw) {
        const int64_t g = off + i;
        const int pg = a.parent[g];
        const cplx* Lp = a.L + int64_t(pg) * KT;
        for (int t = lane; t < KT; t += 32) par[t] = Lp[t];
        __syncwarp();
        const int oct = static_cast<int>(a.key[g] & 7);
        cplx* Lc = a.L + g * KT;
        for (int o = lane; o < KT; o += 32) {
            const int k = o / T, t = o - k * T;
            const cplx v = shift_output<false>(t, a.l2l_ptr, a.l2l_code, a.l2l_g, par + k * T, oct, rpow,
                                               phase + (oct & 3) * (2 * p + 1), p);
            Lc[o].re += v.re;
            Lc[o].im += v.im;
        }
        __syncwarp();
    }
}

// L2P (fmm.hpp:747-771): warp per leaf of level >= 2, lanes over points.
__global__ void __launch_bounds__(kMaxWarps * 32) k_l2p(EvalArgs a)
{
    extern __shared__ double smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int T = a.T, K = a.cs.K, KT = K * T;
    cplx* loc = reinterpret_cast<cplx*>(smem) + w * KT;
    const int64_t nfar = a.n_leaves - a.far_leaf0;
    for (int64_t f = blockIdx.x * int64_t(nw) + w; f < nfar; f += int64_t(gridDim.x) * nw) {
        const int g = a.leaf_node[a.far_leaf0 + f];
        const int l = level_of(a, g);
        double c[3];
        node_center(*a.box, a.key[g], l, c);
        const cplx* Lg = a.L + int64_t(g) * KT;
        for (int t = lane; t < KT; t += 32) loc[t] = Lg[t];
        __syncwarp();
        const int b0 = a.pbeg[g], b1 = a.pend[g];
        for (int i = b0 + lane; i < b1; i += 32) {
            double u[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for_each_harmonic(a.p, a.fx[i] - c[0], a.fy[i] - c[1], a.fz[i] - c[2], c_harm, [&](int n, int m, cplx s) {
                const int t = tri(n, m);
                const double wt = m == 0 ? 1.0 : 2.0;
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    if (k < K) u[k] += wt * (loc[k * T + t].re * s.re + loc[k * T + t].im * s.im);
            });
            for (int k = 0; k < K; ++k) a.out[int64_t(k) * a.n + i] += u[k];
        }
        __syncwarp();
    }
}

// P2P (fmm.hpp:773-809): block per leaf, thread per target, source tiles
// staged in shared memory from the leaf's near-field point ranges.
constexpr int kP2PThreads = 64;

__global__ void __launch_bounds__(kP2PThreads) k_p2p(EvalArgs a)
{
    __shared__ double sx[kP2PThreads], sy[kP2PThreads], sz[kP2PThreads], sq[3][kP2PThreads];
    const int64_t f = blockIdx.x;
    const int g = a.leaf_node[f];
    const int t0 = a.pbeg[g], t1 = a.pend[g];
    const int r0 = a.nr_ptr[f], r1 = a.nr_ptr[f + 1];
    const int qd = a.qdim;
    for (int tb = t0; tb < t1; tb += kP2PThreads) {
        const int i = tb + threadIdx.x;
        const bool on = i < t1;
        const double xi = on ? a.px[i] : 0, yi = on ? a.py[i] : 0, zi = on ? a.pz[i] : 0;
        double pot[3] = {0, 0, 0}, fld[3] = {0, 0, 0};
        for (int r = r0; r < r1; ++r) {
            const int2 rg = a.nr[r];
            for (int sb = rg.x; sb < rg.y; sb += kP2PThreads) {
                const int j = sb + threadIdx.x;
                __syncthreads();
                if (j < rg.y) {
                    sx[threadIdx.x] = a.px[j];
                    sy[threadIdx.x] = a.py[j];
                    sz[threadIdx.x] = a.pz[j];
                    for (int b = 0; b < qd; ++b) sq[b][threadIdx.x] = a.qs[b * a.n + j];
                }
                __syncthreads();
                const int ns = min(kP2PThreads, rg.y - sb);
                if (!on) continue;
                for (int s = 0; s < ns; ++s) {
                    if (sb + s == i) continue;
                    const double dx = xi - sx[s], dy = yi - sy[s], dz = zi - sz[s];
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    const double ir = 1.0 / sqrt(r2);
                    if (a.cs.want_pot)
                        for (int b = 0; b < qd; ++b) pot[b] += sq[b][s] * ir;
                    if (a.cs.want_field) {
                        const double ir3 = ir * ir * ir;
                        if (qd == 1) {
                            const double c = sq[0][s] * ir3;
                            fld[0] += c * dx;
                            fld[1] += c * dy;
                            fld[2] += c * dz;
                        } else {
                            fld[0] += (sq[1][s] * dz - sq[2][s] * dy) * ir3;
                            fld[1] += (sq[2][s] * dx - sq[0][s] * dz) * ir3;
                            fld[2] += (sq[0][s] * dy - sq[1][s] * dx) * ir3;
                        }
                    }
                }
            }
        }
        if (on) {
            if (a.cs.want_pot)
                for (int b = 0; b < qd; ++b) a.out2[int64_t(b) * a.n + i] = pot[b];
            if (a.cs.want_field)
                for (int c = 0; c < 3; ++c) a.out2[int64_t(a.cs.kf + c) * a.n + i] = fld[c];
        }
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
                field[o * 3 + c] += a.out[(a.cs.kf + c) * a.n + i] + a.out2[(a.cs.kf + c) * a.n + i];
    }
}

constexpr size_t kSmemBudget = 200 * 1024;

// Warps per block such that head + warps * per_warp shared bytes fits.
int warps_for(size_t head, size_t per_warp)
{
    int w = kMaxWarps;
    while (w > 1 && head + per_warp * w > kSmemBudget) --w;
    return w;
}

template<typename KernelT>
void launch_cfg(KernelT k, int, size_t smem)
{
    SFMM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
}

}  // namespace

// ------------------------------------------------------------------ plan
void upload_harm_coef(int device)
{
    static bool done[64] = {false};
    if (device >= 0 && device < 64 && done[device]) return;
    HarmCoef h;
    fill_harm_coef(h);
    SFMM_CUDA(cudaMemcpyToSymbol(c_harm, &h, sizeof(h)));
    if (device >= 0 && device < 64) done[device] = true;
}

template<typename T>
static void upload(DevBuf<T>& d, const std::vector<T>& h, cudaStream_t s)
{
    d.alloc(std::max<size_t>(h.size(), 1), s);
    if (!h.empty()) SFMM_CUDA(cudaMemcpyAsync(d.ptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

void plan_init(Plan& pl)
{
    Tree& t = *pl.tree;
    cudaStream_t st = t.ctx->stream;
    upload_harm_coef(t.ctx->device);
    const HostTables tb = make_tables(pl.p);
    pl.T = tb.T;
    pl.rot_len = tb.rot_len;
    pl.tz_len = static_cast<int>(tb.tz.size());
    upload(pl.rot, tb.rot, st);
    upload(pl.rot_off, tb.rot_off, st);
    upload(pl.tz, tb.tz, st);
    upload(pl.tz_off, tb.tz_off, st);
    upload(pl.eil, tb.eil, st);
    upload(pl.echild, tb.echild, st);
    upload(pl.eparent, tb.eparent, st);
    upload(pl.m2m_ptr, tb.m2m_ptr, st);
    upload(pl.m2m_code, tb.m2m_code, st);
    upload(pl.m2m_g, tb.m2m_g, st);
    upload(pl.l2l_ptr, tb.l2l_ptr, st);
    upload(pl.l2l_code, tb.l2l_code, st);
    upload(pl.l2l_g, tb.l2l_g, st);
    // rho^{-(k+1)} per (level, |d|^2), k = 0..2p, as fmm.hpp:629-633 forms them
    std::vector<double> ipw(size_t(t.depth + 1) * 28 * (2 * pl.p + 2), 0.0);
    for (int l = 0; l <= t.depth; ++l)
        for (int d2 = 1; d2 < 28; ++d2) {
            const double rho = t.box.width / (1 << l) * std::sqrt(double(d2));
            double* r = &ipw[(size_t(l) * 28 + d2) * (2 * pl.p + 2)];
            r[0] = 1 / rho;
            for (int k = 0; k < 2 * pl.p + 1; ++k) r[k + 1] = r[k] / rho;
        }
    upload(pl.ipow, ipw, st);
    const int kmax = pl.qdim + 3;
    pl.M.alloc(size_t(t.n_nodes) * pl.qdim * pl.T, st);
    pl.L.alloc(size_t(t.n_nodes) * kmax * pl.T, st);
    pl.qs.alloc(size_t(t.n) * pl.qdim, st);
    pl.out.alloc(size_t(t.n) * kmax, st);
    pl.out2.alloc(size_t(t.n) * kmax, st);
}

void plan_evaluate(Plan& pl, const double* Q, double* pot, double* field)
{
    Tree& t = *pl.tree;
    cudaStream_t st = t.ctx->stream;
    EvalArgs a{};
    a.n = t.n;
    a.depth = t.depth;
    for (int l = 0; l <= t.depth + 1; ++l) a.lvl_off[l] = t.lvl_off[l];
    a.n_leaves = t.n_leaves;
    a.far_leaf0 = t.depth >= 2 ? t.leaf_off[2] : t.n_leaves;
    a.box = t.d_box.ptr;
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
    a.qdim = pl.qdim;
    a.cs.qdim = pl.qdim;
    a.cs.want_pot = pot != nullptr;
    a.cs.want_field = field != nullptr;
    a.cs.kf = a.cs.want_pot ? pl.qdim : 0;
    a.cs.K = a.cs.kf + (a.cs.want_field ? 3 : 0);
    a.rot = pl.rot.ptr;
    a.rot_off = pl.rot_off.ptr;
    a.rot_len = pl.rot_len;
    a.tz = pl.tz.ptr;
    a.tz_off = pl.tz_off.ptr;
    a.tz_len = pl.tz_len;
    a.eil = reinterpret_cast<const cplx*>(pl.eil.ptr);
    a.echild = reinterpret_cast<const cplx*>(pl.echild.ptr);
    a.eparent = reinterpret_cast<const cplx*>(pl.eparent.ptr);
    a.m2m_ptr = pl.m2m_ptr.ptr;
    a.m2m_code = pl.m2m_code.ptr;
    a.m2m_g = pl.m2m_g.ptr;
    a.l2l_ptr = pl.l2l_ptr.ptr;
    a.l2l_code = pl.l2l_code.ptr;
    a.l2l_g = pl.l2l_g.ptr;
    a.ipow = pl.ipow.ptr;
    a.M = reinterpret_cast<cplx*>(pl.M.ptr);
    a.L = reinterpret_cast<cplx*>(pl.L.ptr);
    a.qs = pl.qs.ptr;
    a.out = pl.out.ptr;
    a.out2 = pl.out2.ptr;
    if (a.cs.K == 0) return;
    SFMM_REQUIRE(!(a.cs.want_field && pl.qdim != 1 && pl.qdim != 3), FMM_ERR_UNSUPPORTED,
                 "the field needs scalar (qdim 1) or vector (qdim 3) charges");
    const int K = a.cs.K, T = pl.T;
    const int sms = t.ctx->sm_count;

    SFMM_CUDA(cudaEventRecord(pl.ev[0], st));
    k_gather_q<<<blocks_for(t.n, 256, 8192), 256, 0, st>>>(Q, t.order.ptr, t.n, pl.qdim, pl.qs.ptr);
    SFMM_CHECK_LAUNCH();
    SFMM_CUDA(cudaMemsetAsync(pl.out.ptr, 0, size_t(t.n) * K * sizeof(double), st));
    SFMM_CUDA(cudaMemsetAsync(pl.out2.ptr, 0, size_t(t.n) * K * sizeof(double), st));
    const bool far = t.depth >= 2;
    if (far) {
        SFMM_CUDA(cudaMemsetAsync(pl.M.ptr, 0, size_t(t.n_nodes) * pl.qdim * T * sizeof(cplx), st));
        const int64_t nfar = t.n_leaves - a.far_leaf0;
        const size_t head = (32 + 2 * 4 * (2 * kMaxOrder + 1)) * sizeof(double);
        const size_t sm_p2m_w = size_t(pl.qdim) * T * sizeof(cplx);
        const int w_p2m = warps_for(0, sm_p2m_w);
        launch_cfg(k_p2m, w_p2m, sm_p2m_w * w_p2m);
        k_p2m<<<blocks_for(nfar, w_p2m, 65535), w_p2m * 32, sm_p2m_w * w_p2m, st>>>(a);
        SFMM_CHECK_LAUNCH();
        const size_t sm_m2m_w = 2 * size_t(pl.qdim) * T * sizeof(cplx);
        const int w_m2m = warps_for(head, sm_m2m_w);
        launch_cfg(k_m2m, w_m2m, head + sm_m2m_w * w_m2m);
        for (int l = t.depth - 1; l >= 2; --l) {
            const int64_t c = t.lvl_off[l + 1] - t.lvl_off[l];
            k_m2m<<<blocks_for(c, w_m2m, 65535), w_m2m * 32, head + sm_m2m_w * w_m2m, st>>>(a, l, t.lvl_off[l], c);
            SFMM_CHECK_LAUNCH();
        }
        SFMM_CUDA(cudaEventRecord(pl.ev[1], st));
        const size_t head_m2l = pl.tz_len * sizeof(double) + 49 * (pl.p + 1) * sizeof(cplx);
        const size_t sm_m2l_w = size_t(3 * K * T + pl.qdim * T) * sizeof(cplx);
        const int w_m2l = warps_for(head_m2l, sm_m2l_w);
        launch_cfg(k_m2l, w_m2l, head_m2l + sm_m2l_w * w_m2l);
        const int64_t c2 = t.n_nodes - t.lvl_off[2];
        k_m2l<<<blocks_for(c2, w_m2l, int64_t(sms) * 64), w_m2l * 32, head_m2l + sm_m2l_w * w_m2l, st>>>(a, t.lvl_off[2], c2);
        SFMM_CHECK_LAUNCH();
        SFMM_CUDA(cudaEventRecord(pl.ev[2], st));
        const size_t sm_l2l_w = size_t(K) * T * sizeof(cplx);
        const int w_l2l = warps_for(head, sm_l2l_w);
        launch_cfg(k_l2l, w_l2l, head + sm_l2l_w * w_l2l);
        for (int l = 3; l <= t.depth; ++l) {
            const int64_t c = t.lvl_off[l + 1] - t.lvl_off[l];
            k_l2l<<<blocks_for(c, w_l2l, 65535), w_l2l * 32, head + sm_l2l_w * w_l2l, st>>>(a, l, t.lvl_off[l], c);
            SFMM_CHECK_LAUNCH();
        }
        const size_t sm_l2p_w = size_t(K) * T * sizeof(cplx);
        const int w_l2p = warps_for(0, sm_l2p_w);
        launch_cfg(k_l2p, w_l2p, sm_l2p_w * w_l2p);
        k_l2p<<<blocks_for(nfar, w_l2p, 65535), w_l2p * 32, sm_l2p_w * w_l2p, st>>>(a);
        SFMM_CHECK_LAUNCH();
    } else {
        SFMM_CUDA(cudaEventRecord(pl.ev[1], st));
        SFMM_CUDA(cudaEventRecord(pl.ev[2], st));
    }
    SFMM_CUDA(cudaEventRecord(pl.ev[3], st));
    k_p2p<<<static_cast<unsigned>(t.n_leaves), kP2PThreads, 0, st>>>(a);
    SFMM_CHECK_LAUNCH();
    SFMM_CUDA(cudaEventRecord(pl.ev[4], st));
    k_finalize<<<blocks_for(t.n, 256, 8192), 256, 0, st>>>(a, pot, field);
    SFMM_CHECK_LAUNCH();
    SFMM_CUDA(cudaEventRecord(pl.ev[5], st));
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
    SFMM_CUDA(cudaEventElapsedTime(&v, pl.ev[3], pl.ev[4]));
    ms6[3] = v;
    SFMM_CUDA(cudaEventElapsedTime(&v, pl.ev[0], pl.ev[5]));
    ms6[4] = v;
    ms6[5] = pl.tree->build_ms;
}

}  // namespace sfmm
