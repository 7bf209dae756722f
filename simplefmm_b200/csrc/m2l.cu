// M2L (fmm.hpp:592-712) for the FP64 path: rotation-based, with the potential
// local (order p) and the field local (order p + 1, source orders <= p - 1)
// produced from one rotation and one z-translation per pair.
//
// Kernels: k_m2l_mma (FP64 tensor cores, below) is the path for p >= 2;
// k_m2l_tf32 the mixed-precision one for p >= 11; k_m2l_rows (this header)
// runs p < 2 and any plan whose DMMA kernel does not fit the device, and a
// plan created with SFMM_M2L_KERNEL=rows in the environment (a test switch).
//
// Work decomposition.  One block per sibling group: the children of one node
// (<= 8 targets at level l >= 2).  Their interaction lists are contiguous and
// share most sources.  The group's pairs are stably sorted by rotation class
// (rot_class, fmm.hpp:492-496) and cut into batches of <= kCB columns
// (column = pair x charge component) of one class.
//
// Row ownership.  Thread r owns coefficient row r of the order-(p+1)
// triangle (r = n(n+1)/2 + m).  It keeps in registers its row of every
// operator it applies: the forward rotation rows P/Q (order n, row m), the
// z-translation row (target order n, azimuth m), and the inverse rotation
// rows PB/QB.  The translation row never changes; the rotation rows are
// reloaded only when the batch's rotation class changes.  Batch vectors move
// through small shared buffers:
//   (a) X = e^{i m phi} M_src                       thread r writes X[r]
//   (b) W_n = (P_n Re X_n, Q_n Im X_n) rho^{-n}      reads X of its order
//   (c) LzB_j^k = rho^{-(j+1)} sum_{n<p} tz W_n^k, LzA adds the n = p term
//   (d) L_j^m += e^{-i m phi} (PB Re Lz_j, QB Im Lz_j), for A and B
// In (d) the thread owns output coefficient r of every target of the group,
// so it accumulates without conflicts in a fixed order: deterministic.
// The kernel is instantiated per order p so the register rows are indexed
// statically.
#include "eval_util.cuh"

#include <type_traits>
#include "fmm_tables.h"

namespace sfmm {
namespace {

constexpr int kCB = 4;                    // columns per batch
constexpr int kMaxGroupPairs = 8 * 189;   // <= 8 siblings x n_ilist_max (partition.hpp:149)
constexpr int kNumClasses = 70;           // fmm.hpp:169
constexpr int kTf32MinOrder = 11;         // lowest order at which mixed plans use the TF32 M2L

template<int P>
struct RowCfg {
    static constexpr int T = (P + 1) * (P + 2) / 2;
    static constexpr int T1 = (P + 2) * (P + 3) / 2;
    static constexpr int NT = (T1 + 31) / 32 * 32;
};

struct M2LSmem {
    int ent_src, ent_code, sorted, cls, cls_cnt, cls_off, bat_off, X, W, LzA, LzB, accA, accB, total;
};

__host__ __device__ constexpr int al16(int x) { return (x + 15) & ~15; }

__host__ __device__ inline M2LSmem m2l_smem(int T, int T1, int qd)
{
    M2LSmem s;
    int o = 0;
    s.ent_src = o; o = al16(o + 4 * kMaxGroupPairs);
    s.ent_code = o; o = al16(o + 4 * kMaxGroupPairs);
    s.sorted = o; o = al16(o + 2 * kMaxGroupPairs);
    s.cls = o; o = al16(o + kMaxGroupPairs);
    s.cls_cnt = o; o = al16(o + 4 * 72);
    s.cls_off = o; o = al16(o + 4 * 72);
    s.bat_off = o; o = al16(o + 4 * 72);
    s.X = o; o = al16(o + 16 * kCB * T);
    s.W = o; o = al16(o + 16 * kCB * T);
    s.LzA = o; o = al16(o + 16 * kCB * T);
    s.LzB = o; o = al16(o + 16 * kCB * T1);
    s.accA = o; o = al16(o + 16 * 8 * qd * T);
    s.accB = o; o = al16(o + 16 * 8 * qd * T1);
    s.total = o;
    return s;
}

template<int P>
__global__ void __launch_bounds__(RowCfg<P>::NT) k_m2l_rows(EvalArgs a, int64_t g0, int64_t g1)
{
    constexpr int T = RowCfg<P>::T, T1 = RowCfg<P>::T1;
    extern __shared__ __align__(16) unsigned char sm[];
    const int qd = a.qdim;
    const M2LSmem L = m2l_smem(T, T1, qd);
    int* ent_src = reinterpret_cast<int*>(sm + L.ent_src);
    int* ent_code = reinterpret_cast<int*>(sm + L.ent_code);
    short* sorted = reinterpret_cast<short*>(sm + L.sorted);
    unsigned char* cls = sm + L.cls;
    int* cls_cnt = reinterpret_cast<int*>(sm + L.cls_cnt);
    int* cls_off = reinterpret_cast<int*>(sm + L.cls_off);
    int* bat_off = reinterpret_cast<int*>(sm + L.bat_off);
    cplx* X = reinterpret_cast<cplx*>(sm + L.X);
    cplx* W = reinterpret_cast<cplx*>(sm + L.W);
    cplx* LzA = reinterpret_cast<cplx*>(sm + L.LzA);
    cplx* LzB = reinterpret_cast<cplx*>(sm + L.LzB);
    cplx* accA = reinterpret_cast<cplx*>(sm + L.accA);
    cplx* accB = reinterpret_cast<cplx*>(sm + L.accB);

    const int r = threadIdx.x;
    const int nt = blockDim.x;
    const bool inB = r < T;               // rotation row (order <= p)
    const bool inD = r < T1;              // translation / inverse rotation row
    int n = 0, m = 0;
    if (inD) tri_nm(r, n, m);
    const int base = n * (n + 1) / 2;
    // warp-uniform loop bounds (rows of a warp are consecutive, orders close)
    int nmaxB = inB ? n : 0, nmaxD = inD ? n : 0, mmin = inD ? m : P + 1;
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        nmaxB = max(nmaxB, __shfl_xor_sync(0xffffffffu, nmaxB, o));
        nmaxD = max(nmaxD, __shfl_xor_sync(0xffffffffu, nmaxD, o));
        mmin = min(mmin, __shfl_xor_sync(0xffffffffu, mmin, o));
    }
    // z-translation row (target order n, azimuth m): sources n' = m .. p
    double tz[P + 1];
    {
        const int wd = P + 1 - m;
        const double* row = a.tzx + a.tzx_off[m] + (n - m) * (wd > 0 ? wd : 0);
#pragma unroll
        for (int i = 0; i <= P; ++i) tz[i] = (inD && i < wd) ? __ldg(row + i) : 0.0;
    }
    double Pr[P + 1], Qr[P + 1], PBr[P + 2], QBr[P + 2];
    int cls_b = -1, cls_d = -1;

    for (int64_t g = g0 + blockIdx.x; g < g1; g += gridDim.x) {
        const int nc = a.nchild[g];
        if (nc == 0) continue;
        const int cb = a.child_beg[g];
        const int lt = level_of(a, g) + 1;                      // level of the targets
        const int e0 = a.il_ptr[cb], E = a.il_ptr[cb + nc] - e0;
        for (int s = 0; s < nc; ++s) {
            const int q0 = a.il_ptr[cb + s] - e0, q1 = a.il_ptr[cb + s + 1] - e0;
            for (int e = q0 + r; e < q1; e += nt) {
                const int code = a.il_code[e0 + e];
                ent_src[e] = a.il_src[e0 + e];
                ent_code[e] = code | (s << 9);
                cls[e] = static_cast<unsigned char>(rot_class((code & 7) - 3, ((code >> 3) & 7) - 3, ((code >> 6) & 7) - 3));
            }
        }
        for (int t = r; t < 8 * qd * T; t += nt) accA[t] = cplx{0, 0};
        for (int t = r; t < 8 * qd * T1; t += nt) accB[t] = cplx{0, 0};
        __syncthreads();
        // stable counting sort by class (thread c gathers class c in order)
        for (int cl = r; cl < kNumClasses; cl += nt) {    // blocks may be narrower than 70 threads
            int cnt = 0;
            for (int e = 0; e < E; ++e) cnt += cls[e] == cl;
            cls_cnt[cl] = cnt;
        }
        __syncthreads();
        if (r == 0) {
            int s = 0, k = 0;
            for (int c = 0; c < kNumClasses; ++c) {
                cls_off[c] = s;
                bat_off[c] = k;
                s += cls_cnt[c];
                k += (cls_cnt[c] * qd + kCB - 1) / kCB;
            }
            cls_off[kNumClasses] = s;
            bat_off[kNumClasses] = k;
        }
        __syncthreads();
        for (int cl = r; cl < kNumClasses; cl += nt) {
            int pos = cls_off[cl];
            for (int e = 0; e < E; ++e)
                if (cls[e] == cl) sorted[pos++] = static_cast<short>(e);
        }
        __syncthreads();
        const int nbat = bat_off[kNumClasses];
        int c = 0;
        for (int bi = 0; bi < nbat; ++bi) {
            while (bat_off[c + 1] <= bi) ++c;
            const int col0 = (bi - bat_off[c]) * kCB;
            const int ncol = min(kCB, cls_cnt[c] * qd - col0);
            int src[kCB], bq[kCB], slot[kCB], pidx[kCB];
            int dsq = 0;
#pragma unroll
            for (int cc = 0; cc < kCB; ++cc) {
                src[cc] = 0;
                bq[cc] = 0;
                slot[cc] = 0;
                pidx[cc] = 24;
                if (cc < ncol) {
                    const int col = col0 + cc;
                    const int e = sorted[cls_off[c] + col / qd];
                    const int code = ent_code[e];
                    const int di = (code & 7) - 3, dj = ((code >> 3) & 7) - 3, dk = ((code >> 6) & 7) - 3;
                    src[cc] = ent_src[e];
                    bq[cc] = col - (col / qd) * qd;
                    slot[cc] = (code >> 9) & 7;
                    pidx[cc] = 7 * (dj + 3) + (di + 3);
                    dsq = di * di + dj * dj + dk * dk;
                }
            }
            const double* R = a.rot + int64_t(c) * a.rot_len;
            const double* ipw = a.ipow + (int64_t(lt) * 28 + dsq) * a.ipow_w;
            cplx ph[kCB];
#pragma unroll
            for (int cc = 0; cc < kCB; ++cc) {
                const double2 e = __ldg(reinterpret_cast<const double2*>(a.eil) + pidx[cc] * (P + 2) + (inD ? m : 0));
                ph[cc] = cplx{e.x, e.y};
            }
            // (a) X = e^{i m phi} M
            if (inB) {
#pragma unroll
                for (int cc = 0; cc < kCB; ++cc)
                    if (cc < ncol) {
                        const double2 v = __ldg(reinterpret_cast<const double2*>(a.M) + (int64_t(src[cc]) * qd + bq[cc]) * T + r);
                        X[cc * T + r] = cmul(ph[cc], cplx{v.x, v.y});
                    }
            }
            __syncthreads();
            // (b) forward rotation of order n, row m
            if (inB) {
                if (c != cls_b) {
                    const double* Pp = R + a.rot_off[n] + m * (n + 1);
                    const double* Qp = Pp + (n + 1) * (n + 1);
#pragma unroll
                    for (int b = 0; b <= P; ++b) {
                        Pr[b] = b <= n ? __ldg(Pp + b) : 0.0;
                        Qr[b] = b <= n ? __ldg(Qp + b) : 0.0;
                    }
                    cls_b = c;
                }
                double re[kCB], im[kCB];
#pragma unroll
                for (int cc = 0; cc < kCB; ++cc) re[cc] = im[cc] = 0;
#pragma unroll
                for (int b = 0; b <= P; ++b) {
                    if (b > nmaxB) break;
                    if (b <= n) {
#pragma unroll
                        for (int cc = 0; cc < kCB; ++cc)
                            if (cc < ncol) {
                                const cplx x = X[cc * T + base + b];
                                re[cc] = fma(Pr[b], x.re, re[cc]);
                                im[cc] = fma(Qr[b], x.im, im[cc]);
                            }
                    }
                }
                const double sc = n ? ipw[n - 1] : 1.0;
#pragma unroll
                for (int cc = 0; cc < kCB; ++cc)
                    if (cc < ncol) W[cc * T + r] = cplx{re[cc] * sc, im[cc] * sc};
            }
            __syncthreads();
            // (c) z-translation: target order j = n, azimuth k = m
            if (inD) {
                double bre[kCB], bim[kCB], xre[kCB], xim[kCB];
#pragma unroll
                for (int cc = 0; cc < kCB; ++cc) bre[cc] = bim[cc] = xre[cc] = xim[cc] = 0;
#pragma unroll
                for (int i = 0; i <= P; ++i) {
                    if (i > P - mmin) break;
                    if (i <= P - m) {
                        const int np = m + i;
                        const int tn = np * (np + 1) / 2 + m;
#pragma unroll
                        for (int cc = 0; cc < kCB; ++cc)
                            if (cc < ncol) {
                                const cplx y = W[cc * T + tn];
                                if (i < P - m) {
                                    bre[cc] = fma(tz[i], y.re, bre[cc]);
                                    bim[cc] = fma(tz[i], y.im, bim[cc]);
                                } else {
                                    xre[cc] = tz[i] * y.re;
                                    xim[cc] = tz[i] * y.im;
                                }
                            }
                    }
                }
                const double sc = ipw[n];
#pragma unroll
                for (int cc = 0; cc < kCB; ++cc)
                    if (cc < ncol) {
                        LzB[cc * T1 + r] = cplx{bre[cc] * sc, bim[cc] * sc};
                        if (n <= P) LzA[cc * T + r] = cplx{(bre[cc] + xre[cc]) * sc, (bim[cc] + xim[cc]) * sc};
                    }
            }
            __syncthreads();
            // (d) inverse rotation (order j = n, row m) + phase, accumulate
            if (inD) {
                if (c != cls_d) {
                    const int wd = (n + 1) * (n + 1);
                    const double* PBp = R + a.rot_off[n] + 2 * wd + m * (n + 1);
                    const double* QBp = PBp + wd;
#pragma unroll
                    for (int b = 0; b <= P + 1; ++b) {
                        PBr[b] = b <= n ? __ldg(PBp + b) : 0.0;
                        QBr[b] = b <= n ? __ldg(QBp + b) : 0.0;
                    }
                    cls_d = c;
                }
                const bool doA = a.want_pot && n <= P;
                const bool doB = a.want_field;
                double are[kCB], aim[kCB], bre[kCB], bim[kCB];
#pragma unroll
                for (int cc = 0; cc < kCB; ++cc) are[cc] = aim[cc] = bre[cc] = bim[cc] = 0;
#pragma unroll
                for (int b = 0; b <= P + 1; ++b) {
                    if (b > nmaxD) break;
                    if (b <= n) {
#pragma unroll
                        for (int cc = 0; cc < kCB; ++cc)
                            if (cc < ncol) {
                                if (doB) {
                                    const cplx z = LzB[cc * T1 + base + b];
                                    bre[cc] = fma(PBr[b], z.re, bre[cc]);
                                    bim[cc] = fma(QBr[b], z.im, bim[cc]);
                                }
                                if (doA) {
                                    const cplx x = LzA[cc * T + base + b];
                                    are[cc] = fma(PBr[b], x.re, are[cc]);
                                    aim[cc] = fma(QBr[b], x.im, aim[cc]);
                                }
                            }
                    }
                }
#pragma unroll
                for (int cc = 0; cc < kCB; ++cc)
                    if (cc < ncol) {
                        const cplx e = cconj(ph[cc]);
                        const int sb = slot[cc] * qd + bq[cc];
                        if (doB) {
                            const cplx v = cmul(e, cplx{bre[cc], bim[cc]});
                            accB[sb * T1 + r].re += v.re;
                            accB[sb * T1 + r].im += v.im;
                        }
                        if (doA) {
                            const cplx v = cmul(e, cplx{are[cc], aim[cc]});
                            accA[sb * T + r].re += v.re;
                            accA[sb * T + r].im += v.im;
                        }
                    }
            }
        }
        __syncthreads();
        if (a.want_pot)
            for (int e = r; e < nc * qd * T; e += nt) a.LA[int64_t(cb) * qd * T + e] = accA[e];
        if (a.want_field)
            for (int e = r; e < nc * qd * T1; e += nt) a.LB[int64_t(cb) * qd * T1 + e] = accB[e];
        __syncthreads();
    }
}

template<int P>
void launch_rows_fallback(const EvalArgs& a, int64_t g0, int64_t g1, int sms, cudaStream_t st)
{
    constexpr int T = RowCfg<P>::T, T1 = RowCfg<P>::T1, NT = RowCfg<P>::NT;
    const size_t smem = m2l_smem(T, T1, a.qdim).total;
    allow_max_smem(k_m2l_rows<P>);
    int per_sm = 1;
    SFMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_m2l_rows<P>, NT, smem));
    SFMM_REQUIRE(per_sm > 0, FMM_ERR_UNSUPPORTED, "M2L working set exceeds the device");
    const int64_t groups = g1 - g0;
    const int64_t grid = std::min<int64_t>(std::max<int64_t>(groups, 1), int64_t(sms) * per_sm * 4);
    k_m2l_rows<P><<<static_cast<unsigned>(grid), NT, smem, st>>>(a, g0, g1);
    SFMM_CHECK_LAUNCH();
}


__device__ __forceinline__ void block_barrier() { asm volatile("barrier.sync 0;" ::: "memory"); }

// 16-byte global -> shared copy that completes asynchronously (L2 only);
// the issuing thread waits with cp_async_wait_all before reading it.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem)
{
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ------------------------------------------------------------------ FP64 tensor-core kernel
// The same rotate / translate / rotate-back arithmetic as matrix products on
// the FP64 tensor cores (mma.sync m8n8k4 f64: A 8x4 row-major, B 4x8
// column-major, D 8x8; 256 FMAs per warp instruction with every operand in
// registers).  A tile is up to 8 columns (pair x charge component) of one
// rotation class, the MMA's N.  For a tile:
//   X     = e^{i m phi} M_src                      [coef t][col], re / im apart
//   W_n   = rho^{-n} (P_n Re X_n, Q_n Im X_n)       per order n: A = P_n / Q_n rows
//   LzB^k = rho^{-(j+1)} Tz_k W^k  (sources <= p-1)  per azimuth k: A = Tz_k rows,
//           the same A for the re and im halves
//   LzA^k = LzB^k + rho^{-(j+1)} tz[j][p] W_p^k      (rows j <= p)
//   L_j   = e^{-i m phi} (PB_j Re Lz_j, QB_j Im Lz_j)   for LzA and LzB
// then the tile's columns are added into their target in column order
// (deterministic).  Operators come from tables in fragment order (one
// coalesced 256-byte load per fragment, L1/L2 resident).  Zero-padded
// operator rows and columns make out-of-range operand rows contribute
// nothing; those rows are kept finite.  Four block barriers per tile; two
// blocks per SM overlap each other's barriers; the next tile's source
// moments are copied with cp.async two phases ahead.

__host__ __device__ constexpr int mma_rt(int n) { return (n + 8) / 8; }   // 8-row tiles of order n
__host__ __device__ constexpr int mma_kc(int n) { return (n + 4) / 4; }   // 4-wide K chunks of order n
__host__ __device__ constexpr int mma_foff(int n)                         // fragments of orders < n
{
    int s = 0;
    for (int i = 0; i < n; ++i) s += mma_rt(i) * mma_kc(i);
    return s;
}
// z-translation for azimuth k: rows j = k..P+1, field-local sources n' = k..P-1
__host__ __device__ constexpr int tz_rt(int P, int k) { return (P + 2 - k + 7) / 8; }
__host__ __device__ constexpr int tz_kc(int P, int k) { return k < P ? (P - k + 3) / 4 : 0; }
__host__ __device__ constexpr int tz_foff(int P, int k)
{
    int s = 0;
    for (int i = 0; i < k; ++i) s += tz_rt(P, i) * tz_kc(P, i);
    return s;
}
// first row of azimuth k in the azimuth-major layout of W (n' = k..P)
__host__ __device__ constexpr int az_off(int P, int k) { return k * (P + 1) - k * (k - 1) / 2; }

__device__ __forceinline__ void mma884(double& d0, double& d1, double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

struct MmaMeta {
    int cls, ncol, dsq, pad;
    int src[8], bq[8], sb[8], pidx[8];
};

// column table of a tile of C columns
template<int C>
struct MetaC {
    int cls, ncol, dsq, pad;
    int src[C], bq[C], sb[C], pidx[C];
};

// Compile-time loop: f(std::integral_constant<int, I>) for I in [B, E).
template<int B, int E, typename F>
__device__ __forceinline__ void static_for(F&& f)
{
    if constexpr (B < E) {
        f(std::integral_constant<int, B>{});
        static_for<B + 1, E>(f);
    }
}

// Runs f(std::integral_constant<int, W>) for the calling warp's index W, so
// that a stage's job list is filtered at compile time (each job's code sits
// in the branch of the one warp that runs it).
template<int NW, typename F>
__device__ __forceinline__ void for_warp(int warp, F&& f)
{
    static_for<0, NW>([&](auto ww) {
        if (warp == decltype(ww)::value) f(ww);
    });
}

// padded leading dimension of a [col][row] operand buffer: >= rows + 4 (K
// chunks read up to 3 rows past an order) and = 4 or 12 mod 16 doubles, which
// makes the B-fragment loads (4 rows x 8 columns) bank-conflict free
__host__ __device__ constexpr int mma_ld(int rows)
{
    int ld = rows + 4;
    while (ld % 16 != 4 && ld % 16 != 12) ++ld;
    return ld;
}
// rotation jobs (n, rt), n = P..0: index of the first job of order n
__host__ __device__ constexpr int rot_job0(int P, int n)
{
    int s = 0;
    for (int i = P; i > n; --i) s += mma_rt(i);
    return s;
}
// translation jobs (k, rt), k = 0..P+1: index of the first job of azimuth k
__host__ __device__ constexpr int tz_job0(int P, int k)
{
    int s = 0;
    for (int i = 0; i < k; ++i) s += tz_rt(P, i);
    return s;
}

// Inverse-rotation jobs, orders j = P+1..0: the two locals of a large order
// (LA, LB; RT x KC >= 4 fragments) are separate jobs, a small order is one
// job for both; order P + 1 has only LB.  part: 0 = LA and LB, 1 = LA, 2 = LB.
__host__ __device__ constexpr bool inv_split(int P, int j) { return j <= P && mma_rt(j) * mma_kc(j) >= 4; }
__host__ __device__ constexpr int inv_njobs(int P)
{
    int s = 0;
    for (int j = P + 1; j >= 0; --j) s += inv_split(P, j) ? 2 : 1;
    return s;
}
__host__ __device__ constexpr int inv_job_j(int P, int i)
{
    for (int j = P + 1; j >= 0; --j) {
        const int c = inv_split(P, j) ? 2 : 1;
        if (i < c) return j;
        i -= c;
    }
    return 0;
}
__host__ __device__ constexpr int inv_job_part(int P, int i)
{
    for (int j = P + 1; j >= 0; --j) {
        const int c = inv_split(P, j) ? 2 : 1;
        if (i < c) return c == 2 ? 1 + i : (j <= P ? 0 : 2);
        i -= c;
    }
    return 0;
}
// MMA count of job i of a phase (0: rotation jobs (n, rt), n = P..0;
// 1: translation jobs (k, rt), k = 0..P+1; 2: inverse-rotation jobs)
__host__ __device__ constexpr int job_cost(int P, int phase, int i)
{
    if (phase == 0) {
        for (int n = P; n >= 0; --n) {
            if (i < mma_rt(n)) return 2 * mma_kc(n);
            i -= mma_rt(n);
        }
        return 0;
    }
    if (phase == 1) {
        for (int k = 0; k <= P + 1; ++k) {
            if (i < tz_rt(P, k)) return tz_kc(P, k) > 0 ? 2 * tz_kc(P, k) : 1;
            i -= tz_rt(P, k);
        }
        return 0;
    }
    const int j = inv_job_j(P, i);
    return mma_rt(j) * mma_kc(j) * (inv_job_part(P, i) == 0 ? 4 : 2);
}
// Warp of job i: jobs taken in order, each by the least-loaded warp (the
// orders come largest first, so this is the longest-processing-time rule).
__host__ __device__ constexpr int job_warp(int P, int NW, int phase, int i)
{
    int load[32] = {};
    int w = 0;
    for (int k = 0; k <= i; ++k) {
        w = 0;
        for (int u = 1; u < NW; ++u)
            if (load[u] < load[w]) w = u;
        load[w] += job_cost(P, phase, k);
    }
    return w;
}

// LEAN: no staging buffer for the moments (the phase-in reads them from
// global memory) and the potential local's buffer shares X's (X is dead after
// the rotation; one more barrier between accumulation and the next phase-in),
// for four blocks per SM where that fits.
template<int P, int NS, bool LEAN = false>
struct MmaLayout {
    static constexpr int NC = 8 * NS;                           // columns per tile (NS MMA N-tiles)
    static constexpr int T = (P + 1) * (P + 2) / 2;
    static constexpr int T1 = (P + 2) * (P + 3) / 2;
    static constexpr int LD = mma_ld(T), LD1 = mma_ld(T1);        // column strides (doubles)
    static constexpr int kids = 0;                                 // ilist offsets of the 8 children
    static constexpr int sorted = al16(kids + 4 * 9);
    static constexpr int cls = al16(sorted + 2 * kMaxGroupPairs);
    static constexpr int cls_cnt = al16(cls + kMaxGroupPairs);
    static constexpr int cls_off = al16(cls_cnt + 4 * 72);
    static constexpr int bat_off = al16(cls_off + 4 * 72);
    static constexpr int meta = al16(bat_off + 4 * 72);
    static constexpr int tm = al16(meta + int(sizeof(MetaC<NC>)) * 3);
    static constexpr int Xraw = al16(tm + T1);                    // [col][T] complex (cp.async)
    static constexpr int X = LEAN ? Xraw : al16(Xraw + NC * T * 16); // re, im: [col][LD] doubles each
    static constexpr int W = al16(X + 2 * NC * LD * 8);             // azimuth-major rows
    static constexpr int LzA = LEAN ? X : al16(W + 2 * NC * LD * 8);
    static constexpr int LzB = LEAN ? al16(W + 2 * NC * LD * 8) : al16(LzA + 2 * NC * LD * 8);   // [col][LD1]
    static constexpr int acc = al16(LzB + 2 * NC * LD1 * 8);        // [8 qd][T] then [8 qd][T1] complex
    __host__ __device__ static constexpr int total(int qd) { return al16(acc + 16 * 8 * qd * (T + T1)); }
};

template<int P, int NS, int NW, bool LEAN>
__global__ void __launch_bounds__(32 * NW, NW <= 8 ? (LEAN ? 4 : 3) : 1) k_m2l_mma(EvalArgs a, int64_t g0, int64_t g1)
{
    using L = MmaLayout<P, NS, LEAN>;
    constexpr int T = L::T, T1 = L::T1, LD = L::LD, LD1 = L::LD1, NT = 32 * NW, NC = L::NC;
    using Meta = MetaC<NC>;
    extern __shared__ __align__(16) unsigned char sm[];
    int* kids = reinterpret_cast<int*>(sm + L::kids);
    short* sorted = reinterpret_cast<short*>(sm + L::sorted);
    unsigned char* cls = sm + L::cls;
    int* cls_cnt = reinterpret_cast<int*>(sm + L::cls_cnt);
    int* cls_off = reinterpret_cast<int*>(sm + L::cls_off);
    int* bat_off = reinterpret_cast<int*>(sm + L::bat_off);
    Meta* meta = reinterpret_cast<Meta*>(sm + L::meta);
    unsigned char* tm = sm + L::tm;
    cplx* Xraw = reinterpret_cast<cplx*>(sm + L::Xraw);
    double* Xre = reinterpret_cast<double*>(sm + L::X);
    double* Xim = Xre + NC * LD;
    double* Wre = reinterpret_cast<double*>(sm + L::W);
    double* Wim = Wre + NC * LD;
    double* Are = reinterpret_cast<double*>(sm + L::LzA);
    double* Aim = Are + NC * LD;
    double* Bre = reinterpret_cast<double*>(sm + L::LzB);
    double* Bim = Bre + NC * LD1;
    const int qd = a.qdim;
    cplx* accA = reinterpret_cast<cplx*>(sm + L::acc);
    cplx* accB = accA + 8 * qd * T;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int lr = lane >> 2, lc = lane & 3;                       // fragment row / column group
    // B-fragment element (K row lc, column lr) and D-fragment columns 2 lc + {0, 1}
    const int bofs = lr * LD + lc, bofs1 = lr * LD1 + lc;
    const int d0 = (2 * lc) * LD, d1 = (2 * lc + 1) * LD, e0 = (2 * lc) * LD1, e1 = (2 * lc + 1) * LD1;
    // operand buffers start at zero: padding rows and unused columns must be finite
    for (int e = tid; e < (L::acc - L::X) / 8; e += NT) Xre[e] = 0.0;
    for (int t = tid; t < T1; t += NT) {
        int n, m;
        tri_nm(t, n, m);
        tm[t] = static_cast<unsigned char>(m);
    }
    __syncthreads();
    const double* rf = a.rfrag;
    const int NF = a.rfrag_nf;

    // column table of tile b (threads k < 8); c: class cursor
    auto make_meta = [&](int b, int k, Meta& M, int& c) {
        while (bat_off[c + 1] <= b) ++c;
        const int col0 = (b - bat_off[c]) * NC;
        const int ncol = min(NC, cls_cnt[c] * qd - col0);
        if (k < ncol) {
            const int col = col0 + k;
            const int pair = col / qd;
            const int e = sorted[cls_off[c] + pair];
            const int code = a.il_code[kids[0] + e];
            const int di = (code & 7) - 3, dj = ((code >> 3) & 7) - 3, dk = ((code >> 6) & 7) - 3;
            const int bq = col - pair * qd;
            int slot = 0;
            while (kids[slot + 1] - kids[0] <= e) ++slot;
            M.src[k] = a.il_src[kids[0] + e];
            M.bq[k] = bq;
            M.sb[k] = slot * qd + bq;
            M.pidx[k] = 7 * (dj + 3) + (di + 3);
            if (k == 0) {
                M.cls = c;
                M.ncol = ncol;
                M.dsq = di * di + dj * dj + dk * dk;
            }
        } else {
            M.src[k] = 0;
            M.bq[k] = 0;
            M.sb[k] = 0;
            M.pidx[k] = 24;
        }
    };
    // raw source moments of tile b -> Xraw[b & 1] (asynchronous)
    auto issue = [&](int b) {
        if constexpr (LEAN) return;
        const Meta& M = meta[b % 3];
        const int ncol = M.ncol;
        cplx* xr = Xraw;
        for (int e = tid; e < NC * T; e += NT) {
            const int c = e / T, t = e - c * T;
            if (c < ncol) cp_async16(xr + e, a.M + (int64_t(M.src[c]) * qd + M.bq[c]) * T + t);
        }
        cp_async_commit();
    };
    // X = e^{i m phi} M for tile b, column-major: a warp per column, lanes
    // over its coefficients
    auto phase_in = [&](int b) {
        const Meta& M = meta[b % 3];
        const int ncol = M.ncol;
        for (int c = warp; c < ncol; c += NW) {
            const double2* ph = reinterpret_cast<const double2*>(a.eil) + M.pidx[c] * (P + 2);
            const cplx* src = LEAN ? a.M + (int64_t(M.src[c]) * qd + M.bq[c]) * T : Xraw + c * T;
            for (int t = lane; t < T; t += 32) {
                const double2 f = __ldg(ph + tm[t]);
                const cplx v = cmul(cplx{f.x, f.y}, src[t]);
                Xre[c * LD + t] = v.re;
                Xim[c * LD + t] = v.im;
            }
        }
    };

    // blocks take sibling groups from a counter (group costs vary with the
    // children's interaction lists; the resident blocks stay busy to the end)
    __shared__ int64_t next_group;
    auto take = [&]() -> int64_t {
        if (tid == 0) next_group = g0 + atomicAdd(a.m2l_ctr, 1);
        __syncthreads();
        const int64_t g = next_group;
        __syncthreads();
        return g;
    };
    for (int64_t g = take(); g < g1; g = take()) {
        const int nc = a.nchild[g];
        if (nc == 0) continue;
        const int cb = a.child_beg[g];
        const int lt = level_of(a, g) + 1;
        // ---- group set-up: gather, stable class sort, tiles
        {
            const int e0 = a.il_ptr[cb], E = a.il_ptr[cb + nc] - e0;
            for (int e = tid; e < E; e += NT) {
                const int code = a.il_code[e0 + e];
                cls[e] = static_cast<unsigned char>(rot_class((code & 7) - 3, ((code >> 3) & 7) - 3, ((code >> 6) & 7) - 3));
            }
            if (tid <= 8) kids[tid] = a.il_ptr[cb + min(tid, nc)];
            for (int t = tid; t < 8 * qd * (T + T1); t += NT) accA[t] = cplx{0, 0};
            __syncthreads();
            for (int cl = tid; cl < kNumClasses; cl += NT) {
                int cnt = 0;
                for (int e = 0; e < E; ++e) cnt += cls[e] == cl;
                cls_cnt[cl] = cnt;
            }
            __syncthreads();
            if (tid == 0) {
                int s = 0, k = 0;
                for (int c = 0; c < kNumClasses; ++c) {
                    cls_off[c] = s;
                    bat_off[c] = k;
                    s += cls_cnt[c];
                    k += (cls_cnt[c] * qd + NC - 1) / NC;
                }
                cls_off[kNumClasses] = s;
                bat_off[kNumClasses] = k;
            }
            __syncthreads();
            for (int cl = tid; cl < kNumClasses; cl += NT) {
                int pos = cls_off[cl];
                for (int e = 0; e < E; ++e)
                    if (cls[e] == cl) sorted[pos++] = static_cast<short>(e);
            }
            __syncthreads();
        }
        const int nbat = bat_off[kNumClasses];
        int cur = 0;                                      // class cursor of threads < 8
        if (tid < NC && nbat > 0) make_meta(0, tid, meta[0], cur);
        __syncthreads();
        if (nbat > 0) issue(0);
        if (tid < NC && nbat > 1) make_meta(1, tid, meta[1], cur);
        cp_async_wait_all();
        __syncthreads();
        if (nbat > 0) phase_in(0);
        __syncthreads();

        for (int b = 0; b < nbat; ++b) {
            const Meta& M = meta[b % 3];
            const double* ipw = a.ipow + (int64_t(lt) * 28 + M.dsq) * a.ipow_w;
            const double* rfc = rf + int64_t(M.cls) * NF * 4 * 32 + lane;
            // tile b + 1's moments: the staging buffer is free since phase_in(b)
            if (b + 1 < nbat) issue(b + 1);
            // ---- rotation: jobs (n, rt), largest orders first, round robin over warps
            for_warp<NW>(warp, [&](auto ww) {
            constexpr int W = decltype(ww)::value;
            static_for<0, P + 1>([&](auto nn) {
                constexpr int n = P - decltype(nn)::value;
                constexpr int KC = mma_kc(n), base = n * (n + 1) / 2;
                static_for<0, mma_rt(n)>([&](auto rr) {
                    constexpr int rt = decltype(rr)::value;
                    constexpr int jw = job_warp(P, NW, 0, rot_job0(P, n) + rt);
                    if (jw != W) return;
                    const double* fr = rfc + (mma_foff(n) + rt * KC) * 4 * 32;
                    double aP[KC], aQ[KC];
#pragma unroll
                    for (int kc = 0; kc < KC; ++kc) {
                        aP[kc] = __ldg(fr + (kc * 4 + 0) * 32);
                        aQ[kc] = __ldg(fr + (kc * 4 + 1) * 32);
                    }
                    double r0[NS] = {}, r1[NS] = {}, i0[NS] = {}, i1[NS] = {};
#pragma unroll
                    for (int kc = 0; kc < KC; ++kc)
#pragma unroll
                        for (int q = 0; q < NS; ++q) {
                            mma884(r0[q], r1[q], aP[kc], Xre[bofs + q * 8 * LD + base + 4 * kc]);
                            mma884(i0[q], i1[q], aQ[kc], Xim[bofs + q * 8 * LD + base + 4 * kc]);
                        }
                    const int m = 8 * rt + lr;
                    if (m <= n) {
                        const double sc = n ? ipw[n - 1] : 1.0;
                        const int u = az_off(P, m) + (n - m);
#pragma unroll
                        for (int q = 0; q < NS; ++q) {
                            Wre[d0 + q * 8 * LD + u] = r0[q] * sc;
                            Wre[d1 + q * 8 * LD + u] = r1[q] * sc;
                            Wim[d0 + q * 8 * LD + u] = i0[q] * sc;
                            Wim[d1 + q * 8 * LD + u] = i1[q] * sc;
                        }
                    }
                });
            });
            });
            __syncthreads();
            // ---- z-translation: jobs (k, rt); the same operator for re and im
            for_warp<NW>(warp, [&](auto ww) {
            constexpr int W = decltype(ww)::value;
            static_for<0, P + 2>([&](auto kk) {
                constexpr int k = decltype(kk)::value;
                constexpr int KC = tz_kc(P, k), u0 = az_off(P, k);
                static_for<0, tz_rt(P, k)>([&](auto rr) {
                    constexpr int rt = decltype(rr)::value;
                    constexpr int jw = job_warp(P, NW, 1, tz_job0(P, k) + rt);
                    if (jw != W) return;
                    const double* fz = a.tzfrag + (tz_foff(P, k) + rt * KC) * 32 + lane;
                    double az[KC > 0 ? KC : 1];
#pragma unroll
                    for (int kc = 0; kc < KC; ++kc) az[kc] = __ldg(fz + kc * 32);
                    double r0[NS] = {}, r1[NS] = {}, i0[NS] = {}, i1[NS] = {};
#pragma unroll
                    for (int kc = 0; kc < KC; ++kc)
#pragma unroll
                        for (int q = 0; q < NS; ++q) {
                            mma884(r0[q], r1[q], az[kc], Wre[bofs + q * 8 * LD + u0 + 4 * kc]);
                            mma884(i0[q], i1[q], az[kc], Wim[bofs + q * 8 * LD + u0 + 4 * kc]);
                        }
                    const int j = k + 8 * rt + lr;
                    if (j <= P + 1) {
                        const double sc = ipw[j];
                        const int t1 = j * (j + 1) / 2 + k;
#pragma unroll
                        for (int q = 0; q < NS; ++q) {
                            Bre[e0 + q * 8 * LD1 + t1] = r0[q] * sc;
                            Bre[e1 + q * 8 * LD1 + t1] = r1[q] * sc;
                            Bim[e0 + q * 8 * LD1 + t1] = i0[q] * sc;
                            Bim[e1 + q * 8 * LD1 + t1] = i1[q] * sc;
                        }
                        if constexpr (k <= P) {
                            if (j <= P) {
                                const double tl = a.tzl[k * (P + 2) + j];
                                constexpr int up = u0 + (P - k);          // n' = p
#pragma unroll
                                for (int q = 0; q < NS; ++q) {
                                    const int o0 = d0 + q * 8 * LD, o1 = d1 + q * 8 * LD;
                                    Are[o0 + t1] = fma(tl, Wre[o0 + up], r0[q]) * sc;
                                    Are[o1 + t1] = fma(tl, Wre[o1 + up], r1[q]) * sc;
                                    Aim[o0 + t1] = fma(tl, Wim[o0 + up], i0[q]) * sc;
                                    Aim[o1 + t1] = fma(tl, Wim[o1 + up], i1[q]) * sc;
                                }
                            }
                        }
                    }
                });
            });
            });
            // column table of tile b + 2 (its ring slot is free)
            if (tid < NC && b + 2 < nbat) make_meta(b + 2, tid, meta[(b + 2) % 3], cur);
            __syncthreads();
            // ---- inverse rotation + phase, in place: jobs (order j, local) take all rows of the order
            {
                int pc0[NS], pc1[NS];
#pragma unroll
                for (int q = 0; q < NS; ++q) {
                    pc0[q] = M.pidx[8 * q + 2 * lc] * (P + 2);
                    pc1[q] = M.pidx[8 * q + 2 * lc + 1] * (P + 2);
                }
                for_warp<NW>(warp, [&](auto ww) {
                constexpr int W = decltype(ww)::value;
                static_for<0, inv_njobs(P)>([&](auto jj) {
                    constexpr int job = decltype(jj)::value;
                    constexpr int j = inv_job_j(P, job), part = inv_job_part(P, job);
                    constexpr int jw = job_warp(P, NW, 2, job);
                    if (jw != W) return;
                    constexpr int KC = mma_kc(j), RT = mma_rt(j), base = j * (j + 1) / 2;
                    constexpr bool hasA = j <= P && part != 2, hasB = part != 1;
                    const double* fr = rfc + mma_foff(j) * 4 * 32;
                    double ar[RT][NS][2] = {}, ai[RT][NS][2] = {}, br[RT][NS][2] = {}, bi[RT][NS][2] = {};
#pragma unroll
                    for (int rt = 0; rt < RT; ++rt) {
                        double aPB[KC], aQB[KC];
#pragma unroll
                        for (int kc = 0; kc < KC; ++kc) {
                            aPB[kc] = __ldg(fr + ((rt * KC + kc) * 4 + 2) * 32);
                            aQB[kc] = __ldg(fr + ((rt * KC + kc) * 4 + 3) * 32);
                        }
#pragma unroll
                        for (int kc = 0; kc < KC; ++kc)
#pragma unroll
                            for (int q = 0; q < NS; ++q) {
                                if constexpr (hasB) {
                                    mma884(br[rt][q][0], br[rt][q][1], aPB[kc], Bre[bofs1 + q * 8 * LD1 + base + 4 * kc]);
                                    mma884(bi[rt][q][0], bi[rt][q][1], aQB[kc], Bim[bofs1 + q * 8 * LD1 + base + 4 * kc]);
                                }
                                if constexpr (hasA) {
                                    mma884(ar[rt][q][0], ar[rt][q][1], aPB[kc], Are[bofs + q * 8 * LD + base + 4 * kc]);
                                    mma884(ai[rt][q][0], ai[rt][q][1], aQB[kc], Aim[bofs + q * 8 * LD + base + 4 * kc]);
                                }
                            }
                    }
                    __syncwarp();
#pragma unroll
                    for (int rt = 0; rt < RT; ++rt) {
                        const int m = 8 * rt + lr;
                        if (m > j) continue;
                        const int t = base + m;
#pragma unroll
                        for (int q = 0; q < NS; ++q) {
                            const double2 f0 = __ldg(reinterpret_cast<const double2*>(a.eil) + pc0[q] + m);
                            const double2 f1 = __ldg(reinterpret_cast<const double2*>(a.eil) + pc1[q] + m);
                            if constexpr (hasB) {
                                const int b0 = e0 + q * 8 * LD1 + t, b1 = e1 + q * 8 * LD1 + t;
                                Bre[b0] = f0.x * br[rt][q][0] + f0.y * bi[rt][q][0];
                                Bim[b0] = f0.x * bi[rt][q][0] - f0.y * br[rt][q][0];
                                Bre[b1] = f1.x * br[rt][q][1] + f1.y * bi[rt][q][1];
                                Bim[b1] = f1.x * bi[rt][q][1] - f1.y * br[rt][q][1];
                            }
                            if constexpr (hasA) {
                                const int a0 = d0 + q * 8 * LD + t, a1 = d1 + q * 8 * LD + t;
                                Are[a0] = f0.x * ar[rt][q][0] + f0.y * ai[rt][q][0];
                                Aim[a0] = f0.x * ai[rt][q][0] - f0.y * ar[rt][q][0];
                                Are[a1] = f1.x * ar[rt][q][1] + f1.y * ai[rt][q][1];
                                Aim[a1] = f1.x * ai[rt][q][1] - f1.y * ar[rt][q][1];
                            }
                        }
                    }
                });
                });
            }
            cp_async_wait_all();                          // tile b + 1's moments
            __syncthreads();
            // ---- accumulate tile b into the targets (column order); phase tile b + 1 in
            {
                const int ncol = M.ncol;
                int sb[NC];
#pragma unroll
                for (int c = 0; c < NC; ++c) sb[c] = M.sb[c];
                for (int t = tid; t < T + T1; t += NT) {
                    const bool isA = t < T;
                    const int r = isA ? t : t - T;
                    const double* sre = isA ? Are + r : Bre + r;
                    const double* sim = isA ? Aim + r : Bim + r;
                    const int ld = isA ? LD : LD1;
                    cplx* acc = isA ? accA + r : accB + r;
                    const int stride = isA ? T : T1;
#pragma unroll
                    for (int c = 0; c < NC; ++c)
                        if (c < ncol) {
                            cplx& d = acc[sb[c] * stride];
                            d.re += sre[c * ld];
                            d.im += sim[c * ld];
                        }
                }
                if constexpr (LEAN) __syncthreads();          // X shares the potential local's buffer
                if (b + 1 < nbat) phase_in(b + 1);
            }
            __syncthreads();
        }
        if (a.want_pot)
            for (int e = tid; e < nc * qd * T; e += NT) a.LA[int64_t(cb) * qd * T + e] = accA[e];
        if (a.want_field)
            for (int e = tid; e < nc * qd * T1; e += NT) a.LB[int64_t(cb) * qd * T1 + e] = accB[e];
        __syncthreads();
    }
}

template<int P, int NS, int NW, bool LEAN>
bool try_launch_mma(const EvalArgs& a, int64_t g0, int64_t g1, int sms, cudaStream_t st)
{
    const size_t smem = MmaLayout<P, NS, LEAN>::total(a.qdim);
    int dev = 0, optin = 0;
    SFMM_CUDA(cudaGetDevice(&dev));
    SFMM_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa{};
    SFMM_CUDA(cudaFuncGetAttributes(&fa, k_m2l_mma<P, NS, NW, LEAN>));
    if (smem + fa.sharedSizeBytes > size_t(optin)) return false;
    allow_max_smem(k_m2l_mma<P, NS, NW, LEAN>);
    int per_sm = 0;
    SFMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_m2l_mma<P, NS, NW, LEAN>, 32 * NW, smem));
    if (LEAN && per_sm < 4) return false;
    if (per_sm < 1) return false;
    const int64_t grid = std::min<int64_t>(std::max<int64_t>(g1 - g0, 1), int64_t(sms) * per_sm);
    SFMM_CUDA(cudaMemsetAsync(a.m2l_ctr, 0, sizeof(int), st));
    k_m2l_mma<P, NS, NW, LEAN><<<static_cast<unsigned>(grid), 32 * NW, smem, st>>>(a, g0, g1);
    SFMM_CHECK_LAUNCH();
    return true;
}

// Fragment-order tables (device): rotation matrices of every class for
// orders <= P + 1 and the z-translation operator.
__global__ void k_frag_rot(const double* __restrict__ rot, const int* __restrict__ rot_off, int rot_len, int P, int NF,
                           double* __restrict__ out)
{
    const int64_t total = int64_t(kNumClasses) * NF * 4 * 32;
    for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total; idx += int64_t(gridDim.x) * blockDim.x) {
        const int lane = static_cast<int>(idx & 31), mat = static_cast<int>((idx >> 5) & 3);
        const int64_t rest = idx >> 7;
        const int f = static_cast<int>(rest % NF), c = static_cast<int>(rest / NF);
        int n = 0;
        while (n < P + 1 && mma_foff(n + 1) <= f) ++n;
        const int KC = mma_kc(n);
        const int rt = (f - mma_foff(n)) / KC, kc = (f - mma_foff(n)) - rt * KC;
        const int row = 8 * rt + (lane >> 2), col = 4 * kc + (lane & 3);
        double v = 0.0;
        if (row <= n && col <= n)
            v = rot[int64_t(c) * rot_len + rot_off[n] + mat * (n + 1) * (n + 1) + row * (n + 1) + col];
        out[idx] = v;
    }
}

__global__ void k_frag_tz(const double* __restrict__ tzx, const int* __restrict__ tzx_off, int P, int NFZ,
                          double* __restrict__ out, double* __restrict__ tzl)
{
    const int total = NFZ * 32;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
        const int lane = idx & 31, f = idx >> 5;
        int k = 0;
        while (k < P + 1 && tz_foff(P, k + 1) <= f) ++k;
        const int KC = tz_kc(P, k);
        const int rt = (f - tz_foff(P, k)) / KC, kc = (f - tz_foff(P, k)) - rt * KC;
        const int j = k + 8 * rt + (lane >> 2), np = k + 4 * kc + (lane & 3);
        double v = 0.0;
        if (j <= P + 1 && np <= P - 1) v = tzx[tzx_off[k] + (j - k) * (P + 1 - k) + (np - k)];
        out[idx] = v;
    }
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < (P + 1) * (P + 2); idx += gridDim.x * blockDim.x) {
        const int k = idx / (P + 2), j = idx - k * (P + 2);
        tzl[idx] = (j >= k && j <= P) ? tzx[tzx_off[k] + (j - k) * (P + 1 - k) + (P - k)] : 0.0;
    }
}

// ------------------------------------------------------------------ mixed precision (3xTF32)
// The tensor-core kernel above in FP32 with TF32 tensor cores
// (mma.sync m16n8k8 tf32: A 16x8 row-major, B 8x8 column-major, D 16x8 f32),
// each product taken as three TF32 products of the split operands,
// a b ~ a_hi b_hi + a_hi b_lo + a_lo b_hi (x_hi = tf32(x), x_lo = tf32(x - x_hi)),
// accumulated in FP32.  To keep FP32 in range the expansions are scaled by the
// box size s of the level: X~_n = s^-n X_n in, L_j = s^-(j+1) L~_j out, and
// the z-translation is pre-scaled per class by rho^-(j+n'+1) with rho the
// centre distance in box sizes (2 .. sqrt 27), so every operand is O(1).
// The scaled moments come in FP32 (k_m32, once per evaluation) and the
// per-target sums are FP32, scaled by s^-(j+1) into the FP64 locals at the
// end; four blocks per SM (64 registers, <= 56 KB shared memory at p = 12).

__host__ __device__ constexpr int tf_rt(int n) { return (n + 16) / 16; }   // 16-row tiles of order n
__host__ __device__ constexpr int tf_kc(int n) { return (n + 8) / 8; }     // 8-wide K chunks of order n
__host__ __device__ constexpr int tf_foff(int n)
{
    int s = 0;
    for (int i = 0; i < n; ++i) s += tf_rt(i) * tf_kc(i);
    return s;
}
__host__ __device__ constexpr int tf_zrt(int P, int k) { return (P + 2 - k + 15) / 16; }
__host__ __device__ constexpr int tf_zkc(int P, int k) { return k < P ? (P - k + 7) / 8 : 0; }
__host__ __device__ constexpr int tf_zoff(int P, int k)
{
    int s = 0;
    for (int i = 0; i < k; ++i) s += tf_zrt(P, i) * tf_zkc(P, i);
    return s;
}
__host__ __device__ constexpr int tf_rjob0(int P, int n)
{
    int s = 0;
    for (int i = P; i > n; --i) s += tf_rt(i);
    return s;
}
__host__ __device__ constexpr int tf_zjob0(int P, int k)
{
    int s = 0;
    for (int i = 0; i < k; ++i) s += tf_zrt(P, i);
    return s;
}
// column stride of an FP32 operand buffer: >= rows + 8, = 4 mod 8 (conflict-free fragments)
__host__ __device__ constexpr int tf_ld(int rows)
{
    int ld = rows + 8;
    while (ld % 8 != 4) ++ld;
    return ld;
}
// |d|^2 of a rotation class (class = 7 t2i + dk + 3, fmm.hpp:171)
__host__ __device__ inline int class_dsq(int c)
{
    const int t2[10] = {0, 1, 2, 4, 5, 8, 9, 10, 13, 18};
    const int dk = c % 7 - 3;
    return t2[c / 7] + dk * dk;
}

__device__ __forceinline__ unsigned to_tf32(float x)
{
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

struct Tf32x2 {
    unsigned h, l;
};

__device__ __forceinline__ Tf32x2 split_tf32(float x)
{
    const unsigned h = to_tf32(x);
    return Tf32x2{h, to_tf32(x - __uint_as_float(h))};
}

struct FragA {
    unsigned h[4], l[4];
};


// A fragment stored pre-split: p[0] the TF32 high parts, p[32] the low parts
__device__ __forceinline__ FragA load_a(const float4* p)
{
    const float4 h = __ldg(p), l = __ldg(p + 32);
    return FragA{{__float_as_uint(h.x), __float_as_uint(h.y), __float_as_uint(h.z), __float_as_uint(h.w)},
                 {__float_as_uint(l.x), __float_as_uint(l.y), __float_as_uint(l.z), __float_as_uint(l.w)}};
}

__device__ __forceinline__ void mma1688(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1)
{
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// d += a b in 3xTF32 (small terms first)
__device__ __forceinline__ void mma3x(float (&d)[4], const FragA& a, float b0, float b1)
{
    const Tf32x2 s0 = split_tf32(b0), s1 = split_tf32(b1);
    mma1688(d, a.l, s0.h, s1.h);
    mma1688(d, a.h, s0.l, s1.l);
    mma1688(d, a.h, s0.h, s1.h);
}

template<int P>
struct MixLayout {
    static constexpr int T = (P + 1) * (P + 2) / 2;
    static constexpr int T1 = (P + 2) * (P + 3) / 2;
    static constexpr int LD = tf_ld(T), LD1 = tf_ld(T1);          // column strides (floats)
    static constexpr int kids = 0;                                 // ilist offsets of the 8 children
    static constexpr int sorted = al16(kids + 4 * 9);
    static constexpr int cls = al16(sorted + 2 * kMaxGroupPairs);
    static constexpr int cls_cnt = al16(cls + kMaxGroupPairs);
    static constexpr int cls_off = al16(cls_cnt + 4 * 72);
    static constexpr int bat_off = al16(cls_off + 4 * 72);
    static constexpr int meta = al16(bat_off + 4 * 72);
    static constexpr int tm = al16(meta + int(sizeof(MmaMeta)) * 3);
    static constexpr int tn = al16(tm + T1);                       // order n of coefficient t
    static constexpr int offs = al16(tn + T1);                     // fragment offsets: foff[P+3], zoff[P+3]
    static constexpr int Xraw = al16(offs + 8 * (P + 3));          // [col][T] float2 (cp.async)
    static constexpr int X = al16(Xraw + 8 * T * 8);               // re, im: [col][LD] floats each
    static constexpr int W = al16(X + 2 * 8 * LD * 4);
    static constexpr int LzA = al16(W + 2 * 8 * LD * 4);
    static constexpr int LzB = al16(LzA + 2 * 8 * LD * 4);         // [col][LD1]
    static constexpr int acc = al16(LzB + 2 * 8 * LD1 * 4);        // FP32 complex [8 qd][T] then [8 qd][T1]
    __host__ __device__ static constexpr int total(int qd) { return al16(acc + 8 * 8 * qd * (T + T1)); }
};

template<int P>
__global__ void __launch_bounds__(256, 4) k_m2l_tf32(EvalArgs a, int64_t g0, int64_t g1)
{
    using L = MixLayout<P>;
    constexpr int T = L::T, T1 = L::T1, LD = L::LD, LD1 = L::LD1, NT = 256;
    extern __shared__ __align__(16) unsigned char sm[];
    int* kids = reinterpret_cast<int*>(sm + L::kids);
    short* sorted = reinterpret_cast<short*>(sm + L::sorted);
    unsigned char* cls = sm + L::cls;
    int* cls_cnt = reinterpret_cast<int*>(sm + L::cls_cnt);
    int* cls_off = reinterpret_cast<int*>(sm + L::cls_off);
    int* bat_off = reinterpret_cast<int*>(sm + L::bat_off);
    MmaMeta* meta = reinterpret_cast<MmaMeta*>(sm + L::meta);
    unsigned char* tm = sm + L::tm;
    unsigned char* tn = sm + L::tn;
    int* foff = reinterpret_cast<int*>(sm + L::offs);
    int* zoff = foff + (P + 3);
    float2* Xraw = reinterpret_cast<float2*>(sm + L::Xraw);
    float* Xre = reinterpret_cast<float*>(sm + L::X);
    float* Xim = Xre + 8 * LD;
    float* Wre = reinterpret_cast<float*>(sm + L::W);
    float* Wim = Wre + 8 * LD;
    float* Are = reinterpret_cast<float*>(sm + L::LzA);
    float* Aim = Are + 8 * LD;
    float* Bre = reinterpret_cast<float*>(sm + L::LzB);
    float* Bim = Bre + 8 * LD1;
    const int qd = a.qdim;
    float2* accA = reinterpret_cast<float2*>(sm + L::acc);
    float2* accB = accA + 8 * qd * T;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g8 = lane >> 2, t4 = lane & 3;                      // fragment group / thread in group
    const int bofs = g8 * LD + t4, bofs1 = g8 * LD1 + t4;          // B element (K row t4, column g8)
    const int d0 = (2 * t4) * LD, d1 = (2 * t4 + 1) * LD, e0 = (2 * t4) * LD1, e1 = (2 * t4 + 1) * LD1;
    for (int e = tid; e < (L::acc - L::X) / 4; e += NT) Xre[e] = 0.f;
    for (int t = tid; t < T1; t += NT) {
        int n, m;
        tri_nm(t, n, m);
        tm[t] = static_cast<unsigned char>(m);
        tn[t] = static_cast<unsigned char>(n);
    }
    for (int k = tid; k < P + 3; k += NT) {
        foff[k] = tf_foff(k);
        zoff[k] = tf_zoff(P, k);
    }
    __syncthreads();
    const float4* rf = reinterpret_cast<const float4*>(a.rf32);
    const float4* tzf = reinterpret_cast<const float4*>(a.tz32);
    const int NF = a.rf32_nf, NFZ = a.tz32_nf;

    auto make_meta = [&](int b, int k, MmaMeta& M, int& c) {
        while (bat_off[c + 1] <= b) ++c;
        const int col0 = (b - bat_off[c]) * 8;
        const int ncol = min(8, cls_cnt[c] * qd - col0);
        if (k < ncol) {
            const int col = col0 + k;
            const int pair = col / qd;
            const int e = sorted[cls_off[c] + pair];
            const int code = a.il_code[kids[0] + e];
            const int di = (code & 7) - 3, dj = ((code >> 3) & 7) - 3, dk = ((code >> 6) & 7) - 3;
            const int bq = col - pair * qd;
            int slot = 0;
            while (kids[slot + 1] - kids[0] <= e) ++slot;
            M.src[k] = a.il_src[kids[0] + e];
            M.bq[k] = bq;
            M.sb[k] = slot * qd + bq;
            M.pidx[k] = 7 * (dj + 3) + (di + 3);
            if (k == 0) {
                M.cls = c;
                M.ncol = ncol;
                M.dsq = di * di + dj * dj + dk * dk;
            }
        } else {
            M.src[k] = 0;
            M.bq[k] = 0;
            M.sb[k] = 0;
            M.pidx[k] = 24;
        }
    };
    auto issue = [&](int b) {
        const MmaMeta& M = meta[b % 3];
        const int ncol = M.ncol;
        float2* xr = Xraw;
        for (int e = tid; e < 8 * T; e += NT) {
            const int c = e / T, t = e - c * T;
            if (c < ncol) cp_async8(xr + e, a.m32 + (int64_t(M.src[c]) * qd + M.bq[c]) * T + t);
        }
        cp_async_commit();
    };
    // X~ = e^{i m phi} (s^-n M), column-major
    auto phase_in = [&](int b) {
        const MmaMeta& M = meta[b % 3];
        const int ncol = M.ncol;
        const float2* xr = Xraw;
        for (int e = tid; e < 8 * T; e += NT) {
            const int c = e / T, t = e - c * T;
            if (c < ncol) {
                const double2 ph = __ldg(reinterpret_cast<const double2*>(a.eil) + M.pidx[c] * (P + 2) + tm[t]);
                const float pc = static_cast<float>(ph.x), ps = static_cast<float>(ph.y);
                const float2 v = xr[e];
                Xre[c * LD + t] = pc * v.x - ps * v.y;
                Xim[c * LD + t] = ps * v.x + pc * v.y;
            }
        }
    };

    // blocks take sibling groups from a counter, as in k_m2l_mma
    __shared__ int64_t next_group;
    auto take = [&]() -> int64_t {
        if (tid == 0) next_group = g0 + atomicAdd(a.m2l_ctr, 1);
        __syncthreads();
        const int64_t g = next_group;
        __syncthreads();
        return g;
    };
    for (int64_t g = take(); g < g1; g = take()) {
        const int nc = a.nchild[g];
        if (nc == 0) continue;
        const int cb = a.child_beg[g];
        const int lt = level_of(a, g) + 1;
        {
            const int e0 = a.il_ptr[cb], E = a.il_ptr[cb + nc] - e0;
            for (int e = tid; e < E; e += NT) {
                const int code = a.il_code[e0 + e];
                cls[e] = static_cast<unsigned char>(rot_class((code & 7) - 3, ((code >> 3) & 7) - 3, ((code >> 6) & 7) - 3));
            }
            if (tid <= 8) kids[tid] = a.il_ptr[cb + min(tid, nc)];
            for (int t = tid; t < 8 * qd * (T + T1); t += NT) accA[t] = make_float2(0.f, 0.f);
            __syncthreads();
            for (int cl = tid; cl < kNumClasses; cl += NT) {
                int cnt = 0;
                for (int e = 0; e < E; ++e) cnt += cls[e] == cl;
                cls_cnt[cl] = cnt;
            }
            __syncthreads();
            if (tid == 0) {
                int s = 0, k = 0;
                for (int c = 0; c < kNumClasses; ++c) {
                    cls_off[c] = s;
                    bat_off[c] = k;
                    s += cls_cnt[c];
                    k += (cls_cnt[c] * qd + 7) / 8;
                }
                cls_off[kNumClasses] = s;
                bat_off[kNumClasses] = k;
            }
            __syncthreads();
            for (int cl = tid; cl < kNumClasses; cl += NT) {
                int pos = cls_off[cl];
                for (int e = 0; e < E; ++e)
                    if (cls[e] == cl) sorted[pos++] = static_cast<short>(e);
            }
            __syncthreads();
        }
        const int nbat = bat_off[kNumClasses];
        int cur = 0;
        if (tid < 8 && nbat > 0) make_meta(0, tid, meta[0], cur);
        __syncthreads();
        if (nbat > 0) issue(0);
        if (tid < 8 && nbat > 1) make_meta(1, tid, meta[1], cur);
        cp_async_wait_all();
        __syncthreads();
        if (nbat > 0) phase_in(0);
        __syncthreads();

        for (int b = 0; b < nbat; ++b) {
            const MmaMeta& M = meta[b % 3];
            const float4* rfc = rf + int64_t(M.cls) * NF * 4 * 64 + lane;
            const float4* tzc = tzf + int64_t(M.cls) * NFZ * 64 + lane;
            const float* tlc = a.tzl32 + M.cls * (P + 1) * (P + 2);
            // tile b + 1's moments: the staging buffer is free since phase_in(b)
            if (b + 1 < nbat) issue(b + 1);
            // ---- rotation: jobs (n, rt), largest orders first, round robin over
            // warps; one copy of the job body (runtime n) keeps the code small
            {
                int job = 0;
#pragma unroll 1
                for (int n = P; n >= 0; --n) {
                    const int KC = tf_kc(n), RT = tf_rt(n), base = n * (n + 1) / 2;
#pragma unroll 1
                    for (int rt = 0; rt < RT; ++rt, ++job) {
                        if ((job & 7) != warp) continue;
                        const float4* fr = rfc + (foff[n] + rt * KC) * 4 * 64;
                        float r[4] = {0, 0, 0, 0}, im[4] = {0, 0, 0, 0};
#pragma unroll 1
                        for (int kc = 0; kc < KC; ++kc) {
                            const FragA aP = load_a(fr + (kc * 4 + 0) * 64);
                            const FragA aQ = load_a(fr + (kc * 4 + 1) * 64);
                            const int ro = bofs + base + 8 * kc;
                            mma3x(r, aP, Xre[ro], Xre[ro + 4]);
                            mma3x(im, aQ, Xim[ro], Xim[ro + 4]);
                        }
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int m = 16 * rt + g8 + 8 * h;
                            if (m <= n) {
                                const int u = az_off(P, m) + (n - m);
                                Wre[d0 + u] = r[2 * h];
                                Wre[d1 + u] = r[2 * h + 1];
                                Wim[d0 + u] = im[2 * h];
                                Wim[d1 + u] = im[2 * h + 1];
                            }
                        }
                    }
                }
            }
            __syncthreads();
            // ---- z-translation (class-scaled operator, the same for re and im)
            {
                int job = 0;
#pragma unroll 1
                for (int k = 0; k <= P + 1; ++k) {
                    const int KC = tf_zkc(P, k), RT = tf_zrt(P, k), u0 = az_off(P, k);
#pragma unroll 1
                    for (int rt = 0; rt < RT; ++rt, ++job) {
                        if ((job & 7) != warp) continue;
                        const float4* fz = tzc + (zoff[k] + rt * KC) * 64;
                        float r[4] = {0, 0, 0, 0}, im[4] = {0, 0, 0, 0};
#pragma unroll 1
                        for (int kc = 0; kc < KC; ++kc) {
                            const FragA az = load_a(fz + kc * 64);
                            const int ro = bofs + u0 + 8 * kc;
                            mma3x(r, az, Wre[ro], Wre[ro + 4]);
                            mma3x(im, az, Wim[ro], Wim[ro + 4]);
                        }
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int j = k + 16 * rt + g8 + 8 * h;
                            if (j <= P + 1) {
                                const int t1 = j * (j + 1) / 2 + k;
                                Bre[e0 + t1] = r[2 * h];
                                Bre[e1 + t1] = r[2 * h + 1];
                                Bim[e0 + t1] = im[2 * h];
                                Bim[e1 + t1] = im[2 * h + 1];
                                if (j <= P) {
                                    const float tl = tlc[k * (P + 2) + j];
                                    const int up = u0 + (P - k);          // n' = p
                                    Are[d0 + t1] = fmaf(tl, Wre[d0 + up], r[2 * h]);
                                    Are[d1 + t1] = fmaf(tl, Wre[d1 + up], r[2 * h + 1]);
                                    Aim[d0 + t1] = fmaf(tl, Wim[d0 + up], im[2 * h]);
                                    Aim[d1 + t1] = fmaf(tl, Wim[d1 + up], im[2 * h + 1]);
                                }
                            }
                        }
                    }
                }
            }
            if (tid < 8 && b + 2 < nbat) make_meta(b + 2, tid, meta[(b + 2) % 3], cur);
            __syncthreads();
            // ---- inverse rotation + phase, in place, one warp per order j
            {
                const int pc0 = M.pidx[2 * t4] * (P + 2), pc1 = M.pidx[2 * t4 + 1] * (P + 2);
                constexpr int RTM = tf_rt(P + 1);
#pragma unroll 1
                for (int j = P + 1 - warp; j >= 0; j -= 8) {
                    const int KC = tf_kc(j), RT = tf_rt(j), base = j * (j + 1) / 2;
                    const bool hasA = j <= P;
                    const float4* fr = rfc + foff[j] * 4 * 64;
                    float ar[RTM][4] = {}, ai[RTM][4] = {}, br[RTM][4] = {}, bi[RTM][4] = {};
#pragma unroll
                    for (int rt = 0; rt < RTM; ++rt) {
                        if (rt >= RT) break;
#pragma unroll 1
                        for (int kc = 0; kc < KC; ++kc) {
                            const FragA aPB = load_a(fr + ((rt * KC + kc) * 4 + 2) * 64);
                            const FragA aQB = load_a(fr + ((rt * KC + kc) * 4 + 3) * 64);
                            const int ro1 = bofs1 + base + 8 * kc;
                            mma3x(br[rt], aPB, Bre[ro1], Bre[ro1 + 4]);
                            mma3x(bi[rt], aQB, Bim[ro1], Bim[ro1 + 4]);
                            if (hasA) {
                                const int ro = bofs + base + 8 * kc;
                                mma3x(ar[rt], aPB, Are[ro], Are[ro + 4]);
                                mma3x(ai[rt], aQB, Aim[ro], Aim[ro + 4]);
                            }
                        }
                    }
                    __syncwarp();
#pragma unroll
                    for (int rt = 0; rt < RTM; ++rt)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int m = 16 * rt + g8 + 8 * h;
                            if (rt >= RT || m > j) continue;
                            const int t = base + m;
                            const double2 f0 = __ldg(reinterpret_cast<const double2*>(a.eil) + pc0 + m);
                            const double2 f1 = __ldg(reinterpret_cast<const double2*>(a.eil) + pc1 + m);
                            const float c0 = static_cast<float>(f0.x), s0 = static_cast<float>(f0.y);
                            const float c1 = static_cast<float>(f1.x), s1 = static_cast<float>(f1.y);
                            const float b0r = br[rt][2 * h], b0i = bi[rt][2 * h], b1r = br[rt][2 * h + 1], b1i = bi[rt][2 * h + 1];
                            Bre[e0 + t] = c0 * b0r + s0 * b0i;
                            Bim[e0 + t] = c0 * b0i - s0 * b0r;
                            Bre[e1 + t] = c1 * b1r + s1 * b1i;
                            Bim[e1 + t] = c1 * b1i - s1 * b1r;
                            if (hasA) {
                                const float a0r = ar[rt][2 * h], a0i = ai[rt][2 * h], a1r = ar[rt][2 * h + 1], a1i = ai[rt][2 * h + 1];
                                Are[d0 + t] = c0 * a0r + s0 * a0i;
                                Aim[d0 + t] = c0 * a0i - s0 * a0r;
                                Are[d1 + t] = c1 * a1r + s1 * a1i;
                                Aim[d1 + t] = c1 * a1i - s1 * a1r;
                            }
                        }
                }
            }
            cp_async_wait_all();
            __syncthreads();
            // ---- accumulate (FP32, scaled at the end) in column order; phase tile b + 1 in
            {
                const int ncol = M.ncol;
                int sb[8];
#pragma unroll
                for (int c = 0; c < 8; ++c) sb[c] = M.sb[c];
                for (int t = tid; t < T + T1; t += NT) {
                    const bool isA = t < T;
                    const int r = isA ? t : t - T;
                    const float* sre = isA ? Are + r : Bre + r;
                    const float* sim = isA ? Aim + r : Bim + r;
                    const int ld = isA ? LD : LD1;
                    float2* acc = isA ? accA + r : accB + r;
                    const int stride = isA ? T : T1;
#pragma unroll
                    for (int c = 0; c < 8; ++c)
                        if (c < ncol) {
                            float2& d = acc[sb[c] * stride];
                            d.x += sre[c * ld];
                            d.y += sim[c * ld];
                        }
                }
                if (b + 1 < nbat) phase_in(b + 1);
            }
            __syncthreads();
        }
        // L_j = s^-(j+1) L~_j for the box size s of the targets' level
        const double sinv = double(1 << lt) / a.box->width;
        if (a.want_pot)
            for (int e = tid; e < nc * qd * T; e += NT) {
                const float2 v = accA[e];
                const double sc = pow(sinv, double(tn[e % T] + 1));
                a.LA[int64_t(cb) * qd * T + e] = cplx{sc * v.x, sc * v.y};
            }
        if (a.want_field)
            for (int e = tid; e < nc * qd * T1; e += NT) {
                const float2 v = accB[e];
                const double sc = pow(sinv, double(tn[e % T1] + 1));
                a.LB[int64_t(cb) * qd * T1 + e] = cplx{sc * v.x, sc * v.y};
            }
        __syncthreads();
    }
}

// s^-n M in FP32 (the mixed kernel's source moments), nodes [n0, n1)
__global__ void k_m32(EvalArgs a, int64_t n0, int64_t n1)
{
    const int T = a.T;
    const int64_t per = int64_t(a.qdim) * T, total = (n1 - n0) * per;
    for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total; idx += int64_t(gridDim.x) * blockDim.x) {
        const int64_t node = n0 + idx / per, e = node * per + idx % per;
        int n, m;
        tri_nm(static_cast<int>(idx % per % T), n, m);
        const double sc = pow(double(1 << level_of(a, node)) / a.box->width, double(n));
        const cplx v = a.M[e];
        a.m32[e] = make_float2(static_cast<float>(v.re * sc), static_cast<float>(v.im * sc));
    }
}

template<int P>
bool try_launch_tf32(const EvalArgs& a, int64_t g0, int64_t g1, int sms, cudaStream_t st)
{
    const size_t smem = MixLayout<P>::total(a.qdim);
    int dev = 0, optin = 0;
    SFMM_CUDA(cudaGetDevice(&dev));
    SFMM_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa{};
    SFMM_CUDA(cudaFuncGetAttributes(&fa, k_m2l_tf32<P>));
    if (smem + fa.sharedSizeBytes > size_t(optin)) return false;
    allow_max_smem(k_m2l_tf32<P>);
    int per_sm = 0;
    SFMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_m2l_tf32<P>, 256, smem));
    if (per_sm < 1 || a.m32 == nullptr) return false;
    // sources of every interaction are boxes of levels >= 2
    const int64_t n0 = a.lvl_off[2], n1 = a.lvl_off[a.depth + 1];
    k_m32<<<static_cast<unsigned>(std::min<int64_t>((n1 - n0) * a.qdim * a.T / 256 + 1, int64_t(sms) * 16)), 256, 0, st>>>(a, n0,
                                                                                                                        n1);
    SFMM_CHECK_LAUNCH();
    const int64_t grid = std::min<int64_t>(std::max<int64_t>(g1 - g0, 1), int64_t(sms) * per_sm);
    SFMM_CUDA(cudaMemsetAsync(a.m2l_ctr, 0, sizeof(int), st));
    k_m2l_tf32<P><<<static_cast<unsigned>(grid), 256, smem, st>>>(a, g0, g1);
    SFMM_CHECK_LAUNCH();
    return true;
}

// FP32 TF32-fragment tables: rotation matrices per class (orders <= P+1) and
// the class-scaled z-translation and order-p column.
__global__ void k_frag_rot32(const double* __restrict__ rot, const int* __restrict__ rot_off, int rot_len, int P, int NF,
                             float4* __restrict__ out)
{
    const int64_t total = int64_t(kNumClasses) * NF * 4 * 32;
    for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total; idx += int64_t(gridDim.x) * blockDim.x) {
        const int lane = static_cast<int>(idx & 31), mat = static_cast<int>((idx >> 5) & 3);
        const int64_t rest = idx >> 7;
        const int f = static_cast<int>(rest % NF), c = static_cast<int>(rest / NF);
        int n = 0;
        while (n < P + 1 && tf_foff(n + 1) <= f) ++n;
        const int KC = tf_kc(n);
        const int rt = (f - tf_foff(n)) / KC, kc = (f - tf_foff(n)) - rt * KC;
        const int g = lane >> 2, t = lane & 3;
        float v[4];
        for (int q = 0; q < 4; ++q) {
            const int row = 16 * rt + g + 8 * (q & 1), col = 8 * kc + t + 4 * (q >> 1);
            v[q] = (row <= n && col <= n)
                       ? static_cast<float>(rot[int64_t(c) * rot_len + rot_off[n] + mat * (n + 1) * (n + 1) + row * (n + 1) + col])
                       : 0.f;
        }
        float h[4], l[4];
        for (int q = 0; q < 4; ++q) {
            h[q] = __uint_as_float(to_tf32(v[q]));
            l[q] = __uint_as_float(to_tf32(v[q] - h[q]));
        }
        const int64_t o = (idx >> 5) * 64 + lane;       // [fragment][hi, lo][lane]
        out[o] = make_float4(h[0], h[1], h[2], h[3]);
        out[o + 32] = make_float4(l[0], l[1], l[2], l[3]);
    }
}

__global__ void k_frag_tz32(const double* __restrict__ tzx, const int* __restrict__ tzx_off, int P, int NFZ,
                            float4* __restrict__ out, float* __restrict__ tzl)
{
    const int64_t total = int64_t(kNumClasses) * NFZ * 32;
    for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total; idx += int64_t(gridDim.x) * blockDim.x) {
        const int lane = static_cast<int>(idx & 31);
        const int f = static_cast<int>((idx >> 5) % NFZ), c = static_cast<int>((idx >> 5) / NFZ);
        const double rho = sqrt(double(class_dsq(c)));
        int k = 0;
        while (k < P + 1 && tf_zoff(P, k + 1) <= f) ++k;
        const int KC = tf_zkc(P, k);
        const int rt = (f - tf_zoff(P, k)) / KC, kc = (f - tf_zoff(P, k)) - rt * KC;
        const int g = lane >> 2, t = lane & 3;
        float v[4];
        for (int q = 0; q < 4; ++q) {
            const int j = k + 16 * rt + g + 8 * (q & 1), np = k + 8 * kc + t + 4 * (q >> 1);
            v[q] = (j <= P + 1 && np <= P - 1)
                       ? static_cast<float>(tzx[tzx_off[k] + (j - k) * (P + 1 - k) + (np - k)] * pow(rho, -(j + np + 1)))
                       : 0.f;
        }
        float h[4], l[4];
        for (int q = 0; q < 4; ++q) {
            h[q] = __uint_as_float(to_tf32(v[q]));
            l[q] = __uint_as_float(to_tf32(v[q] - h[q]));
        }
        const int64_t o = (idx >> 5) * 64 + lane;
        out[o] = make_float4(h[0], h[1], h[2], h[3]);
        out[o + 32] = make_float4(l[0], l[1], l[2], l[3]);
    }
    const int ntl = kNumClasses * (P + 1) * (P + 2);
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ntl; idx += gridDim.x * blockDim.x) {
        const int c = idx / ((P + 1) * (P + 2)), r = idx - c * (P + 1) * (P + 2);
        const int k = r / (P + 2), j = r - k * (P + 2);
        const double rho = sqrt(double(class_dsq(c)));
        tzl[idx] = (j >= k && j <= P)
                       ? static_cast<float>(tzx[tzx_off[k] + (j - k) * (P + 1 - k) + (P - k)] * pow(rho, -(j + P + 1)))
                       : 0.f;
    }
}

template<int P>
void launch_m2l_p(const EvalArgs& a, int64_t g0, int64_t g1, int sms, cudaStream_t st)
{
    if (a.m2l_force_rows) {
        launch_rows_fallback<P>(a, g0, g1, sms, st);
        return;
    }
    if constexpr (P >= 2) {
        // mixed plans take the TF32 kernel where it is the faster one (p = 12:
        // 281 ms against 364 ms on 16M uniform points; p = 10: 92 ms against
        // 81 ms on 4M Plummer points, where the FP64 kernel runs instead)
        if (a.mixed && P >= kTf32MinOrder && try_launch_tf32<P>(a, g0, g1, sms, st)) return;
        if (try_launch_mma<P, 1, 8, true>(a, g0, g1, sms, st)) return;
        if (try_launch_mma<P, 1, 8, false>(a, g0, g1, sms, st)) return;
    }
    launch_rows_fallback<P>(a, g0, g1, sms, st);
}

}  // namespace

void build_m2l_fragments(PlanTables& tb, int P, bool mixed, cudaStream_t st)
{
    tb.rfrag_nf = mma_foff(P + 2);
    tb.rfrag.alloc(size_t(kNumClasses) * tb.rfrag_nf * 4 * 32, st);
    const int nfz = std::max(tz_foff(P, P + 2), 1);
    tb.tzfrag.alloc(size_t(nfz) * 32, st);
    tb.tzl.alloc(size_t(P + 1) * (P + 2), st);
    k_frag_rot<<<256, 256, 0, st>>>(tb.rot.ptr, tb.rot_off.ptr, tb.rot_len, P, tb.rfrag_nf, tb.rfrag.ptr);
    SFMM_CHECK_LAUNCH();
    k_frag_tz<<<16, 256, 0, st>>>(tb.tzx.ptr, tb.tzx_off.ptr, P, tz_foff(P, P + 2), tb.tzfrag.ptr, tb.tzl.ptr);
    SFMM_CHECK_LAUNCH();
    if (mixed) {
        tb.rf32_nf = tf_foff(P + 2);
        tb.tz32_nf = std::max(tf_zoff(P, P + 2), 1);
        tb.rf32.alloc(size_t(kNumClasses) * tb.rf32_nf * 4 * 64 * 4, st);     // float4, high and low parts
        tb.tz32.alloc(size_t(kNumClasses) * tb.tz32_nf * 64 * 4, st);
        tb.tzl32.alloc(size_t(kNumClasses) * (P + 1) * (P + 2), st);
        k_frag_rot32<<<256, 256, 0, st>>>(tb.rot.ptr, tb.rot_off.ptr, tb.rot_len, P, tb.rf32_nf,
                                          reinterpret_cast<float4*>(tb.rf32.ptr));
        SFMM_CHECK_LAUNCH();
        k_frag_tz32<<<64, 256, 0, st>>>(tb.tzx.ptr, tb.tzx_off.ptr, P, tf_zoff(P, P + 2),
                                        reinterpret_cast<float4*>(tb.tz32.ptr), tb.tzl32.ptr);
        SFMM_CHECK_LAUNCH();
    }
}

void launch_m2l(const EvalArgs& a, int64_t g0, int64_t g1, int sms, cudaStream_t st)
{
    if (g1 <= g0) return;
    switch (a.p) {
#define SFMM_M2L_CASE(P) case P: launch_m2l_p<P>(a, g0, g1, sms, st); break;
        SFMM_M2L_CASE(0) SFMM_M2L_CASE(1) SFMM_M2L_CASE(2) SFMM_M2L_CASE(3) SFMM_M2L_CASE(4) SFMM_M2L_CASE(5)
        SFMM_M2L_CASE(6) SFMM_M2L_CASE(7) SFMM_M2L_CASE(8) SFMM_M2L_CASE(9) SFMM_M2L_CASE(10) SFMM_M2L_CASE(11)
        SFMM_M2L_CASE(12) SFMM_M2L_CASE(13) SFMM_M2L_CASE(14) SFMM_M2L_CASE(15) SFMM_M2L_CASE(16)
#undef SFMM_M2L_CASE
    default:
        throw Error(FMM_ERR_UNSUPPORTED, "expansion order must be in [0, 16]");
    }
}

}  // namespace sfmm
