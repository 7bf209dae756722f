// M2L (fmm.hpp:592-712) for the FP64 path: rotation-based, with the potential
// local (order p) and the field local (order p + 1, source orders <= p - 1)
// produced from one rotation and one z-translation per pair.
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
#include "fmm_tables.h"

namespace sfmm {
namespace {

constexpr int kCB = 4;                    // columns per batch
constexpr int kMaxGroupPairs = 8 * 189;   // <= 8 siblings x n_ilist_max (partition.hpp:149)
constexpr int kNumClasses = 70;           // fmm.hpp:169

template<int P>
struct RowCfg {
    static constexpr int T = (P + 1) * (P + 2) / 2;
    static constexpr int T1 = (P + 2) * (P + 3) / 2;
    static constexpr int NT = (T1 + 31) / 32 * 32;
};

struct M2LSmem {
    int ent_src, ent_code, sorted, cls, cls_cnt, cls_off, bat_off, X, W, LzA, LzB, accA, accB, total;
};

__host__ __device__ inline int al16(int x) { return (x + 15) & ~15; }

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
void launch_rows(const EvalArgs& a, int64_t g0, int64_t g1, int sms, cudaStream_t st)
{
    constexpr int T = RowCfg<P>::T, T1 = RowCfg<P>::T1, NT = RowCfg<P>::NT;
    const size_t smem = m2l_smem(T, T1, a.qdim).total;
    SFMM_CUDA(cudaFuncSetAttribute(k_m2l_rows<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    int per_sm = 1;
    SFMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_m2l_rows<P>, NT, smem));
    SFMM_REQUIRE(per_sm > 0, FMM_ERR_UNSUPPORTED, "M2L working set exceeds the device");
    const int64_t groups = g1 - g0;
    const int64_t grid = std::min<int64_t>(std::max<int64_t>(groups, 1), int64_t(sms) * per_sm * 4);
    k_m2l_rows<P><<<static_cast<unsigned>(grid), NT, smem, st>>>(a, g0, g1);
    SFMM_CHECK_LAUNCH();
}

}  // namespace

void launch_m2l(const EvalArgs& a, int64_t g0, int64_t g1, int sms, cudaStream_t st)
{
    if (g1 <= g0) return;
    switch (a.p) {
#define SFMM_M2L_CASE(P) case P: launch_rows<P>(a, g0, g1, sms, st); break;
        SFMM_M2L_CASE(0) SFMM_M2L_CASE(1) SFMM_M2L_CASE(2) SFMM_M2L_CASE(3) SFMM_M2L_CASE(4) SFMM_M2L_CASE(5)
        SFMM_M2L_CASE(6) SFMM_M2L_CASE(7) SFMM_M2L_CASE(8) SFMM_M2L_CASE(9) SFMM_M2L_CASE(10) SFMM_M2L_CASE(11)
        SFMM_M2L_CASE(12) SFMM_M2L_CASE(13) SFMM_M2L_CASE(14) SFMM_M2L_CASE(15) SFMM_M2L_CASE(16)
#undef SFMM_M2L_CASE
    default:
        throw Error(FMM_ERR_UNSUPPORTED, "expansion order must be in [0, 16]");
    }
}

}  // namespace sfmm
