// Direct M2L: the reference's compile-time alternative M2Lc_direct
// (its build option FMM_M2L_DIRECT, fmm.hpp:592-618 with the tables of fmm.hpp:317-337),
// selected per plan with fmm_plan_set_m2l(plan, FMM_M2L_METHOD_DIRECT).
//
// For each (target, source, offset d) of the interaction list, every output
// coefficient is the dense sum over the source's coefficients
//   L[j][k] += sum_{n, m} coef(j,k,n,m) rho^-(j+n+1) Z(j+n, |m-k|, theta_d)
//              e^{i (m-k) phi_d} M[n][m]
// with theta_d = acos(|dk| / |d|) and a parity sign (-1)^((j+n)-(m-k)) for
// dk < 0 (the reference's _m2l_cl table).  Charges are real, so
// M[n][-m] = conj(M[n][m]) and only k >= 0 is formed.  The potential local
// (orders j <= p) sums source orders n <= p; the field local (j <= p + 1)
// n <= p - 1, as the rotation kernels do.
//
// Work decomposition: one block per sibling group, a thread per output
// coefficient (the potential local's T rows, then the field local's T1
// rows); per target its interaction-list entries in list order, the source's
// moments and the offset's Z / phase / rho rows staged in shared memory.
// Each thread accumulates its coefficient in registers in a fixed order, so
// results are deterministic.  It computes (p+1)^2 terms per coefficient and
// pair, an order of p more than the rotation scheme: an alternative kept for
// parity with the reference's option, not a fast path.
#include "eval_util.cuh"

namespace sfmm {
namespace {

__global__ void __launch_bounds__(512) k_m2l_direct(EvalArgs a, int64_t g0, int64_t g1)
{
    extern __shared__ double sm[];
    const int T = a.T, T1 = a.T1, qd = a.qdim, p = a.p;
    const int nz = a.dnz, ne = a.dne;
    cplx* Ms = reinterpret_cast<cplx*>(sm);                  // qd x T
    double* Zs = sm + 2 * qd * T;                             // nz
    cplx* Es = reinterpret_cast<cplx*>(Zs + nz + (nz & 1));   // ne
    double* Pw = reinterpret_cast<double*>(Es + ne);          // 2p + 3
    const int r = threadIdx.x;
    const bool isA = r < T, on = r < T + T1;
    const int row = isA ? r : r - T;                           // (j, k) in the m >= 0 triangle
    int j = 0, k = 0;
    if (on) tri_nm(row, j, k);
    const int nmax = isA ? p : p - 1;
    const bool want = isA ? a.want_pot : a.want_field;
    const double* cf = a.dcoef + int64_t(on ? row : 0) * a.dncoef;
    for (int64_t g = g0 + blockIdx.x; g < g1; g += gridDim.x) {
        const int nc = a.nchild[g];
        if (nc == 0) continue;
        const int cb = a.child_beg[g];
        const int lt = level_of(a, g) + 1;
        for (int c = cb; c < cb + nc; ++c) {
            cplx acc[3] = {{0, 0}, {0, 0}, {0, 0}};
            for (int e = a.il_ptr[c]; e < a.il_ptr[c + 1]; ++e) {
                const int src = a.il_src[e], code = a.il_code[e];
                const int di = (code & 7) - 3, dj = ((code >> 3) & 7) - 3, dk = ((code >> 6) & 7) - 3;
                const int zrow = 16 * abs(dk) + 4 * abs(dj) + abs(di);
                const int erow = 7 * (dj + 3) + (di + 3);
                const int d2 = di * di + dj * dj + dk * dk;
                __syncthreads();                                  // the previous pair's rows are consumed
                for (int t = threadIdx.x; t < qd * T; t += blockDim.x) Ms[t] = a.M[int64_t(src) * qd * T + t];
                for (int t = threadIdx.x; t < nz; t += blockDim.x) Zs[t] = a.dzil[int64_t(zrow) * nz + t];
                for (int t = threadIdx.x; t < ne; t += blockDim.x) Es[t] = a.deil2[int64_t(erow) * ne + t];
                for (int t = threadIdx.x; t < 2 * p + 3; t += blockDim.x)
                    Pw[t] = a.ipow[(int64_t(lt) * 28 + d2) * a.ipow_w + t];
                __syncthreads();
                if (!on || !want) continue;
                for (int n = 0; n <= nmax; ++n) {
                    const int jn = j + n;
                    const double pw = Pw[jn];
                    const int zb = jn * (jn + 1) / 2;
                    for (int m = -n; m <= n; ++m) {
                        const int q = m - k;
                        double v = cf[n * (n + 1) + m] * pw * Zs[zb + (q < 0 ? -q : q)];
                        if (dk < 0 && ((jn - q) & 1)) v = -v;
                        const cplx ep = Es[q + (ne >> 1)];
                        const cplx w{v * ep.re, v * ep.im};
                        const int tnm = n * (n + 1) / 2 + (m < 0 ? -m : m);
                        for (int b = 0; b < qd; ++b) {
                            cplx x = Ms[b * T + tnm];
                            if (m < 0) x.im = -x.im;
                            acc[b].re += w.re * x.re - w.im * x.im;
                            acc[b].im += w.re * x.im + w.im * x.re;
                        }
                    }
                }
            }
            if (on && want)
                for (int b = 0; b < qd; ++b) {
                    if (isA) a.LA[(int64_t(c) * qd + b) * T + row] = acc[b];
                    else a.LB[(int64_t(c) * qd + b) * T1 + row] = acc[b];
                }
        }
    }
}

}  // namespace

void launch_m2l_direct(const EvalArgs& a, int64_t g0, int64_t g1, int sms, cudaStream_t st)
{
    if (g1 <= g0) return;
    const int threads = (a.T + a.T1 + 31) / 32 * 32;
    SFMM_REQUIRE(threads <= 512, FMM_ERR_UNSUPPORTED, "direct M2L: order too high");
    const size_t smem = (2 * size_t(a.qdim) * a.T + a.dnz + 1 + 2 * size_t(a.dne) + 2 * a.p + 3) * sizeof(double);
    const int64_t grid = std::min<int64_t>(g1 - g0, int64_t(sms) * 8);
    k_m2l_direct<<<static_cast<unsigned>(grid), threads, smem, st>>>(a, g0, g1);
    SFMM_CHECK_LAUNCH();
}

}  // namespace sfmm
