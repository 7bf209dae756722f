// CPU checks of the tensor-core M2L's arithmetic (simplefmm_b200/csrc/i8_ops.h):
// the digit split, the dense per-offset operator against direct sums of the
// potential and field, the int8-slice products against the FP64 operator,
// and the int32 bound that fixes the highest order.
#include <cmath>
#include <complex>
#include <cstdio>
#include <random>
#include <vector>

#include "fmm_tables.h"
#include "i8_ops.h"

using namespace sfmm;

static int fails = 0;
#define CHECK(c, ...)                 \
    do {                              \
        if (!(c)) {                   \
            std::printf(__VA_ARGS__); \
            std::printf("\n");        \
            ++fails;                  \
        }                             \
    } while (0)

static HarmCoef H;

static std::vector<cplx> harmonics(int p, double x, double y, double z)
{
    std::vector<cplx> s((p + 1) * (p + 2) / 2);
    for_each_harmonic(p, x, y, z, H, [&](int n, int m, cplx v) { s[tri(n, m)] = v; });
    return s;
}

// U = sum_n [Re(L_n^0 S_n^0) + 2 sum_{m>0} Re(L_n^m conj S_n^m)]
static double eval_local(const std::vector<cplx>& L, const std::vector<cplx>& S, int p)
{
    double u = 0;
    for (int n = 0; n <= p; ++n)
        for (int m = 0; m <= n; ++m) {
            const cplx l = L[tri(n, m)], s = S[tri(n, m)];
            const double v = l.re * s.re + l.im * s.im;
            u += m == 0 ? v : 2 * v;
        }
    return u;
}

int main()
{
    fill_harm_coef(H);
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> U(-1.0, 1.0);

    // 1. digits: sum_i d_i 2^(8(3-i)) == round(x Q), ranges
    for (int i = 0; i < 300000; ++i) {
        double x = U(rng) * (i % 3 == 0 ? 1e-4 : 1.0);
        if (i == 0) x = 1.0;
        if (i == 1) x = -1.0;
        int8_t d[4];
        split_digits<4>(x, d);
        const int64_t X = static_cast<int64_t>(std::nearbyint(x * double(I8Digits<4>::Q)));
        int64_t r = 0;
        for (int k = 0; k < 4; ++k) r = r * 256 + d[k];
        CHECK(r == X && std::abs(int(d[0])) <= 127, "digits of %.17g: %lld vs %lld", x, (long long)r, (long long)X);
    }

    // 2. dense operator against direct sums, and 3. int8 slices against the dense operator
    const int P[] = {4, 8, 12};
    for (int p : P) {
        const DirectTables h = make_direct_tables(p);
        const DirectArgs da{h.coef.data(), h.ncoef, h.zil.data(), h.nz, reinterpret_cast<const cplx*>(h.eil2.data()), h.ne};
        const int RA = (p + 1) * (p + 1), RB = (p + 2) * (p + 2), R = RA + RB, K = RA;
        const int T = (p + 1) * (p + 2) / 2, T1 = (p + 2) * (p + 3) / 2;
        // source box of width 1 at the origin, 40 charges
        std::vector<double> xs(40), ys(40), zs(40), qs(40);
        for (int i = 0; i < 40; ++i) {
            xs[i] = 0.5 * U(rng);
            ys[i] = 0.5 * U(rng);
            zs[i] = 0.5 * U(rng);
            qs[i] = U(rng);
        }
        std::vector<cplx> M(T, cplx{0, 0});
        for (int i = 0; i < 40; ++i) {
            const auto s = harmonics(p, xs[i], ys[i], zs[i]);
            for (int t = 0; t < T; ++t) {
                M[t].re += qs[i] * s[t].re;
                M[t].im += qs[i] * s[t].im;
            }
        }
        std::vector<double> Mr(K);
        for (int k = 0; k < K; ++k) {
            int n, m, im;
            real_nm(k, n, m, im);
            Mr[k] = im ? M[tri(n, m)].im : M[tri(n, m)].re;
        }
        // beta over every offset (as the device tables), alpha over this box
        std::vector<double> beta(R, 0.0);
        for (int c = 0; c < 343; ++c) {
            if (!offset_valid(c)) continue;
            for (int r = 0; r < R; ++r)
                for (int k = 0; k < K; ++k) {
                    int n, m, im;
                    real_nm(k, n, m, im);
                    beta[r] = std::max(beta[r], std::fabs(op_entry(da, p, RA, c, r, k)) * i8_gamma(n));
                }
        }
        double alpha = 0;
        for (int k = 0; k < K; ++k) {
            int n, m, im;
            real_nm(k, n, m, im);
            alpha = std::max(alpha, std::fabs(Mr[k]) / i8_gamma(n));
        }
        std::vector<int8_t> md(4 * K);
        for (int k = 0; k < K; ++k) {
            int n, m, im;
            real_nm(k, n, m, im);
            split_digits<4>(Mr[k] / i8_gamma(n) / alpha, &md[4 * k]);
        }
        const int offs[][3] = {{2, 0, 0}, {3, -2, 1}, {-2, 3, -3}, {0, 0, -2}, {1, -3, 2}};
        double worst_pot = 0, worst_fld = 0, worst_i8 = 0;
        for (const auto& o : offs) {
            const int c = (o[0] + 3) + 7 * (o[1] + 3) + 49 * (o[2] + 3);
            std::vector<double> L(R, 0.0), Le(R, 0.0);
            for (int r = 0; r < R; ++r) {
                int64_t S[4] = {0, 0, 0, 0};
                for (int k = 0; k < K; ++k) {
                    int n, m, im;
                    real_nm(k, n, m, im);
                    const double t = op_entry(da, p, RA, c, r, k);
                    L[r] += t * Mr[k];
                    int8_t od[4];
                    split_digits<4>(beta[r] > 0 ? t * i8_gamma(n) / beta[r] : 0.0, od);
                    for (int g = 0; g < 4; ++g)
                        for (int i = 0; i <= g; ++i) S[g] += int64_t(od[i]) * md[4 * k + (g - i)];
                }
                for (int g = 0; g < 4; ++g) CHECK(std::llabs(S[g]) < (int64_t(1) << 31), "S%d overflows", g);
                double v = 0;
                for (int g = 3; g >= 0; --g) v = v / 256 + double(S[g]);
                Le[r] = alpha * beta[r] * v / (127.0 * 127.0);
            }
            double lmax = 0, dmax = 0;
            for (int r = 0; r < R; ++r) {
                lmax = std::max(lmax, std::fabs(L[r]));
                dmax = std::max(dmax, std::fabs(L[r] - Le[r]));
            }
            worst_i8 = std::max(worst_i8, dmax / lmax);
            // target box centre -d; points inside it
            std::vector<cplx> LA(T), LB(T1);
            for (int r = 0; r < R; ++r) {
                int j, kk, po;
                real_nm(r < RA ? r : r - RA, j, kk, po);
                cplx& e = r < RA ? LA[tri(j, kk)] : LB[tri(j, kk)];
                (po ? e.im : e.re) = L[r];
            }
            for (int trial = 0; trial < 4; ++trial) {
                const double y[3] = {-o[0] + 0.5 * U(rng), -o[1] + 0.5 * U(rng), -o[2] + 0.5 * U(rng)};
                const double yr[3] = {y[0] + o[0], y[1] + o[1], y[2] + o[2]};     // from the target centre
                double pot = 0, fd[3] = {0, 0, 0};
                for (int i = 0; i < 40; ++i) {
                    const double dx = y[0] - xs[i], dy = y[1] - ys[i], dz = y[2] - zs[i];
                    const double ir = 1 / std::sqrt(dx * dx + dy * dy + dz * dz);
                    pot += qs[i] * ir;
                    fd[0] += qs[i] * dx * ir * ir * ir;
                    fd[1] += qs[i] * dy * ir * ir * ir;
                    fd[2] += qs[i] * dz * ir * ir * ir;
                }
                const auto S = harmonics(p + 1, yr[0], yr[1], yr[2]);
                const double up = eval_local(LA, S, p);
                worst_pot = std::max(worst_pot, std::fabs(up - pot) / std::fabs(pot));
                // field = -grad of the order-(p+1) local
                std::vector<cplx> gx(T), gy(T), gz(T);
                for (int n = 0; n <= p; ++n)
                    for (int m = 0; m <= n; ++m) grad_local(LB.data(), n, m, &gx[tri(n, m)], &gy[tri(n, m)], &gz[tri(n, m)]);
                const double f[3] = {-eval_local(gx, S, p), -eval_local(gy, S, p), -eval_local(gz, S, p)};
                const double fn = std::sqrt(fd[0] * fd[0] + fd[1] * fd[1] + fd[2] * fd[2]);
                const double en = std::sqrt((f[0] - fd[0]) * (f[0] - fd[0]) + (f[1] - fd[1]) * (f[1] - fd[1]) + (f[2] - fd[2]) * (f[2] - fd[2]));
                worst_fld = std::max(worst_fld, en / fn);
            }
        }
        std::printf("p=%d: potential %.2e field %.2e (truncation), int8 slices vs FP64 operator %.2e\n", p, worst_pot, worst_fld,
                    worst_i8);
        const double trunc = p == 4 ? 2e-2 : p == 8 ? 2e-3 : 5e-4;
        CHECK(worst_pot < trunc && worst_fld < 5 * trunc, "p=%d truncation error too large", p);
        CHECK(worst_i8 < 1e-8, "p=%d int8 slices off by %.2e", p, worst_i8);
    }

    // 4. no int32 overflow up to the highest order the library takes it at
    CHECK(i8_sum_bound(kI8MaxOrder, 4) < (int64_t(1) << 31), "bound at p = %d", kI8MaxOrder);
    CHECK(i8_sum_bound(kI8MaxOrder + 1, 4) >= (int64_t(1) << 31), "p = %d would also fit", kI8MaxOrder + 1);

    if (fails) {
        std::printf("%d failures\n", fails);
        return 1;
    }
    std::printf("i8 ok\n");
    return 0;
}
