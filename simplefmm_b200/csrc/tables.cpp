// Host-side generation of the FMM operator tables for expansion order p.
//
// The coefficient values follow the reference constructor (fmm.hpp:264-396):
// A(n,m) = 1/sqrt((n-m)!(n+m)!) via tgamma, Z(n,m,theta) via
// std::sph_legendre, Wigner small-d rotations by the explicit factorial sum
// in long double for the 70 rotation classes (i^2+j^2 in 10 values) x 7 dk,
// and the z-translation coefficients.  They are then reshaped for a device
// formulation that stores only m >= 0 coefficients (real charges give
// M_n^{-m} = conj(M_n^m), and the rotation tables satisfy
// R[-a][-b] = R[a][b], R[-a][b] = R[a][-b]):
//   rotation of order n  ->  four real (n+1)x(n+1) matrices [out][in]
//       forward  P[a][b] = R[a][b] + R[a][-b],  Q[a][b] = R[a][b] - R[a][-b]  (b >= 1),
//                P[a][0] = Q[a][0] = R[a][0]:   Re W = P Re Mt,  Im W = Q Im Mt;
//       inverse  PB[a][b] = R[b][a] + R[-b][a], QB[a][b] = R[b][a] - R[-b][a] (b >= 1),
//                PB[a][0] = QB[a][0] = R[0][a]  (fmm.hpp:669-686 sums R[b][a] over b).
//   M2M / L2L (fmm.hpp:558-576, 714-733) -> per-output term lists whose
//       octant-independent factor is precomputed; the octant enters through
//       a sign (-1)^(n-|m|) and a phase e^{i q phi}.
#include <algorithm>
#include <cmath>
#include <complex>
#include <stdexcept>
#include <vector>

#include "fmm_tables.h"

namespace sfmm {
namespace {

int sgn_pow(int e) { return (e % 2 == 0) ? 1 : -1; }
int fkm(int k, int m) { return (std::abs(k) - std::abs(m) - std::abs(k - m)) >> 1; }
int tri(int n, int m) { return n * (n + 1) / 2 + m; }

double Afun(int n, int m) { return 1 / std::sqrt(std::tgamma(n - m + 1) * std::tgamma(n + m + 1)); }

double Zfun(int n, int m, double theta) { return std::sqrt(4 * M_PI / (2 * n + 1)) * std::sph_legendre(n, std::abs(m), theta); }

long double wigner_small_d(int n, int a, int b, const long double* f, const long double* c, const long double* s)
{
    const long double pref = std::sqrt(f[n + a] * f[n - a] * f[n + b] * f[n - b]);
    long double acc = 0;
    const int t0 = std::max(0, b - a), t1 = std::min(n + b, n - a);
    for (int t = t0; t <= t1; ++t) {
        const long double term = pref / (f[n + b - t] * f[t] * f[a - b + t] * f[n - a - t]) *
                                 c[2 * n + b - a - 2 * t] * s[a - b + 2 * t];
        acc += ((a - b + t) % 2 == 0) ? term : -term;
    }
    return acc;
}

double child_phi(int c)    // fmm.hpp:444-455 (c % 4)
{
    static const double v[4] = {-0.75 * M_PI, -0.25 * M_PI, 0.75 * M_PI, 0.25 * M_PI};
    return v[c];
}

double parent_phi(int c)   // fmm.hpp:462-473 (c % 4)
{
    static const double v[4] = {0.25 * M_PI, 0.75 * M_PI, -0.25 * M_PI, -0.75 * M_PI};
    return v[c];
}

}  // namespace

HostTables make_tables(int p)
{
    HostTables t;
    t.p = p;
    t.T = (p + 1) * (p + 2) / 2;
    const double th_diag = std::acos(1 / std::sqrt(3.0));
    std::vector<double> A((2 * p + 3) * (2 * p + 4) / 2);
    for (int n = 0; n <= 2 * p + 2; ++n)
        for (int m = 0; m <= n; ++m) A[tri(n, m)] = Afun(n, m);
    auto a = [&](int n, int m) { return A[tri(n, std::abs(m))]; };
    std::vector<double> Znear(t.T);
    for (int n = 0; n <= p; ++n)
        for (int m = 0; m <= n; ++m) Znear[tri(n, m)] = Zfun(n, m, th_diag);

    // ---- rotations
    t.rot_off.resize(p + 2);
    t.rot_off[0] = 0;
    for (int n = 0; n <= p; ++n) t.rot_off[n + 1] = t.rot_off[n] + 4 * (n + 1) * (n + 1);
    t.rot_len = t.rot_off[p + 1];
    t.rot.assign(size_t(kRotClasses) * t.rot_len, 0.0);
    std::vector<long double> f(2 * p + 2), cb(2 * p + 1), sb(2 * p + 1);
    f[0] = 1;
    for (int k = 1; k < 2 * p + 2; ++k) f[k] = f[k - 1] * k;
    const int tvals[10] = {0, 1, 2, 4, 5, 8, 9, 10, 13, 18};
    auto sg = [](int m) { return m < 0 ? sgn_pow(m) : 1; };
    for (int ti = 0; ti < 10; ++ti)
        for (int dk = -3; dk <= 3; ++dk) {
            if (tvals[ti] == 0 && dk == 0) continue;
            const long double th = std::acos(dk / std::sqrt(static_cast<long double>(tvals[ti] + dk * dk)));
            cb[0] = sb[0] = 1;
            for (int e = 0; e < 2 * p; ++e) {
                cb[e + 1] = cb[e] * std::cos(-th / 2);
                sb[e + 1] = sb[e] * std::sin(-th / 2);
            }
            double* blk = t.rot.data() + size_t(7 * ti + dk + 3) * t.rot_len;
            for (int n = 0; n <= p; ++n) {
                auto R = [&](int aa, int bb) {
                    return static_cast<double>(sg(aa) * sg(bb) * wigner_small_d(n, aa, bb, f.data(), cb.data(), sb.data()));
                };
                const int w = (n + 1) * (n + 1);
                double* P = blk + t.rot_off[n];
                double* Q = P + w;
                double* PB = Q + w;
                double* QB = PB + w;
                for (int aa = 0; aa <= n; ++aa)
                    for (int bb = 0; bb <= n; ++bb) {
                        const int o = aa * (n + 1) + bb;
                        if (bb == 0) {
                            P[o] = Q[o] = R(aa, 0);
                            PB[o] = QB[o] = R(0, aa);
                        } else {
                            P[o] = R(aa, bb) + R(aa, -bb);
                            Q[o] = R(aa, bb) - R(aa, -bb);
                            PB[o] = R(bb, aa) + R(-bb, aa);
                            QB[o] = R(bb, aa) - R(-bb, aa);
                        }
                    }
            }
        }

    // ---- z-translation (fmm.hpp:379-396), k >= 0 only
    t.tz_off.resize(p + 2);
    t.tz_off[0] = 0;
    for (int k = 0; k <= p; ++k) t.tz_off[k + 1] = t.tz_off[k] + (p + 1 - k) * (p + 1 - k);
    t.tz.resize(t.tz_off[p + 1]);
    for (int k = 0; k <= p; ++k) {
        const int w = p + 1 - k;
        for (int j = k; j <= p; ++j)
            for (int n = k; n <= p; ++n)
                t.tz[t.tz_off[k] + (j - k) * w + (n - k)] = sgn_pow(n + k) * a(n, k) * a(j, k) / a(j + n, 0);
    }

    t.tzx_off.resize(p + 3);
    t.tzx_off[0] = 0;
    for (int k = 0; k <= p + 1; ++k) t.tzx_off[k + 1] = t.tzx_off[k] + (p + 2 - k) * std::max(p + 1 - k, 0);
    t.tzx.resize(std::max(t.tzx_off[p + 2], 1));
    for (int k = 0; k <= p + 1; ++k) {
        const int w = p + 1 - k;
        for (int j = k; j <= p + 1; ++j)
            for (int n = k; n <= p; ++n)
                t.tzx[t.tzx_off[k] + (j - k) * w + (n - k)] = sgn_pow(n + k) * a(n, k) * a(j, k) / a(j + n, 0);
    }

    // ---- M2L phases e^{i q atan2(dj, di)}, q = 0..p (fmm.hpp:285-292)
    t.eil.resize(size_t(49) * (p + 1) * 2);
    for (int dj = -3; dj <= 3; ++dj)
        for (int di = -3; di <= 3; ++di) {
            const double ph = std::atan2(double(dj), double(di));
            for (int q = 0; q <= p; ++q) {
                const std::complex<double> e = std::polar(1.0, q * ph);
                const size_t o = (size_t(7 * (dj + 3) + (di + 3)) * (p + 1) + q) * 2;
                t.eil[o] = e.real();
                t.eil[o + 1] = e.imag();
            }
        }

    // ---- child / parent phases e^{i q phi_c}, q = -p..p (fmm.hpp:294-299)
    t.echild.resize(size_t(4) * (2 * p + 1) * 2);
    t.eparent.resize(size_t(4) * (2 * p + 1) * 2);
    for (int c = 0; c < 4; ++c)
        for (int q = -p; q <= p; ++q) {
            const std::complex<double> ec = std::polar(1.0, q * child_phi(c));
            const std::complex<double> ep = std::polar(1.0, q * parent_phi(c));
            const size_t o = (size_t(c) * (2 * p + 1) + (q + p)) * 2;
            t.echild[o] = ec.real();
            t.echild[o + 1] = ec.imag();
            t.eparent[o] = ep.real();
            t.eparent[o + 1] = ep.imag();
        }

    // ---- M2M terms (fmm.hpp:564-573): output (j,k>=0) gets
    //   g * rho^n * s_c(n,m) * e^{-i m phi_c} * Mc[j-n, k-m]
    t.m2m_ptr.assign(1, 0);
    for (int j = 0; j <= p; ++j)
        for (int k = 0; k <= j; ++k) {
            for (int n = 0; n <= j; ++n)
                for (int m = std::max(-n, k - (j - n)); m <= std::min(n, k + (j - n)); ++m) {
                    const double g = sgn_pow(fkm(k, m)) * a(n, m) * a(j - n, k - m) / a(j, k) * Znear[tri(n, std::abs(m))];
                    const int q = -m;
                    const int km = k - m;
                    const int in = tri(j - n, std::abs(km));
                    if (!term_fits(n, q, in)) throw std::length_error("M2M term outside its code's fields");
                    t.m2m_code.push_back(pack_term(n, q, in, km < 0));
                    t.m2m_g.push_back(g);
                }
            t.m2m_ptr.push_back(static_cast<int>(t.m2m_g.size()));
        }

    // ---- L2L terms (fmm.hpp:720-730): output (j,k>=0) gets
    //   g * rho^(n-j) * s_c(n-j,m-k) * e^{i (m-k) phi_c} * Lp[n, m]
    t.l2l_ptr.assign(1, 0);
    for (int j = 0; j <= p; ++j)
        for (int k = 0; k <= j; ++k) {
            for (int n = j; n <= p; ++n)
                for (int m = std::max(-n, k - (n - j)); m <= std::min(n, k + (n - j)); ++m) {
                    const double g = sgn_pow(fkm(m, m - k) + n + j) * a(n - j, m - k) * a(j, k) / a(n, m) *
                                     Znear[tri(n - j, std::abs(m - k))];
                    const int q = m - k;
                    const int in = tri(n, std::abs(m));
                    if (!term_fits(n - j, q, in)) throw std::length_error("L2L term outside its code's fields");
                    t.l2l_code.push_back(pack_term(n - j, q, in, m < 0));
                    t.l2l_g.push_back(g);
                }
            t.l2l_ptr.push_back(static_cast<int>(t.l2l_g.size()));
        }
    return t;
}

DirectTables make_direct_tables(int p)
{
    DirectTables d;
    d.p = p;
    const int jmax = p + 1, nzmax = 2 * p + 1;
    std::vector<double> A((2 * nzmax + 2) * (2 * nzmax + 3) / 2);
    for (int n = 0; n <= 2 * nzmax; ++n)
        for (int m = 0; m <= n; ++m) A[tri(n, m)] = Afun(n, m);
    auto a = [&](int n, int m) { return A[tri(n, std::abs(m))]; };
    d.ncoef = (p + 1) * (p + 1);
    const int T1 = (jmax + 1) * (jmax + 2) / 2;
    d.coef.assign(size_t(T1) * d.ncoef, 0.0);
    for (int j = 0; j <= jmax; ++j)
        for (int k = 0; k <= j; ++k)
            for (int n = 0; n <= p; ++n)
                for (int m = -n; m <= n; ++m)
                    d.coef[size_t(tri(j, k)) * d.ncoef + n * (n + 1) + m] =
                        sgn_pow(fkm(k - m, k) + n) * a(n, m) * a(j, k) / a(j + n, m - k);
    d.nz = (nzmax + 1) * (nzmax + 2) / 2;
    d.zil.assign(size_t(64) * d.nz, 0.0);
    for (int k = 0; k < 4; ++k)
        for (int j = 0; j < 4; ++j)
            for (int i = 0; i < 4; ++i) {
                if (i + j + k < 2) continue;
                const double th = std::acos(k / std::sqrt(double(i * i + j * j + k * k)));
                for (int n = 0; n <= nzmax; ++n)
                    for (int m = 0; m <= n; ++m) d.zil[size_t(16 * k + 4 * j + i) * d.nz + tri(n, m)] = Zfun(n, m, th);
            }
    d.ne = 2 * nzmax + 1;
    d.eil2.assign(size_t(49) * d.ne * 2, 0.0);
    for (int dj = -3; dj <= 3; ++dj)
        for (int di = -3; di <= 3; ++di) {
            const double ph = std::atan2(double(dj), double(di));
            for (int q = -nzmax; q <= nzmax; ++q) {
                const std::complex<double> e = std::polar(1.0, q * ph);
                const size_t o = (size_t(7 * (dj + 3) + (di + 3)) * d.ne + (q + nzmax)) * 2;
                d.eil2[o] = e.real();
                d.eil2[o + 1] = e.imag();
            }
        }
    return d;
}

}  // namespace sfmm
