// Per-coefficient FMM operator math, usable from device kernels and from the
// host (the CPU unit tests compile this header with g++ to check the m >= 0
// formulation against the oracle before it runs on a GPU).
//
// Expansion layout: per component T = (p+1)(p+2)/2 complex coefficients
// (n, m) with 0 <= m <= n <= p at index tri(n, m) = n(n+1)/2 + m.  Negative
// orders are implied: X_n^{-m} = conj(X_n^m) (real charges).
//
// Regular solid harmonics in the reference's normalization
//   S_n^m(r) = rho^n Z(n, m, theta) e^{-i m phi},
//   Z(n, m, theta) = sqrt(4 pi/(2n+1)) Y_n^{|m|}(theta, 0)   (fmm.hpp:107-111)
// -- P2M accumulates q S_n^m (fmm.hpp:545-548), L2P evaluates
// sum Re(L_n^m conj(S_n^m)) (fmm.hpp:765-768).  They are generated by the
// three-term recurrences of the normalized associated Legendre functions in
// Cartesian form (no trigonometric calls):
//   S_m^m     = S_{m-1}^{m-1} (-x + i y) sqrt((2m-1)/(2m))
//   S_{m+1}^m = sqrt(2m+1) z S_m^m
//   S_n^m     = [(2n-1) z S_{n-1}^m - sqrt((n+m-1)(n-m-1)) r^2 S_{n-2}^m] / sqrt((n-m)(n+m)).
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define SFMM_HD __host__ __device__ __forceinline__
#else
#define SFMM_HD inline
#endif

namespace sfmm {

constexpr int kMaxOrder = 16;
constexpr int kMaxTri = (kMaxOrder + 1) * (kMaxOrder + 2) / 2;

struct cplx {
    double re, im;
};

SFMM_HD cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
SFMM_HD cplx cconj(cplx a) { return {a.re, -a.im}; }
SFMM_HD int tri(int n, int m) { return n * (n + 1) / 2 + m; }

// Morton keys: bit b of axis a -> key bit 3b + a (zorder.hpp:26-58), by the
// usual 21-bit mask-and-shift spread.
SFMM_HD uint64_t spread3(uint32_t v)
{
    uint64_t x = v & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}

SFMM_HD uint32_t compact3(uint64_t x)
{
    x &= 0x1249249249249249ULL;
    x = (x ^ (x >> 2)) & 0x10c30c30c30c30c3ULL;
    x = (x ^ (x >> 4)) & 0x100f00f00f00f00fULL;
    x = (x ^ (x >> 8)) & 0x1f0000ff0000ffULL;
    x = (x ^ (x >> 16)) & 0x1f00000000ffffULL;
    x = (x ^ (x >> 32)) & 0x1fffffULL;
    return static_cast<uint32_t>(x);
}

// Recurrence coefficients of the solid harmonics (order-independent of p).
struct HarmCoef {
    double diag[kMaxOrder + 1];
    double sub[kMaxOrder + 1];
    double ra[kMaxTri];
    double rb[kMaxTri];
    signed char tn[kMaxTri];             // tri index -> n
    signed char tm[kMaxTri];             // tri index -> m
};

inline void fill_harm_coef(HarmCoef& h)
{
    for (int m = 0; m <= kMaxOrder; ++m) {
        h.diag[m] = m == 0 ? 1.0 : std::sqrt((2.0 * m - 1) / (2.0 * m));
        h.sub[m] = std::sqrt(2.0 * m + 1);
    }
    for (int n = 0; n <= kMaxOrder; ++n)
        for (int m = 0; m <= n; ++m) {
            const int t = tri(n, m);
            h.tn[t] = static_cast<signed char>(n);
            h.tm[t] = static_cast<signed char>(m);
            if (n >= m + 2) {
                const double d = std::sqrt(double(n - m) * double(n + m));
                h.ra[t] = (2.0 * n - 1) / d;
                h.rb[t] = std::sqrt(double(n + m - 1) * double(n - m - 1)) / d;
            } else {
                h.ra[t] = h.rb[t] = 0;
            }
        }
}

// Calls f(n, m, S_n^m) for m = 0..p, n = m..p at offset (x, y, z).
template<typename F>
SFMM_HD void for_each_harmonic(int p, double x, double y, double z, const HarmCoef& h, F&& f)
{
    const double r2 = x * x + y * y + z * z;
    cplx d{1.0, 0.0};
    for (int m = 0; m <= p; ++m) {
        if (m > 0) {
            d = cmul(d, cplx{-x, y});
            d.re *= h.diag[m];
            d.im *= h.diag[m];
        }
        f(m, m, d);
        if (m == p) break;
        cplx s0 = d;
        cplx s1{h.sub[m] * z * d.re, h.sub[m] * z * d.im};
        f(m + 1, m, s1);
        for (int n = m + 2; n <= p; ++n) {
            const int t = tri(n, m);
            const double a = h.ra[t] * z, b = h.rb[t] * r2;
            const cplx s{a * s1.re - b * s0.re, a * s1.im - b * s0.im};
            f(n, m, s);
            s0 = s1;
            s1 = s;
        }
    }
}

// Source-gradient moments from plain moments (one charge component):
// with D+- = d/dx +- i d/dy the ladder relations of S_n^m give, for m >= 0,
//   dz S_n^m = sqrt((n-m)(n+m)) S_{n-1}^m
//   D- S_n^m = sqrt((n-m)(n-m-1)) S_{n-1}^{m+1}
//   D+ S_n^m = -sqrt((n+m)(n+m-1)) S_{n-1}^{m-1}  (m >= 1),
//   D+ S_n^0 = sqrt(n(n-1)) conj(S_{n-1}^1),
// so sum_i q_i grad S_n^m(x_i - c) -- the moments of Q x Zgrho / q Zgrho in
// fmm.hpp:234-253, 549-551 -- is a linear map of the plain moments of order
// n - 1.  Returns the (x, y, z) derivative moments of coefficient (n, m).
SFMM_HD void grad_moment(const cplx* M, int n, int m, cplx* gx, cplx* gy, cplx* gz)
{
    cplx z{0, 0}, dm{0, 0}, dp{0, 0};
    if (n >= 1) {
        if (m <= n - 1) {
            const double c = sqrt(double(n - m) * double(n + m));
            const cplx v = M[tri(n - 1, m)];
            z = {c * v.re, c * v.im};
        }
        if (m + 1 <= n - 1) {
            const double c = sqrt(double(n - m) * double(n - m - 1));
            const cplx v = M[tri(n - 1, m + 1)];
            dm = {c * v.re, c * v.im};
        }
        if (m >= 1) {
            const double c = -sqrt(double(n + m) * double(n + m - 1));
            const cplx v = M[tri(n - 1, m - 1)];
            dp = {c * v.re, c * v.im};
        } else if (n >= 2) {
            const double c = sqrt(double(n) * double(n - 1));
            const cplx v = M[tri(n - 1, 1)];
            dp = {c * v.re, -c * v.im};
        }
    }
    // dx = (D+ + D-)/2, dy = (D+ - D-)/(2i)
    *gx = {0.5 * (dp.re + dm.re), 0.5 * (dp.im + dm.im)};
    *gy = {0.5 * (dp.im - dm.im), -0.5 * (dp.re - dm.re)};
    *gz = z;
}

// Target-side gradient of a local expansion.  With
//   U(x) = sum_{j, |k| <= j} Re(B_j^k conj(S_j^k(x - c)))      (fmm.hpp:765-768)
// and the ladder relations above extended to k < 0 through
// S_j^{-k} = conj(S_j^k), dU/dx_c = sum_{n,m} Re(G_c[n,m] conj(S_n^m)) with
//   G_z[n,m] = sqrt((n+1-m)(n+1+m)) B_{n+1}^m
//   G_x[n,m] = (t1 + t2)/2,   G_y[n,m] = (i/2)(t1 - t2)
//   t1 = -sqrt((n+m+2)(n+m+1)) B_{n+1}^{m+1}
//   t2 =  sqrt((n-m+2)(n-m+1)) B_{n+1}^{m-1}   (m >= 1)
//   t2 = -sqrt((n+2)(n+1)) conj(B_{n+1}^1)      (m = 0).
// The source-gradient M2L of the reference (moments of Q x Zgrho, order p,
// from plain moments of order p - 1) equals, term by term, minus this
// gradient of the order-(p+1) local expansion of the order-(p-1) plain
// moments: grad_s 1/|t - s| = -grad_t 1/|t - s| matches every coefficient of
// the two-centre expansion.  B is stored with order p + 1 (tri indexing).
SFMM_HD void grad_local(const cplx* B, int n, int m, cplx* gx, cplx* gy, cplx* gz)
{
    const cplx b0 = B[tri(n + 1, m)];
    const double cz = sqrt(double(n + 1 - m) * double(n + 1 + m));
    *gz = {cz * b0.re, cz * b0.im};
    const cplx bp = B[tri(n + 1, m + 1)];
    const double c1 = -sqrt(double(n + m + 2) * double(n + m + 1));
    const cplx t1{c1 * bp.re, c1 * bp.im};
    cplx t2;
    if (m >= 1) {
        const cplx bm = B[tri(n + 1, m - 1)];
        const double c2 = sqrt(double(n - m + 2) * double(n - m + 1));
        t2 = {c2 * bm.re, c2 * bm.im};
    } else {
        const cplx b1 = B[tri(n + 1, 1)];
        const double c2 = -sqrt(double(n + 2) * double(n + 1));
        t2 = {c2 * b1.re, -c2 * b1.im};
    }
    *gx = {0.5 * (t1.re + t2.re), 0.5 * (t1.im + t2.im)};
    // (i/2)(t1 - t2)
    *gy = {-0.5 * (t1.im - t2.im), 0.5 * (t1.re - t2.re)};
}

// Component layout of an evaluation: `qdim` plain-moment components come
// out of P2M/M2M; `K` components go through M2L/L2L/L2P:
//   [0, qdim)      potential of each charge component (if want_pot)
//   [kf, kf + 3)   field: q grad (qdim 1) or Q x grad (qdim 3, rinv<true>)
struct CompSpec {
    int qdim;
    int K;
    int want_pot;
    int want_field;
    int kf;                               // first field component
};

// Derived M2L component k of coefficient (n, m) from the plain moments
// (qdim arrays of T coefficients, stride T).
SFMM_HD cplx derive_component(const CompSpec& cs, const cplx* M, int T, int k, int n, int m)
{
    if (cs.want_pot && k < cs.qdim) return M[k * T + tri(n, m)];
    const int a = k - cs.kf;
    if (cs.qdim == 1) {
        cplx g[3];
        grad_moment(M, n, m, &g[0], &g[1], &g[2]);
        return g[a];
    }
    // Q x grad: component a = sum eps_abc D_c M^{b}
    const int b1 = (a + 1) % 3, c1 = (a + 2) % 3;
    cplx g1[3], g2[3];
    grad_moment(M + b1 * T, n, m, &g1[0], &g1[1], &g1[2]);
    grad_moment(M + c1 * T, n, m, &g2[0], &g2[1], &g2[2]);
    return {g1[c1].re - g2[b1].re, g1[c1].im - g2[b1].im};
}

// Term decode for the M2M / L2L term lists (see fmm_tables.h pack_term).
SFMM_HD void unpack_term(int code, int* power, int* q, int* in, bool* conj_in)
{
    *power = code & 31;
    *q = ((code >> 5) & 127) - 32;
    *in = (code >> 12) & 511;
    *conj_in = (code >> 21) & 1;
}

// One output coefficient of M2M (child -> parent, fmm.hpp:558-576) or L2L
// (parent -> child, fmm.hpp:714-733) for a child of octant `oct` (the low 3
// key bits).  rpow[k] = rho^k; phase[q + p] = e^{i q phi_oct}.
template<bool kM2M>
SFMM_HD cplx shift_output(int o, const int* ptr, const int* code, const double* g, const cplx* X, int oct,
                          const double* rpow, const cplx* phase, int p)
{
    const bool zup = (oct >> 2) & 1;
    const bool flip_parity = kM2M ? !zup : zup;
    cplx acc{0, 0};
    for (int e = ptr[o]; e < ptr[o + 1]; ++e) {
        int pw, q, in;
        bool cj;
        unpack_term(code[e], &pw, &q, &in, &cj);
        double s = g[e] * rpow[pw];
        if (flip_parity && ((pw - (q < 0 ? -q : q)) & 1)) s = -s;
        cplx v = X[in];
        if (cj) v.im = -v.im;
        v = cmul(phase[q + p], v);
        acc.re += s * v.re;
        acc.im += s * v.im;
    }
    return acc;
}

// M2L rotation class of an offset (fmm.hpp:171, 492-496).
SFMM_HD int rot_class(int di, int dj, int dk)
{
    const int t = di * di + dj * dj;
    const int t2i = t == 0 ? 0 : t == 1 ? 1 : t == 2 ? 2 : t == 4 ? 3 : t == 5 ? 4 : t == 8 ? 5 : t == 9 ? 6 : t == 10 ? 7 : t == 13 ? 8 : 9;
    return 7 * t2i + (dk + 3);
}

}  // namespace sfmm
