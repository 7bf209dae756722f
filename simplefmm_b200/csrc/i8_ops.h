// Arithmetic of the tensor-core M2L of the mixed plans (m2l_i8.cu), usable on
// the device and on the host (a CPU test compiles this header with g++ and
// checks the dense operator against direct sums and the digit products
// against exact ones).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdlib>

#include "fmm_ops.cuh"

namespace sfmm {

constexpr int kI8MaxOrder = 12;

// Direct-M2L tables (tables.cpp make_direct_tables) seen through pointers.
struct DirectArgs {
    const double* coef;
    int ncoef;
    const double* zil;
    int nz;
    const cplx* eil2;
    int ne;
};

// Real form of an expansion of order P: per order n, Re X_n^0, then Re and Im
// of X_n^m for m = 1..n at n^2 + 2m - 1 (+1): (P+1)^2 values.
SFMM_HD void real_nm(int r, int& n, int& m, int& im)
{
    n = 0;
    while ((n + 1) * (n + 1) <= r) ++n;
    const int o = r - n * n;
    m = (o + 1) / 2;
    im = (o > 0 && (o & 1) == 0) ? 1 : 0;
}

// Byte offset of element (row, k) of a K-major operand slab of the MMA with no
// swizzle: 8-row x 16-byte core matrices, the two 16-byte K halves 128 B apart
// (leading byte offset), row groups 256 B apart (stride byte offset).
SFMM_HD int canon_off(int row, int k) { return (row >> 3) * 256 + (k >> 4) * 128 + (row & 7) * 16 + (k & 15); }

// Digit number scale of ND signed 8-bit digits: |x| <= 1 -> |round(x Q)| <= Q.
template<int ND>
struct I8Digits {
    static constexpr int64_t Q = int64_t(127) << (8 * (ND - 1));
};

// x in [-1, 1] -> ND balanced digits, most significant first:
// round(x Q) = sum_i d_i 2^(8 (ND-1-i)), |d_0| <= 127, d_i in [-128, 127].
template<int ND>
SFMM_HD void split_digits(double x, int8_t* d)
{
    x = x < -1.0 ? -1.0 : (x > 1.0 ? 1.0 : x);
#ifdef __CUDA_ARCH__
    int X = __double2int_rn(x * double(I8Digits<ND>::Q));
#else
    int X = static_cast<int>(std::nearbyint(x * double(I8Digits<ND>::Q)));
#endif
    for (int i = ND - 1; i > 0; --i) {
        const int di = ((X + 128) & 255) - 128;
        d[i] = static_cast<int8_t>(di);
        X = (X - di) >> 8;
    }
    d[0] = static_cast<int8_t>(X);
}

// gamma_n: bound of a scaled order-n moment |w^-n M_n| / sum |q| (a charge at
// a corner of the box, at distance sqrt(3)/2 w from its centre).
SFMM_HD double i8_gamma(int n) { return pow(0.8660254037844386, double(n)); }

// Offset index c = (dx+3) + 7 (dy+3) + 49 (dz+3) of d = source - target.
SFMM_HD bool offset_valid(int c)
{
    const int dx = c % 7 - 3, dy = (c / 7) % 7 - 3, dz = c / 49 - 3;
    return abs(dx) > 1 || abs(dy) > 1 || abs(dz) > 1;
}

// Entry (r, k) of the dense M2L of offset c between scaled expansions:
// L~ = T M~, M~_n = w^-n M_n, L_j = w^-(j+1) L~_j.  Rows r < RA are the
// potential local (order p), the rest the field local (order p + 1 from
// source orders <= p - 1); columns are the real form of M~.  The terms are
// those of the direct M2L (fmm.hpp:592-618, m2l_direct.cu) with
// rho^-(j+n+1) -> |d|^-(j+n+1); M_n^-m = conj(M_n^m) folds the m < 0 terms
// into the columns of Re and Im M_n^m.
SFMM_HD double op_entry(const DirectArgs& t, int p, int RA, int c, int r, int k)
{
    const int dx = c % 7 - 3, dy = (c / 7) % 7 - 3, dz = c / 49 - 3;
    int j, kk, po, n, m, pi;
    int nmax = p;
    if (r < RA) {
        real_nm(r, j, kk, po);
    } else {
        real_nm(r - RA, j, kk, po);
        nmax = p - 1;
    }
    if (k >= (p + 1) * (p + 1)) return 0.0;
    real_nm(k, n, m, pi);
    if (n > nmax) return 0.0;
    const int d2 = dx * dx + dy * dy + dz * dz;
    const double rho = sqrt(double(d2));
    const int zrow = 16 * abs(dz) + 4 * abs(dy) + abs(dx);
    const int erow = 7 * (dy + 3) + (dx + 3);
    const int jn = j + n;
    const double pw = pow(rho, -double(jn + 1));
    auto w = [&](int mm) {
        const int q = mm - kk;
        double v = t.coef[int64_t(j * (j + 1) / 2 + kk) * t.ncoef + n * (n + 1) + mm] * pw *
                   t.zil[int64_t(zrow) * t.nz + jn * (jn + 1) / 2 + (q < 0 ? -q : q)];
        if (dz < 0 && ((jn - q) & 1)) v = -v;
        const cplx e = t.eil2[int64_t(erow) * t.ne + q + (t.ne >> 1)];
        return cplx{v * e.re, v * e.im};
    };
    cplx cf;
    if (m == 0) {
        cf = w(0);
    } else {
        const cplx a = w(m), b = w(-m);
        cf = pi == 0 ? cplx{a.re + b.re, a.im + b.im} : cplx{-(a.im - b.im), a.re - b.re};
    }
    return po == 0 ? cf.re : cf.im;
}

// Largest |S_g| the int32 sums can reach: a target has at most 189 sources,
// each with at most (p+1)^2 nonzero terms; S_g has g + 1 products per term
// (g <= ND - 1), each at most 128 x 128 in magnitude.
inline int64_t i8_sum_bound(int p, int ND)
{
    return int64_t(189) * (p + 1) * (p + 1) * ND * 128 * 128;
}

}  // namespace sfmm
