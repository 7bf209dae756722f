// Operator tables shared by the host generator (tables.cpp) and the device code.
#pragma once

#include <vector>

namespace sfmm {

constexpr int kMaxP = 16;
constexpr int kRotClasses = 70;          // fmm.hpp:169

// M2M / L2L term code: power of rho (5 bits, 0..31), phase index q + 32
// (7 bits, |q| <= 32), input coefficient index (9 bits, < 512), conjugate-input
// flag (1 bit).  The L2L of the field local runs at order p + 1 <= 17, where
// q = m - k reaches -17: the phase field must hold it without a sign.
inline constexpr bool term_fits(int power, int q, int in)
{
    return power >= 0 && power < 32 && q >= -32 && q < 96 && in >= 0 && in < 512;
}
inline constexpr int pack_term(int power, int q, int in, bool conj_in)
{
    return power | ((q + 32) << 5) | (in << 12) | (conj_in ? 1 << 21 : 0);
}

struct HostTables {
    int p = 0, T = 0;
    int rot_len = 0;                     // doubles per rotation class
    std::vector<int> rot_off;            // per order n: offset of P_n (then Q_n, PB_n, QB_n)
    std::vector<double> rot;             // kRotClasses x rot_len
    std::vector<int> tz_off;             // per k >= 0
    std::vector<double> tz;
    // z-translation with target orders j <= p+1 and source orders n <= p
    // (rows j = k..p+1, columns n = k..p), for the field's order-(p+1) local
    std::vector<int> tzx_off;
    std::vector<double> tzx;
    std::vector<double> eil;             // 49 x (p+1) complex (re, im)
    std::vector<double> echild, eparent; // 4 x (2p+1) complex
    std::vector<int> m2m_ptr, m2m_code;  // per output (tri order) term ranges
    std::vector<double> m2m_g;
    std::vector<int> l2l_ptr, l2l_code;
    std::vector<double> l2l_g;
};

HostTables make_tables(int p);

// Tables of the direct (dense) M2L, the reference's M2Lc_direct
// (fmm.hpp:317-337, 592-618), for target orders j <= p + 1 (the field local)
// and source orders n <= p:
//   coef  [tri(j, k)][n (n + 1) + m]  (-1)^(fkm(k - m, k) + n) A(n,m) A(j,k) / A(j+n, m-k)
//         (the dk >= 0 form; dk < 0 multiplies by (-1)^((j+n) - (m-k)))
//   zil   [16 |dk| + 4 |dj| + |di|][tri(n, m)]  Z(n, m, acos(|dk| / |d|)), n <= 2p + 1
//   eil2  [7 (dj + 3) + (di + 3)][q + 2p + 1]  e^{i q atan2(dj, di)}, |q| <= 2p + 1 (re, im)
struct DirectTables {
    int p = 0;
    int ncoef = 0, nz = 0, ne = 0;       // row lengths of coef / zil / eil2
    std::vector<double> coef, zil, eil2;
};

DirectTables make_direct_tables(int p);

}  // namespace sfmm
