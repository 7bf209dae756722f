// Operator tables shared by the host generator (tables.cpp) and the device code.
#pragma once

#include <vector>

namespace sfmm {

constexpr int kMaxP = 16;
constexpr int kRotClasses = 70;          // fmm.hpp:169

// M2M / L2L term code: power of rho (5 bits), phase index q + 16 (6 bits),
// input coefficient index (9 bits), conjugate-input flag (1 bit).
inline constexpr int pack_term(int power, int q, int in, bool conj_in)
{
    return power | ((q + 16) << 5) | (in << 11) | (conj_in ? 1 << 20 : 0);
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

}  // namespace sfmm
