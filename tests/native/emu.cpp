// Test harness: the device operator math (simplefmm_b200/csrc/fmm_ops.cuh and
// the tables of tables.cpp) executed serially on the CPU over a tree given as
// the reference-format per-level arrays.  Used by tests/test_ops_host.py to
// check the m >= 0 formulation against the oracle without a GPU.  Not part of
// the library.
#include <cmath>
#include <complex>
#include <cstdint>
#include <vector>

#include "fmm_ops.cuh"
#include "fmm_tables.h"

using namespace sfmm;

namespace {

struct Lv {
    int64_t nn, nl;
    const int64_t* keys;
    const int* leaf;
    const int* idxp;
    const int* idxv;
    const int* ilp;
    const int* ilv;
    const int* clp;
    const int64_t* clv;
    const int64_t* pl;
    const int* nlp;
    const int* nlv;
};

void ijk(int64_t k, int* o)
{
    o[0] = int(compact3(uint64_t(k)));
    o[1] = int(compact3(uint64_t(k) >> 1));
    o[2] = int(compact3(uint64_t(k) >> 2));
}

}  // namespace

extern "C" int emu_fmm(int depth, const int64_t* nnode, const int64_t* nleaf, void** keys, void** leafnode, void** idxp,
                       void** idxv, void** ilp, void** ilv, void** clp, void** clv, void** pl, void** nlp, void** nlv,
                       const double* box4, int va, double phideg, const double* pos, int64_t n, int p, int qdim,
                       int want_pot, int want_field, const double* Q, double* pot, double* field, int split)
{
    if (p < 0 || p > kMaxOrder) return -1;
    std::vector<Lv> L(depth + 1);
    for (int l = 0; l <= depth; ++l) {
        L[l] = Lv{nnode[l], nleaf[l], (const int64_t*)keys[l], (const int*)leafnode[l], (const int*)idxp[l],
                  (const int*)idxv[l], (const int*)ilp[l], (const int*)ilv[l], (const int*)clp[l],
                  (const int64_t*)clv[l], (const int64_t*)pl[l], (const int*)nlp[l], (const int*)nlv[l]};
    }
    const HostTables tb = make_tables(p);
    HarmCoef hc;
    fill_harm_coef(hc);
    const int T = tb.T;
    CompSpec cs;
    cs.qdim = qdim;
    cs.want_pot = want_pot;
    cs.want_field = want_field;
    cs.kf = want_pot ? qdim : 0;
    cs.K = cs.kf + (want_field ? 3 : 0);
    const int K = cs.K;
    const double width = box4[0];
    const double corner[3] = {box4[1], box4[2], box4[3]};
    const int X = (va + 1) % 3, Y = (va + 2) % 3, Z = va;
    const double phi = phideg * (M_PI / 180), cp = std::cos(phi), sp = std::sin(phi);
    auto rot = [&](const double* v, double* r) {
        r[0] = cp * v[X] - sp * v[Y];
        r[1] = sp * v[X] + cp * v[Y];
        r[2] = v[Z];
    };
    auto center = [&](int l, int64_t key, double* c) {
        int g[3];
        ijk(key, g);
        for (int a = 0; a < 3; ++a) c[a] = corner[a] + width * ((g[a] + 0.5) / (1 << l));
    };
    std::vector<std::vector<cplx>> M(depth + 1), Lx(depth + 1);
    for (int l = 0; l <= depth; ++l) {
        M[l].assign(size_t(L[l].nn) * qdim * T, cplx{0, 0});
        Lx[l].assign(size_t(L[l].nn) * K * T, cplx{0, 0});
    }
    std::vector<cplx> echild(4 * (2 * p + 1)), eparent(4 * (2 * p + 1)), eil(49 * (p + 1));
    for (size_t i = 0; i < echild.size(); ++i) {
        echild[i] = {tb.echild[2 * i], tb.echild[2 * i + 1]};
        eparent[i] = {tb.eparent[2 * i], tb.eparent[2 * i + 1]};
    }
    for (size_t i = 0; i < eil.size(); ++i) eil[i] = {tb.eil[2 * i], tb.eil[2 * i + 1]};

    if (depth >= 2) {
        // P2M at leaves of levels >= 2
        for (int l = 2; l <= depth; ++l)
            for (int64_t f = 0; f < L[l].nl; ++f) {
                const int node = L[l].leaf[f];
                double c[3];
                center(l, L[l].keys[node], c);
                cplx* Mn = &M[l][size_t(node) * qdim * T];
                for (int e = L[l].idxp[f]; e < L[l].idxp[f + 1]; ++e) {
                    const int i = L[l].idxv[e];
                    double r[3];
                    rot(pos + 3 * size_t(i), r);
                    for_each_harmonic(p, r[0] - c[0], r[1] - c[1], r[2] - c[2], hc, [&](int nn, int m, cplx s) {
                        for (int b = 0; b < qdim; ++b) {
                            const double q = Q[size_t(i) * qdim + b];
                            Mn[b * T + tri(nn, m)].re += q * s.re;
                            Mn[b * T + tri(nn, m)].im += q * s.im;
                        }
                    });
                }
            }
        // M2M, levels depth-1 .. 2
        for (int l = depth - 1; l >= 2; --l) {
            const double rho = std::sqrt(0.75) * width / (1 << (l + 1));
            double rp[kMaxOrder + 1];
            rp[0] = 1;
            for (int k = 1; k <= p; ++k) rp[k] = rp[k - 1] * rho;
            for (int64_t ip = 0; ip < L[l].nn; ++ip)
                for (int e = L[l].clp[ip]; e < L[l].clp[ip + 1]; ++e) {
                    const int ic = int(L[l].clv[2 * e]);
                    const int oct = int(L[l].clv[2 * e + 1] & 7);
                    for (int b = 0; b < qdim; ++b) {
                        const cplx* Mc = &M[l + 1][(size_t(ic) * qdim + b) * T];
                        cplx* Mp = &M[l][(size_t(ip) * qdim + b) * T];
                        for (int o = 0; o < T; ++o) {
                            const cplx v = shift_output<true>(o, tb.m2m_ptr.data(), tb.m2m_code.data(), tb.m2m_g.data(), Mc,
                                                              oct, rp, &echild[(oct & 3) * (2 * p + 1)], p);
                            Mp[o].re += v.re;
                            Mp[o].im += v.im;
                        }
                    }
                }
        }
        if (split) {
            // Field through the order-(p+1) local B of the order-(p-1) moments
            // (grad_local), sharing rotation and translation with the potential.
            const HostTables tb1 = make_tables(p + 1);
            const int T1 = tb1.T;
            std::vector<std::vector<cplx>> LA(depth + 1), LB(depth + 1);
            for (int l = 0; l <= depth; ++l) {
                LA[l].assign(size_t(L[l].nn) * qdim * T, cplx{0, 0});
                LB[l].assign(size_t(L[l].nn) * qdim * T1, cplx{0, 0});
            }
            std::vector<cplx> Mt(T), W(T), LzA(T), LzB(T1);
            for (int l = 2; l <= depth; ++l)
                for (int64_t it = 0; it < L[l].nn; ++it)
                    for (int e = L[l].ilp[it]; e < L[l].ilp[it + 1]; ++e) {
                        const int src = L[l].ilv[4 * e];
                        const int di = L[l].ilv[4 * e + 1], dj = L[l].ilv[4 * e + 2], dk = L[l].ilv[4 * e + 3];
                        const double rho = width / (1 << l) * std::sqrt(double(di * di + dj * dj + dk * dk));
                        const double* R = tb1.rot.data() + size_t(rot_class(di, dj, dk)) * tb1.rot_len;
                        const cplx* ph = &eil[(7 * (dj + 3) + (di + 3)) * (p + 1)];
                        double ip[2 * kMaxOrder + 4];
                        ip[0] = 1;
                        for (int k = 1; k <= 2 * p + 3; ++k) ip[k] = ip[k - 1] / rho;
                        for (int b = 0; b < qdim; ++b) {
                            const cplx* Ms = &M[l][(size_t(src) * qdim + b) * T];
                            for (int nn = 0; nn <= p; ++nn)
                                for (int m = 0; m <= nn; ++m) Mt[tri(nn, m)] = cmul(ph[m], Ms[tri(nn, m)]);
                            for (int nn = 0; nn <= p; ++nn) {
                                const double* P = R + tb1.rot_off[nn];
                                const double* Qm = P + (nn + 1) * (nn + 1);
                                for (int a = 0; a <= nn; ++a) {
                                    double re = 0, im = 0;
                                    for (int bb = 0; bb <= nn; ++bb) {
                                        re += P[a * (nn + 1) + bb] * Mt[tri(nn, bb)].re;
                                        im += Qm[a * (nn + 1) + bb] * Mt[tri(nn, bb)].im;
                                    }
                                    W[tri(nn, a)] = {re * ip[nn], im * ip[nn]};
                                }
                            }
                            for (int kk = 0; kk <= p + 1; ++kk) {
                                const int w = p + 1 - kk;
                                const double* tz = tb.tzx.data() + tb.tzx_off[kk];
                                for (int j = kk; j <= p + 1; ++j) {
                                    double re = 0, im = 0;
                                    for (int nn = kk; nn <= p - 1; ++nn) {
                                        re += tz[(j - kk) * w + (nn - kk)] * W[tri(nn, kk)].re;
                                        im += tz[(j - kk) * w + (nn - kk)] * W[tri(nn, kk)].im;
                                    }
                                    LzB[tri(j, kk)] = {re * ip[j + 1], im * ip[j + 1]};
                                    if (j <= p && kk <= p) {
                                        const double c = tz[(j - kk) * w + (p - kk)];
                                        LzA[tri(j, kk)] = {(re + c * W[tri(p, kk)].re) * ip[j + 1], (im + c * W[tri(p, kk)].im) * ip[j + 1]};
                                    }
                                }
                            }
                            auto back = [&](const std::vector<cplx>& Lz, int order, cplx* out) {
                                for (int j = 0; j <= order; ++j) {
                                    const int w = (j + 1) * (j + 1);
                                    const double* PB = R + tb1.rot_off[j] + 2 * w;
                                    const double* QB = PB + w;
                                    for (int a = 0; a <= j; ++a) {
                                        double re = 0, im = 0;
                                        for (int bb = 0; bb <= j; ++bb) {
                                            re += PB[a * (j + 1) + bb] * Lz[tri(j, bb)].re;
                                            im += QB[a * (j + 1) + bb] * Lz[tri(j, bb)].im;
                                        }
                                        const cplx e2 = a <= p ? ph[a] : cmul(ph[a - 1], ph[1]);
                                        const cplx v = cmul(cconj(e2), cplx{re, im});
                                        out[tri(j, a)].re += v.re;
                                        out[tri(j, a)].im += v.im;
                                    }
                                }
                            };
                            if (want_pot) back(LzA, p, &LA[l][(size_t(it) * qdim + b) * T]);
                            if (want_field) back(LzB, p + 1, &LB[l][(size_t(it) * qdim + b) * T1]);
                        }
                    }
            // L2L: A at order p, B at order p + 1
            for (int l = 3; l <= depth; ++l) {
                const double rho = std::sqrt(0.75) * width / (1 << l);
                double rp[kMaxOrder + 2];
                rp[0] = 1;
                for (int k = 1; k <= p + 1; ++k) rp[k] = rp[k - 1] * rho;
                std::vector<cplx> ep1(4 * (2 * p + 3));
                for (size_t i = 0; i < ep1.size(); ++i) ep1[i] = {tb1.eparent[2 * i], tb1.eparent[2 * i + 1]};
                for (int64_t ic = 0; ic < L[l].nn; ++ic) {
                    const int ipar = int(L[l].pl[2 * ic]);
                    const int oct = int(L[l].pl[2 * ic + 1] & 7);
                    for (int b = 0; b < qdim; ++b) {
                        const cplx* Ap = &LA[l - 1][(size_t(ipar) * qdim + b) * T];
                        cplx* Ac = &LA[l][(size_t(ic) * qdim + b) * T];
                        for (int o = 0; o < T; ++o) {
                            const cplx v = shift_output<false>(o, tb.l2l_ptr.data(), tb.l2l_code.data(), tb.l2l_g.data(), Ap,
                                                               oct, rp, &eparent[(oct & 3) * (2 * p + 1)], p);
                            Ac[o].re += v.re;
                            Ac[o].im += v.im;
                        }
                        const cplx* Bp = &LB[l - 1][(size_t(ipar) * qdim + b) * T1];
                        cplx* Bc = &LB[l][(size_t(ic) * qdim + b) * T1];
                        for (int o = 0; o < T1; ++o) {
                            const cplx v = shift_output<false>(o, tb1.l2l_ptr.data(), tb1.l2l_code.data(), tb1.l2l_g.data(), Bp,
                                                               oct, rp, &ep1[(oct & 3) * (2 * p + 3)], p + 1);
                            Bc[o].re += v.re;
                            Bc[o].im += v.im;
                        }
                    }
                }
            }
            // L2P: potential from A, field from the gradient of B
            std::vector<cplx> F(3 * T), G(3 * size_t(qdim) * T);
            for (int l = 2; l <= depth; ++l)
                for (int64_t f = 0; f < L[l].nl; ++f) {
                    const int node = L[l].leaf[f];
                    double c[3];
                    center(l, L[l].keys[node], c);
                    if (want_field) {
                        for (int b = 0; b < qdim; ++b) {
                            const cplx* Bn = &LB[l][(size_t(node) * qdim + b) * T1];
                            for (int nn = 0; nn <= p; ++nn)
                                for (int m = 0; m <= nn; ++m)
                                    grad_local(Bn, nn, m, &G[(3 * b + 0) * T + tri(nn, m)], &G[(3 * b + 1) * T + tri(nn, m)],
                                               &G[(3 * b + 2) * T + tri(nn, m)]);
                        }
                        for (int t = 0; t < T; ++t)
                            for (int a = 0; a < 3; ++a) {
                                if (qdim == 1) {
                                    F[a * T + t] = {-G[a * T + t].re, -G[a * T + t].im};
                                } else {
                                    const int b1 = (a + 1) % 3, c1 = (a + 2) % 3;
                                    const cplx x1 = G[(3 * c1 + b1) * T + t], x2 = G[(3 * b1 + c1) * T + t];
                                    F[a * T + t] = {x1.re - x2.re, x1.im - x2.im};
                                }
                            }
                    }
                    const cplx* An = &LA[l][size_t(node) * qdim * T];
                    for (int e = L[l].idxp[f]; e < L[l].idxp[f + 1]; ++e) {
                        const int i = L[l].idxv[e];
                        double r[3];
                        rot(pos + 3 * size_t(i), r);
                        double up[3] = {0, 0, 0}, uf[3] = {0, 0, 0};
                        for_each_harmonic(p, r[0] - c[0], r[1] - c[1], r[2] - c[2], hc, [&](int nn, int m, cplx sv) {
                            const double w = m == 0 ? 1.0 : 2.0;
                            const int t = tri(nn, m);
                            for (int b = 0; b < qdim; ++b) up[b] += w * (An[b * T + t].re * sv.re + An[b * T + t].im * sv.im);
                            for (int a = 0; a < 3; ++a) uf[a] += w * (F[a * T + t].re * sv.re + F[a * T + t].im * sv.im);
                        });
                        if (want_pot)
                            for (int b = 0; b < qdim; ++b) pot[size_t(i) * qdim + b] += up[b];
                        if (want_field)
                            for (int a = 0; a < 3; ++a) field[size_t(i) * 3 + a] += uf[a];
                    }
                }
        } else {
        // M2L, levels 2 .. depth
        std::vector<cplx> Mt(T), W(T), Lz(T);
        for (int l = 2; l <= depth; ++l)
            for (int64_t it = 0; it < L[l].nn; ++it)
                for (int e = L[l].ilp[it]; e < L[l].ilp[it + 1]; ++e) {
                    const int src = L[l].ilv[4 * e];
                    const int di = L[l].ilv[4 * e + 1], dj = L[l].ilv[4 * e + 2], dk = L[l].ilv[4 * e + 3];
                    const double rho = width / (1 << l) * std::sqrt(double(di * di + dj * dj + dk * dk));
                    const double* R = tb.rot.data() + size_t(rot_class(di, dj, dk)) * tb.rot_len;
                    const cplx* ph = &eil[(7 * (dj + 3) + (di + 3)) * (p + 1)];
                    double ip[2 * kMaxOrder + 2];
                    ip[0] = 1;
                    for (int k = 1; k <= 2 * p + 1; ++k) ip[k] = ip[k - 1] / rho;
                    for (int k = 0; k < K; ++k) {
                        for (int nn = 0; nn <= p; ++nn)
                            for (int m = 0; m <= nn; ++m)
                                Mt[tri(nn, m)] = cmul(ph[m], derive_component(cs, &M[l][size_t(src) * qdim * T], T, k, nn, m));
                        for (int nn = 0; nn <= p; ++nn) {
                            const double* P = R + tb.rot_off[nn];
                            const double* Qm = P + (nn + 1) * (nn + 1);
                            for (int a = 0; a <= nn; ++a) {
                                double re = 0, im = 0;
                                for (int b = 0; b <= nn; ++b) {
                                    re += P[a * (nn + 1) + b] * Mt[tri(nn, b)].re;
                                    im += Qm[a * (nn + 1) + b] * Mt[tri(nn, b)].im;
                                }
                                W[tri(nn, a)] = {re * ip[nn], im * ip[nn]};
                            }
                        }
                        for (int kk = 0; kk <= p; ++kk) {
                            const int w = p + 1 - kk;
                            const double* tz = tb.tz.data() + tb.tz_off[kk];
                            for (int j = kk; j <= p; ++j) {
                                double re = 0, im = 0;
                                for (int nn = kk; nn <= p; ++nn) {
                                    re += tz[(j - kk) * w + (nn - kk)] * W[tri(nn, kk)].re;
                                    im += tz[(j - kk) * w + (nn - kk)] * W[tri(nn, kk)].im;
                                }
                                Lz[tri(j, kk)] = {re * ip[j + 1], im * ip[j + 1]};
                            }
                        }
                        cplx* Lt = &Lx[l][(size_t(it) * K + k) * T];
                        for (int j = 0; j <= p; ++j) {
                            const int w = (j + 1) * (j + 1);
                            const double* PB = R + tb.rot_off[j] + 2 * w;
                            const double* QB = PB + w;
                            for (int a = 0; a <= j; ++a) {
                                double re = 0, im = 0;
                                for (int b = 0; b <= j; ++b) {
                                    re += PB[a * (j + 1) + b] * Lz[tri(j, b)].re;
                                    im += QB[a * (j + 1) + b] * Lz[tri(j, b)].im;
                                }
                                const cplx v = cmul(cconj(ph[a]), cplx{re, im});
                                Lt[tri(j, a)].re += v.re;
                                Lt[tri(j, a)].im += v.im;
                            }
                        }
                    }
                }
        // L2L, child levels 3 .. depth
        for (int l = 3; l <= depth; ++l) {
            const double rho = std::sqrt(0.75) * width / (1 << l);
            double rp[kMaxOrder + 1];
            rp[0] = 1;
            for (int k = 1; k <= p; ++k) rp[k] = rp[k - 1] * rho;
            for (int64_t ic = 0; ic < L[l].nn; ++ic) {
                const int ipar = int(L[l].pl[2 * ic]);
                const int oct = int(L[l].pl[2 * ic + 1] & 7);
                for (int k = 0; k < K; ++k) {
                    const cplx* Lp = &Lx[l - 1][(size_t(ipar) * K + k) * T];
                    cplx* Lc = &Lx[l][(size_t(ic) * K + k) * T];
                    for (int o = 0; o < T; ++o) {
                        const cplx v = shift_output<false>(o, tb.l2l_ptr.data(), tb.l2l_code.data(), tb.l2l_g.data(), Lp,
                                                           oct, rp, &eparent[(oct & 3) * (2 * p + 1)], p);
                        Lc[o].re += v.re;
                        Lc[o].im += v.im;
                    }
                }
            }
        }
        // L2P at leaves of levels >= 2
        for (int l = 2; l <= depth; ++l)
            for (int64_t f = 0; f < L[l].nl; ++f) {
                const int node = L[l].leaf[f];
                double c[3];
                center(l, L[l].keys[node], c);
                const cplx* Ln = &Lx[l][size_t(node) * K * T];
                for (int e = L[l].idxp[f]; e < L[l].idxp[f + 1]; ++e) {
                    const int i = L[l].idxv[e];
                    double r[3];
                    rot(pos + 3 * size_t(i), r);
                    double u[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                    for_each_harmonic(p, r[0] - c[0], r[1] - c[1], r[2] - c[2], hc, [&](int nn, int m, cplx s) {
                        const double w = m == 0 ? 1.0 : 2.0;
                        for (int k = 0; k < K; ++k) {
                            const cplx v = Ln[k * T + tri(nn, m)];
                            u[k] += w * (v.re * s.re + v.im * s.im);
                        }
                    });
                    if (want_pot)
                        for (int b = 0; b < qdim; ++b) pot[size_t(i) * qdim + b] += u[b];
                    if (want_field)
                        for (int a = 0; a < 3; ++a) field[size_t(i) * 3 + a] += u[cs.kf + a];
                }
            }
        }
    }
    // P2P over the nlist (fmm.hpp:773-809)
    for (int l = 0; l <= depth; ++l)
        for (int64_t f = 0; f < L[l].nl; ++f)
            for (int e = L[l].idxp[f]; e < L[l].idxp[f + 1]; ++e) {
                const int i = L[l].idxv[e];
                for (int s = L[l].nlp[f]; s < L[l].nlp[f + 1]; ++s) {
                    const int lj = L[l].nlv[2 * s], fj = L[l].nlv[2 * s + 1];
                    for (int e2 = L[lj].idxp[fj]; e2 < L[lj].idxp[fj + 1]; ++e2) {
                        const int j = L[lj].idxv[e2];
                        if (j == i) continue;
                        const double R[3] = {pos[3 * size_t(i)] - pos[3 * size_t(j)], pos[3 * size_t(i) + 1] - pos[3 * size_t(j) + 1],
                                             pos[3 * size_t(i) + 2] - pos[3 * size_t(j) + 2]};
                        const double r2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
                        const double ir = 1 / std::sqrt(r2), ir3 = ir * ir * ir;
                        if (want_pot)
                            for (int b = 0; b < qdim; ++b) pot[size_t(i) * qdim + b] += Q[size_t(j) * qdim + b] * ir;
                        if (want_field) {
                            if (qdim == 1) {
                                for (int a = 0; a < 3; ++a) field[size_t(i) * 3 + a] += Q[j] * ir3 * R[a];
                            } else {
                                const double* q = Q + 3 * size_t(j);
                                field[3 * size_t(i)] += (q[1] * R[2] - q[2] * R[1]) * ir3;
                                field[3 * size_t(i) + 1] += (q[2] * R[0] - q[0] * R[2]) * ir3;
                                field[3 * size_t(i) + 2] += (q[0] * R[1] - q[1] * R[0]) * ir3;
                            }
                        }
                    }
                }
            }
    return 0;
}

// Decodes every M2M / L2L term code of order p and counts the codes whose
// fields fall outside what an order-p shift can hold (|phase index| <= p,
// rho power <= p, input coefficient < T(p)): a field too narrow for its
// value shows up here, where on the device it would index past the arrays.
extern "C" int emu_check_term_codes(int p)
{
    const HostTables tb = make_tables(p);
    const int T = (p + 1) * (p + 2) / 2;
    int bad = 0;
    auto check = [&](const std::vector<int>& codes) {
        for (int c : codes) {
            int pw, q, in;
            bool cj;
            unpack_term(c, &pw, &q, &in, &cj);
            if (q < -p || q > p || pw < 0 || pw > p || in < 0 || in >= T) ++bad;
        }
    };
    check(tb.m2m_code);
    check(tb.l2l_code);
    return bad;
}

// Every M2M / L2L term of order p carries the rho power |n(out) - n(in)|,
// the order difference of its output and input coefficients.  The plan
// set-up relies on it: a level's shift maps are the maps at rho = 1 with
// entry (out, in) scaled by rho^|n(out) - n(in)|.  Returns the number of
// terms that break it.
extern "C" int emu_check_term_powers(int p)
{
    const HostTables tb = make_tables(p);
    auto order = [](int t) {
        int n = 0;
        while ((n + 1) * (n + 2) / 2 <= t) ++n;
        return n;
    };
    int bad = 0;
    auto check = [&](const std::vector<int>& ptr, const std::vector<int>& codes) {
        for (size_t o = 0; o + 1 < ptr.size(); ++o)
            for (int e = ptr[o]; e < ptr[o + 1]; ++e) {
                int pw, q, in;
                bool cj;
                unpack_term(codes[e], &pw, &q, &in, &cj);
                if (pw != std::abs(order(static_cast<int>(o)) - order(in))) ++bad;
            }
    };
    check(tb.m2m_ptr, tb.m2m_code);
    check(tb.l2l_ptr, tb.l2l_code);
    return bad;
}
