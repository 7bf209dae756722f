// CPU restatement of the reference FMM evaluation path -- TEST ORACLE ONLY.
//
// Only the test suite, __graft_entry__.smoke() and bench.py's CPU-baseline leg
// load this library (through ctypes).  It is a test oracle, never the product:
// the product path is the CUDA library and fails loudly without it.
//
// Written from the reference's algorithm, step by step, with runtime p and
// flat arrays.  Each function cites the reference lines it restates
// (paths are relative to the reference checkout).  It is itself checked
// against the compiled reference (oracle/_ref) by tests/test_oracle.py.
#include "shard_ranges.h"   // the library's work split (simplefmm_b200/csrc), restated stages below
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <memory>
#include <tuple>
#include <utility>
#include <vector>

namespace {

using cd = std::complex<double>;
constexpr int kMaxKeyLevel = 20;          // box.hpp:26 (bits_per_index<int32,int64,3> - 1)
constexpr int kKeyBits = 20;              // zorder.hpp:36 interleaves bits 0..19 of each axis

// ---------------------------------------------------------------- Morton keys
// zorder.hpp:26-44: bit b of axis a goes to bit 3b + a of the key.
int64_t interleave(int32_t i, int axis)
{
    int64_t z = 0;
    for (int b = 0; b < kKeyBits; ++b) z |= static_cast<int64_t>((i >> b) & 1) << (3 * b + axis);
    return z;
}

// zorder.hpp:47-58: inverse of interleave for one axis.
int32_t deinterleave(int64_t z, int axis)
{
    int32_t i = 0;
    for (int b = 0; b < kKeyBits; ++b) i |= static_cast<int32_t>((z >> (3 * b + axis)) & 1) << b;
    return i;
}

struct I3 { int i, j, k; };
I3 key_ijk(int64_t z) { return {deinterleave(z, 0), deinterleave(z, 1), deinterleave(z, 2)}; }
int64_t ijk_key(int i, int j, int k) { return interleave(i, 0) | interleave(j, 1) | interleave(k, 2); }

// ---------------------------------------------------------------- bounding cube
struct Cube {
    int X, Y, Z;
    double phi, width, corner[3];

    // box.hpp:152-157
    void rotate(const double* v, double* r) const
    {
        r[0] = std::cos(phi) * v[X] - std::sin(phi) * v[Y];
        r[1] = std::sin(phi) * v[X] + std::cos(phi) * v[Y];
        r[2] = v[Z];
    }

    // box.hpp:58-63 and 119-122: key of the level-l cell holding v
    int64_t key(int level, const double* v) const
    {
        double r[3];
        rotate(v, r);
        const int32_t imax = (int32_t(1) << level) - 1;
        int64_t z = 0;
        for (int a = 0; a < 3; ++a) {
            const double u = (r[a] - corner[a]) / width;
            int32_t ia = static_cast<int32_t>(u * (1 << level));
            ia = std::min(std::max(ia, 0), imax);
            z |= interleave(ia, a);
        }
        return z;
    }

    // box.hpp:66-70 and 147-150: centre of cell (level, c)
    void center(int level, int64_t c, double* out) const
    {
        const I3 ijk = key_ijk(c);
        const int idx[3] = {ijk.i, ijk.j, ijk.k};
        for (int a = 0; a < 3; ++a) out[a] = corner[a] + width * ((idx[a] + 0.5) / (1 << level));
    }
};

// box.hpp:84-107: the root cube.  Width from the vertical extent grown by the
// margin, doubled (moving the centre up) until it covers every extent.
Cube make_cube(const double* pos, int64_t n, int vertical_axis, double phideg)
{
    Cube b;
    b.X = (vertical_axis + 1) % 3;
    b.Y = (vertical_axis + 2) % 3;
    b.Z = vertical_axis;
    b.phi = phideg * (M_PI / 180);
    double lo[3], hi[3], r[3];
    b.rotate(pos, r);
    for (int a = 0; a < 3; ++a) lo[a] = hi[a] = r[a];
    for (int64_t i = 0; i < n; ++i) {
        b.rotate(pos + 3 * i, r);
        for (int a = 0; a < 3; ++a) {
            lo[a] = lo[a] > r[a] ? r[a] : lo[a];
            hi[a] = hi[a] < r[a] ? r[a] : hi[a];
        }
    }
    double dl[3], c[3];
    for (int a = 0; a < 3; ++a) { dl[a] = hi[a] - lo[a]; c[a] = (hi[a] + lo[a]) / 2; }
    const double dmax = std::max(dl[0], std::max(dl[1], dl[2]));
    b.width = (1 + 2 * 1e-3) * dl[2];
    while (b.width < dmax) {
        c[2] += b.width / 2;
        b.width *= 2;
    }
    for (int a = 0; a < 3; ++a) b.corner[a] = c[a] - b.width / 2;
    return b;
}

// ---------------------------------------------------------------- octree
struct Node {
    int level;
    int64_t key;
    std::vector<int> pts;                 // non-empty only for leaves
    std::vector<std::unique_ptr<Node>> kids;
};

// partition.hpp:47-61 + 93-103 + 134-143: split a node into its non-empty
// children in Morton order (points sorted by (child key, index), so each
// child keeps ascending original indices), recursing while
// level < max_level and count > max_ppn.
void refine(Node* nd, const Cube& cube, const double* pos, int max_level, int max_ppn)
{
    if (!(nd->level < max_level && static_cast<int>(nd->pts.size()) > max_ppn)) return;
    std::vector<std::pair<int64_t, int>> ci;
    ci.reserve(nd->pts.size());
    for (int idx : nd->pts) ci.push_back({cube.key(nd->level + 1, pos + 3 * static_cast<int64_t>(idx)), idx});
    std::sort(ci.begin(), ci.end());
    size_t a = 0;
    for (int64_t c = nd->key << 3; c < (nd->key << 3) + 8; ++c) {
        size_t b = a;
        while (b < ci.size() && ci[b].first == c) ++b;
        if (b > a) {
            auto kid = std::make_unique<Node>();
            kid->level = nd->level + 1;
            kid->key = c;
            for (size_t t = a; t < b; ++t) kid->pts.push_back(ci[t].second);
            nd->kids.push_back(std::move(kid));
        }
        a = b;
    }
    nd->pts.clear();
    for (auto& k : nd->kids) refine(k.get(), cube, pos, max_level, max_ppn);
}

struct Level {
    std::vector<int64_t> keys;            // _c_node: sorted keys of all nodes (partition.hpp:158)
    std::vector<int> leaf_node;           // _i_leaf (partition.hpp:159)
    std::vector<int> idx_ptr{0}, idx;     // _indices CSR (partition.hpp:160)
    std::vector<int> il_ptr{0};           // _ilist CSR: (src node, dijk)
    std::vector<int> il_src;
    std::vector<I3> il_d;
    std::vector<int> cl_ptr{0}, cl_idx;   // _clist: (child node, child key)
    std::vector<int64_t> cl_key;
    std::vector<int> pl_idx;              // _plist: (parent node, own key)
    std::vector<int> nl_ptr{0};           // _nlist: (level, leaf)
    std::vector<std::pair<int, int>> nl;

    bool has(int64_t c) const { return std::binary_search(keys.begin(), keys.end(), c); }
    int index(int64_t c) const { return int(std::lower_bound(keys.begin(), keys.end(), c) - keys.begin()); }
    bool is_leaf(int i) const { return std::binary_search(leaf_node.begin(), leaf_node.end(), i); }
    int to_leaf(int i) const { return int(std::lower_bound(leaf_node.begin(), leaf_node.end(), i) - leaf_node.begin()); }
};

struct Tree {
    Cube cube;
    int64_t n = 0;
    std::vector<double> pos;              // caller's positions, AoS
    std::unique_ptr<Node> root;
    int depth = 0;
    std::vector<Level> lv;
    std::vector<std::pair<int, int>> part; // point -> (leaf level, leaf index)
};

// tree.hpp:83-95 + 103-113: clipped 3x3x3 neighbourhood of cell (l, c),
// visited with i fastest, then j, then k.
template<typename F>
void for_neighbours(int l, int64_t c, F&& f)
{
    const I3 p = key_ijk(c);
    const int imax = 1 << l;
    const int b[3] = {std::max(p.i - 1, 0), std::max(p.j - 1, 0), std::max(p.k - 1, 0)};
    const int e[3] = {std::min(p.i + 2, imax), std::min(p.j + 2, imax), std::min(p.k + 2, imax)};
    for (int k = b[2]; k < e[2]; ++k)
        for (int j = b[1]; j < e[1]; ++j)
            for (int i = b[0]; i < e[0]; ++i) f(I3{i, j, k});
}

bool adjacent(const I3& a, const I3& b)      // tree.hpp:142-147
{
    return std::abs(a.i - b.i) <= 1 && std::abs(a.j - b.j) <= 1 && std::abs(a.k - b.k) <= 1;
}

void collect_level(const Node* nd, int l, Level& L)   // partition.hpp:168-211 (preorder)
{
    if (nd->level > l) return;
    if (nd->level == l) {
        L.keys.push_back(nd->key);
        if (!nd->pts.empty()) {
            L.leaf_node.push_back(int(L.keys.size()) - 1);
            for (int i : nd->pts) L.idx.push_back(i);
            L.idx_ptr.push_back(int(L.idx.size()));
        }
        return;
    }
    for (const auto& k : nd->kids) collect_level(k.get(), l, L);
}

// partition.hpp:283-297 with tree.hpp:122-174: for each node, the children of
// its parent's neighbours that exist and are not adjacent; row sorted by
// (source index, dijk) -- the source index alone decides, it is unique.
void build_ilist(int l, Level& L)
{
    for (int64_t c : L.keys) {
        const I3 t = key_ijk(c);
        std::vector<std::pair<int, I3>> row;
        for_neighbours(l - 1, c >> 3, [&](I3 pn) {
            const int64_t pz = ijk_key(pn.i, pn.j, pn.k);
            for (int o = 0; o < 8; ++o) {
                const int64_t cz = (pz << 3) | o;
                const I3 s = key_ijk(cz);
                if (adjacent(t, s) || !L.has(cz)) continue;
                row.push_back({L.index(cz), I3{s.i - t.i, s.j - t.j, s.k - t.k}});
            }
        });
        std::sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (const auto& e : row) { L.il_src.push_back(e.first); L.il_d.push_back(e.second); }
        L.il_ptr.push_back(int(L.il_src.size()));
    }
}

void add_descendants(const Tree& T, int l, int node, std::vector<std::pair<int, int>>& row)  // partition.hpp:331-341
{
    const Level& L = T.lv[l];
    if (L.is_leaf(node)) {
        row.push_back({l, L.to_leaf(node)});
        return;
    }
    for (int e = L.cl_ptr[node]; e < L.cl_ptr[node + 1]; ++e) add_descendants(T, l + 1, L.cl_idx[e], row);
}

// partition.hpp:343-366: per leaf, the coarser leaves among every ancestor's
// neighbours plus every same-level neighbour (self included) expanded to its
// descendant leaves; rows sorted by (level, leaf).
void build_nlist(Tree& T, int lvl)
{
    Level& L = T.lv[lvl];
    for (int node : L.leaf_node) {
        const int64_t c = L.keys[node];
        std::vector<std::pair<int, int>> row;
        for (int l = 0; l < lvl; ++l) {
            for_neighbours(l, c >> (3 * (lvl - l)), [&](I3 nb) {
                const int64_t z = ijk_key(nb.i, nb.j, nb.k);
                const Level& A = T.lv[l];
                if (A.has(z)) {
                    const int i = A.index(z);
                    if (A.is_leaf(i)) row.push_back({l, A.to_leaf(i)});
                }
            });
        }
        for_neighbours(lvl, c, [&](I3 nb) {
            const int64_t z = ijk_key(nb.i, nb.j, nb.k);
            if (L.has(z)) add_descendants(T, lvl, L.index(z), row);
        });
        std::sort(row.begin(), row.end());
        for (const auto& e : row) L.nl.push_back(e);
        L.nl_ptr.push_back(int(L.nl.size()));
    }
}

// partition.hpp:406-446; box = {corner x, y, z, width} gives the cube of
// Box(corner, width, vertical_axis, phideg) (box.hpp:73-82), else it is fitted.
Tree* build_tree(const double* pos, int64_t n, int max_level, int max_ppn, int vertical_axis, double phideg,
                 const double* box = nullptr)
{
    auto* T = new Tree;
    T->n = n;
    T->pos.assign(pos, pos + 3 * n);
    if (box) {
        Cube& b = T->cube;
        b.X = (vertical_axis + 1) % 3;
        b.Y = (vertical_axis + 2) % 3;
        b.Z = vertical_axis;
        b.phi = phideg * (M_PI / 180);
        for (int a = 0; a < 3; ++a) b.corner[a] = box[a];
        b.width = box[3];
    } else {
        T->cube = make_cube(pos, n, vertical_axis, phideg);
    }
    T->root = std::make_unique<Node>();
    T->root->level = 0;
    T->root->key = 0;
    for (int64_t i = 0; i < n; ++i) T->root->pts.push_back(int(i));
    refine(T->root.get(), T->cube, T->pos.data(), std::min(max_level, kMaxKeyLevel), max_ppn);
    // depth = deepest node (partition.hpp:410-417)
    std::vector<const Node*> stack{T->root.get()};
    while (!stack.empty()) {
        const Node* nd = stack.back();
        stack.pop_back();
        T->depth = std::max(T->depth, nd->level);
        for (const auto& k : nd->kids) stack.push_back(k.get());
    }
    T->lv.resize(T->depth + 1);
    for (int l = 0; l <= T->depth; ++l) {
        collect_level(T->root.get(), l, T->lv[l]);
        if (l >= 2) build_ilist(l, T->lv[l]);
    }
    for (int l = 0; l < T->depth; ++l) {                   // partition.hpp:299-313
        Level& L = T->lv[l];
        const Level& C = T->lv[l + 1];
        for (int64_t c : L.keys) {
            for (int o = 0; o < 8; ++o) {
                const int64_t z = (c << 3) | o;
                if (C.has(z)) { L.cl_idx.push_back(C.index(z)); L.cl_key.push_back(z); }
            }
            L.cl_ptr.push_back(int(L.cl_idx.size()));
        }
    }
    for (int l = 1; l <= T->depth; ++l)                     // partition.hpp:315-322
        for (int64_t c : T->lv[l].keys) T->lv[l].pl_idx.push_back(T->lv[l - 1].index(c >> 3));
    for (int l = 0; l <= T->depth; ++l) build_nlist(*T, l);
    T->part.assign(n, {0, 0});                              // partition.hpp:436-445
    for (int l = 0; l <= T->depth; ++l) {
        const Level& L = T->lv[l];
        for (size_t f = 0; f + 1 < L.idx_ptr.size(); ++f)
            for (int e = L.idx_ptr[f]; e < L.idx_ptr[f + 1]; ++e) T->part[L.idx[e]] = {l, int(f)};
    }
    return T;
}

// ---------------------------------------------------------------- FMM tables
int nm2i(int n, int m) { return n * (n + 1) + m; }          // fmm.hpp:69-72
int npos(int n, int m) { return n * (n + 1) / 2 + std::abs(m); }  // fmm.hpp:87-90
int sgn1(int e) { return e % 2 == 0 ? 1 : -1; }             // fmm.hpp:93-96
int fkm(int k, int m) { return (std::abs(k) - std::abs(m) - std::abs(k - m)) >> 1; }  // fmm.hpp:128-131

// fmm.hpp:99-104
double Apos(int n, int m) { return 1 / std::sqrt(std::tgamma(n - m + 1) * std::tgamma(n + m + 1)); }

// fmm.hpp:107-111: sqrt(4 pi / (2n+1)) Y_n^{|m|}(theta, 0)
double Zf(int n, int m, double theta) { return std::sqrt(4 * M_PI / (2 * n + 1)) * std::sph_legendre(n, std::abs(m), theta); }

// fmm.hpp:114-125: Wigner small-d by the explicit factorial sum
long double wigner_d(int n, int a, int b, const long double* f, const long double* cbp, const long double* sbp)
{
    const long double pref = std::sqrt(f[n + a] * f[n - a] * f[n + b] * f[n - b]);
    long double s = 0;
    for (int t = std::max(0, b - a); t <= std::min(n + b, n - a); ++t) {
        const long double term = pref / (f[n + b - t] * f[t] * f[a - b + t] * f[n - a - t]) *
                                 cbp[2 * n + b - a - 2 * t] * sbp[a - b + 2 * t];
        s += (a - b + t) % 2 == 0 ? term : -term;
    }
    return s;
}

struct Tables {
    int p, n2;
    std::vector<double> A;                // A(n,m), n <= 2p (fmm.hpp:301-306)
    std::vector<double> Znear;            // Z at the cube-diagonal angle (fmm.hpp:264-268)
    std::vector<cd> eil;                  // e^{i q phi(di,dj)}, 49 x (4p+1) (fmm.hpp:285-292)
    std::vector<cd> echild, eparent;      // 4 x (2p+1) (fmm.hpp:294-299)
    std::vector<int> rot_off;             // fmm.hpp:339-342
    int n_rot;
    std::vector<double> rot;              // 70 classes x n_rot (fmm.hpp:344-377)
    std::vector<int> tz_off;              // fmm.hpp:379-396
    std::vector<double> tz;

    double a(int n, int m) const { return A[npos(n, m)]; }
    double zchild(int64_t c, int n, int m) const { return (((c >> 2) % 2 == 0) ? sgn1(n - std::abs(m)) : 1) * Znear[npos(n, m)]; }   // fmm.hpp:457-460
    double zparent(int64_t c, int n, int m) const { return (((c >> 2) % 2 == 0) ? 1 : sgn1(n - std::abs(m))) * Znear[npos(n, m)]; } // fmm.hpp:475-478
};

double phi_child(int64_t c)   // fmm.hpp:444-455
{
    const int r = int(c % 4);
    return r == 0 ? -0.75 * M_PI : r == 1 ? -0.25 * M_PI : r == 2 ? 0.75 * M_PI : 0.25 * M_PI;
}

double phi_parent(int64_t c)  // fmm.hpp:462-473
{
    const int r = int(c % 4);
    return r == 0 ? 0.25 * M_PI : r == 1 ? 0.75 * M_PI : r == 2 ? -0.25 * M_PI : -0.75 * M_PI;
}

Tables make_tables(int p)
{
    Tables t;
    t.p = p;
    t.n2 = (p + 1) * (p + 1);
    t.A.resize(npos(2 * p, 2 * p) + 1);
    for (int n = 0; n <= 2 * p; ++n)
        for (int m = 0; m <= n; ++m) t.A[npos(n, m)] = Apos(n, m);
    t.Znear.resize(npos(p, p) + 1);
    for (int n = 0; n <= p; ++n)
        for (int m = 0; m <= n; ++m) t.Znear[npos(n, m)] = Zf(n, m, std::acos(1 / std::sqrt(3.0)));
    t.eil.resize(49 * (4 * p + 1));
    for (int j = -3; j <= 3; ++j)
        for (int i = -3; i <= 3; ++i) {
            const double ph = std::atan2(double(j), double(i));
            for (int q = -2 * p; q <= 2 * p; ++q) t.eil[(7 * (j + 3) + (i + 3)) * (4 * p + 1) + q + 2 * p] = std::polar(1.0, q * ph);
        }
    t.echild.resize(4 * (2 * p + 1));
    t.eparent.resize(4 * (2 * p + 1));
    for (int c = 0; c < 4; ++c)
        for (int q = -p; q <= p; ++q) {
            t.echild[c * (2 * p + 1) + q + p] = std::polar(1.0, q * phi_child(c));
            t.eparent[c * (2 * p + 1) + q + p] = std::polar(1.0, q * phi_parent(c));
        }
    t.rot_off.resize(p + 1);
    t.rot_off[0] = 0;
    for (int n = 1; n <= p; ++n) t.rot_off[n] = t.rot_off[n - 1] + (2 * n - 1) * (2 * n - 1);
    t.n_rot = (p + 1) * (2 * p + 1) * (2 * p + 3) / 3;
    std::vector<long double> f(2 * p + 2), cbp(2 * p + 1), sbp(2 * p + 1);
    f[0] = 1;
    for (int n = 1; n < 2 * p + 2; ++n) f[n] = f[n - 1] * n;
    t.rot.assign(size_t(70) * t.n_rot, 0.0);
    const int tvals[10] = {0, 1, 2, 4, 5, 8, 9, 10, 13, 18};
    auto sgnm = [](int m) { return m < 0 ? sgn1(m) : 1; };
    for (int ti = 0; ti < 10; ++ti)
        for (int dk = -3; dk <= 3; ++dk) {
            if (tvals[ti] == 0 && dk == 0) continue;
            const long double th = std::acos(dk / std::sqrt(static_cast<long double>(tvals[ti] + dk * dk)));
            cbp[0] = sbp[0] = 1;
            for (int e = 0; e < 2 * p; ++e) {
                cbp[e + 1] = cbp[e] * std::cos(-th / 2);
                sbp[e + 1] = sbp[e] * std::sin(-th / 2);
            }
            double* R = t.rot.data() + size_t(7 * ti + dk + 3) * t.n_rot;
            for (int n = 0; n <= p; ++n)
                for (int a = -n; a <= n; ++a)
                    for (int b = -n; b <= n; ++b)
                        R[t.rot_off[n] + (a + n) * (2 * n + 1) + (b + n)] =
                            double(sgnm(a) * sgnm(b) * wigner_d(n, a, b, f.data(), cbp.data(), sbp.data()));
        }
    t.tz_off.resize(2 * p + 1);
    int off = 0;
    for (int k = -p; k <= p; ++k) {
        t.tz_off[k + p] = off;
        off += (p + 1 - std::abs(k)) * (p + 1 - std::abs(k));
    }
    t.tz.resize(off);
    for (int k = -p; k <= p; ++k) {
        const int ak = std::abs(k), w = p + 1 - ak;
        for (int j = ak; j <= p; ++j)
            for (int n = ak; n <= p; ++n)
                t.tz[t.tz_off[k + p] + (j - ak) * w + (n - ak)] = sgn1(n + ak) * t.a(n, ak) * t.a(j, ak) / t.a(j + n, 0);
    }
    return t;
}

int rot_class(const I3& d)    // fmm.hpp:171 + 492-496
{
    static const int t2i[19] = {0, 1, 2, -1, 3, 4, -1, -1, 5, 6, 7, -1, -1, 8, -1, -1, -1, -1, 9};
    return 7 * t2i[d.i * d.i + d.j * d.j] + (d.k + 3);
}

// ---------------------------------------------------------------- evaluation
struct Eval {
    const Tree& T;
    const Tables& t;
    int p, n2, nc;                        // nc = number of components
    bool grad;
    std::vector<double> phi;              // per point
    std::vector<double> Zrho;             // per point x n2 (fmm.hpp:152)
    std::vector<cd> Zg;                   // per point x n2 x 3 (fmm.hpp:153)
    std::vector<std::vector<cd>> M, L;    // per level: node x n2 x nc
    // sharded stages (oracle_eval_*): this shard's leaves per level, its
    // parents of M2L targets per level, its points; empty = everything
    std::vector<std::vector<char>> own_leaf;
    std::vector<int64_t> own_par_b, own_par_e;
    std::vector<char> own_pt;

    bool leaf_mine(int l, size_t f) const { return own_leaf.empty() || own_leaf[l][f]; }
    bool target_mine(int l, size_t i) const
    {
        if (own_par_b.empty()) return true;
        const int64_t ip = T.lv[l].pl_idx[i];
        return ip >= own_par_b[l - 1] && ip < own_par_e[l - 1];
    }

    cd& m(int l, int node, int nm, int c) { return M[l][(size_t(node) * n2 + nm) * nc + c]; }
    cd& lc(int l, int node, int nm, int c) { return L[l][(size_t(node) * n2 + nm) * nc + c]; }

    // fmm.hpp:217-257: per-point harmonics relative to its leaf centre
    void precompute()
    {
        phi.assign(T.n, 0);
        Zrho.assign(size_t(T.n) * n2, 0);
        if (grad) Zg.assign(size_t(T.n) * n2 * 3, 0);
        for (int l = 0; l <= T.depth; ++l) {
            const Level& Lv = T.lv[l];
            for (size_t f = 0; f < Lv.leaf_node.size(); ++f) {
                double ctr[3];
                T.cube.center(l, Lv.keys[Lv.leaf_node[f]], ctr);
                for (int e = Lv.idx_ptr[f]; e < Lv.idx_ptr[f + 1]; ++e) {
                    const int i = Lv.idx[e];
                    double r[3], d[3];
                    T.cube.rotate(&T.pos[3 * size_t(i)], r);
                    for (int a = 0; a < 3; ++a) d[a] = r[a] - ctr[a];
                    const double rho = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                    const double th = std::acos(d[2] / rho);
                    phi[i] = std::atan2(d[1], d[0]);
                    double rn = 1;
                    for (int n = 0; n <= p; ++n) {
                        for (int mm = -n; mm <= n; ++mm) Zrho[size_t(i) * n2 + nm2i(n, mm)] = rn * Zf(n, mm, th);
                        rn *= rho;
                    }
                    if (!grad) continue;
                    const double st = std::sin(th), ct = std::cos(th), sp = std::sin(phi[i]), cp = std::cos(phi[i]);
                    // rows: e_rho, e_theta, e_phi in Cartesian components
                    const double E[3][3] = {{st * cp, st * sp, ct}, {ct * cp, ct * sp, -st}, {-sp, cp, 0}};
                    double rm1 = 1;
                    for (int n = 1; n <= p; ++n) {
                        for (int mm = -n; mm <= n; ++mm) {
                            const cd v0 = std::polar(n * rm1 * Zf(n, mm, th), -mm * phi[i]);
                            const cd v1 = std::polar(rm1 / st * (std::sqrt(double((n + 1) * (n + 1) - mm * mm)) * Zf(n + 1, mm, th) -
                                                                 (n + 1) * ct * Zf(n, mm, th)), -mm * phi[i]);
                            const cd v2 = std::polar(mm * rm1 / st * Zf(n, mm, th), -(mm * phi[i] + M_PI / 2));
                            for (int a = 0; a < 3; ++a)
                                Zg[(size_t(i) * n2 + nm2i(n, mm)) * 3 + a] = E[0][a] * v0 + E[1][a] * v1 + E[2][a] * v2;
                        }
                        rm1 *= rho;
                    }
                }
            }
        }
    }

    // fmm.hpp:524-556
    void N2M(int l, const double* Q)
    {
        const Level& Lv = T.lv[l];
        for (size_t f = 0; f < Lv.leaf_node.size(); ++f) {
            if (!leaf_mine(l, f)) continue;
            const int node = Lv.leaf_node[f];
            for (int e = Lv.idx_ptr[f]; e < Lv.idx_ptr[f + 1]; ++e) {
                const int i = Lv.idx[e];
                std::vector<cd> Ep(p + 1);
                const cd step(std::cos(phi[i]), -std::sin(phi[i]));
                Ep[0] = 1;
                for (int k = 1; k <= p; ++k) Ep[k] = Ep[k - 1] * step;
                for (int nm = 0; nm < n2; ++nm) {
                    const int n = int(std::sqrt(double(nm)) + 1e-9), mm = nm - n * (n + 1);
                    if (!grad) {
                        const cd e = mm >= 0 ? Ep[mm] : std::conj(Ep[-mm]);
                        for (int c = 0; c < nc; ++c) m(l, node, nm, c) += (Q[size_t(i) * nc + c] * Zrho[size_t(i) * n2 + nm]) * e;
                    } else {
                        const cd* g = &Zg[(size_t(i) * n2 + nm) * 3];
                        const double* q = &Q[size_t(i) * 3];
                        m(l, node, nm, 0) += q[1] * g[2] - q[2] * g[1];
                        m(l, node, nm, 1) += q[2] * g[0] - q[0] * g[2];
                        m(l, node, nm, 2) += q[0] * g[1] - q[1] * g[0];
                    }
                }
            }
        }
    }

    // fmm.hpp:558-590
    void M2M(int lp)
    {
        const Level& Lv = T.lv[lp];
        const double rho = std::sqrt(0.75) * T.cube.width / (1 << (lp + 1));
        for (size_t ip = 0; ip < Lv.keys.size(); ++ip)
            for (int e = Lv.cl_ptr[ip]; e < Lv.cl_ptr[ip + 1]; ++e) {
                const int ic = Lv.cl_idx[e];
                const int64_t cc = Lv.cl_key[e];
                const cd* eph = &t.echild[(cc % 4) * (2 * p + 1)];
                for (int j = 0; j <= p; ++j)
                    for (int k = -j; k <= j; ++k) {
                        double rn = 1;
                        for (int n = 0; n <= j; ++n) {
                            for (int mm = std::max(-n, k - (j - n)); mm <= std::min(n, k + (j - n)); ++mm) {
                                const double v = sgn1(fkm(k, mm)) * t.a(n, mm) * t.a(j - n, k - mm) / t.a(j, k) * rn * t.zchild(cc, n, -mm);
                                for (int c = 0; c < nc; ++c) m(lp, int(ip), nm2i(j, k), c) += v * eph[p - mm] * m(lp + 1, ic, nm2i(j - n, k - mm), c);
                            }
                            rn *= rho;
                        }
                    }
            }
    }

    // fmm.hpp:620-688: rotate, translate along z, rotate back
    void M2L_pair(int l, const I3& d, int src, int tgt)
    {
        const double rho = T.cube.width / (1 << l) * std::sqrt(double(d.i * d.i + d.j * d.j + d.k * d.k));
        const cd* eph = &t.eil[(7 * (d.j + 3) + (d.i + 3)) * (4 * p + 1)];
        const double* R = &t.rot[size_t(rot_class(d)) * t.n_rot];
        std::vector<double> pw(2 * p + 1);
        pw[0] = 1 / rho;
        for (int i = 0; i < 2 * p; ++i) pw[i + 1] = pw[i] / rho;
        std::vector<cd> Mt(size_t(n2) * nc), W(size_t(n2) * nc), Lz(size_t(n2) * nc);
        for (int nm = 0; nm < n2; ++nm) {
            const int n = int(std::sqrt(double(nm)) + 1e-9), mm = nm - n * (n + 1);
            for (int c = 0; c < nc; ++c) Mt[size_t(nm) * nc + c] = eph[mm + 2 * p] * m(l, src, nm, c);
        }
        for (int n = 0; n <= p; ++n) {
            const double* Rn = R + t.rot_off[n];
            const int base = nm2i(n, -n);
            for (int a = 0; a < 2 * n + 1; ++a)
                for (int c = 0; c < nc; ++c) {
                    cd acc = 0;
                    for (int b = 0; b < 2 * n + 1; ++b) acc += Rn[a * (2 * n + 1) + b] * Mt[size_t(base + b) * nc + c];
                    W[size_t(base + a) * nc + c] = acc;
                }
        }
        for (int k = -p; k <= p; ++k) {
            const int ak = std::abs(k), w = p + 1 - ak;
            const double* tz = &t.tz[t.tz_off[k + p]];
            for (int j = ak; j <= p; ++j)
                for (int c = 0; c < nc; ++c) {
                    cd acc = 0;
                    for (int n = ak; n <= p; ++n) acc += (tz[(j - ak) * w + (n - ak)] * pw[j + n]) * W[size_t(nm2i(n, k)) * nc + c];
                    Lz[size_t(nm2i(j, k)) * nc + c] = acc;
                }
        }
        for (int j = 0; j <= p; ++j) {
            const double* Rj = R + t.rot_off[j];
            const int base = nm2i(j, -j);
            for (int a = 0; a < 2 * j + 1; ++a)
                for (int c = 0; c < nc; ++c) {
                    cd acc = 0;
                    for (int b = 0; b < 2 * j + 1; ++b) acc += Rj[b * (2 * j + 1) + a] * Lz[size_t(base + b) * nc + c];
                    lc(l, tgt, base + a, c) += eph[(j - a) + 2 * p] * acc;
                }
        }
    }

    void M2L(int l)   // fmm.hpp:700-712
    {
        const Level& Lv = T.lv[l];
        for (size_t i = 0; i < Lv.keys.size(); ++i) {
            if (!target_mine(l, i)) continue;
            for (int e = Lv.il_ptr[i]; e < Lv.il_ptr[i + 1]; ++e) M2L_pair(l, Lv.il_d[e], Lv.il_src[e], int(i));
        }
    }

    // fmm.hpp:714-745
    void L2L(int lc_)
    {
        const Level& Lv = T.lv[lc_];
        const double rho = std::sqrt(0.75) * T.cube.width / (1 << lc_);
        for (size_t ic = 0; ic < Lv.keys.size(); ++ic) {
            const int ip = Lv.pl_idx[ic];
            const int64_t cc = Lv.keys[ic];
            const cd* eph = &t.eparent[(cc % 4) * (2 * p + 1)];
            for (int j = 0; j <= p; ++j)
                for (int k = -j; k <= j; ++k) {
                    double rn = 1;
                    for (int n = j; n <= p; ++n) {
                        for (int mm = std::max(-n, k - (n - j)); mm <= std::min(n, k + (n - j)); ++mm) {
                            const double v = sgn1(fkm(mm, mm - k) + n + j) * t.a(n - j, mm - k) * t.a(j, k) / t.a(n, mm) * rn * t.zparent(cc, n - j, mm - k);
                            for (int c = 0; c < nc; ++c) lc(lc_, int(ic), nm2i(j, k), c) += v * eph[(mm - k) + p] * lc(lc_ - 1, ip, nm2i(n, mm), c);
                        }
                        rn *= rho;
                    }
                }
        }
    }

    // fmm.hpp:747-771
    void L2N(int l, double* U)
    {
        const Level& Lv = T.lv[l];
        for (size_t f = 0; f < Lv.leaf_node.size(); ++f) {
            if (!leaf_mine(l, f)) continue;
            const int node = Lv.leaf_node[f];
            for (int e = Lv.idx_ptr[f]; e < Lv.idx_ptr[f + 1]; ++e) {
                const int i = Lv.idx[e];
                std::vector<cd> F(p + 1);
                const cd step(std::cos(phi[i]), std::sin(phi[i]));
                F[0] = 1;
                for (int k = 1; k <= p; ++k) F[k] = F[k - 1] * step;
                for (int jk = 0; jk < n2; ++jk) {
                    const int j = int(std::sqrt(double(jk)) + 1e-9), mm = jk - j * (j + 1);
                    const cd e = mm >= 0 ? F[mm] : std::conj(F[-mm]);
                    for (int c = 0; c < nc; ++c) {
                        const cd v = lc(l, node, jk, c);
                        U[size_t(i) * nc + c] += Zrho[size_t(i) * n2 + jk] * (v.real() * e.real() - v.imag() * e.imag());
                    }
                }
            }
        }
    }

    // fmm.hpp:773-809 with the default is_self (i == j) and an empty slist
    void N2N(const double* Q, double* U)
    {
        const double* X = T.pos.data();
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t i = 0; i < T.n; ++i) {
            if (!own_pt.empty() && !own_pt[i]) continue;
            const auto [li, fi] = T.part[i];
            const Level& Lv = T.lv[li];
            for (int e = Lv.nl_ptr[fi]; e < Lv.nl_ptr[fi + 1]; ++e) {
                const auto [lj, fj] = Lv.nl[e];
                const Level& S = T.lv[lj];
                for (int s = S.idx_ptr[fj]; s < S.idx_ptr[fj + 1]; ++s) {
                    const int j = S.idx[s];
                    if (j == i) continue;
                    const double R[3] = {X[3 * i] - X[3 * size_t(j)], X[3 * i + 1] - X[3 * size_t(j) + 1], X[3 * i + 2] - X[3 * size_t(j) + 2]};
                    const double r = std::sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]);
                    if (!grad) {
                        for (int c = 0; c < nc; ++c) U[i * nc + c] += Q[size_t(j) * nc + c] / r;
                    } else {
                        const double* q = &Q[size_t(j) * 3];
                        const double r3 = std::pow(r, 3.0);
                        U[i * 3 + 0] += (q[1] * R[2] - q[2] * R[1]) / r3;
                        U[i * 3 + 1] += (q[2] * R[0] - q[0] * R[2]) / r3;
                        U[i * 3 + 2] += (q[0] * R[1] - q[1] * R[0]) / r3;
                    }
                }
            }
        }
    }

    // fmm.hpp:811-881
    void rinv(const double* Q, double* U)
    {
        const int D = T.depth;
        if (D >= 2) {
            precompute();
            M.assign(D + 1, {});
            L.assign(D + 1, {});
            for (int l = 0; l <= D; ++l) {
                M[l].assign(T.lv[l].keys.size() * n2 * nc, 0);
                L[l].assign(T.lv[l].keys.size() * n2 * nc, 0);
            }
            N2M(D, Q);
            for (int l = D - 1; l >= 2; --l) {
                M2M(l);
                N2M(l, Q);
            }
            for (int l = 2; l <= D; ++l) M2L(l);
            for (int l = 2; l < D; ++l) {
                L2N(l, U);
                L2L(l + 1);
            }
            L2N(D, U);
        }
        N2N(Q, U);
    }

    // One shard's share (shard_ranges.h): leaves per level balanced by points,
    // M2L targets by contiguous ranges of their parents per level.
    void set_shard(int index, int count)
    {
        own_leaf.assign(T.depth + 1, {});
        own_par_b.assign(T.depth + 1, 0);
        own_par_e.assign(T.depth + 1, 0);
        own_pt.assign(T.n, 0);
        for (int l = 0; l <= T.depth; ++l) {
            const Level& Lv = T.lv[l];
            const int64_t nl = int64_t(Lv.leaf_node.size());
            std::vector<int64_t> prefix(Lv.idx_ptr.begin(), Lv.idx_ptr.end());
            const auto r = sfmm::balanced_leaf_range(prefix.data(), nl, count, index);
            own_leaf[l].assign(nl, 0);
            for (int64_t f = r.first; f < r.second; ++f) {
                own_leaf[l][f] = 1;
                for (int e = Lv.idx_ptr[f]; e < Lv.idx_ptr[f + 1]; ++e) own_pt[Lv.idx[e]] = 1;
            }
            const int64_t nn = int64_t(Lv.keys.size());
            own_par_b[l] = sfmm::shard_begin(nn, count, index);
            own_par_e[l] = sfmm::shard_end(nn, count, index);
        }
    }

    // The stages of the sharded solve; the caller sums every level's M
    // across shards after stage 0 and every level's L after stage 1.
    void stage(int s, const double* Q, double* U)
    {
        const int D = T.depth;
        if (s == 0) {
            M.assign(D + 1, {});
            L.assign(D + 1, {});
            if (D >= 2) {
                precompute();
                for (int l = 0; l <= D; ++l) {
                    M[l].assign(T.lv[l].keys.size() * n2 * nc, 0);
                    L[l].assign(T.lv[l].keys.size() * n2 * nc, 0);
                }
                for (int l = D; l >= 2; --l) N2M(l, Q);
            }
        } else if (s == 1) {
            if (D >= 2) {
                for (int l = D - 1; l >= 2; --l) M2M(l);
                for (int l = 2; l <= D; ++l) M2L(l);
            }
        } else {
            if (D >= 2) {
                for (int l = 2; l < D; ++l) {
                    L2N(l, U);
                    L2L(l + 1);
                }
                L2N(D, U);
            }
            N2N(Q, U);
        }
    }
};

}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" {

int oracle_cube(const double* pos, int64_t n, int vertical_axis, double phideg, double* out4)
{
    if (n <= 0) return -1;
    const Cube b = make_cube(pos, n, vertical_axis, phideg);
    out4[0] = b.width;
    for (int a = 0; a < 3; ++a) out4[1 + a] = b.corner[a];
    return 0;
}

int64_t oracle_key(const double* pos, int64_t n, int vertical_axis, double phideg, int level, int64_t* keys)
{
    const Cube b = make_cube(pos, n, vertical_axis, phideg);
    for (int64_t i = 0; i < n; ++i) keys[i] = b.key(level, pos + 3 * i);
    return n;
}

void* oracle_tree_build(const double* pos, int64_t n, int max_level, int max_ppn, int vertical_axis, double phideg)
{
    return build_tree(pos, n, max_level, max_ppn, vertical_axis, phideg);
}

void* oracle_tree_build_box(const double* pos, int64_t n, int max_level, int max_ppn, int vertical_axis,
                            double phideg, const double* box4)
{
    return build_tree(pos, n, max_level, max_ppn, vertical_axis, phideg, box4);
}

void oracle_tree_free(void* t) { delete static_cast<Tree*>(t); }

int oracle_tree_depth(void* t) { return static_cast<Tree*>(t)->depth; }

// what: 0 keys, 1 leaf nodes, 2 idx ptr, 3 idx, 4 ilist ptr, 5 ilist (src,di,dj,dk),
//       6 clist ptr, 7 clist (idx,key) as int64 pairs, 8 plist (idx,key) int64 pairs,
//       9 nlist ptr, 10 nlist (level, leaf), 11 partitions (level, leaf) per point
int64_t oracle_tree_export(void* tp, int l, int what, void* out)
{
    const Tree& T = *static_cast<Tree*>(tp);
    if (what == 11) {
        if (out) for (int64_t i = 0; i < T.n; ++i) { static_cast<int*>(out)[2 * i] = T.part[i].first; static_cast<int*>(out)[2 * i + 1] = T.part[i].second; }
        return 2 * T.n;
    }
    if (l < 0 || l > T.depth) return -1;
    const Level& L = T.lv[l];
    auto copy_i = [&](const std::vector<int>& v) -> int64_t { if (out) std::memcpy(out, v.data(), v.size() * 4); return int64_t(v.size()); };
    switch (what) {
    case 0: if (out) std::memcpy(out, L.keys.data(), L.keys.size() * 8); return int64_t(L.keys.size());
    case 1: return copy_i(L.leaf_node);
    case 2: return copy_i(L.idx_ptr);
    case 3: return copy_i(L.idx);
    case 4: return l >= 2 ? copy_i(L.il_ptr) : 0;
    case 5:
        if (out) for (size_t e = 0; e < L.il_src.size(); ++e) {
            int* o = static_cast<int*>(out) + 4 * e;
            o[0] = L.il_src[e]; o[1] = L.il_d[e].i; o[2] = L.il_d[e].j; o[3] = L.il_d[e].k;
        }
        return int64_t(4 * L.il_src.size());
    case 6: return l < T.depth ? copy_i(L.cl_ptr) : 0;
    case 7:
        if (out) for (size_t e = 0; e < L.cl_idx.size(); ++e) { static_cast<int64_t*>(out)[2 * e] = L.cl_idx[e]; static_cast<int64_t*>(out)[2 * e + 1] = L.cl_key[e]; }
        return int64_t(2 * L.cl_idx.size());
    case 8:
        if (out) for (size_t e = 0; e < L.pl_idx.size(); ++e) { static_cast<int64_t*>(out)[2 * e] = L.pl_idx[e]; static_cast<int64_t*>(out)[2 * e + 1] = L.keys[e]; }
        return int64_t(2 * L.pl_idx.size());
    case 9: return copy_i(L.nl_ptr);
    case 10:
        if (out) for (size_t e = 0; e < L.nl.size(); ++e) { static_cast<int*>(out)[2 * e] = L.nl[e].first; static_cast<int*>(out)[2 * e + 1] = L.nl[e].second; }
        return int64_t(2 * L.nl.size());
    default: return -1;
    }
}

// mode 0: rinv (potential), Q/U have ncomp components per point;
// mode 1: rinv<true> (Q x grad form), ncomp must be 3.  U is accumulated.
int oracle_rinv(void* tp, int p, int mode, int ncomp, const double* Q, double* U)
{
    if (p < 0 || p > 30 || (mode == 1 && ncomp != 3) || ncomp < 1) return -1;
    const Tree& T = *static_cast<Tree*>(tp);
    const Tables tb = make_tables(p);
    Eval ev{T, tb, p, (p + 1) * (p + 1), ncomp, mode == 1, {}, {}, {}, {}, {}, {}, {}, {}, {}};
    ev.rinv(Q, U);
    return 0;
}

// Sharded stages (the library's fmm_plan_set_shard / fmm_evaluate_stage,
// restated): an evaluator object keeps M and L between stages.
struct StagedEval {
    Tables tb;
    Eval ev;
    StagedEval(const Tree& T, int p, int mode, int ncomp)
        : tb(make_tables(p)), ev{T, tb, p, (p + 1) * (p + 1), ncomp, mode == 1, {}, {}, {}, {}, {}, {}, {}, {}, {}}
    {
    }
};

void* oracle_eval_create(void* tp, int p, int mode, int ncomp)
{
    if (p < 0 || p > 30 || (mode == 1 && ncomp != 3) || ncomp < 1) return nullptr;
    return new StagedEval(*static_cast<Tree*>(tp), p, mode, ncomp);
}

void oracle_eval_free(void* e) { delete static_cast<StagedEval*>(e); }

int oracle_eval_set_shard(void* e, int index, int count)
{
    if (count < 1 || index < 0 || index >= count) return -1;
    static_cast<StagedEval*>(e)->ev.set_shard(index, count);
    return 0;
}

int oracle_eval_stage(void* e, int stage, const double* Q, double* U)
{
    if (stage < 0 || stage > 2) return -1;
    static_cast<StagedEval*>(e)->ev.stage(stage, Q, U);
    return 0;
}

// Level l's moments (which 0) or locals (which 1) as count doubles (complex
// pairs), for the caller's sum across shards; NULL if not allocated.
double* oracle_eval_buffer(void* e, int which, int l, int64_t* count)
{
    Eval& ev = static_cast<StagedEval*>(e)->ev;
    auto& v = which == 0 ? ev.M : ev.L;
    if (l < 0 || l >= int(v.size())) {
        *count = 0;
        return nullptr;
    }
    *count = int64_t(v[l].size()) * 2;
    return reinterpret_cast<double*>(v[l].data());
}

// O(N^2)-per-target direct sums (main.cpp:70-96) for the listed targets:
// mode 0 potential sum_j q_j/|R| (ncomp comps), mode 1 sum_j Q_j x R/|R|^3
// (ncomp 3), mode 2 scalar-charge field sum_j q_j R/|R|^3 (ncomp 1, 3 outputs),
// mode 3 the magnitude sums (sum_j |Q_j|/|R|, sum_j |Q_j|/|R|^2) that scale
// the rounding error of the potential and of the field at each target.
int oracle_direct(const double* pos, int64_t n, int mode, int ncomp, const double* Q,
                  const int64_t* targets, int64_t nt, double* out)
{
    const int nout = mode == 2 ? 3 : mode == 3 ? 2 : ncomp;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < nt; ++t) {
        const int64_t i = targets[t];
        std::vector<double> acc(nout, 0.0);
        for (int64_t j = 0; j < n; ++j) {
            if (j == i) continue;
            const double R[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
            const double r = std::sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]);
            if (mode == 0) {
                for (int c = 0; c < ncomp; ++c) acc[c] += Q[j * ncomp + c] / r;
            } else if (mode == 1) {
                const double* q = &Q[3 * j];
                const double r3 = r * r * r;
                acc[0] += (q[1] * R[2] - q[2] * R[1]) / r3;
                acc[1] += (q[2] * R[0] - q[0] * R[2]) / r3;
                acc[2] += (q[0] * R[1] - q[1] * R[0]) / r3;
            } else if (mode == 2) {
                const double s = Q[j] / (r * r * r);
                for (int a = 0; a < 3; ++a) acc[a] += s * R[a];
            } else {
                double qq = 0;
                for (int c = 0; c < ncomp; ++c) qq += Q[j * ncomp + c] * Q[j * ncomp + c];
                acc[0] += std::sqrt(qq) / r;
                acc[1] += std::sqrt(qq) / (r * r);
            }
        }
        for (int c = 0; c < nout; ++c) out[t * nout + c] = acc[c];
    }
    return 0;
}

}  // extern "C"
