// The reference's example driver flow (main.cpp:22-111) written against the
// header-only facade: vector charges, rinv and rinv<true>, then the relative
// L2 error against a direct sum on a subset of targets; and (argument
// "exclude") the self_generator / is_self forms on a given input, whose
// outputs tests/test_facade.py compares with the reference's.  Built and run
// by tests/test_facade.py on a GPU.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

#include "simplefmm_b200.hpp"

using namespace simplefmm_b200;

constexpr size_t N = 20000;
constexpr int dim = 3;
using Vector_t = Vector<double, dim>;

// Exclusion forms through the facade (fmm.hpp:204, 398-408, 773-807):
// FMM3D(partitioner, comm, self_generator) with self_generator(i) =
// {i, i+s1, i+s2} (mod n), then rinv(Q, U, is_self) with the matching
// is_self (near_too = 1) or rinv(Q, U) (near_too = 0), for the potential
// (N = 1) and, as the reference's driver forms it, the field of scalar
// charges from two rinv<true> runs with Q = (q,0,0) and (0,0,q).
// Input file: int64 n, int32 max_ppn, s1, s2, near_too, double pos[3n],
// double q[n]; output: double pot[n], field[3n].
static int run_exclusions(const char* in_path, const char* out_path)
{
    FILE* f = std::fopen(in_path, "rb");
    if (!f) return 2;
    int64_t n = 0;
    int32_t hdr[4] = {0, 0, 0, 0};
    if (std::fread(&n, 8, 1, f) != 1 || std::fread(hdr, 4, 4, f) != 4) return 2;
    const int ppn = hdr[0], s1 = hdr[1], s2 = hdr[2], near_too = hdr[3];
    std::vector<Vector<double, 3>> pos(n);
    std::vector<double> q(n);
    if (std::fread(pos.data(), 24, n, f) != size_t(n) || std::fread(q.data(), 8, n, f) != size_t(n)) return 2;
    std::fclose(f);
    Box<double, 3, Vector> box(pos, 2);
    OctreePartitioner<double, Vector> part(pos, box);
    part.refine(20, ppn);
    const int nn = static_cast<int>(n);
    auto gen = [&](int i) { return std::vector<int>{i, (i + s1) % nn, (i + s2) % nn}; };
    auto is_self = [&](int i, int j) { return j == i || j == (i + s1) % nn || j == (i + s2) % nn; };
    FMM3D<double, 1, 6, Vector> fmm1(part, 0, gen);
    std::vector<Vector<double, 1>> Q1(n), U(n, Vector<double, 1>{{0.0}});
    for (int64_t i = 0; i < n; ++i) Q1[i] = Vector<double, 1>{{q[i]}};
    if (near_too) fmm1.rinv(Q1.data(), U.data(), is_self);
    else fmm1.rinv(Q1.data(), U.data());
    FMM3D<double, 3, 6, Vector, true> fmm3(part, 0, gen);
    std::vector<Vector<double, 3>> Qx(n), Qz(n), Ux(n, Vector<double, 3>{{0, 0, 0}}), Uz(n, Vector<double, 3>{{0, 0, 0}});
    for (int64_t i = 0; i < n; ++i) {
        Qx[i] = Vector<double, 3>{{q[i], 0.0, 0.0}};
        Qz[i] = Vector<double, 3>{{0.0, 0.0, q[i]}};
    }
    if (near_too) {
        fmm3.rinv<true>(Qx.data(), Ux.data(), is_self);
        fmm3.rinv<true>(Qz.data(), Uz.data(), is_self);
    } else {
        fmm3.rinv<true>(Qx.data(), Ux.data());
        fmm3.rinv<true>(Qz.data(), Uz.data());
    }
    FILE* o = std::fopen(out_path, "wb");
    if (!o) return 2;
    for (int64_t i = 0; i < n; ++i) std::fwrite(&U[i][0], 8, 1, o);
    for (int64_t i = 0; i < n; ++i) {
        const double E[3] = {Uz[i][1], -Uz[i][0], -Ux[i][1]};
        std::fwrite(E, 8, 3, o);
    }
    std::fclose(o);
    std::printf("exclusions ok: n %lld depth %d\n", static_cast<long long>(n), part.level());
    return 0;
}

int main(int argc, char** argv)
{
    if (argc == 4 && std::string(argv[1]) == "exclude") return run_exclusions(argv[2], argv[3]);
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    std::vector<Vector_t> positions(N), charges(N);
    for (size_t i = 0; i < N; ++i) {
        positions[i] = Vector_t{{u(rng), u(rng), u(rng)}};
        charges[i] = Vector_t{{u(rng), u(rng), u(rng)}};
    }
    Box<double, dim, Vector> box(positions, 2);
    OctreePartitioner<double, Vector> partitioner(positions, box);
    partitioner.refine(20, 128);
    FMM3D<double, dim, 8, Vector, true> fmm(partitioner, 0);
    std::vector<Vector_t> pot(N, Vector_t{{0, 0, 0}}), fld(N, Vector_t{{0, 0, 0}});
    fmm.rinv(charges.data(), pot.data());
    fmm.rinv<true>(charges.data(), fld.data());
    double np = 0, dp = 0, nf = 0, df = 0;
    for (size_t i = 0; i < N; i += 97) {
        double P[3] = {0, 0, 0}, F[3] = {0, 0, 0};
        for (size_t j = 0; j < N; ++j) {
            if (i == j) continue;
            const double R[3] = {positions[i][0] - positions[j][0], positions[i][1] - positions[j][1],
                                 positions[i][2] - positions[j][2]};
            const double r = std::sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]);
            const double* q = charges[j].data();
            for (int a = 0; a < 3; ++a) P[a] += q[a] / r;
            F[0] += (q[1] * R[2] - q[2] * R[1]) / (r * r * r);
            F[1] += (q[2] * R[0] - q[0] * R[2]) / (r * r * r);
            F[2] += (q[0] * R[1] - q[1] * R[0]) / (r * r * r);
        }
        for (int a = 0; a < 3; ++a) {
            np += (P[a] - pot[i][a]) * (P[a] - pot[i][a]);
            dp += P[a] * P[a];
            nf += (F[a] - fld[i][a]) * (F[a] - fld[i][a]);
            df += F[a] * F[a];
        }
    }
    std::printf("depth %d width %.6f\n", partitioner.level(), box.width());
    std::printf("Relative l2 error of potential = %.3e\n", std::sqrt(np / dp));
    std::printf("Relative l2 error of field = %.3e\n", std::sqrt(nf / df));
    return (std::sqrt(np / dp) < 1e-4 && std::sqrt(nf / df) < 1e-3) ? 0 : 1;
}
