// The reference's example driver flow (main.cpp:22-111) written against the
// header-only facade: vector charges, rinv and rinv<true>, then the relative
// L2 error against a direct sum on a subset of targets.  Built and run by
// tests/test_facade.py on a GPU.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "simplefmm_b200.hpp"

using namespace simplefmm_b200;

constexpr size_t N = 20000;
constexpr int dim = 3;
using Vector_t = Vector<double, dim>;

int main()
{
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

// Compile-time check of the rest of the facade API (explicit cube,
// self_generator / is_self); exercised through the C ABI by the GPU tests.
[[maybe_unused]] static void facade_api_compiles(std::vector<Vector<double, 3>>& pos, std::vector<Vector<double, 1>>& q,
                                                 std::vector<Vector<double, 1>>& u)
{
    Box<double, 3, Vector> box(Vector<double, 3>{{0.0, 0.0, 0.0}}, 1.0, 2, 0.0);
    OctreePartitioner<double, Vector> part(pos, box);
    part.refine(20, 64);
    FMM3D<double, 1, 6, Vector> fmm(part, 0, [](int i) { return std::vector<int>{i, i + 1}; });
    fmm.rinv(q.data(), u.data());
    fmm.rinv(q.data(), u.data(), [](int i, int j) { return j == i || j == i + 1; });
}
