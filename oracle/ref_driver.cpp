// Driver around the UNMODIFIED reference headers (compiled from the read-only
// reference checkout by oracle/Makefile; nothing here is shipped).
//
// It performs the reference's own API sequence (main.cpp:36-68):
//   Box(positions, vertical_axis, phideg)            box.hpp:84-107
//   OctreePartitioner(positions, box).refine(L, ppn)  partition.hpp:397-446
//   FMM3D<double, N, p, Vector, grad>(part, comm)     fmm.hpp:204-427
//   rinv / rinv<true>                                 fmm.hpp:864-881
// followed by MPI_Allreduce of U (main.cpp:62), and dumps what the tests
// compare against: the box, every per-level list, and U.
//
// Input  (little-endian): "SFMMIN01", int64 n, int32 p, max_level, max_ppn,
//        vertical_axis, double phideg, int32 qdim, int32 flags,
//        double pos[3n], double q[qdim*n].
// flags: 1 tree dump, 2 scalar potential (qdim 1), 4 scalar field via two
//        rinv<true> runs with Q=(q,0,0),(0,0,q) (qdim 1), 8 vector potential
//        (qdim 3), 16 rinv<true> with vector charges (qdim 3), 32 skip the
//        evaluation, only time the tree, 64 explicit cube (Box(corner, width,
//        vertical_axis, phideg), box.hpp:73-82): double corner[3], width follow
//        the charges, 128 / 256 exclusions: int32 s1, s2 follow (after the
//        cube if any); FMM3D gets self_generator(i) = {i, (i+s1)%n, (i+s2)%n}
//        (fmm.hpp:204, 398-408) and rinv runs with the matching is_self (128)
//        or with the default is_self i == j, so only the non-neighbour
//        exclusions (slist) are removed (256).
// Output: "SFMMOUT1" then sections: char tag[8], int64 nbytes, payload.
#include <mpi.h>

#include "box.hpp"
#include "fmm.hpp"
#include "matrix.hpp"
#include "partition.hpp"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#ifndef REF_P
#define REF_DRIVER_MAIN 1
#endif

using V3 = Vector<double, 3>;
using V1 = Vector<double, 1>;
using Part = OctreePartitioner<double, Vector>;
using BoxT = Box<double, 3, Vector>;

struct Out {
    FILE* f = nullptr;
    void section(const char* tag, const void* data, int64_t nbytes)
    {
        if (!f) return;
        char t[8] = {0};
        std::strncpy(t, tag, 8);
        std::fwrite(t, 1, 8, f);
        std::fwrite(&nbytes, 8, 1, f);
        if (nbytes) std::fwrite(data, 1, static_cast<size_t>(nbytes), f);
    }
    void scalar(const char* tag, double v) { section(tag, &v, 8); }
    template<typename T>
    void vec(const char* tag, const std::vector<T>& v) { section(tag, v.data(), int64_t(v.size() * sizeof(T))); }
};

inline double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

inline double timed_barrier()
{
    MPI_Barrier(MPI_COMM_WORLD);
    return now_s();
}

struct Job {
    int64_t n;
    int p, max_level, max_ppn, vertical_axis;
    double phideg;
    int qdim, flags;
    std::vector<V3> pos;
    std::vector<double> q;
    double corner[3] = {0, 0, 0}, width = 0;
    int s1 = 0, s2 = 0;

    std::vector<int> self(int i) const
    {
        if (!(flags & (128 | 256))) return {i};
        const int n = static_cast<int>(this->n);
        return {i, (i + s1) % n, (i + s2) % n};
    }
    bool is_self(int i, int j) const
    {
        if (!(flags & 128)) return i == j;
        const int n = static_cast<int>(this->n);
        return j == i || j == (i + s1) % n || j == (i + s2) % n;
    }
};

// per-p evaluation entry points (one translation unit per p, see Makefile)
#define DECL(P) void run_p##P(const Job&, const Part&, Out&, int rank);
DECL(2) DECL(3) DECL(4) DECL(5) DECL(6) DECL(7) DECL(8) DECL(9) DECL(10) DECL(11) DECL(12) DECL(13) DECL(16)
#undef DECL

template<int p>
void run_p(const Job& job, const Part& part, Out& out, int rank)
{
    const size_t n = static_cast<size_t>(job.n);
    if (job.flags & 2) {
        double t0 = timed_barrier();
        FMM3D<double, 1, p, Vector> fmm(part, MPI_COMM_WORLD, [&](int i) { return job.self(i); });
        double t1 = timed_barrier();
        std::vector<V1> Q(n), U(n);
        for (size_t i = 0; i < n; ++i) { Q[i][0] = job.q[i]; U[i][0] = 0; }
        double t2 = timed_barrier();
        fmm.rinv(Q.data(), U.data(), [&](int i, int j) { return job.is_self(i, j); });
        MPI_Allreduce(MPI_IN_PLACE, U.data(), int(n), MPI_DOUBLE, MPI_SUM, MPI_COMM_WORLD);
        double t3 = timed_barrier();
        if (rank == 0) {
            out.scalar("T_CTOR1", t1 - t0);
            out.scalar("T_POT", t3 - t2);
            out.section("POT", U.data(), int64_t(n * 8));
        }
    }
    if ((job.flags & 4) || (job.flags & 16)) {
        double t0 = timed_barrier();
        FMM3D<double, 3, p, Vector, true> fmm(part, MPI_COMM_WORLD, [&](int i) { return job.self(i); });
        double t1 = timed_barrier();
        if (rank == 0) out.scalar("T_CTOR3G", t1 - t0);
        std::vector<V3> Q(n), U(n);
        if (job.flags & 4) {
            std::vector<double> E(3 * n);
            double tt = 0;
            for (int run = 0; run < 2; ++run) {
                for (size_t i = 0; i < n; ++i) {
                    Q[i] = V3{{run == 0 ? job.q[i] : 0.0, 0.0, run == 1 ? job.q[i] : 0.0}};
                    U[i] = V3{{0, 0, 0}};
                }
                double t2 = timed_barrier();
                fmm.template rinv<true>(Q.data(), U.data(), [&](int i, int j) { return job.is_self(i, j); });
                MPI_Allreduce(MPI_IN_PLACE, U.data(), int(3 * n), MPI_DOUBLE, MPI_SUM, MPI_COMM_WORLD);
                double t3 = timed_barrier();
                tt += t3 - t2;
                for (size_t i = 0; i < n; ++i) {
                    if (run == 0) {
                        E[3 * i + 2] = -U[i][1];          // Q=(q,0,0): Q x R = (0, -qRz, qRy)
                    } else {
                        E[3 * i + 0] = U[i][1];           // Q=(0,0,q): Q x R = (-qRy, qRx, 0)
                        E[3 * i + 1] = -U[i][0];
                    }
                }
            }
            if (rank == 0) {
                out.scalar("T_FIELD", tt);
                out.vec("FIELD", E);
            }
        }
        if (job.flags & 16) {
            for (size_t i = 0; i < n; ++i) {
                Q[i] = V3{{job.q[3 * i], job.q[3 * i + 1], job.q[3 * i + 2]}};
                U[i] = V3{{0, 0, 0}};
            }
            double t2 = timed_barrier();
            fmm.template rinv<true>(Q.data(), U.data(), [&](int i, int j) { return job.is_self(i, j); });
            MPI_Allreduce(MPI_IN_PLACE, U.data(), int(3 * n), MPI_DOUBLE, MPI_SUM, MPI_COMM_WORLD);
            double t3 = timed_barrier();
            if (rank == 0) {
                out.scalar("T_BIOT", t3 - t2);
                out.section("BIOT", U.data(), int64_t(n * 24));
            }
        }
    }
    if (job.flags & 8) {
        double t0 = timed_barrier();
        FMM3D<double, 3, p, Vector> fmm(part, MPI_COMM_WORLD);
        double t1 = timed_barrier();
        std::vector<V3> Q(n), U(n);
        for (size_t i = 0; i < n; ++i) {
            Q[i] = V3{{job.q[3 * i], job.q[3 * i + 1], job.q[3 * i + 2]}};
            U[i] = V3{{0, 0, 0}};
        }
        double t2 = timed_barrier();
        fmm.rinv(Q.data(), U.data());
        MPI_Allreduce(MPI_IN_PLACE, U.data(), int(3 * n), MPI_DOUBLE, MPI_SUM, MPI_COMM_WORLD);
        double t3 = timed_barrier();
        if (rank == 0) {
            out.scalar("T_CTOR3", t1 - t0);
            out.scalar("T_VECPOT", t3 - t2);
            out.section("VECPOT", U.data(), int64_t(n * 24));
        }
    }
}

#ifdef REF_P
#define INST2(P) void run_p##P(const Job& j, const Part& t, Out& o, int r) { run_p<P>(j, t, o, r); }
#define INST(P) INST2(P)
INST(REF_P)
#endif

#ifdef REF_DRIVER_MAIN
static void dump_tree(const Part& part, const BoxT& box, Out& out, int64_t n)
{
    const double bx[4] = {box.width(), box.corner()[0], box.corner()[1], box.corner()[2]};
    out.section("BOX", bx, sizeof(bx));
    const int depth = part.level();
    for (int l = 0; l <= depth; ++l) {
        const auto& lv = part.octreeLevel(l);
        const std::string s = std::to_string(l);
        out.vec(("CNODE" + s).c_str(), lv.c_node());
        std::vector<int> ileaf;
        for (int i = 0; i < lv.n_leaf(); ++i) ileaf.push_back(lv.from_leaf(i));
        out.vec(("ILEAF" + s).c_str(), ileaf);
        // leaf -> particle CSR (partition.hpp:192-210)
        std::vector<int> rp{0}, v;
        for (int i = 0; i < lv.n_leaf(); ++i) {
            for (int k = 0; k < lv.indices().nnz(i); ++k) v.push_back(std::get<0>(lv.indices().value(i, k)));
            rp.push_back(int(v.size()));
        }
        out.vec(("IDXP" + s).c_str(), rp);
        out.vec(("IDXV" + s).c_str(), v);
        if (l >= 2) {
            std::vector<int> irp{0}, iv;
            const auto& il = lv.ilist();
            for (int i = 0; i < lv.n_node(); ++i) {
                for (int k = 0; k < il.nnz(i); ++k) {
                    const auto& e = il.value(i, k);
                    const auto& d = std::get<1>(e);
                    iv.push_back(std::get<0>(e));
                    iv.push_back(d.i);
                    iv.push_back(d.j);
                    iv.push_back(d.k);
                }
                irp.push_back(int(iv.size() / 4));
            }
            out.vec(("ILP" + s).c_str(), irp);
            out.vec(("ILV" + s).c_str(), iv);
        }
        if (l < depth) {
            std::vector<int> crp{0};
            std::vector<int64_t> cv;
            const auto& cl = lv.clist();
            for (int i = 0; i < lv.n_node(); ++i) {
                for (int k = 0; k < cl.nnz(i); ++k) {
                    cv.push_back(std::get<0>(cl.value(i, k)));
                    cv.push_back(std::get<1>(cl.value(i, k)));
                }
                crp.push_back(int(cv.size() / 2));
            }
            out.vec(("CLP" + s).c_str(), crp);
            out.vec(("CLV" + s).c_str(), cv);
        }
        if (l >= 1) {
            std::vector<int64_t> pv;
            for (const auto& e : lv.plist()) { pv.push_back(e.first); pv.push_back(e.second); }
            out.vec(("PL" + s).c_str(), pv);
        }
        std::vector<int> nrp{0}, nv;
        const auto& nl = lv.nlist();
        for (int i = 0; i < lv.n_leaf(); ++i) {
            for (int k = 0; k < nl.nnz(i); ++k) {
                nv.push_back(std::get<0>(nl.value(i, k)));
                nv.push_back(std::get<1>(nl.value(i, k)));
            }
            nrp.push_back(int(nv.size() / 2));
        }
        out.vec(("NLP" + s).c_str(), nrp);
        out.vec(("NLV" + s).c_str(), nv);
    }
    std::vector<int> parts;
    for (int64_t i = 0; i < n; ++i) {
        const auto& pr = part.get_partition(int(i));
        parts.push_back(pr.first);
        parts.push_back(pr.second);
    }
    out.vec("PARTS", parts);
}

int main(int argc, char** argv)
{
    MPI_Init(&argc, &argv);
    int rank = 0, size = 1;
    MPI_Comm_rank(MPI_COMM_WORLD, &rank);
    MPI_Comm_size(MPI_COMM_WORLD, &size);
    if (argc < 3) {
        if (rank == 0) std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
        MPI_Finalize();
        return 2;
    }
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) { std::fprintf(stderr, "cannot open %s\n", argv[1]); return 2; }
    char magic[8];
    Job job;
    int32_t hdr[4];
    bool ok = std::fread(magic, 1, 8, in) == 8 && std::memcmp(magic, "SFMMIN01", 8) == 0;
    ok = ok && std::fread(&job.n, 8, 1, in) == 1 && std::fread(hdr, 4, 4, in) == 4;
    job.p = hdr[0]; job.max_level = hdr[1]; job.max_ppn = hdr[2]; job.vertical_axis = hdr[3];
    int32_t qf[2];
    ok = ok && std::fread(&job.phideg, 8, 1, in) == 1 && std::fread(qf, 4, 2, in) == 2;
    job.qdim = qf[0]; job.flags = qf[1];
    std::vector<double> raw(static_cast<size_t>(job.n) * 3);
    ok = ok && std::fread(raw.data(), 8, raw.size(), in) == raw.size();
    job.q.resize(static_cast<size_t>(job.n) * job.qdim);
    ok = ok && std::fread(job.q.data(), 8, job.q.size(), in) == job.q.size();
    if (ok && (job.flags & 64)) {
        double cw[4];
        ok = std::fread(cw, 8, 4, in) == 4;
        job.corner[0] = cw[0]; job.corner[1] = cw[1]; job.corner[2] = cw[2]; job.width = cw[3];
    }
    if (ok && (job.flags & (128 | 256))) {
        int32_t ss[2];
        ok = std::fread(ss, 4, 2, in) == 2;
        job.s1 = ss[0]; job.s2 = ss[1];
    }
    std::fclose(in);
    if (!ok) { std::fprintf(stderr, "bad input file\n"); return 2; }
    job.pos.resize(static_cast<size_t>(job.n));
    for (int64_t i = 0; i < job.n; ++i) job.pos[i] = V3{{raw[3 * i], raw[3 * i + 1], raw[3 * i + 2]}};

    Out out;
    if (rank == 0) {
        out.f = std::fopen(argv[2], "wb");
        if (!out.f) { std::fprintf(stderr, "cannot open %s\n", argv[2]); return 2; }
        std::fwrite("SFMMOUT1", 1, 8, out.f);
    }
    const double t0 = timed_barrier();
    BoxT box = (job.flags & 64) ? BoxT(V3{{job.corner[0], job.corner[1], job.corner[2]}}, job.width, job.vertical_axis,
                                       job.phideg)
                                  : BoxT(job.pos, job.vertical_axis, job.phideg);
    Part part(job.pos, box);
    part.refine(job.max_level, job.max_ppn);
    const double t1 = timed_barrier();
    if (rank == 0) out.scalar("T_TREE", t1 - t0);
    const int32_t info[2] = {part.level(), size};
    if (rank == 0) out.section("DEPTH", info, sizeof(info));
    if (rank == 0 && (job.flags & 1)) dump_tree(part, box, out, job.n);
    if (!(job.flags & 32)) {
        switch (job.p) {
#define CASE(P) case P: run_p##P(job, part, out, rank); break;
            CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9) CASE(10) CASE(11) CASE(12) CASE(13)
            CASE(16)
#undef CASE
        default:
            if (rank == 0) std::fprintf(stderr, "unsupported p=%d\n", job.p);
            return 2;
        }
    }
    if (rank == 0) std::fclose(out.f);
    MPI_Finalize();
    return 0;
}
#endif
