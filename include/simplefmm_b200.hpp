// Header-only C++ facade with the reference library's API (SimpleFMM,
// box.hpp / partition.hpp / fmm.hpp), implemented over the C ABI of
// simplefmm_b200.h.  Code written against the reference compiles against
// this header with the same class names, template parameters, constructor
// arguments and rinv / rinv<true> calls:
//
//   Box<double, 3, Vector> box(positions, vertical_axis);            // box.hpp:84
//   OctreePartitioner<double, Vector> part(positions, box);           // partition.hpp:397
//   part.refine(max_level, max_particles_per_node);                   // partition.hpp:406
//   FMM3D<double, N, p, Vector, grad> fmm(part, MPI_COMM_WORLD);      // fmm.hpp:423
//   fmm.rinv(Q, U);  fmm.rinv<true>(Q, U);                            // fmm.hpp:864-881
//
// Differences: the communicator argument is accepted and ignored (one GPU
// holds the whole problem, so every rank would compute the full U; call it
// on one rank or skip the MPI_Allreduce of main.cpp:62); failures throw
// simplefmm_b200::Error instead of being silently ignored.  U is accumulated
// exactly as in the reference.
#pragma once

#include <array>
#include <cstddef>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "simplefmm_b200.h"

namespace simplefmm_b200 {

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(int rc)
{
    if (rc != FMM_OK) throw Error(rc, std::string(fmm_status_string(rc)) + ": " + fmm_last_error());
}

// Minimal fixed-size vector with the memory layout of the reference's
// Vector<T, N> (matrix.hpp:164-165: a std::array of N elements).
template<typename T, size_t N>
struct Vector : std::array<T, N> {};

// One process-wide context per device, created on first use.
inline fmm_context* default_context(int device = 0)
{
    struct Holder {
        fmm_context* c = nullptr;
        ~Holder() { if (c) fmm_context_destroy(c); }
    };
    static Holder h;
    if (!h.c) check(fmm_context_create(device, &h.c));
    return h.c;
}

template<typename T, int dim, template<typename, size_t> typename Container>
class Box {
    static_assert(dim == 3, "the FMM is three-dimensional");
    static_assert(sizeof(Container<T, dim>) == dim * sizeof(double), "positions must be 3 contiguous doubles");

public:
    using Coord_t = Container<T, dim>;

    Box(const std::vector<Coord_t>& positions, int vertical_axis = dim - 1, T phideg = 0)
        : positions_(&positions), vertical_axis_(vertical_axis), phideg_(phideg) {}
    // box.hpp:73-82: the cube given explicitly (corner in the rotated frame)
    Box(const Coord_t& corner, T width, int vertical_axis = dim - 1, T phideg = 0)
        : positions_(nullptr), vertical_axis_(vertical_axis), phideg_(phideg), explicit_(true), width0_(width)
    {
        for (int a = 0; a < dim; ++a) corner0_[a] = corner[a];
    }

    int vertical_axis() const noexcept { return vertical_axis_; }
    T phideg() const noexcept { return phideg_; }
    bool is_explicit() const noexcept { return explicit_; }
    const double* explicit_corner() const noexcept { return corner0_; }
    double explicit_width() const noexcept { return width0_; }
    // box.hpp:109-117; available once a partitioner has refined the tree
    T width() const { need(); double w, c[3]; check(fmm_tree_box(tree_, &w, c)); return w; }
    Coord_t corner() const
    {
        need();
        double w, c[3];
        check(fmm_tree_box(tree_, &w, c));
        Coord_t r;
        for (int a = 0; a < 3; ++a) r[a] = c[a];
        return r;
    }
    void attach(const fmm_tree* t) const noexcept { tree_ = t; }

private:
    void need() const { if (!tree_) throw Error(FMM_ERR_INVALID_ARGUMENT, "the box is computed by OctreePartitioner::refine"); }
    const std::vector<Coord_t>* positions_;
    int vertical_axis_;
    T phideg_;
    bool explicit_ = false;
    double corner0_[3] = {0, 0, 0}, width0_ = 0;
    mutable const fmm_tree* tree_ = nullptr;
};

template<typename T, template<typename, size_t> typename Container>
class OctreePartitioner {
public:
    using Coord_t = Container<T, 3>;
    using Box_t = Box<T, 3, Container>;

    OctreePartitioner(const std::vector<Coord_t>& positions, const Box_t& box) : positions_(positions), box_(box) {}

    void refine(int max_level = 20, int max_particles_per_node = 64)
    {
        fmm_tree* t = nullptr;
        const double* xyz = reinterpret_cast<const double*>(positions_.data());
        const int64_t n = static_cast<int64_t>(positions_.size());
        if (box_.is_explicit())
            check(fmm_tree_build_box(default_context(), xyz, n, FMM_HOST, box_.explicit_corner(), box_.explicit_width(),
                                     max_level, max_particles_per_node, box_.vertical_axis(),
                                     static_cast<double>(box_.phideg()), &t));
        else
            check(fmm_tree_build(default_context(), xyz, n, FMM_HOST, max_level, max_particles_per_node,
                                 box_.vertical_axis(), static_cast<double>(box_.phideg()), &t));
        tree_.reset(t);
        box_.attach(t);
    }

    int level() const { int d = 0; check(fmm_tree_depth(tree_.get(), &d)); return d; }
    const std::vector<Coord_t>& positions() const noexcept { return positions_; }
    const Box_t& box() const noexcept { return box_; }
    fmm_tree* handle() const noexcept { return tree_.get(); }

    // per-level node keys (OctreeLevel::c_node, partition.hpp:228-231)
    std::vector<int64_t> c_node(int l) const { return exported<int64_t>(l, FMM_EXPORT_NODE_KEYS); }
    // point -> (leaf level, leaf index) (partition.hpp:479-482)
    std::pair<int, int> get_partition(int i) const
    {
        const auto v = exported<int32_t>(0, FMM_EXPORT_PARTITIONS);
        return {v[2 * i], v[2 * i + 1]};
    }

private:
    template<typename I>
    std::vector<I> exported(int l, int what) const
    {
        int64_t n = 0;
        check(fmm_tree_export_size(tree_.get(), l, what, &n));
        std::vector<I> v(n > 0 ? n : 0);
        if (n > 0) check(fmm_tree_export(tree_.get(), l, what, v.data()));
        return v;
    }
    struct Del { void operator()(fmm_tree* t) const { fmm_tree_destroy(t); } };
    const std::vector<Coord_t>& positions_;
    const Box_t& box_;
    std::unique_ptr<fmm_tree, Del> tree_;
};

template<typename T, size_t N, int p, template<typename, size_t> typename Container, bool support_gradient = false>
class FMM3D {
    static_assert(N >= 1 && N <= 3, "N charge components: 1, 2 or 3");
    static_assert(p >= 0 && p <= 16, "expansion order 0..16");
    static_assert(sizeof(Container<T, N>) == N * sizeof(double), "charges must be N contiguous doubles");

public:
    using Partitioner_t = OctreePartitioner<T, Container>;

    template<typename Comm = int>
    explicit FMM3D(const Partitioner_t& partitioner, Comm = Comm{}, int precision = FMM_PRECISION_FP64)
        : n_(static_cast<int64_t>(partitioner.positions().size()))
    {
        fmm_plan* pl = nullptr;
        check(fmm_plan_create(partitioner.handle(), p, static_cast<int>(N), precision, &pl));
        plan_.reset(pl);
#ifdef FMM_M2L_DIRECT
        // the reference's build option for the dense M2L (fmm.hpp:700-712)
        check(fmm_plan_set_m2l(plan_.get(), FMM_M2L_METHOD_DIRECT));
#endif
    }

    // fmm.hpp:204, 398-408: self_generator(i) names the sources whose
    // interaction with target i is removed.  rinv(Q, U) removes those outside
    // i's near field (the reference's slist); rinv(Q, U, is_self) removes all
    // of them, and is_self must be true on every generated pair (other
    // is_self predicates are not supported: they are checked and rejected).
    template<typename Comm, typename Generator,
             typename = decltype(std::declval<Generator>()(0).size())>
    FMM3D(const Partitioner_t& partitioner, Comm comm, const Generator& self_generator,
          int precision = FMM_PRECISION_FP64)
        : FMM3D(partitioner, comm, precision)
    {
        ex_ptr_.assign(1, 0);
        for (int64_t i = 0; i < n_; ++i) {
            for (int j : self_generator(static_cast<int>(i))) ex_col_.push_back(j);
            ex_ptr_.push_back(static_cast<int64_t>(ex_col_.size()));
        }
        set_exclusions(0);
    }

    // fmm.hpp:864-881: U += sum_j Q_j / |x_i - x_j|  or (gradient) sum_j Q_j x R / |R|^3
    template<bool gradient = false>
    void rinv(const Container<T, N>* Q, Container<T, N>* U) const
    {
        static_assert(support_gradient || !gradient, "rinv<true> needs support_gradient (fmm.hpp:867)");
        static_assert(!gradient || N == 3, "rinv<true> needs N == 3 (fmm.hpp:550)");
        if (!ex_ptr_.empty()) set_exclusions(0);
        check(fmm_rinv(plan_.get(), reinterpret_cast<const double*>(Q), reinterpret_cast<double*>(U), gradient ? 1 : 0,
                       FMM_HOST));
    }

    // fmm.hpp:864-873 with a custom is_self (see the self_generator constructor)
    template<bool gradient = false, typename IsSelf>
    void rinv(const Container<T, N>* Q, Container<T, N>* U, const IsSelf& is_self) const
    {
        static_assert(support_gradient || !gradient, "rinv<true> needs support_gradient (fmm.hpp:867)");
        for (int64_t i = 0; i < n_; ++i) {
            if (!is_self(static_cast<int>(i), static_cast<int>(i)))
                throw Error(FMM_ERR_UNSUPPORTED, "is_self(i, i) must be true");
            for (int64_t e = ex_ptr_.empty() ? 0 : ex_ptr_[i]; e < (ex_ptr_.empty() ? 0 : ex_ptr_[i + 1]); ++e)
                if (!is_self(static_cast<int>(i), ex_col_[e]))
                    throw Error(FMM_ERR_UNSUPPORTED, "is_self must be true on every self_generator pair");
        }
        if (!ex_ptr_.empty()) set_exclusions(1);
        check(fmm_rinv(plan_.get(), reinterpret_cast<const double*>(Q), reinterpret_cast<double*>(U), gradient ? 1 : 0,
                       FMM_HOST));
    }

    // potential and field in one pass (either output may be null)
    void evaluate(const Container<T, N>* Q, Container<T, N>* potential, Container<T, 3>* field) const
    {
        check(fmm_evaluate(plan_.get(), reinterpret_cast<const double*>(Q), reinterpret_cast<double*>(potential),
                           reinterpret_cast<double*>(field), FMM_HOST));
    }

    fmm_plan* handle() const noexcept { return plan_.get(); }

private:
    void set_exclusions(int near_too) const
    {
        if (mode_ == near_too) return;
        check(fmm_plan_set_exclusions(plan_.get(), ex_ptr_.data(), ex_col_.data(), FMM_HOST, near_too));
        mode_ = near_too;
    }
    struct Del { void operator()(fmm_plan* q) const { fmm_plan_destroy(q); } };
    int64_t n_;
    std::unique_ptr<fmm_plan, Del> plan_;
    std::vector<int64_t> ex_ptr_;
    std::vector<int32_t> ex_col_;
    mutable int mode_ = -1;
};

}  // namespace simplefmm_b200
