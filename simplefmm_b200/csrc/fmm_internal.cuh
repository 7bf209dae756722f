// Internal declarations of the B200 FMM library (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "alloc_meter.h"
#include "csr_limits.h"
#include "fmm_ops.cuh"
#include "simplefmm_b200.h"

namespace sfmm {

// ------------------------------------------------------------------ errors
struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line);

#define SFMM_CUDA(x)                                                     \
    do {                                                                 \
        cudaError_t e_ = (x);                                            \
        if (e_ != cudaSuccess) ::sfmm::throw_cuda(e_, #x, __FILE__, __LINE__); \
    } while (0)

extern std::atomic<long long> g_launches;

// Records the calling thread's last-error message (fmm_last_error) and returns status.
int record_failure(int status, const char* msg);

#define SFMM_CHECK_LAUNCH()                   \
    do {                                      \
        ::sfmm::g_launches.fetch_add(1);      \
        SFMM_CUDA(cudaGetLastError());        \
    } while (0)

#define SFMM_REQUIRE(cond, status, msg)                 \
    do {                                                \
        if (!(cond)) throw ::sfmm::Error((status), (msg)); \
    } while (0)

// Lets kernel k use up to the device's opt-in shared memory per block.  The
// attribute belongs to the function, not the launch, so it is always set to
// the same maximum: host threads launching k concurrently with different
// shared-memory sizes (a server running several solves) cannot undo each
// other's setting between the attribute call and the launch.
template<typename KernelT>
inline void allow_max_smem(KernelT k)
{
    int dev = 0, optin = 0;
    SFMM_CUDA(cudaGetDevice(&dev));
    SFMM_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa{};
    SFMM_CUDA(cudaFuncGetAttributes(&fa, k));                 // static + dynamic <= opt-in limit
    SFMM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   optin - static_cast<int>(fa.sharedSizeBytes)));
}

// ------------------------------------------------------------------ device memory
// Stream-ordered device allocation from a memory pool owned by this library
// (one per device, created on first use, kept until exit, release threshold
// unlimited): repeated trees and plans reuse the pool's memory, and no other
// user of the device's default pool can trim it between evaluations.
cudaMemPool_t device_pool(int device);

// Device allocation for DevBuf (memory.cu): blocks of at least 4 MiB are
// cached by exact size when released and handed back to the next request of
// that size on the same device, after the requesting stream has waited for
// the releasing stream (an event recorded at release).  Repeated solves of
// one size (time stepping, the bench) then reuse their own buffers and the
// pool never grows between them: growing it stalled single allocations for
// 0.4-0.9 s once several GB were in play.  The cache holds at most a third of
// the device's memory (oldest blocks are freed first) and is emptied when an
// allocation fails, before the allocation is retried.
void* device_alloc(size_t bytes, int device, cudaStream_t s);        // throws FMM_ERR_OUT_OF_MEMORY
void device_free(void* p, size_t bytes, int device, cudaStream_t s) noexcept;



template<typename T>
struct DevBuf {
    T* ptr = nullptr;
    size_t count = 0;
    cudaStream_t stream = nullptr;
    int device = 0;

    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), count(o.count), stream(o.stream), device(o.device) { o.ptr = nullptr; o.count = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept
    {
        if (this != &o) {
            release();
            ptr = o.ptr; count = o.count; stream = o.stream; device = o.device;
            o.ptr = nullptr; o.count = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }

    void alloc(size_t n, cudaStream_t s)
    {
        release();
        stream = s;
        if (n) {
            SFMM_CUDA(cudaGetDevice(&device));
            ptr = static_cast<T*>(device_alloc(n * sizeof(T), device, s));
            count = n;
        }
    }
    // grow keeping the first `keep` elements
    void grow(size_t n, size_t keep, cudaStream_t s)
    {
        if (n <= count) return;
        DevBuf<T> nb;
        nb.alloc(n, s);
        if (keep && ptr) SFMM_CUDA(cudaMemcpyAsync(nb.ptr, ptr, keep * sizeof(T), cudaMemcpyDeviceToDevice, s));
        *this = std::move(nb);
    }
    void release() noexcept
    {
        if (ptr) device_free(ptr, count * sizeof(T), device, stream);
        ptr = nullptr;
        count = 0;
    }
    size_t bytes() const { return count * sizeof(T); }
};

constexpr int kKeyLevel = 20;             // box.hpp:26 -- deepest keyed level

// Root cube (box.hpp:24-31, 84-107) as used on the device.
struct BoxDev {
    double width;
    double corner[3];
    double cphi, sphi;                    // cos / sin of the rotation about the vertical axis
    int X, Y, Z;                          // axis permutation (box.hpp:74-76)
    int rotated;                          // phideg != 0
    int status;                           // FMM_OK or FMM_ERR_DEGENERATE_INPUT
};

// rotate(v) of box.hpp:152-157, without contraction so the rounding is the
// plain product/sum sequence of the source.
__host__ __device__ inline void box_rotate(const BoxDev& b, const double* v, double* r)
{
    if (!b.rotated) {
        r[0] = v[b.X];
        r[1] = v[b.Y];
        r[2] = v[b.Z];
        return;
    }
#ifdef __CUDA_ARCH__
    r[0] = __dsub_rn(__dmul_rn(b.cphi, v[b.X]), __dmul_rn(b.sphi, v[b.Y]));
    r[1] = __dadd_rn(__dmul_rn(b.sphi, v[b.X]), __dmul_rn(b.cphi, v[b.Y]));
#else
    r[0] = b.cphi * v[b.X] - b.sphi * v[b.Y];
    r[1] = b.sphi * v[b.X] + b.cphi * v[b.Y];
#endif
    r[2] = v[b.Z];
}

// ------------------------------------------------------------------ objects
struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t retired = nullptr;       // the context's own stream after the caller set theirs:
                                          // buffers allocated before still free on it
    cudaStream_t copy = nullptr;          // host-array evaluations copy the accumulated outputs in on it,
                                          // beside the far field
    cudaStream_t side = nullptr;          // the library's second stream: the near field runs
                                          // on it beside the far field (forked from and joined
                                          // back into `stream` with events)
    int sm_count = 148;
    // batched solves (fmm_solve_batch): executable graphs of the batch
    // evaluation kept per launch shape, updated in place for the next batch
    std::vector<std::pair<uint64_t, cudaGraphExec_t>> batch_graphs;
    int64_t batch_graph_instantiations = 0, batch_graph_updates = 0;
};

// Device-resident octree: nodes of all levels concatenated level by level
// (within a level in key order, the reference's _c_node order), points in
// leaf order (leaves in Morton order, each leaf's points by ascending
// original index -- the order OctreeNode::subdivide leaves them in).
struct Tree {
    Context* ctx = nullptr;
    int64_t n = 0;
    int depth = 0;
    int max_level = 20, max_ppn = 64, vertical_axis = 2;
    double phideg = 0;
    BoxDev box{};                         // host copy
    DevBuf<BoxDev> d_box;

    std::vector<int64_t> lvl_off;         // node offset per level (depth + 2)
    std::vector<int64_t> leaf_off;        // leaf offset per level (depth + 2)
    int64_t n_nodes = 0, n_leaves = 0;

    // points (sorted order)
    DevBuf<int32_t> order;                // sorted position -> original index
    DevBuf<double> pts;                   // 3 x n SoA: x | y | z, original frame (near field)
    DevBuf<double> rpts;                  // 3 x n SoA rotated frame, only when box.rotated
    const double* far_x = nullptr;        // rotated-frame coordinates used by the far field
    const double* far_y = nullptr;
    const double* far_z = nullptr;

    // nodes
    DevBuf<uint64_t> key;
    DevBuf<int32_t> pbeg, pend, parent, child_beg, nchild, leaf_id;
    DevBuf<int32_t> leaf_node;            // global leaf id -> global node id
    DevBuf<int32_t> colleague;            // 27 per node: same-level neighbours (tree.hpp:66-119)

    // interaction list (partition.hpp:283-297), rows = all nodes, sorted by source
    DevBuf<int32_t> il_ptr, il_src, il_code;
    int64_t il_nnz = 0;

    // near-field source point ranges per leaf (the point sets of _nlist rows)
    DevBuf<int32_t> nr_ptr;
    DevBuf<int2> nr;
    int64_t nr_nnz = 0;
    int64_t near_pairs = 0;

    float build_ms = 0;
    // device time of the build's phases: keys, refinement, leaves and points,
    // colleagues, interaction lists, near-field lists.  The single-launch
    // refinement also numbers the leaves and fills the colleague lists: its
    // phase then holds them, "leaves and points" only the point gather, and
    // "colleagues" nothing.
    float phase_ms[6] = {};
    bool single_refine = false;

    // a forest of independent trees (forest.cu): the member of each node; empty
    // for a single tree
    DevBuf<int32_t> node_tree;
    int n_trees = 1;
    std::vector<double> member_width;     // root-cube width of each member
};

struct Plan;

// tree.cu
// corner3 / width: an explicit root cube (Box(corner, width, ...), box.hpp:73-82)
// instead of the one fitted to the points (box.hpp:84-107); corner3 == nullptr fits.
void build_tree(Tree& t, const double* xyz_dev, int max_level, int max_ppn, int vertical_axis, double phideg,
                const double* corner3 = nullptr, double width = 0.0);
int64_t tree_export(const Tree& t, int level, int what, void* host_out);
// forest.cu: merge trees built on one context into a forest F (member points
// scaled into the unit cube, each by its own box; lists never cross members)
void build_forest(Tree& F, const std::vector<const Tree*>& members);
void tree_phase_bytes(const Tree& t, double* bytes6);

// direct.cu: a target index outside [0, n) is not read; its outputs are NaN
// and *bad (a device int, may be NULL) is set to 1
void direct_sum(Context& c, const double* xyz, int64_t n, const double* Q, int qdim, const int64_t* targets, int64_t nt,
                double* pot, double* field, int* bad = nullptr);

// scan.cu: out[0..n] (n + 1 entries; out[n] is the total) of non-negative
// counts, one launch.  total64 (a device int64, may be NULL) receives the
// total in 64 bits, so that an int32 scan that overflowed can be refused.
void exclusive_scan_i32(const int32_t* in, int32_t* out, int64_t n, cudaStream_t s, int64_t* total64 = nullptr);
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s, int64_t* total64 = nullptr);
// Throws if a scan's bounded wait gave up since the last call (a scan's
// result is then wrong); call after synchronizing the scans' stream.
void check_scan_error();

// A CSR list whose row pointers are int32 must have at most 2^31 - 1
// entries; the total is summed in 64 bits and checked before the list is
// allocated (csr_limits.h).
inline void require_i32_total(int64_t total, const char* what)
{
    if (!csr_total_fits(total)) throw Error(FMM_ERR_UNSUPPORTED, csr_overflow_message(what, total));
}

inline unsigned blocks_for(int64_t n, int threads, int64_t cap = 1 << 20)
{
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return static_cast<unsigned>(b);
}

}  // namespace sfmm
