// C ABI of the library (include/simplefmm_b200.h).  Every entry point
// converts exceptions to an fmm_status and records a per-thread message.
#include <algorithm>
#include <atomic>
#include <memory>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "fmm_eval.cuh"

namespace sfmm {

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line)
{
    const int st = e == cudaErrorMemoryAllocation ? FMM_ERR_OUT_OF_MEMORY : FMM_ERR_CUDA;
    throw Error(st, std::string(cudaGetErrorString(e)) + " in " + what + " (" + file + ":" + std::to_string(line) + ")");
}

}  // namespace sfmm

// Handles are reference counted: a tree holds its context and a plan holds
// its tree, so the caller may destroy them in any order (garbage-collected
// bindings finalize objects in arbitrary order).
struct fmm_context {
    sfmm::Context c;
    std::atomic<int> refs{1};
};

struct fmm_tree {
    sfmm::Tree t;
    fmm_context* owner = nullptr;
    std::atomic<int> refs{1};
};

struct fmm_plan {
    sfmm::Plan pl;
    fmm_tree* owner = nullptr;
};

namespace {

thread_local std::string g_last_error;

int fail(int status, const std::string& msg)
{
    g_last_error = msg;
    return status;
}

}  // namespace

namespace sfmm {
// For entry points defined outside this file.
int record_failure(int status, const char* msg) { return fail(status, msg); }
}  // namespace sfmm

namespace {

#define API_TRY try {
#define API_CATCH                                                              \
    }                                                                          \
    catch (const sfmm::Error& e) { return fail(e.status, e.what()); }          \
    catch (const std::bad_alloc&) { return fail(FMM_ERR_OUT_OF_MEMORY, "host allocation failed"); } \
    catch (const std::exception& e) { return fail(FMM_ERR_CUDA, e.what()); }   \
    return FMM_OK;

void bind(const sfmm::Context& c) { SFMM_CUDA(cudaSetDevice(c.device)); }

void release_context(fmm_context* ctx)
{
    if (!ctx || --ctx->refs > 0) return;
    cudaSetDevice(ctx->c.device);
    cudaStreamSynchronize(ctx->c.stream);
    if (ctx->c.side) {
        cudaStreamSynchronize(ctx->c.side);
        cudaStreamDestroy(ctx->c.side);
    }
    if (ctx->c.copy) {
        cudaStreamSynchronize(ctx->c.copy);
        cudaStreamDestroy(ctx->c.copy);
    }
    if (ctx->c.retired) {
        cudaStreamSynchronize(ctx->c.retired);
        cudaStreamDestroy(ctx->c.retired);
    }
    for (auto& e : ctx->c.batch_graphs)
        if (e.second) cudaGraphExecDestroy(e.second);
    if (ctx->c.own_stream) cudaStreamDestroy(ctx->c.stream);
    delete ctx;
}

void release_tree(fmm_tree* tree)
{
    if (!tree || --tree->refs > 0) return;
    fmm_context* ctx = tree->owner;
    cudaSetDevice(ctx->c.device);
    delete tree;
    release_context(ctx);
}

}  // namespace

extern "C" {

const char* fmm_status_string(int s)
{
    switch (s) {
    case FMM_OK: return "ok";
    case FMM_ERR_INVALID_ARGUMENT: return "invalid argument";
    case FMM_ERR_UNSUPPORTED: return "unsupported";
    case FMM_ERR_CUDA: return "CUDA error";
    case FMM_ERR_OUT_OF_MEMORY: return "out of memory";
    case FMM_ERR_DEGENERATE_INPUT: return "degenerate input";
    case FMM_ERR_OVER_BUDGET: return "over memory budget";
    case FMM_ERR_TIMEOUT: return "timeout";
    default: return "unknown status";
    }
}

const char* fmm_last_error(void) { return g_last_error.c_str(); }

const char* fmm_version(void) { return "0.1.0"; }

int fmm_context_create(int device, fmm_context** out)
{
    API_TRY
    if (!out) return fail(FMM_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    SFMM_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(FMM_ERR_INVALID_ARGUMENT, "no such device");
    auto* ctx = new fmm_context;
    ctx->c.device = device;
    try {
        SFMM_CUDA(cudaSetDevice(device));
        SFMM_CUDA(cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking));
        ctx->c.own_stream = true;
        SFMM_CUDA(cudaStreamCreateWithFlags(&ctx->c.side, cudaStreamNonBlocking));
        SFMM_CUDA(cudaStreamCreateWithFlags(&ctx->c.copy, cudaStreamNonBlocking));
        SFMM_CUDA(cudaDeviceGetAttribute(&ctx->c.sm_count, cudaDevAttrMultiProcessorCount, device));
        (void)sfmm::device_pool(device);
    } catch (...) {
        if (ctx->c.stream) cudaStreamDestroy(ctx->c.stream);
        if (ctx->c.side) cudaStreamDestroy(ctx->c.side);
        if (ctx->c.copy) cudaStreamDestroy(ctx->c.copy);
        delete ctx;
        throw;
    }
    *out = ctx;
    API_CATCH
}

int fmm_context_destroy(fmm_context* ctx)
{
    API_TRY
    release_context(ctx);
    API_CATCH
}

int fmm_context_set_stream(fmm_context* ctx, void* stream)
{
    API_TRY
    if (!ctx) return fail(FMM_ERR_INVALID_ARGUMENT, "ctx is NULL");
    bind(ctx->c);
    SFMM_CUDA(cudaStreamSynchronize(ctx->c.stream));
    if (ctx->c.own_stream) ctx->c.retired = ctx->c.stream;   // destroyed with the context
    ctx->c.stream = static_cast<cudaStream_t>(stream);
    ctx->c.own_stream = false;
    API_CATCH
}

int fmm_context_synchronize(fmm_context* ctx)
{
    API_TRY
    if (!ctx) return fail(FMM_ERR_INVALID_ARGUMENT, "ctx is NULL");
    bind(ctx->c);
    SFMM_CUDA(cudaStreamSynchronize(ctx->c.stream));
    API_CATCH
}

int fmm_host_register(void* ptr, size_t bytes)
{
    API_TRY
    if (!ptr || !bytes) return fail(FMM_ERR_INVALID_ARGUMENT, "empty range");
    SFMM_CUDA(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
    API_CATCH
}

int fmm_host_unregister(void* ptr)
{
    API_TRY
    SFMM_CUDA(cudaHostUnregister(ptr));
    API_CATCH
}

static int tree_build(fmm_context* ctx, const double* xyz, int64_t n, int where, int max_level, int max_ppn,
                      int vertical_axis, double phideg, const double* corner3, double width, fmm_tree** out)
{
    API_TRY
    if (!ctx || !out || !xyz) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    if (where != FMM_HOST && where != FMM_DEVICE) return fail(FMM_ERR_INVALID_ARGUMENT, "where must be FMM_HOST or FMM_DEVICE");
    *out = nullptr;
    bind(ctx->c);
    auto* tr = new fmm_tree;
    tr->owner = ctx;
    ++ctx->refs;
    try {
        tr->t.ctx = &ctx->c;
        tr->t.n = n;
        if (n <= 0) throw sfmm::Error(FMM_ERR_INVALID_ARGUMENT, "n must be positive");
        sfmm::DevBuf<double> staged;
        const double* dxyz = xyz;
        if (where == FMM_HOST) {
            staged.alloc(size_t(3) * n, ctx->c.stream);
            SFMM_CUDA(cudaMemcpyAsync(staged.ptr, xyz, size_t(3) * n * sizeof(double), cudaMemcpyHostToDevice, ctx->c.stream));
            dxyz = staged.ptr;
        }
        sfmm::build_tree(tr->t, dxyz, max_level, max_ppn, vertical_axis, phideg, corner3, width);
    } catch (...) {
        release_tree(tr);
        throw;
    }
    *out = tr;
    API_CATCH
}

int fmm_tree_build(fmm_context* ctx, const double* xyz, int64_t n, int where, int max_level, int max_ppn,
                   int vertical_axis, double phideg, fmm_tree** out)
{
    return tree_build(ctx, xyz, n, where, max_level, max_ppn, vertical_axis, phideg, nullptr, 0.0, out);
}

int fmm_tree_build_box(fmm_context* ctx, const double* xyz, int64_t n, int where, const double* corner3,
                       double width, int max_level, int max_ppn, int vertical_axis, double phideg, fmm_tree** out)
{
    if (!corner3) return fail(FMM_ERR_INVALID_ARGUMENT, "corner is NULL");
    return tree_build(ctx, xyz, n, where, max_level, max_ppn, vertical_axis, phideg, corner3, width, out);
}

int fmm_plan_set_exclusions(fmm_plan* plan, const int64_t* row_ptr, const int32_t* cols, int where, int near_too)
{
    API_TRY
    if (!plan) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL plan");
    if (where != FMM_HOST && where != FMM_DEVICE) return fail(FMM_ERR_INVALID_ARGUMENT, "where must be FMM_HOST or FMM_DEVICE");
    sfmm::Plan& pl = plan->pl;
    bind(*pl.tree->ctx);
    if (!row_ptr) {
        sfmm::plan_clear_exclusions(pl);
        return FMM_OK;
    }
    const int64_t n = pl.tree->n;
    if (where == FMM_DEVICE) {
        if (!cols) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL cols");
        sfmm::plan_set_exclusions(pl, row_ptr, cols, near_too);
        SFMM_CUDA(cudaStreamSynchronize(pl.tree->ctx->stream));
        return FMM_OK;
    }
    if (row_ptr[0] != 0) return fail(FMM_ERR_INVALID_ARGUMENT, "row_ptr[0] must be 0");
    for (int64_t i = 0; i < n; ++i)
        if (row_ptr[i + 1] < row_ptr[i]) return fail(FMM_ERR_INVALID_ARGUMENT, "row_ptr must be non-decreasing");
    const int64_t nnz = row_ptr[n];
    if (nnz > 0 && !cols) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL cols");
    for (int64_t e = 0; e < nnz; ++e)
        if (cols[e] < 0 || cols[e] >= n) return fail(FMM_ERR_INVALID_ARGUMENT, "excluded index out of range");
    cudaStream_t st = pl.tree->ctx->stream;
    sfmm::DevBuf<int64_t> dptr;
    sfmm::DevBuf<int32_t> dcol;
    dptr.alloc(n + 1, st);
    dcol.alloc(std::max<int64_t>(nnz, 1), st);
    SFMM_CUDA(cudaMemcpyAsync(dptr.ptr, row_ptr, size_t(n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    if (nnz) SFMM_CUDA(cudaMemcpyAsync(dcol.ptr, cols, size_t(nnz) * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    sfmm::plan_set_exclusions(pl, dptr.ptr, dcol.ptr, near_too);
    SFMM_CUDA(cudaStreamSynchronize(st));
    API_CATCH
}

int fmm_plan_set_m2l(fmm_plan* plan, int method)
{
    API_TRY
    if (!plan) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL plan");
    bind(*plan->pl.tree->ctx);
    sfmm::plan_set_m2l(plan->pl, method);
    API_CATCH
}

int fmm_plan_set_shard(fmm_plan* plan, int index, int count)
{
    API_TRY
    if (!plan) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL plan");
    bind(*plan->pl.tree->ctx);
    sfmm::plan_set_shard(plan->pl, index, count);
    API_CATCH
}

int fmm_evaluate_stage(fmm_plan* plan, const double* Q, double* pot, double* field, int stage)
{
    API_TRY
    if (!plan || !Q) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    sfmm::Plan& pl = plan->pl;
    if (field && pl.qdim == 2) return fail(FMM_ERR_UNSUPPORTED, "the field needs N = 1 or N = 3 charges");
    bind(*pl.tree->ctx);
    sfmm::plan_evaluate_stage(pl, Q, pot, field, stage);
    API_CATCH
}

int fmm_plan_exchange_buffer(fmm_plan* plan, int which, void** device_ptr, int64_t* count)
{
    if (!plan || !device_ptr || !count) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    sfmm::Plan& pl = plan->pl;
    sfmm::DevBuf<double2>* b = which == 0 ? &pl.M : which == 1 ? &pl.LA : which == 2 ? &pl.LB : nullptr;
    if (!b) return fail(FMM_ERR_INVALID_ARGUMENT, "which must be 0 (moments), 1 (potential locals) or 2 (field locals)");
    *device_ptr = b->ptr;
    *count = static_cast<int64_t>(b->count) * 2;
    return FMM_OK;
}

int fmm_tree_destroy(fmm_tree* tree)
{
    API_TRY
    release_tree(tree);
    API_CATCH
}

int fmm_tree_depth(const fmm_tree* tree, int* depth)
{
    if (!tree || !depth) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    *depth = tree->t.depth;
    return FMM_OK;
}

int fmm_tree_box(const fmm_tree* tree, double* width, double* corner3)
{
    if (!tree || !width || !corner3) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    *width = tree->t.box.width;
    for (int a = 0; a < 3; ++a) corner3[a] = tree->t.box.corner[a];
    return FMM_OK;
}

int fmm_tree_export_size(const fmm_tree* tree, int level, int what, int64_t* count)
{
    API_TRY
    if (!tree || !count) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    bind(*tree->t.ctx);
    *count = sfmm::tree_export(tree->t, level, what, nullptr);
    API_CATCH
}

int fmm_tree_export(const fmm_tree* tree, int level, int what, void* host_out)
{
    API_TRY
    if (!tree || !host_out) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    bind(*tree->t.ctx);
    if (sfmm::tree_export(tree->t, level, what, host_out) < 0) return fail(FMM_ERR_INVALID_ARGUMENT, "export not defined at this level");
    API_CATCH
}

int fmm_tree_stats(const fmm_tree* tree, int64_t* s)
{
    if (!tree || !s) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    s[0] = tree->t.n_nodes;
    s[1] = tree->t.n_leaves;
    s[2] = tree->t.il_nnz;
    s[3] = tree->t.near_pairs;
    s[4] = tree->t.nr_nnz;
    return FMM_OK;
}

int fmm_tree_build_phases(const fmm_tree* tree, double* ms6, double* bytes6)
{
    API_TRY
    if (!tree || !ms6) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    for (int k = 0; k < 6; ++k) ms6[k] = tree->t.phase_ms[k];
    if (bytes6) {
        bind(*tree->t.ctx);
        sfmm::tree_phase_bytes(tree->t, bytes6);
    }
    API_CATCH
}

int fmm_plan_create(fmm_tree* tree, int p, int qdim, int precision, fmm_plan** out)
{
    API_TRY
    if (!tree || !out) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (p < 0 || p > sfmm::kMaxOrder) return fail(FMM_ERR_UNSUPPORTED, "expansion order must be in [0, 16]");
    if (qdim < 1 || qdim > 3) return fail(FMM_ERR_UNSUPPORTED, "charge components N must be 1, 2 or 3");
    if (precision != FMM_PRECISION_FP64 && precision != FMM_PRECISION_MIXED)
        return fail(FMM_ERR_INVALID_ARGUMENT, "precision must be FMM_PRECISION_FP64 or FMM_PRECISION_MIXED");
    bind(*tree->t.ctx);
    auto* pl = new fmm_plan;
    pl->owner = tree;
    ++tree->refs;
    try {
        pl->pl.tree = &tree->t;
        pl->pl.p = p;
        pl->pl.qdim = qdim;
        pl->pl.precision = precision;
        for (auto& e : pl->pl.ev) SFMM_CUDA(cudaEventCreate(&e));
        SFMM_CUDA(cudaEventCreateWithFlags(&pl->pl.fork, cudaEventDisableTiming));
        SFMM_CUDA(cudaEventCreateWithFlags(&pl->pl.join, cudaEventDisableTiming));
        SFMM_CUDA(cudaEventCreateWithFlags(&pl->pl.io_start, cudaEventDisableTiming));
        SFMM_CUDA(cudaEventCreateWithFlags(&pl->pl.io_done, cudaEventDisableTiming));
        sfmm::plan_init(pl->pl);
        SFMM_CUDA(cudaStreamSynchronize(tree->t.ctx->stream));
        sfmm::check_scan_error();
    } catch (...) {
        for (auto& e : pl->pl.ev)
            if (e) cudaEventDestroy(e);
        if (pl->pl.fork) cudaEventDestroy(pl->pl.fork);
        if (pl->pl.join) cudaEventDestroy(pl->pl.join);
        if (pl->pl.io_start) cudaEventDestroy(pl->pl.io_start);
        if (pl->pl.io_done) cudaEventDestroy(pl->pl.io_done);
        delete pl;
        release_tree(tree);
        throw;
    }
    *out = pl;
    API_CATCH
}

int fmm_plan_destroy(fmm_plan* plan)
{
    API_TRY
    if (!plan) return FMM_OK;
    bind(*plan->pl.tree->ctx);
    SFMM_CUDA(cudaStreamSynchronize(plan->pl.tree->ctx->stream));
    for (auto& e : plan->pl.ev)
        if (e) cudaEventDestroy(e);
    if (plan->pl.fork) cudaEventDestroy(plan->pl.fork);
    if (plan->pl.join) cudaEventDestroy(plan->pl.join);
    if (plan->pl.io_start) cudaEventDestroy(plan->pl.io_start);
    if (plan->pl.io_done) cudaEventDestroy(plan->pl.io_done);
    if (plan->pl.graph_exec) cudaGraphExecDestroy(plan->pl.graph_exec);
    if (plan->pl.graph) cudaGraphDestroy(plan->pl.graph);
    fmm_tree* owner = plan->owner;
    delete plan;
    release_tree(owner);
    API_CATCH
}

int fmm_plan_capture(fmm_plan* plan, const double* Q, double* pot, double* field)
{
    API_TRY
    if (!plan || !Q) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!pot && !field) return fail(FMM_ERR_INVALID_ARGUMENT, "nothing to evaluate");
    sfmm::Plan& pl = plan->pl;
    if (field && pl.qdim == 2) return fail(FMM_ERR_UNSUPPORTED, "the field needs N = 1 or N = 3 charges");
    sfmm::Context& c = *pl.tree->ctx;
    bind(c);
    if (c.stream == nullptr || c.stream == cudaStreamLegacy || c.stream == cudaStreamPerThread)
        return fail(FMM_ERR_UNSUPPORTED, "capture needs the context's own stream, not a default stream");
    SFMM_CUDA(cudaStreamSynchronize(c.stream));
    if (pl.graph_exec) {
        cudaGraphExecDestroy(pl.graph_exec);
        pl.graph_exec = nullptr;
    }
    if (pl.graph) {
        cudaGraphDestroy(pl.graph);
        pl.graph = nullptr;
    }
    SFMM_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    try {
        sfmm::plan_evaluate(pl, Q, pot, field);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(c.stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    SFMM_CUDA(cudaStreamEndCapture(c.stream, &pl.graph));
    SFMM_CUDA(cudaGraphInstantiate(&pl.graph_exec, pl.graph, 0));
    API_CATCH
}

// One evaluation of the batch's forest plan through the context's graph
// executable for its launch shape (a new one when none can be updated).
static void evaluate_graph(sfmm::Plan& pl, const double* Q, double* pot, double* field)
{
    sfmm::Context& c = *pl.tree->ctx;
    cudaGraph_t g = nullptr;
    SFMM_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    try {
        sfmm::plan_evaluate(pl, Q, pot, field);
    } catch (...) {
        cudaStreamEndCapture(c.stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    SFMM_CUDA(cudaStreamEndCapture(c.stream, &g));
    // launch shape: the kernel sequence depends on the depth, the order, the
    // precision, the charge components and the outputs
    const uint64_t shape = uint64_t(pl.tree->depth) | uint64_t(pl.p) << 8 | uint64_t(pl.precision) << 16 |
                           uint64_t(pl.qdim) << 20 | uint64_t(pot != nullptr) << 24 | uint64_t(field != nullptr) << 25 |
                           uint64_t(pl.i8 != nullptr) << 26;
    cudaGraphExec_t exec = nullptr;
    for (auto& e : c.batch_graphs)
        if (e.first == shape) {
            cudaGraphExecUpdateResultInfo info{};
            if (cudaGraphExecUpdate(e.second, g, &info) == cudaSuccess) {
                exec = e.second;
                ++c.batch_graph_updates;
            } else {
                cudaGetLastError();
                cudaGraphExecDestroy(e.second);
                e.second = nullptr;
            }
            break;
        }
    if (!exec) {
        const cudaError_t rc = cudaGraphInstantiate(&exec, g, 0);
        if (rc != cudaSuccess) {
            cudaGraphDestroy(g);
            SFMM_CUDA(rc);
        }
        ++c.batch_graph_instantiations;
        bool placed = false;
        for (auto& e : c.batch_graphs)
            if (e.first == shape) {
                e.second = exec;
                placed = true;
            }
        if (!placed) {
            if (c.batch_graphs.size() >= 64) {           // a few dozen shapes are live at a time
                cudaGraphExecDestroy(c.batch_graphs.front().second);
                c.batch_graphs.erase(c.batch_graphs.begin());
            }
            c.batch_graphs.emplace_back(shape, exec);
        }
    }
    cudaGraphDestroy(g);
    SFMM_CUDA(cudaGraphLaunch(exec, c.stream));
}

int fmm_solve_batch(fmm_context* ctx, const fmm_batch_item* items, int count, int p, int qdim, int precision, int max_level)
{
    API_TRY
    if (!ctx || !items || count < 1) return fail(FMM_ERR_INVALID_ARGUMENT, "need a context and at least one item");
    if (qdim < 1 || qdim > 3 || p < 0 || p > 16 || max_level < 1 || max_level > sfmm::kKeyLevel)
        return fail(FMM_ERR_INVALID_ARGUMENT, "bad qdim, p or max_level");
    if (precision != FMM_PRECISION_FP64 && precision != FMM_PRECISION_MIXED)
        return fail(FMM_ERR_INVALID_ARGUMENT, "precision must be FMM_PRECISION_FP64 or FMM_PRECISION_MIXED");
    const bool want_pot = items[0].pot != nullptr, want_field = items[0].field != nullptr;
    if (!want_pot && !want_field) return fail(FMM_ERR_INVALID_ARGUMENT, "items ask for no output");
    if (want_field && qdim == 2) return fail(FMM_ERR_UNSUPPORTED, "the field needs N = 1 or N = 3 charges");
    int64_t N = 0;
    for (int r = 0; r < count; ++r) {
        const fmm_batch_item& it = items[r];
        if (!it.xyz || !it.Q || it.n <= 0 || it.leaf < 1) return fail(FMM_ERR_INVALID_ARGUMENT, "bad batch item");
        if ((it.pot != nullptr) != want_pot || (it.field != nullptr) != want_field)
            return fail(FMM_ERR_INVALID_ARGUMENT, "all items must ask for the same outputs");
        N += it.n;
    }
    if (N >= (int64_t(1) << 31)) return fail(FMM_ERR_UNSUPPORTED, "a batch holds fewer than 2^31 points");
    sfmm::Context& c = ctx->c;
    bind(c);
    if (c.stream == nullptr || c.stream == cudaStreamLegacy || c.stream == cudaStreamPerThread)
        return fail(FMM_ERR_UNSUPPORTED, "batches need the context's own stream, not a default stream");
    cudaStream_t st = c.stream;
    // inputs, concatenated
    std::vector<double> hx(size_t(3) * N), hq(size_t(N) * qdim);
    std::vector<int64_t> base(count + 1, 0);
    for (int r = 0; r < count; ++r) {
        base[r + 1] = base[r] + items[r].n;
        std::copy(items[r].xyz, items[r].xyz + 3 * items[r].n, hx.begin() + 3 * base[r]);
        std::copy(items[r].Q, items[r].Q + qdim * items[r].n, hq.begin() + qdim * base[r]);
    }
    sfmm::DevBuf<double> dx, dq, dpot, dfield;
    dx.alloc(size_t(3) * N, st);
    dq.alloc(size_t(N) * qdim, st);
    SFMM_CUDA(cudaMemcpyAsync(dx.ptr, hx.data(), hx.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    SFMM_CUDA(cudaMemcpyAsync(dq.ptr, hq.data(), hq.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    // member trees, each as a single solve builds it.  A build waits on the
    // host four times (the cube, the refinement's totals, the two list
    // sizes), so several members are built at once: worker threads, each on a
    // stream of its own, take every kBuilders-th member.
    constexpr int kBuilders = 4;
    const int nb = std::min(count, kBuilders);
    std::vector<std::unique_ptr<sfmm::Tree>> trees(count);
    std::vector<sfmm::Context> wc(nb);
    sfmm::Tree F;
    cudaEvent_t uploaded = nullptr;
    SFMM_CUDA(cudaEventCreateWithFlags(&uploaded, cudaEventDisableTiming));
    SFMM_CUDA(cudaEventRecord(uploaded, st));
    for (int w = 0; w < nb; ++w) {
        wc[w].device = c.device;
        wc[w].sm_count = c.sm_count;
        if (nb == 1) {
            wc[w].stream = st;
        } else {
            SFMM_CUDA(cudaStreamCreateWithFlags(&wc[w].stream, cudaStreamNonBlocking));
            SFMM_CUDA(cudaStreamWaitEvent(wc[w].stream, uploaded, 0));
        }
    }
    auto destroy_streams = [&] {
        if (nb > 1)
            for (auto& x : wc)
                if (x.stream) {
                    cudaStreamSynchronize(x.stream);
                    cudaStreamDestroy(x.stream);
                    x.stream = nullptr;
                }
        cudaEventDestroy(uploaded);
    };
    try {
        sfmm::AllocMeter *meter_req = nullptr, *meter_srv = nullptr;
        sfmm::get_thread_alloc_meters(&meter_req, &meter_srv);
        const bool cache = sfmm::thread_block_cache();
        std::vector<std::exception_ptr> fault(nb);
        auto build = [&](int w) {
            try {
                SFMM_CUDA(cudaSetDevice(c.device));
                sfmm::set_thread_alloc_meters(meter_req, meter_srv);
                sfmm::set_thread_block_cache(cache);
                for (int r = w; r < count; r += nb) {
                    trees[r].reset(new sfmm::Tree);
                    sfmm::Tree& t = *trees[r];
                    t.ctx = &wc[w];
                    t.n = items[r].n;
                    sfmm::build_tree(t, dx.ptr + 3 * base[r], max_level, items[r].leaf, 2, 0.0);
                }
                SFMM_CUDA(cudaStreamSynchronize(wc[w].stream));
            } catch (...) {
                fault[w] = std::current_exception();
            }
        };
        if (nb == 1) {
            build(0);
        } else {
            std::vector<std::thread> th;
            for (int w = 0; w < nb; ++w) th.emplace_back(build, w);
            for (auto& x : th) x.join();
        }
        for (auto& f : fault)
            if (f) std::rethrow_exception(f);
        std::vector<const sfmm::Tree*> members;
        for (auto& t : trees) {
            t->ctx = &c;                                 // the forest is built on the batch's stream
            members.push_back(t.get());
        }
        sfmm::build_forest(F, members);
    } catch (...) {
        trees.clear();
        destroy_streams();
        throw;
    }
    trees.clear();
    destroy_streams();
    {
        sfmm::Plan pl;
        // the plan's events, destroyed when the batch is done (after the sync below)
        struct Events {
            sfmm::Plan& pl;
            explicit Events(sfmm::Plan& q) : pl(q)
            {
                for (auto& e : pl.ev) SFMM_CUDA(cudaEventCreate(&e));
                for (cudaEvent_t* e : {&pl.fork, &pl.join, &pl.io_start, &pl.io_done})
                    SFMM_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
            }
            ~Events()
            {
                for (auto& e : pl.ev)
                    if (e) cudaEventDestroy(e);
                for (cudaEvent_t e : {pl.fork, pl.join, pl.io_start, pl.io_done})
                    if (e) cudaEventDestroy(e);
            }
        } events(pl);
        pl.tree = &F;
        pl.p = p;
        pl.qdim = qdim;
        pl.precision = precision;
        sfmm::plan_init(pl);
        if (want_pot) {
            dpot.alloc(size_t(N) * qdim, st);
            SFMM_CUDA(cudaMemsetAsync(dpot.ptr, 0, dpot.bytes(), st));
        }
        if (want_field) {
            dfield.alloc(size_t(N) * 3, st);
            SFMM_CUDA(cudaMemsetAsync(dfield.ptr, 0, dfield.bytes(), st));
        }
        // a batch of several sets runs through the context's graph of its launch
        // shape; a set alone launches directly (the same kernels, one use)
        if (count > 1) evaluate_graph(pl, dq.ptr, dpot.ptr, dfield.ptr);
        else sfmm::plan_evaluate(pl, dq.ptr, dpot.ptr, dfield.ptr);
        if (want_pot) SFMM_CUDA(cudaMemcpyAsync(hq.data(), dpot.ptr, size_t(N) * qdim * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (want_field) {
            hx.resize(size_t(3) * N);
            SFMM_CUDA(cudaMemcpyAsync(hx.data(), dfield.ptr, size_t(N) * 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
        }
        SFMM_CUDA(cudaStreamSynchronize(st));
        sfmm::m2l_i8_check(pl);
    }
    // back to each set's units: potential / width, field / width^2
    for (int r = 0; r < count; ++r) {
        const double w = F.member_width.empty() ? 1.0 : F.member_width[r];
        const double s1 = 1.0 / w, s2 = s1 * s1;
        if (want_pot)
            for (int64_t i = 0; i < items[r].n * qdim; ++i) items[r].pot[i] += s1 * hq[qdim * base[r] + i];
        if (want_field)
            for (int64_t i = 0; i < items[r].n * 3; ++i) items[r].field[i] += s2 * hx[3 * base[r] + i];
    }
    API_CATCH
}

int fmm_batch_graph_stats(const fmm_context* ctx, int64_t* instantiated, int64_t* updated)
{
    if (!ctx || !instantiated || !updated) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    *instantiated = ctx->c.batch_graph_instantiations;
    *updated = ctx->c.batch_graph_updates;
    return FMM_OK;
}

int fmm_plan_replay(fmm_plan* plan)
{
    API_TRY
    if (!plan) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL plan");
    sfmm::Plan& pl = plan->pl;
    if (!pl.graph_exec) return fail(FMM_ERR_INVALID_ARGUMENT, "nothing captured (fmm_plan_capture)");
    bind(*pl.tree->ctx);
    SFMM_CUDA(cudaGraphLaunch(pl.graph_exec, pl.tree->ctx->stream));
    API_CATCH
}

int fmm_evaluate(fmm_plan* plan, const double* Q, double* pot, double* field, int where)
{
    API_TRY
    if (!plan || !Q) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    if (where != FMM_HOST && where != FMM_DEVICE) return fail(FMM_ERR_INVALID_ARGUMENT, "where must be FMM_HOST or FMM_DEVICE");
    sfmm::Plan& pl = plan->pl;
    if (field && pl.qdim == 2) return fail(FMM_ERR_UNSUPPORTED, "the field needs N = 1 or N = 3 charges");
    if (!pot && !field) return FMM_OK;
    sfmm::Context& c = *pl.tree->ctx;
    bind(c);
    const int64_t n = pl.tree->n;
    if (where == FMM_DEVICE) {
        sfmm::plan_evaluate(pl, Q, pot, field);
        return FMM_OK;
    }
    cudaStream_t st = c.stream;
    const size_t qb = size_t(n) * pl.qdim * sizeof(double);
    if (pl.qin.count < size_t(n) * pl.qdim) pl.qin.alloc(size_t(n) * pl.qdim, st);
    double* dpot = nullptr;
    double* dfield = nullptr;
    if (pot && pl.uio_pot.count < size_t(n) * pl.qdim) pl.uio_pot.alloc(size_t(n) * pl.qdim, st);
    if (field && pl.uio_field.count < size_t(n) * 3) pl.uio_field.alloc(size_t(n) * 3, st);
    SFMM_CUDA(cudaMemcpyAsync(pl.qin.ptr, Q, qb, cudaMemcpyHostToDevice, st));
    // the accumulated outputs are only needed by the final sums: copy them in
    // on the context's copy stream while the far field runs (after the
    // stream's earlier work, which may still read the staging buffers)
    cudaEvent_t io = nullptr;
    if (pot || field) {
        cudaStream_t cp = c.copy ? c.copy : st;
        SFMM_CUDA(cudaEventRecord(pl.io_start, st));
        SFMM_CUDA(cudaStreamWaitEvent(cp, pl.io_start, 0));
        if (pot) {
            SFMM_CUDA(cudaMemcpyAsync(pl.uio_pot.ptr, pot, qb, cudaMemcpyHostToDevice, cp));
            dpot = pl.uio_pot.ptr;
        }
        if (field) {
            SFMM_CUDA(cudaMemcpyAsync(pl.uio_field.ptr, field, size_t(n) * 3 * sizeof(double), cudaMemcpyHostToDevice, cp));
            dfield = pl.uio_field.ptr;
        }
        SFMM_CUDA(cudaEventRecord(pl.io_done, cp));
        io = pl.io_done;
    }
    sfmm::plan_evaluate(pl, pl.qin.ptr, dpot, dfield, io);
    if (pot) SFMM_CUDA(cudaMemcpyAsync(pot, dpot, qb, cudaMemcpyDeviceToHost, st));
    if (field) SFMM_CUDA(cudaMemcpyAsync(field, dfield, size_t(n) * 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    SFMM_CUDA(cudaStreamSynchronize(st));
    sfmm::m2l_i8_check(pl);
    API_CATCH
}

int fmm_rinv(fmm_plan* plan, const double* Q, double* U, int gradient, int where)
{
    if (!plan) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL plan");
    if (gradient && plan->pl.qdim != 3) return fail(FMM_ERR_UNSUPPORTED, "rinv<true> needs N = 3 (fmm.hpp:550)");
    return gradient ? fmm_evaluate(plan, Q, nullptr, U, where) : fmm_evaluate(plan, Q, U, nullptr, where);
}

int fmm_plan_timings(const fmm_plan* plan, double* ms6)
{
    API_TRY
    if (!plan || !ms6) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    bind(*plan->pl.tree->ctx);
    sfmm::plan_read_timings(const_cast<sfmm::Plan&>(plan->pl), ms6);
    sfmm::m2l_i8_check(const_cast<sfmm::Plan&>(plan->pl));
    API_CATCH
}

int fmm_direct(fmm_context* ctx, const double* xyz, int64_t n, const double* Q, int qdim, const int64_t* targets,
               int64_t nt, double* pot, double* field, int where)
{
    API_TRY
    if (!ctx || !xyz || !Q || !targets) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    if (qdim < 1 || qdim > 3) return fail(FMM_ERR_UNSUPPORTED, "qdim must be 1, 2 or 3");
    if (field && qdim == 2) return fail(FMM_ERR_UNSUPPORTED, "the field needs qdim 1 or 3");
    if (n <= 0 || nt < 0) return fail(FMM_ERR_INVALID_ARGUMENT, "bad sizes");
    if (where != FMM_HOST && where != FMM_DEVICE) return fail(FMM_ERR_INVALID_ARGUMENT, "where must be FMM_HOST or FMM_DEVICE");
    bind(ctx->c);
    cudaStream_t st = ctx->c.stream;
    if (where == FMM_DEVICE) {
        // the targets are device memory: the kernels skip an index outside
        // [0, n) and flag it; the flag is read back after the sums
        sfmm::DevBuf<int> bad;
        bad.alloc(1, st);
        SFMM_CUDA(cudaMemsetAsync(bad.ptr, 0, sizeof(int), st));
        sfmm::direct_sum(ctx->c, xyz, n, Q, qdim, targets, nt, pot, field, bad.ptr);
        int h_bad = 0;
        SFMM_CUDA(cudaMemcpyAsync(&h_bad, bad.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
        SFMM_CUDA(cudaStreamSynchronize(st));
        if (h_bad) return fail(FMM_ERR_INVALID_ARGUMENT, "target index out of range [0, n)");
        return FMM_OK;
    }
    for (int64_t t = 0; t < nt; ++t)
        if (targets[t] < 0 || targets[t] >= n) return fail(FMM_ERR_INVALID_ARGUMENT, "target index out of range [0, n)");
    sfmm::DevBuf<double> dx, dq, dp, df;
    sfmm::DevBuf<int64_t> dt;
    dx.alloc(size_t(3) * n, st);
    dq.alloc(size_t(qdim) * n, st);
    dt.alloc(std::max<int64_t>(nt, 1), st);
    SFMM_CUDA(cudaMemcpyAsync(dx.ptr, xyz, size_t(3) * n * 8, cudaMemcpyHostToDevice, st));
    SFMM_CUDA(cudaMemcpyAsync(dq.ptr, Q, size_t(qdim) * n * 8, cudaMemcpyHostToDevice, st));
    SFMM_CUDA(cudaMemcpyAsync(dt.ptr, targets, size_t(nt) * 8, cudaMemcpyHostToDevice, st));
    if (pot) dp.alloc(size_t(qdim) * std::max<int64_t>(nt, 1), st);
    if (field) df.alloc(size_t(3) * std::max<int64_t>(nt, 1), st);
    sfmm::direct_sum(ctx->c, dx.ptr, n, dq.ptr, qdim, dt.ptr, nt, pot ? dp.ptr : nullptr, field ? df.ptr : nullptr);
    if (pot) SFMM_CUDA(cudaMemcpyAsync(pot, dp.ptr, size_t(qdim) * nt * 8, cudaMemcpyDeviceToHost, st));
    if (field) SFMM_CUDA(cudaMemcpyAsync(field, df.ptr, size_t(3) * nt * 8, cudaMemcpyDeviceToHost, st));
    SFMM_CUDA(cudaStreamSynchronize(st));
    API_CATCH
}

int fmm_launch_count(int64_t* count)
{
    if (!count) return fail(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    *count = sfmm::g_launches.load();
    return FMM_OK;
}

}  // extern "C"
