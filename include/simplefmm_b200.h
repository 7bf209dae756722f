/*
 * simplefmm_b200 -- C ABI of the B200 (sm_100a) 3D Laplace FMM.
 *
 * The reference library (SimpleFMM) is header-only C++ templates; its
 * evaluation path is the sequence
 *     Box(positions, vertical_axis, phideg)                 box.hpp:84-107
 *     OctreePartitioner(positions, box).refine(L, ppn)       partition.hpp:397-446
 *     FMM3D<double, N, p, Vector, grad>(partitioner, comm)   fmm.hpp:204-427
 *     fmm.rinv(Q, U) / fmm.rinv<true>(Q, U)                  fmm.hpp:864-881
 * Each entry point below replaces one step of that sequence (cited per
 * function).  Arguments are plain pointers and sizes; no C++ or CUDA types
 * cross the boundary (a cudaStream_t is passed as void*).
 *
 * Conventions
 *  - Every function returns an fmm_status (0 = FMM_OK).  fmm_last_error()
 *    returns a message for the calling thread's last failure.
 *  - Positions are n x 3 doubles, row-major (x0 y0 z0 x1 ...), exactly the
 *    memory of the reference's std::vector<Vector<double,3>>.
 *  - Charges Q are n x qdim doubles (the reference's Vector<double,N>*);
 *    outputs are accumulated (U += ...), as the reference's rinv does.
 *  - `where` says whether pointers are host (FMM_HOST) or device
 *    (FMM_DEVICE) memory.
 *  - The library keeps the tree, lists and expansions resident on the
 *    device; one context = one device + one stream.  Calls on one context
 *    are not re-entrant (like the reference's mutable _M/_L, fmm.hpp:178-179).
 *  - Handles may be destroyed in any order: a tree keeps its context alive
 *    and a plan keeps its tree alive until they are destroyed themselves.
 */
#ifndef SIMPLEFMM_B200_H
#define SIMPLEFMM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fmm_status {
    FMM_OK = 0,
    FMM_ERR_INVALID_ARGUMENT = 1,
    FMM_ERR_UNSUPPORTED = 2,
    FMM_ERR_CUDA = 3,
    FMM_ERR_OUT_OF_MEMORY = 4,
    /* All points share the vertical coordinate: the reference's Box loops
       forever doubling a zero width (box.hpp:101-105); rejected here. */
    FMM_ERR_DEGENERATE_INPUT = 5,
    FMM_ERR_OVER_BUDGET = 6,
    FMM_ERR_TIMEOUT = 7
} fmm_status;

enum { FMM_HOST = 0, FMM_DEVICE = 1 };

/* Plan precision: FP64 throughout (matches the reference to 1e-12), or the
   mixed-precision form: near field in FP32 with compensated sums; M2L (orders
   2..12) as dense per-offset operators in four 8-bit slices on the int8
   tensor cores with exact int32 sums (about 1e-7 relative to the FP64 path);
   moments, locals and the final sums in FP64.  A pipeline wait of that M2L
   that expires is reported as FMM_ERR_TIMEOUT by the next host-array
   fmm_evaluate or fmm_plan_timings of the plan. */
enum { FMM_PRECISION_FP64 = 0, FMM_PRECISION_MIXED = 1 };

/* M2L formulation: rotate / z-translate / rotate back (the reference's
   default M2Lc_rtr, fmm.hpp:620-688), or the dense direct sum the reference
   compiles with -DFMM_M2L_DIRECT (M2Lc_direct, fmm.hpp:592-618). */
enum { FMM_M2L_METHOD_ROTATION = 0, FMM_M2L_METHOD_DIRECT = 1 };

/* Tree export selectors for fmm_tree_export (one level at a time). */
enum {
    FMM_EXPORT_NODE_KEYS = 0,   /* int64[n_node]  OctreeLevel::_c_node      partition.hpp:158 */
    FMM_EXPORT_LEAF_NODES = 1,  /* int32[n_leaf]  OctreeLevel::_i_leaf      partition.hpp:159 */
    FMM_EXPORT_INDEX_PTR = 2,   /* int32[n_leaf+1] _indices row pointers    partition.hpp:160 */
    FMM_EXPORT_INDEX = 3,       /* int32[nnz]     _indices (original ids)  */
    FMM_EXPORT_ILIST_PTR = 4,   /* int32[n_node+1] _ilist rows (level>=2)   partition.hpp:283-297 */
    FMM_EXPORT_ILIST = 5,       /* int32[4*nnz]   (src node, di, dj, dk)   */
    FMM_EXPORT_CLIST_PTR = 6,   /* int32[n_node+1] _clist rows (level<depth) partition.hpp:299-313 */
    FMM_EXPORT_CLIST = 7,       /* int64[2*nnz]   (child node, child key)  */
    FMM_EXPORT_PLIST = 8,       /* int64[2*n_node] (parent node, own key), level>=1  partition.hpp:315-322 */
    FMM_EXPORT_NLIST_PTR = 9,   /* int32[n_leaf+1] _nlist rows              partition.hpp:343-366 */
    FMM_EXPORT_NLIST = 10,      /* int32[2*nnz]   (level, leaf)            */
    FMM_EXPORT_PARTITIONS = 11  /* int32[2*n]     point -> (level, leaf)   partition.hpp:436-445 */
};

typedef struct fmm_context fmm_context;
typedef struct fmm_tree fmm_tree;
typedef struct fmm_plan fmm_plan;

const char* fmm_status_string(int status);
const char* fmm_last_error(void);
/* Library version, e.g. "0.1.0". */
const char* fmm_version(void);

/* Create a context on `device` with its own stream. */
int fmm_context_create(int device, fmm_context** out);
int fmm_context_destroy(fmm_context* ctx);
/* Use the caller's stream (a cudaStream_t) for all work of this context.
   The call first waits for the context's current stream.  Device buffers of
   trees and plans are released in stream order on the stream they were
   allocated on: a caller stream set earlier must outlive the trees and plans
   built while it was set (the context's own stream lives as long as the
   context). */
int fmm_context_set_stream(fmm_context* ctx, void* stream);
int fmm_context_synchronize(fmm_context* ctx);
/* Page-lock host memory so host<->device copies run at full speed. */
int fmm_host_register(void* ptr, size_t bytes);
int fmm_host_unregister(void* ptr);

/* Box(positions, vertical_axis, phideg) + OctreePartitioner::refine(max_level,
   max_particles_per_node): box.hpp:84-107, partition.hpp:397-446.  The tree
   (nodes, leaf point lists, interaction/neighbour lists) is built on the
   device and stays resident.  max_level is clamped to 20 (box.hpp:26).
   The tree copies the positions it needs; the caller's array may be freed. */
int fmm_tree_build(fmm_context* ctx, const double* xyz, int64_t n, int where, int max_level,
                   int max_particles_per_node, int vertical_axis, double phideg, fmm_tree** out);
/* Box(corner, width, vertical_axis, phideg) + refine: box.hpp:73-82 -- the
   caller's root cube (corner in the rotated frame of the keys, as the
   reference stores it) instead of the one fitted to the points.  Points
   outside the cube are clamped into its boundary cells, as the reference's
   keys are (box.hpp:58-63). */
int fmm_tree_build_box(fmm_context* ctx, const double* xyz, int64_t n, int where, const double* corner3,
                       double width, int max_level, int max_particles_per_node, int vertical_axis, double phideg,
                       fmm_tree** out);
int fmm_tree_destroy(fmm_tree* tree);
/* Deepest level (OctreePartitioner::level(), partition.hpp:463-466). */
int fmm_tree_depth(const fmm_tree* tree, int* depth);
/* Box::width() and Box::corner() (box.hpp:109-117). */
int fmm_tree_box(const fmm_tree* tree, double* width, double* corner3);
/* Element count of an export (see FMM_EXPORT_*), or -1 if not defined at this level. */
int fmm_tree_export_size(const fmm_tree* tree, int level, int what, int64_t* count);
/* Copy one export to host memory sized by fmm_tree_export_size. */
int fmm_tree_export(const fmm_tree* tree, int level, int what, void* host_out);
/* Total element counts of the device lists: [0] nodes, [1] leaves, [2] ilist
   pairs, [3] near-field point pairs (self excluded), [4] near-field ranges. */
int fmm_tree_stats(const fmm_tree* tree, int64_t* stats5);
/* Device time (ms) of the phases of the tree build -- [0] root cube and
   Morton keys, [1] refinement (the subdivision of partition.hpp:47-104, level
   by level), [2] leaves and points in leaf order, [3] same-level neighbours,
   [4] interaction lists, [5] near-field lists -- and, if bytes6 is not NULL,
   the device-memory bytes each phase must move at least once (its
   algorithmic traffic), for achieved-bandwidth figures.  The refinement runs
   as one cooperative launch that also numbers the leaves and fills the
   neighbour lists: [1] then holds that work, [2] only the point gather and
   [3] nothing (0 bytes).  No counterpart in the reference (its tree build is
   timed as one step). */
int fmm_tree_build_phases(const fmm_tree* tree, double* ms6, double* bytes6);

/* FMM3D<double, qdim, p, Vector, support_gradient>(partitioner, comm):
   fmm.hpp:204-427.  Builds the operator tables for order p (0..16) and
   allocates device expansions.  qdim is the number of charge components N. */
int fmm_plan_create(fmm_tree* tree, int p, int qdim, int precision, fmm_plan** out);
int fmm_plan_destroy(fmm_plan* plan);
/* Excluded interactions: FMM3D(partitioner, comm, self_generator) and
   rinv(Q, U, is_self), fmm.hpp:204, 398-408, 773-807.  row_ptr (n + 1
   int64) and cols (row_ptr[n] int32, original indices) list for each target
   i the sources j whose interaction is removed from every later evaluation
   (j == i is always excluded).  near_too = 0 removes only the listed sources
   outside i's near field -- the reference's slist with the default is_self
   (rinv(Q, U)); near_too = 1 removes all of them -- rinv(Q, U, is_self) with
   an is_self true exactly on the listed pairs.  row_ptr = NULL clears. */
int fmm_plan_set_exclusions(fmm_plan* plan, const int64_t* row_ptr, const int32_t* cols, int where, int near_too);
/* Chooses the plan's M2L formulation for later evaluations: FMM_M2L_METHOD_ROTATION
   (default) or FMM_M2L_METHOD_DIRECT, the reference's FMM_M2L_DIRECT build option
   (fmm.hpp:700-712 calling M2Lc_direct, fmm.hpp:592-618; tables
   fmm.hpp:317-337).  The direct form is FP64 only and costs (p+1)^2 terms
   per coefficient and pair; its tables are built on first use per device
   and order (synchronous). */
int fmm_plan_set_m2l(fmm_plan* plan, int method);

/* fmm.rinv(Q, U) (gradient = 0) or fmm.rinv<true>(Q, U) (gradient = 1,
   qdim must be 3): fmm.hpp:864-881.  U (n x qdim, or n x 3) is accumulated. */
int fmm_rinv(fmm_plan* plan, const double* Q, double* U, int gradient, int where);

/* One pass computing any of: pot (n x qdim) += sum_j Q_j/|x_i-x_j|, and
   field (n x 3) += sum_j q_j R/|R|^3 for qdim = 1, or sum_j Q_j x R/|R|^3 for
   qdim = 3 (the reference's rinv<true>).  NULL skips an output.  Both are
   accumulated.  The far field of the field uses source-gradient moments, the
   formulation of fmm.hpp:234-253 and 549-551. */
int fmm_evaluate(fmm_plan* plan, const double* Q, double* pot, double* field, int where);

/* ---- One solve split over several devices (no counterpart in the
   reference's API; it mirrors the reference's MPI work split, fmm.hpp:503-522
   and distributed.hpp:14-25, and its per-level MPI_Allreduce of moments and
   locals, fmm.hpp:832-859).  Each process builds the same tree and a plan,
   calls fmm_plan_set_shard(plan, index, count) and then evaluates in three
   stages on device arrays, summing two exchange buffers across all shards
   between them (an all-reduce, e.g. NCCL, on the context's stream):
       fmm_evaluate_stage(plan, Q, pot, field, 0)   near field and moments of
                                                    this shard's leaves
       sum buffer 0 (moments) over the shards
       fmm_evaluate_stage(plan, Q, pot, field, 1)   M2M, M2L into this shard's
                                                    targets
       sum buffers 1 and 2 (potential / field locals) over the shards
       fmm_evaluate_stage(plan, Q, pot, field, 2)   L2L, L2P of this shard's
                                                    leaves, sums into pot/field
   pot / field then hold this shard's points' results added to their input
   (other points unchanged); summing the shards' increments gives the solve.
   Leaves are split level by level, balanced by points; M2L targets by
   contiguous ranges of their parents.  Excluded interactions are removed by
   shard 0.  The same pot / field pointers (or NULLs) must be passed to all
   three stages.  count = 1 returns the plan to fmm_evaluate. */
int fmm_plan_set_shard(fmm_plan* plan, int index, int count);
int fmm_evaluate_stage(fmm_plan* plan, const double* Q, double* pot, double* field, int stage);
/* Device address and length (doubles) of exchange buffer `which`: 0 the
   moments, 1 the potential locals, 2 the field locals of every node. */
int fmm_plan_exchange_buffer(fmm_plan* plan, int which, void** device_ptr, int64_t* count);

/* Capture one evaluation of device arrays Q / pot / field (what fmm_evaluate
   with FMM_DEVICE does) as a CUDA graph, and launch it again on the context's
   stream with fmm_plan_replay -- for callers that evaluate the same tree
   repeatedly with new charges written into Q (no counterpart in the
   reference).  Capturing computes nothing; each replay computes and, like
   fmm_evaluate, accumulates into pot / field.  Needs a context on its own
   stream (not a default stream). */
int fmm_plan_capture(fmm_plan* plan, const double* Q, double* pot, double* field);
int fmm_plan_replay(fmm_plan* plan);

/* ---- Batched solves (no counterpart in the reference): several independent
   point sets, each with its own charges, solved by one plan and one set of
   kernel launches.  Each set's tree is built exactly as fmm_tree_build builds
   it (its own fitted root cube, max_particles_per_node = leaf); the trees are
   merged into one forest, the points of each scaled into the unit cube by
   its own box, and evaluated at once: the persistent near-field and M2L
   kernels take the work of all sets.  A batch of two or more sets runs its
   evaluation as a CUDA graph that the context keeps per launch shape and
   updates in place for the next batch of that shape (a set alone launches
   directly).  pot (n x qdim) / field (n x 3) are accumulated like
   fmm_evaluate's; all items of a batch pass pot (or all NULL) and field (or
   all NULL).  Each set's result is the same as that set solved by a batch of
   one (bit for bit in FP64); against fmm_evaluate of the set's own tree it
   differs by the rounding of the scaled coordinates (1e-14 to 1e-12
   relative in FP64).  Host
   arrays; the axis is z and phideg 0. */
typedef struct {
    const double* xyz;        /* n x 3 */
    int64_t n;
    const double* Q;          /* n x qdim */
    int leaf;                 /* max_particles_per_node of this set's tree */
    double* pot;              /* n x qdim, or NULL */
    double* field;            /* n x 3, or NULL */
} fmm_batch_item;
int fmm_solve_batch(fmm_context* ctx, const fmm_batch_item* items, int count, int p, int qdim, int precision, int max_level);
/* Graph executables instantiated and updated in place by this context's
   batches so far. */
int fmm_batch_graph_stats(const fmm_context* ctx, int64_t* instantiated, int64_t* updated);

/* Device time (ms) of each phase of the last evaluation: [0] P2M+M2M,
   [1] M2L, [2] L2L+L2P, [3] P2P (it runs on a second stream beside the far
   field, so [0] + [1] + [2] + [3] can exceed [4]), [4] total; and of the last
   tree build [5]. */
int fmm_plan_timings(const fmm_plan* plan, double* ms6);

/* Direct O(n * nt) FP64 sums at nt target indices (the reference's own
   accuracy check, main.cpp:70-111): pot (nt x qdim) = sum_{j != i} Q_j/|R|,
   field (nt x 3) = sum_j q_j R/|R|^3 (qdim 1) or sum_j Q_j x R/|R|^3 (qdim 3).
   Outputs are overwritten.  Synchronous.  A target index outside [0, n)
   returns FMM_ERR_INVALID_ARGUMENT (checked before any copy for FMM_HOST,
   on the device for FMM_DEVICE: nothing out of range is read). */
int fmm_direct(fmm_context* ctx, const double* xyz, int64_t n, const double* Q, int qdim, const int64_t* targets,
               int64_t nt, double* pot, double* field, int where);

/* Direct sums that allocate nothing (no counterpart in the reference).
   For callers that cannot allocate device memory while they run: a service
   that holds a fixed device-memory budget for its lifetime, or a caller that
   cannot wait on an allocation.  Same sums and output layout as fmm_direct;
   every pointer is device memory of the current device; the work is queued
   on `stream` (a cudaStream_t) and the call returns without waiting.
   Scratch is one fixed 8 MiB device array per device, held from the first
   call until the process exits; the first call on a device looks up its
   address (set-up), so make that first call before any stream capture.
   Limit: nt <= 174762 targets per call (FMM_ERR_OVER_BUDGET above it).
   The call cannot wait for the GPU, so a target index outside [0, n) is not
   reported by the status: nothing out of range is read and that target's
   outputs are NaN.
   Every call shares the array: calls that overlap on the GPU (other streams,
   other host threads) race and corrupt each other's results. */
int fmm_direct_noalloc(const double* xyz, int64_t n, const double* Q, int qdim, const int64_t* targets,
                       int64_t nt, double* pot, double* field, void* stream);

/* ---- Serving loop (no counterpart in the reference: its API solves one
   problem per call).  Solves of different N, p and precision are submitted
   as they arrive and run concurrently on one device: `slots` workers, each
   with its own stream, admit queued requests in arrival order as a slot and
   `memory_budget` bytes of estimated device memory become free, so the
   kernels of admitted requests overlap.  A request keeps its host pointers
   (xyz, Q, pot, field) until fmm_server_wait returns; pot / field are
   accumulated as by fmm_evaluate.  max_particles_per_node = 0 lets the
   server's autotuner pick the leaf size per (p, precision, log2 N). */
typedef struct fmm_server fmm_server;
int fmm_server_create(int device, int slots, size_t memory_budget, fmm_server** out);
/* Finishes every queued request, then frees the server. */
int fmm_server_destroy(fmm_server* server);
int fmm_server_submit(fmm_server* server, const double* xyz, int64_t n, const double* Q, int qdim, int p,
                      int precision, int max_particles_per_node, double* pot, double* field, int64_t* id);
int fmm_server_poll(fmm_server* server, int64_t id, int* done);
/* Blocks until request `id` is done; returns its status and its latency
   (submission to completion, ms).  The id is released. */
int fmm_server_wait(fmm_server* server, int64_t id, double* latency_ms);
/* [0] completed requests, [1] p50 latency ms, [2] p99 latency ms, [3] mean
   latency ms, [4] most requests running at once, [5] most budgeted bytes in
   use at once, [6] budget bytes, [7] requests queued now. */
int fmm_server_stats(fmm_server* server, double* stats8);
/* Measured device memory: [0] peak of the bytes allocated at once by the
   running requests (every device allocation of their tree, plan and
   evaluation, metered on the worker threads; the workers return freed blocks
   to the pool rather than to the library's block cache), [1] budget bytes,
   [2] largest ratio of a completed request's measured peak to the estimate
   that admission used for it.  Shared operator tables (one copy per device,
   p and precision, built by the first request that needs them) count toward
   that request. */
int fmm_server_memory(fmm_server* server, double* out3);
/* Small requests (at most 65,536 points) are solved in batches with the
   queued requests that can share their plan (fmm_solve_batch); the number of
   batches and of requests solved in them so far. */
int fmm_server_batch_stats(fmm_server* server, int64_t* batches, int64_t* batched_requests);

/* Number of kernels this library has launched in this process. */
int fmm_launch_count(int64_t* count);

#ifdef __cplusplus
}
#endif

#endif
