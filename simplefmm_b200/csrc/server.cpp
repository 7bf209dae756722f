// Serving loop: FMM solves of different N, p and precision submitted as they
// arrive, run concurrently on one device.
//
// Continuous batching at the request level: `slots` worker threads each own
// a context (a device + its own CUDA stream).  A submitted request waits in
// a FIFO queue until a slot is free and its estimated device memory fits the
// budget beside the requests already running; it is then admitted, builds
// its tree, sets up its plan and evaluates on its slot's stream, so the
// kernels of all admitted requests overlap on the device.  When it finishes
// its memory and slot return to the pool and the next queued request that
// fits is admitted.  A request larger than the whole budget is rejected at
// submission (FMM_ERR_OVER_BUDGET).
//
// Memory: admission sums per-request estimates (estimate_bytes) against the
// budget.  Every device allocation a request makes is metered on its worker
// thread (its own peak, and the server's live total over running requests),
// and a server's workers bypass the library's block cache, so freed blocks go
// back to the pool: fmm_server_memory reports the measured peak of the
// running requests' device memory beside the budget, and the largest ratio
// of a request's measured peak to its estimate.
//
// Leaf size: a request may name max_particles_per_node, or pass 0 to let the
// server's autotuner choose: per (p, precision, log2 N) bucket it tries each
// candidate leaf size twice, timing the solve's own tree build and
// evaluation on the device (CUDA events on its stream, after the operator
// tables exist), keeps each candidate's best rate, and then uses the fastest.
//
// Small solves are batched: a worker that admits a request of at most
// kBatchMaxPoints points also takes the queued requests that can share its
// plan (same order, precision, charge components and outputs), up to
// kBatchMaxCount requests or kBatchPoints points in all, scanning the first
// kBatchScan queued requests, and solves them together with fmm_solve_batch:
// their trees merged into one forest, one plan, one graph-launched evaluation
// whose persistent near-field and M2L kernels take the work of all of them.
// A small request always goes this way, alone or with others, so its result
// does not depend on its company (bit for bit: no sum crosses two requests).
//
// Latency is measured from submission to completion (queueing included);
// fmm_server_stats reports its p50 / p99 over completed requests.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "alloc_meter.h"
#include "i8_ops.h"
#include "simplefmm_b200.h"

namespace sfmm {
int record_failure(int status, const char* msg);
}

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t id = 0;
    const double* xyz = nullptr;
    int64_t n = 0;
    const double* Q = nullptr;
    int qdim = 1, p = 0, precision = 0, leaf = 0;
    double* pot = nullptr;
    double* field = nullptr;
    size_t bytes = 0;                 // estimated device memory (admission)
    int64_t measured = 0;             // measured peak of its device allocations
    bool tuned = false;               // leaf size chosen by the autotuner
    Clock::time_point t_submit, t_done;
    int status = FMM_OK;
    std::string error;
    bool done = false;
};

constexpr int kLeafCandidates[] = {32, 64, 128};
constexpr int64_t kBatchMaxPoints = 65536;      // requests batched with others
constexpr int kBatchMaxCount = 32;
constexpr int64_t kBatchPoints = 1 << 20;
constexpr size_t kBatchScan = 256;

// Device memory of one solve: tree (points, keys, lists) and plan
// (expansions of order p for qdim components, outputs).  Nodes per point and
// interaction-list entries per node are taken at their high end (Plummer-like
// clustering) so the budget is not overrun.
size_t estimate_bytes(int64_t n, int p, int qdim, int leaf, int precision)
{
    const double T = (p + 1) * (p + 2) / 2.0, T1 = (p + 2) * (p + 3) / 2.0;
    const double nodes = std::max<double>(64.0, 2.5 * double(n) / std::max(leaf, 8));
    // points (two frames), sort scratch, I/O; colleague lists and leaf ids
    // are first allocated for n / 8 nodes (15 B per point)
    const double per_point = 48 + 48 + 48 + 8.0 * (qdim + 3) * 3 + 16;
    double per_node = 16.0 * qdim * (2 * T + T1) + 190 * 8 + 64;         // M, LA, LB, ilist, node arrays
    // mixed plans' tensor-core M2L (m2l_i8.cu): slot table, block lists and
    // four digits of the padded real moments per node
    if (precision == FMM_PRECISION_MIXED && p <= sfmm::kI8MaxOrder)
        per_node += 216 * 4 + 16 + 4.0 * 32 * ((p + 1) * (p + 1) / 32 + 1) * qdim;
    return static_cast<size_t>(per_point * double(n) + per_node * nodes + (64 << 20));
}

constexpr int kTrialsPerCandidate = 2;

struct Autotuner {
    std::mutex mu;
    struct Bucket {
        double best_rate[3] = {0, 0, 0};
        int tried = 0;                // trials handed out, candidate tried % 3
    };
    std::map<std::tuple<int, int, int>, Bucket> buckets;

    static std::tuple<int, int, int> key(const Request& r)
    {
        return {r.p, r.precision, static_cast<int>(std::log2(double(std::max<int64_t>(r.n, 1))))};
    }
    // Called once a request has been accepted (after the budget check), so a
    // rejected request takes no trial.
    int choose(const Request& r)
    {
        std::lock_guard<std::mutex> lk(mu);
        Bucket& b = buckets[key(r)];
        if (b.tried < 3 * kTrialsPerCandidate) return kLeafCandidates[b.tried++ % 3];
        int best = 1;
        for (int i = 0; i < 3; ++i)
            if (b.best_rate[i] > b.best_rate[best]) best = i;
        return kLeafCandidates[best];
    }
    // device_ms: the request's tree build + evaluation on its stream
    void report(const Request& r, double device_ms)
    {
        if (!(device_ms > 0)) return;
        std::lock_guard<std::mutex> lk(mu);
        Bucket& b = buckets[key(r)];
        for (int i = 0; i < 3; ++i)
            if (kLeafCandidates[i] == r.leaf) b.best_rate[i] = std::max(b.best_rate[i], double(r.n) / device_ms);
    }
};

}  // namespace

struct fmm_server {
    int device = 0;
    size_t budget = 0;
    std::vector<fmm_context*> ctx;
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::unordered_map<int64_t, std::shared_ptr<Request>> all;
    size_t in_use = 0, peak_in_use = 0;
    int running = 0, peak_running = 0;
    sfmm::AllocMeter meter;               // measured device bytes of the running requests
    double worst_ratio = 0;               // largest measured / estimated over completed requests
    int64_t next_id = 1;
    bool stopping = false;
    std::vector<double> latencies_ms;
    int64_t batches = 0, batched = 0;
    Autotuner tuner;

    void worker(int slot);
    void run(fmm_context* c, Request& r);
    void run_batch(fmm_context* c, std::vector<std::shared_ptr<Request>>& rs);
    void finish(Request& r);
};

void fmm_server::run_batch(fmm_context* c, std::vector<std::shared_ptr<Request>>& rs)
{
    sfmm::AllocMeter own;
    sfmm::set_thread_alloc_meters(&own, &meter);
    std::vector<fmm_batch_item> items(rs.size());
    for (size_t k = 0; k < rs.size(); ++k) {
        const Request& r = *rs[k];
        items[k] = fmm_batch_item{r.xyz, r.n, r.Q, r.leaf, r.pot, r.field};
    }
    const Request& r0 = *rs[0];
    const int rc = fmm_solve_batch(c, items.data(), static_cast<int>(items.size()), r0.p, r0.qdim, r0.precision, 20);
    const std::string err = rc == FMM_OK ? std::string() : std::string(fmm_last_error());
    sfmm::set_thread_alloc_meters(nullptr, nullptr);
    // the batch's measured peak, shared in proportion to the requests' estimates
    size_t total = 0;
    for (auto& r : rs) total += r->bytes;
    for (auto& r : rs) {
        r->status = rc;
        r->error = err;
        r->measured = total ? int64_t(double(own.peak.load()) * double(r->bytes) / double(total)) : 0;
    }
}

void fmm_server::finish(Request& r)
{
    r.t_done = Clock::now();
    r.done = true;
    in_use -= r.bytes;
    --running;
    if (r.bytes) worst_ratio = std::max(worst_ratio, double(r.measured) / double(r.bytes));
    if (r.status == FMM_OK) latencies_ms.push_back(std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count());
}

void fmm_server::run(fmm_context* c, Request& r)
{
    fmm_tree* tree = nullptr;
    fmm_plan* plan = nullptr;
    sfmm::AllocMeter own;
    sfmm::set_thread_alloc_meters(&own, &meter);
    int rc = fmm_tree_build(c, r.xyz, r.n, FMM_HOST, 20, r.leaf, 2, 0.0, &tree);
    if (rc == FMM_OK) rc = fmm_plan_create(tree, r.p, r.qdim, r.precision, &plan);
    if (rc == FMM_OK) rc = fmm_evaluate(plan, r.Q, r.pot, r.field, FMM_HOST);
    if (rc != FMM_OK) r.error = fmm_last_error();
    double ms6[6] = {0, 0, 0, 0, 0, 0};
    if (rc == FMM_OK && r.tuned && fmm_plan_timings(plan, ms6) != FMM_OK) ms6[4] = ms6[5] = 0;
    if (plan) fmm_plan_destroy(plan);
    if (tree) fmm_tree_destroy(tree);
    sfmm::set_thread_alloc_meters(nullptr, nullptr);
    r.measured = own.peak.load();
    r.status = rc;
    if (rc == FMM_OK && r.tuned) tuner.report(r, ms6[4] + ms6[5]);
}

void fmm_server::worker(int slot)
{
    fmm_context* c = ctx[slot];
    sfmm::set_thread_block_cache(false);
    for (;;) {
        std::vector<std::shared_ptr<Request>> rs;
        {
            std::unique_lock<std::mutex> lk(mu);
            // admit the oldest queued request once its memory fits beside the running ones
            cv_work.wait(lk, [&] {
                return (!queue.empty() && in_use + queue.front()->bytes <= budget) || (stopping && queue.empty());
            });
            if (queue.empty()) return;                      // stopping and drained
            rs.push_back(queue.front());
            queue.pop_front();
            in_use += rs[0]->bytes;
            const Request& r0 = *rs[0];
            if (r0.n <= kBatchMaxPoints) {
                // the queued small requests that can share its plan, while memory allows
                int64_t pts = r0.n;
                for (auto it = queue.begin(); it != queue.end() && size_t(it - queue.begin()) < kBatchScan &&
                                              rs.size() < size_t(kBatchMaxCount);) {
                    const Request& q = **it;
                    if (q.n <= kBatchMaxPoints && q.p == r0.p && q.precision == r0.precision && q.qdim == r0.qdim &&
                        (q.pot != nullptr) == (r0.pot != nullptr) && (q.field != nullptr) == (r0.field != nullptr) &&
                        pts + q.n <= kBatchPoints && in_use + q.bytes <= budget) {
                        pts += q.n;
                        in_use += q.bytes;
                        rs.push_back(*it);
                        it = queue.erase(it);
                    } else {
                        ++it;
                    }
                }
                ++batches;
                batched += int64_t(rs.size());
            }
            peak_in_use = std::max(peak_in_use, in_use);
            running += int(rs.size());
            peak_running = std::max(peak_running, running);
        }
        if (rs[0]->n <= kBatchMaxPoints) run_batch(c, rs);
        else run(c, *rs[0]);
        {
            std::lock_guard<std::mutex> lk(mu);
            for (auto& r : rs) finish(*r);
        }
        cv_done.notify_all();
        cv_work.notify_all();
    }
}

extern "C" {

int fmm_server_create(int device, int slots, size_t memory_budget, fmm_server** out)
{
    if (!out || slots < 1 || slots > 64 || memory_budget == 0)
        return sfmm::record_failure(FMM_ERR_INVALID_ARGUMENT, "need out != NULL, 1 <= slots <= 64, memory_budget > 0");
    *out = nullptr;
    auto* s = new fmm_server;
    s->device = device;
    s->budget = memory_budget;
    for (int i = 0; i < slots; ++i) {
        fmm_context* c = nullptr;
        const int rc = fmm_context_create(device, &c);
        if (rc != FMM_OK) {
            for (auto* x : s->ctx) fmm_context_destroy(x);
            delete s;
            return rc;
        }
        s->ctx.push_back(c);
    }
    for (int i = 0; i < slots; ++i) s->workers.emplace_back(&fmm_server::worker, s, i);
    *out = s;
    return FMM_OK;
}

int fmm_server_destroy(fmm_server* s)
{
    if (!s) return FMM_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    for (auto* c : s->ctx) fmm_context_destroy(c);
    delete s;
    return FMM_OK;
}

int fmm_server_submit(fmm_server* s, const double* xyz, int64_t n, const double* Q, int qdim, int p, int precision,
                      int max_particles_per_node, double* pot, double* field, int64_t* id)
{
    if (!s || !xyz || !Q || !id || n <= 0 || qdim < 1 || qdim > 3 || p < 0 || p > 16 || max_particles_per_node < 0)
        return sfmm::record_failure(FMM_ERR_INVALID_ARGUMENT, "bad request arguments");
    if (!pot && !field) return sfmm::record_failure(FMM_ERR_INVALID_ARGUMENT, "request asks for no output");
    auto r = std::make_shared<Request>();
    r->xyz = xyz;
    r->n = n;
    r->Q = Q;
    r->qdim = qdim;
    r->p = p;
    r->precision = precision;
    r->pot = pot;
    r->field = field;
    r->tuned = max_particles_per_node == 0;
    // the budget check takes the smallest candidate leaf (the largest
    // estimate) for an autotuned request, before it takes a trial
    r->leaf = r->tuned ? kLeafCandidates[0] : max_particles_per_node;
    r->bytes = estimate_bytes(n, p, qdim, r->leaf, r->precision);
    if (r->bytes > s->budget)
        return sfmm::record_failure(FMM_ERR_OVER_BUDGET, "request's estimated device memory exceeds the server budget");
    if (r->tuned) r->leaf = s->tuner.choose(*r);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stopping) return sfmm::record_failure(FMM_ERR_INVALID_ARGUMENT, "server is stopping");
        r->id = s->next_id++;
        r->t_submit = Clock::now();
        s->all[r->id] = r;
        s->queue.push_back(r);
        *id = r->id;
    }
    s->cv_work.notify_all();
    return FMM_OK;
}

int fmm_server_poll(fmm_server* s, int64_t id, int* done)
{
    if (!s || !done) return FMM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return sfmm::record_failure(FMM_ERR_INVALID_ARGUMENT, "unknown request id");
    *done = it->second->done ? 1 : 0;
    return FMM_OK;
}

int fmm_server_wait(fmm_server* s, int64_t id, double* latency_ms)
{
    if (!s) return FMM_ERR_INVALID_ARGUMENT;
    std::shared_ptr<Request> r;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->all.find(id);
        if (it == s->all.end()) return sfmm::record_failure(FMM_ERR_INVALID_ARGUMENT, "unknown request id");
        r = it->second;
        s->cv_done.wait(lk, [&] { return r->done; });
        s->all.erase(it);
    }
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    if (r->status != FMM_OK) return sfmm::record_failure(r->status, r->error.c_str());
    return FMM_OK;
}

int fmm_server_stats(fmm_server* s, double* stats8)
{
    if (!s || !stats8) return FMM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    std::vector<double> v = s->latencies_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) {
        if (v.empty()) return 0.0;
        const size_t i = std::min(v.size() - 1, static_cast<size_t>(std::ceil(q * v.size())) - (q > 0 ? 1 : 0));
        return v[i];
    };
    double mean = 0;
    for (double x : v) mean += x;
    stats8[0] = double(v.size());
    stats8[1] = pct(0.50);
    stats8[2] = pct(0.99);
    stats8[3] = v.empty() ? 0.0 : mean / v.size();
    stats8[4] = double(s->peak_running);
    stats8[5] = double(s->peak_in_use);
    stats8[6] = double(s->budget);
    stats8[7] = double(s->queue.size());
    return FMM_OK;
}

int fmm_server_batch_stats(fmm_server* s, int64_t* batches, int64_t* batched_requests)
{
    if (!s || !batches || !batched_requests) return sfmm::record_failure(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *batches = s->batches;
    *batched_requests = s->batched;
    return FMM_OK;
}

int fmm_server_memory(fmm_server* s, double* out3)
{
    if (!s || !out3) return sfmm::record_failure(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    out3[0] = double(s->meter.peak.load());
    out3[1] = double(s->budget);
    out3[2] = s->worst_ratio;
    return FMM_OK;
}

}  // extern "C"
