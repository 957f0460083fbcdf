// BFS query server: resident graphs, continuous batching, a device-memory
// budget (include/b40c_server.h).
//
// One dispatcher thread owns all GPU work of a server.  Each in-flight slot
// has a CUDA stream of its own, so batches of different graphs (and the label
// read-back of one with the search of another) overlap on the device; a
// batch's persistent grid takes a share of every SM (ctas_per_sm), so several
// grids are resident side by side.  The dispatcher's loop:
//   1. queries whose arrival time has come move from the arrival heap to their
//      graph's FIFO;
//   2. finished batches (any slot, in whatever order they finish) are retired:
//      results, latencies, labels already copied;
//   3. while a slot is free and some graph with waiting queries has no batch in
//      flight, the graph whose oldest waiting query arrived first gets a batch
//      of up to its width on that slot's stream: the batched kernel for two or
//      more queries, the plain search for one;
//   4. it spins (yielding) while batches are in flight, otherwise sleeps until
//      the next arrival or a submit.
// Queries for a graph that already has a batch in flight wait and gather into
// its next batch: that is the continuous batching.  Removing a graph returns
// its bytes to the budget and widens the other graphs' batches again.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <queue>
#include <thread>
#include <vector>

#include "b40c_server.h"
#include "problem.h"

extern "C" int b40c_bfs_enact_limited(b40c_bfs_problem *p, int strategy, int mode, int32_t src, int32_t depth_limit,
                                      int max_grid_size, const b40c_bfs_policy *policy);
extern "C" int b40c_msbfs_enact(b40c_bfs_problem *p, const int32_t *sources, const int32_t *depth_limits, int k,
                                int max_grid_size, const b40c_bfs_policy *policy);
extern "C" int b40c_bfs_problem_create(const int32_t *row_offsets, const int32_t *column_indices, int64_t nodes,
                                       int64_t edges, int mark_predecessors, int stream_from_host, int device,
                                       b40c_bfs_problem **out);
extern "C" int b40c_bfs_problem_destroy(b40c_bfs_problem *p);

namespace b40c {
namespace server {

constexpr double kQueueSizing = 1.3;

struct Query {
    int64_t ticket;
    int32_t graph, source, depth_limit;
    int32_t *h_labels;
    bool pinned;  // h_labels is page-locked: copied asynchronously behind the search
    int64_t arrival_ns;
};

struct LaterArrival {
    bool operator()(const Query &a, const Query &b) const
    {
        return a.arrival_ns != b.arrival_ns ? a.arrival_ns > b.arrival_ns : a.ticket > b.ticket;
    }
};

struct Graph {
    b40c_bfs_problem *p = nullptr;
    int64_t nodes = 0, edges = 0;
    int32_t width = 0;        // batch width admitted
    int64_t bytes = 0;        // device bytes charged to the budget
    bool busy = false;        // a batch of this graph is in flight
    bool removed = false;
    int64_t pending = 0;      // queries submitted and not yet finished
    std::deque<Query> ready;  // arrived, waiting for a batch
    bool has_single = false, has_batch = false;
    b40c_bfs_policy single{}, batch{};  // tuned policies (else the library defaults)
};

// Page-locked landing area of one in-flight batch.
struct Landing {
    int32_t depth[64];
    uint32_t error;
    int32_t max_level;
    int32_t taken;  // join requests the batched search took
};

struct Batch {
    int graph;
    std::vector<Query> queries;  // the batch's own k, then the ones sent to join it
    std::vector<int64_t> join_ns;  // when each joining query was sent
    int k = 0;                   // queries the batch was launched with
    bool single;
    int slot;
    int64_t launch_ns;
};

}  // namespace server
}  // namespace b40c

using namespace b40c;
using namespace b40c::server;

struct b40c_server {
    int device = 0;
    int32_t max_batch = 64, single_strategy = B40C_DIRECTION_OPTIMIZING, max_in_flight = 2;
    int32_t ctas_per_sm = 0;  // of each batch's persistent grid (0: the policy's)
    int64_t budget = 0, used = 0;
    cudaStream_t *streams = nullptr;  // [max_in_flight]: one per in-flight slot
    std::chrono::steady_clock::time_point t0;
    std::vector<Graph *> graphs;
    std::mutex mu;
    std::mutex admin;  // serialises add_graph / remove_graph (admission reads then charges the budget)
    std::condition_variable cv_work, cv_done;
    std::priority_queue<Query, std::vector<Query>, LaterArrival> arrivals;
    std::vector<b40c_server_result> results;  // by ticket
    std::deque<Batch> in_flight;
    Landing *landing = nullptr;               // [max_in_flight], page-locked
    cudaEvent_t *done_ev = nullptr;           // [max_in_flight]
    cudaEvent_t *gpu_ev = nullptr;            // [2 * max_in_flight]: timing events around each slot's search
    cudaEvent_t base_ev = nullptr;            // device-clock origin (recorded at creation)
    std::vector<int> free_slots;
    int64_t submitted = 0, completed = 0, failed = 0, batches = 0, batched_queries = 0, single_queries = 0;
    int64_t joined_queries = 0;  // queries answered by joining a batch in flight
    bool stop = false;
    int thread_error = 0;
    std::thread worker;

    int64_t now() const
    {
        return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

// Marks the queries of a batch finished (called with the lock held): its own
// and the joining ones the search took; joining queries it did not take go
// back to the head of their graph's queue, in order.
void finish_batch(b40c_server *s, Batch &b, int status, int64_t finish_ns)
{
    Graph &g = *s->graphs[b.graph];
    const Landing &l = s->landing[b.slot];
    const int joined = (int)b.queries.size() - b.k;
    const int taken = (status == B40C_SUCCESS && joined > 0) ? std::max(0, std::min(joined, l.taken)) : 0;
    if (status == B40C_SUCCESS && taken < joined) {
        for (int i = (int)b.queries.size() - 1; i >= b.k + taken; i--) g.ready.push_front(b.queries[i]);
        b.queries.resize(b.k + taken);
    }
    s->joined_queries += taken;
    s->batched_queries += taken;
    // labels bound for pageable host memory: copied now, from the rows the batch
    // left on the device (its graph's next batch cannot start before this
    // returns); a copy queued behind the search would have made the dispatcher
    // wait for the whole search
    if (status == B40C_SUCCESS) {
        for (size_t i = 0; i < b.queries.size(); i++) {
            const Query &q = b.queries[i];
            if (!q.h_labels || q.pinned) continue;
            const int32_t *src = b.single ? g.p->d_labels : g.p->d_ms_labels + i * (size_t)g.nodes;
            if (cudaMemcpy(q.h_labels, src, sizeof(int32_t) * g.nodes, cudaMemcpyDeviceToHost) != cudaSuccess) {
                cudaGetLastError();
                status = B40C_ERROR_INVALID_VALUE;
            }
        }
    }
    float t0 = 0.f, t1 = 0.f;
    if (status == B40C_SUCCESS &&
        (cudaEventElapsedTime(&t0, s->base_ev, s->gpu_ev[2 * b.slot]) != cudaSuccess ||
         cudaEventElapsedTime(&t1, s->base_ev, s->gpu_ev[2 * b.slot + 1]) != cudaSuccess)) {
        cudaGetLastError();
        t0 = t1 = 0.f;
    }
    for (size_t i = 0; i < b.queries.size(); i++) {
        const Query &q = b.queries[i];
        b40c_server_result &r = s->results[q.ticket];
        r.status = status;
        r.search_depth = status ? 0 : (b.single ? l.max_level + 1 : l.depth[i]);
        r.batch_size = (int32_t)b.queries.size();
        r.launch_ns = i < (size_t)b.k ? b.launch_ns : b.join_ns[i - b.k];
        r.finish_ns = finish_ns;
        r.gpu_start_ns = (int64_t)((double)t0 * 1e6);
        r.gpu_end_ns = (int64_t)((double)t1 * 1e6);
        g.pending--;
        s->completed++;
        if (status) s->failed++;
    }
    g.busy = false;
    s->free_slots.push_back(b.slot);
}

// The policy of one batch: the graph's (or the library default) with the
// grid share of the server applied.
const b40c_bfs_policy *batch_policy(const b40c_server *s, const Graph &g, bool single, b40c_bfs_policy *buf)
{
    const bool has = single ? g.has_single : g.has_batch;
    if (!has && s->ctas_per_sm == 0) return nullptr;
    *buf = has ? (single ? g.single : g.batch) : b40c_bfs_policy{};
    if (s->ctas_per_sm > 0 && (buf->ctas_per_sm == 0 || buf->ctas_per_sm > s->ctas_per_sm))
        buf->ctas_per_sm = s->ctas_per_sm;
    return buf;
}

// Issues one batch on its slot's stream (lock held; the calls only queue work).
int issue(b40c_server *s, Batch &b)
{
    Graph &g = *s->graphs[b.graph];
    b40c_bfs_problem *p = g.p;
    Landing *l = s->landing + b.slot;
    cudaStream_t st = s->streams[b.slot];
    p->stream = st;  // a graph has at most one batch in flight: its buffers are this stream's alone
    const int k = (int)b.queries.size();
    b40c_bfs_policy pol;
    int rc;
    CUDA_TRY(cudaEventRecord(s->gpu_ev[2 * b.slot], st), "event record");
    if (b.single) {
        const Query &q = b.queries[0];
        rc = b40c_bfs_enact_limited(p, s->single_strategy, B40C_ENACT_FUSED, q.source, q.depth_limit, 0,
                                    batch_policy(s, g, true, &pol));
        if (rc) return rc;
        CUDA_TRY(cudaEventRecord(s->gpu_ev[2 * b.slot + 1], st), "event record");
        CUDA_TRY(cudaMemcpyAsync(&l->max_level, &p->st->max_level, sizeof(int32_t), cudaMemcpyDeviceToHost, st),
                 "depth copy");
        if (q.h_labels && q.pinned)
            CUDA_TRY(cudaMemcpyAsync(q.h_labels, p->d_labels, sizeof(int32_t) * g.nodes, cudaMemcpyDeviceToHost, st),
                     "label copy");
    } else {
        int32_t src[64], lim[64];
        for (int i = 0; i < k; i++) {
            src[i] = b.queries[i].source;
            lim[i] = b.queries[i].depth_limit;
        }
        rc = b40c_msbfs_enact(p, src, lim, k, 0, batch_policy(s, g, false, &pol));
        if (rc) return rc;
        CUDA_TRY(cudaEventRecord(s->gpu_ev[2 * b.slot + 1], st), "event record");
        CUDA_TRY(cudaMemcpyAsync(l->depth, p->d_ms_depth, sizeof(int32_t) * 64, cudaMemcpyDeviceToHost, st),
                 "depth copy");
        CUDA_TRY(cudaMemcpyAsync(&l->taken, &p->d_ms_join->taken, sizeof(int32_t), cudaMemcpyDeviceToHost, st),
                 "join count copy");
        for (int i = 0; i < k; i++)
            if (b.queries[i].h_labels && b.queries[i].pinned)
                CUDA_TRY(cudaMemcpyAsync(b.queries[i].h_labels, p->d_ms_labels + (size_t)i * (size_t)g.nodes,
                                         sizeof(int32_t) * g.nodes, cudaMemcpyDeviceToHost, st),
                         "label copy");
    }
    CUDA_TRY(cudaMemcpyAsync(&l->error, &p->st->error, sizeof(uint32_t), cudaMemcpyDeviceToHost, st),
             "error word copy");
    CUDA_TRY(cudaEventRecord(s->done_ev[b.slot], st), "event record");
    return B40C_SUCCESS;
}

// Sends the waiting queries of a graph whose batched search is in flight to
// join it, while it has free slots (lock held).  Each joining query's labels
// are copied from its slot after the search (queued on the batch's stream
// behind the search), then the batch's depths, join count and error word are
// copied again and its completion event re-recorded, so the batch retires
// only after all of them.  Returns true when any query was sent.
bool join_waiting(b40c_server *s, Batch &b)
{
    if (b.single) return false;
    Graph &g = *s->graphs[b.graph];
    b40c_bfs_problem *p = g.p;
    Landing *l = s->landing + b.slot;
    cudaStream_t st = s->streams[b.slot];
    const int rows = std::min(64, (int)std::min<int64_t>(g.width, p->ms_labels_k));
    bool sent = false;
    while (!g.ready.empty() && (int)b.queries.size() < rows) {
        const Query q = g.ready.front();
        const int slot = (int)b.queries.size();
        if (b40c_msbfs_join(p, slot, q.source, q.depth_limit) != B40C_SUCCESS) break;
        g.ready.pop_front();
        b.queries.push_back(q);
        b.join_ns.push_back(s->now());
        if (q.h_labels && q.pinned &&
            cudaMemcpyAsync(q.h_labels, p->d_ms_labels + (size_t)slot * (size_t)g.nodes, sizeof(int32_t) * g.nodes,
                            cudaMemcpyDeviceToHost, st) != cudaSuccess)
            cudaGetLastError();  // the query then reports the batch's status with stale labels: not expected
        sent = true;
    }
    if (sent) {
        if (cudaMemcpyAsync(l->depth, p->d_ms_depth, sizeof(int32_t) * 64, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(&l->taken, &p->d_ms_join->taken, sizeof(int32_t), cudaMemcpyDeviceToHost, st) !=
                cudaSuccess ||
            cudaMemcpyAsync(&l->error, &p->st->error, sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaEventRecord(s->done_ev[b.slot], st) != cudaSuccess)
            cudaGetLastError();
    }
    return sent;
}

// The graph whose oldest waiting query arrived first among graphs without a
// batch in flight, or -1.
int next_graph(b40c_server *s)
{
    int best = -1;
    int64_t best_t = 0;
    for (size_t i = 0; i < s->graphs.size(); i++) {
        Graph *g = s->graphs[i];
        if (!g || g->removed || g->busy || g->ready.empty()) continue;
        const Query &q = g->ready.front();
        if (best < 0 || q.arrival_ns < best_t || (q.arrival_ns == best_t && q.ticket < s->graphs[best]->ready.front().ticket)) {
            best = (int)i;
            best_t = q.arrival_ns;
        }
    }
    return best;
}

void dispatcher(b40c_server *s)
{
    if (cudaSetDevice(s->device) != cudaSuccess) {
        cudaGetLastError();
        std::lock_guard<std::mutex> lk(s->mu);
        s->thread_error = B40C_ERROR_NO_DEVICE;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        int64_t t = s->now();
        // 1. arrivals that are due
        while (!s->arrivals.empty() && s->arrivals.top().arrival_ns <= t) {
            Query q = s->arrivals.top();
            s->arrivals.pop();
            s->graphs[q.graph]->ready.push_back(q);
        }
        // 2. retire finished batches (slots run on their own streams: any order)
        bool retired = false;
        for (auto it = s->in_flight.begin(); it != s->in_flight.end();) {
            Batch &b = *it;
            const cudaError_t e = cudaEventQuery(s->done_ev[b.slot]);
            if (e == cudaErrorNotReady) {
                ++it;
                continue;
            }
            int status = B40C_SUCCESS;
            if (e != cudaSuccess) {
                cudaGetLastError();
                status = (int)e;
            } else {
                const uint32_t w = s->landing[b.slot].error;
                if (w & dev::kErrOverflow)
                    status = B40C_ERROR_INVALID_CONFIGURATION;
                else if (w)
                    status = B40C_ERROR_LAUNCH_TIMEOUT;
            }
            finish_batch(s, b, status, s->now());
            it = s->in_flight.erase(it);
            retired = true;
        }
        // a dispatcher without a device fails what is waiting instead of issuing it
        if (s->thread_error) {
            for (size_t gi = 0; gi < s->graphs.size(); gi++) {
                Graph *g = s->graphs[gi];
                while (g && !g->ready.empty()) {
                    b40c_server_result &r = s->results[g->ready.front().ticket];
                    r.status = s->thread_error;
                    r.finish_ns = s->now();
                    g->ready.pop_front();
                    g->pending--;
                    s->completed++;
                    s->failed++;
                    retired = true;
                }
            }
        }
        if (retired) s->cv_done.notify_all();
        // 3. waiting queries of a graph whose batch is running join it (its free
        // slots), the rest wait for a batch of their own
        if (!s->thread_error)
            for (Batch &b : s->in_flight) join_waiting(s, b);
        // 4. issue batches
        while ((int)s->in_flight.size() < s->max_in_flight && !s->free_slots.empty() && !s->thread_error) {
            const int gi = next_graph(s);
            if (gi < 0) break;
            Graph &g = *s->graphs[gi];
            Batch b;
            b.graph = gi;
            b.slot = s->free_slots.back();
            s->free_slots.pop_back();
            const int k = std::min<int>(g.width, (int)g.ready.size());
            for (int i = 0; i < k; i++) {
                b.queries.push_back(g.ready.front());
                g.ready.pop_front();
            }
            b.k = k;
            b.single = (k == 1 && s->single_strategy >= 0);
            b.launch_ns = s->now();
            g.busy = true;
            const int rc = issue(s, b);
            if (rc) {
                finish_batch(s, b, rc, s->now());
                s->cv_done.notify_all();
                continue;
            }
            s->batches++;
            if (b.single)
                s->single_queries++;
            else
                s->batched_queries += k;
            s->in_flight.push_back(std::move(b));
        }
        // 5. wait
        bool waiting = false;
        for (Graph *g : s->graphs)
            if (g && !g->ready.empty()) waiting = true;
        if (s->stop && s->in_flight.empty() && s->arrivals.empty() && !waiting) break;
        if (!s->in_flight.empty()) {
            lk.unlock();
            std::this_thread::yield();
            lk.lock();
        } else if (!s->arrivals.empty()) {
            const int64_t dt = s->arrivals.top().arrival_ns - s->now();
            if (dt > 200000) {
                s->cv_work.wait_for(lk, std::chrono::nanoseconds(dt - 100000));
            } else {
                lk.unlock();
                std::this_thread::yield();
                lk.lock();
            }
        } else {
            s->cv_work.wait(lk);
        }
    }
}

int check_query(b40c_server *s, int32_t graph, int32_t source)
{
    if (graph < 0 || graph >= (int32_t)s->graphs.size() || !s->graphs[graph] || s->graphs[graph]->removed)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "no graph %d in the server", graph);
    if (source < 0 || source >= s->graphs[graph]->nodes)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "source %d out of range for graph %d", source, graph);
    return B40C_SUCCESS;
}

// Queues one checked query (lock held).
int64_t enqueue(b40c_server *s, int32_t graph, int32_t source, int32_t depth_limit, int32_t *h_labels,
                int64_t arrival_ns)
{
    Query q;
    q.ticket = (int64_t)s->results.size();
    q.graph = graph;
    q.source = source;
    q.depth_limit = depth_limit < 0 ? -1 : depth_limit;
    q.h_labels = h_labels;
    q.pinned = false;
    if (h_labels) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, h_labels) == cudaSuccess)
            q.pinned = a.type == cudaMemoryTypeHost;
        else
            cudaGetLastError();
    }
    q.arrival_ns = arrival_ns < 0 ? s->now() : arrival_ns;
    b40c_server_result r{};
    r.ticket = q.ticket;
    r.graph = graph;
    r.source = source;
    r.depth_limit = q.depth_limit;
    r.status = B40C_ERROR_NOT_READY;
    r.arrival_ns = q.arrival_ns;
    s->results.push_back(r);
    s->graphs[graph]->pending++;
    s->submitted++;
    s->arrivals.push(q);
    return q.ticket;
}

}  // namespace

extern "C" {

int b40c_server_plan_bytes(int64_t nodes, int64_t edges, int32_t max_batch, int64_t *device_bytes)
{
    b40c::clear_error();
    if (!device_bytes || nodes < 1 || edges < 0 || max_batch < 1 || max_batch > 64)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "bad arguments");
    *device_bytes = rt::planned_bytes(nodes, edges, max_batch, kQueueSizing);
    return B40C_SUCCESS;
}

int b40c_server_create(int device, const b40c_server_options *options, b40c_server **out)
{
    b40c::clear_error();
    if (!out) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null out");
    *out = nullptr;
    b40c_server_options o{};
    if (options) o = *options;
    if (o.max_batch < 0 || o.max_batch > 64) return b40c::fail(B40C_ERROR_INVALID_VALUE, "max_batch must be in 0..64");
    if (o.single_strategy == 0) o.single_strategy = B40C_DIRECTION_OPTIMIZING;
    if (o.single_strategy != -1 && o.single_strategy != B40C_DIRECTION_OPTIMIZING &&
        o.single_strategy != B40C_EXPAND_CONTRACT)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "single_strategy must be -1, B40C_EXPAND_CONTRACT or "
                                                    "B40C_DIRECTION_OPTIMIZING");
    if (o.max_in_flight < 0 || o.max_in_flight > 16)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "max_in_flight must be in 0..16");
    if (o.memory_budget_bytes < 0) return b40c::fail(B40C_ERROR_INVALID_VALUE, "negative memory budget");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) {
        cudaGetLastError();
        return b40c::fail(B40C_ERROR_NO_DEVICE, "no CUDA device");
    }
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return b40c::fail(B40C_ERROR_NO_DEVICE, "no current CUDA device");
    }
    if (device >= count) return b40c::fail(B40C_ERROR_INVALID_VALUE, "device %d out of range", device);
    rt::DeviceGuard guard(device);
    auto *s = new b40c_server();
    s->device = device;
    s->max_batch = o.max_batch ? o.max_batch : 64;
    s->single_strategy = o.single_strategy;
    s->max_in_flight = o.max_in_flight ? o.max_in_flight : 2;
    // by default the slots split each SM evenly (the kernels are resident at 4 CTAs per SM)
    s->ctas_per_sm = o.ctas_per_sm > 0 ? o.ctas_per_sm : std::max(1, 4 / s->max_in_flight);
    if (o.ctas_per_sm < 0) s->ctas_per_sm = 0;  // -1: every batch takes the whole device
    s->t0 = std::chrono::steady_clock::now();
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        delete s;
        return b40c::fail(B40C_ERROR_NO_DEVICE, "cudaMemGetInfo failed");
    }
    s->budget = o.memory_budget_bytes ? o.memory_budget_bytes : (int64_t)(0.9 * (double)free_b);
    s->streams = new cudaStream_t[s->max_in_flight]();
    s->done_ev = new cudaEvent_t[s->max_in_flight]();
    s->gpu_ev = new cudaEvent_t[2 * s->max_in_flight]();
    auto undo = [s]() {
        for (int j = 0; j < s->max_in_flight; j++) {
            if (s->done_ev[j]) cudaEventDestroy(s->done_ev[j]);
            if (s->gpu_ev[2 * j]) cudaEventDestroy(s->gpu_ev[2 * j]);
            if (s->gpu_ev[2 * j + 1]) cudaEventDestroy(s->gpu_ev[2 * j + 1]);
            if (s->streams[j]) cudaStreamDestroy(s->streams[j]);
        }
        if (s->base_ev) cudaEventDestroy(s->base_ev);
        delete[] s->done_ev;
        delete[] s->gpu_ev;
        delete[] s->streams;
        if (s->landing) cudaFreeHost(s->landing);
        cudaGetLastError();
        delete s;
    };
    if (cudaMallocHost((void **)&s->landing, sizeof(Landing) * s->max_in_flight) != cudaSuccess) {
        s->landing = nullptr;
        undo();
        return b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "server landing area allocation failed");
    }
    for (int i = 0; i < s->max_in_flight; i++) {
        if (cudaStreamCreateWithFlags(&s->streams[i], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&s->done_ev[i], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreate(&s->gpu_ev[2 * i]) != cudaSuccess || cudaEventCreate(&s->gpu_ev[2 * i + 1]) != cudaSuccess) {
            undo();
            return b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "server stream or event creation failed");
        }
        s->free_slots.push_back(s->max_in_flight - 1 - i);
    }
    if (cudaEventCreate(&s->base_ev) != cudaSuccess || cudaEventRecord(s->base_ev, s->streams[0]) != cudaSuccess) {
        undo();
        return b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "server event creation failed");
    }
    s->worker = std::thread(dispatcher, s);
    *out = s;
    return B40C_SUCCESS;
}

int b40c_server_drain(b40c_server *s)
{
    b40c::clear_error();
    if (!s) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_work.notify_all();
    s->cv_done.wait(lk, [s] { return s->completed == s->submitted; });
    return B40C_SUCCESS;
}

int b40c_server_destroy(b40c_server *s)
{
    b40c::clear_error();
    if (!s) return B40C_SUCCESS;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    rt::DeviceGuard guard(s->device);
    for (int i = 0; i < s->max_in_flight; i++) cudaStreamSynchronize(s->streams[i]);
    for (Graph *g : s->graphs) {
        if (g && g->p) b40c_bfs_problem_destroy(g->p);
        delete g;
    }
    for (int i = 0; i < s->max_in_flight; i++) {
        cudaEventDestroy(s->done_ev[i]);
        cudaEventDestroy(s->gpu_ev[2 * i]);
        cudaEventDestroy(s->gpu_ev[2 * i + 1]);
        cudaStreamDestroy(s->streams[i]);
    }
    cudaEventDestroy(s->base_ev);
    delete[] s->done_ev;
    delete[] s->gpu_ev;
    delete[] s->streams;
    cudaFreeHost(s->landing);
    cudaGetLastError();
    delete s;
    return B40C_SUCCESS;
}

int b40c_server_add_graph(b40c_server *s, const int32_t *row_offsets, const int32_t *column_indices, int64_t nodes,
                          int64_t edges, int32_t *graph_id)
{
    b40c::clear_error();
    if (!s || !row_offsets || (!column_indices && edges > 0) || !graph_id || nodes < 1 || edges < 0)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "bad arguments");
    std::lock_guard<std::mutex> admin(s->admin);
    int64_t free_budget;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        free_budget = s->budget - s->used;
    }
    int width = s->max_batch;
    // widest power-of-two batch (at most max_batch) whose buffers fit the budget
    while (width > 1 && rt::planned_bytes(nodes, edges, width, kQueueSizing) > free_budget) {
        int w = 1;
        while (w * 2 < width) w *= 2;
        width = w;
    }
    const int64_t need = rt::planned_bytes(nodes, edges, width, kQueueSizing);
    if (need > free_budget)
        return b40c::fail(B40C_ERROR_MEMORY_ALLOCATION,
                          "graph of %lld vertices and %lld edges needs %lld device bytes; %lld of the budget left",
                          (long long)nodes, (long long)edges, (long long)need, (long long)free_budget);
    rt::DeviceGuard guard(s->device);
    b40c_bfs_problem *p = nullptr;
    int rc = b40c_bfs_problem_create(row_offsets, column_indices, nodes, edges, 0, 0, s->device, &p);
    if (rc) return rc;
    auto bail = [&](int code) {
        b40c_bfs_problem_destroy(p);
        return code;
    };
    p->stream = s->streams[0];  // set-up only; each batch runs on its slot's stream
    p->queue_sizing = kQueueSizing;
    // allocate everything a batch of full width and a single search use, now
    // rather than while serving; the searches also run the symmetry test once
    std::vector<int32_t> warm(width, 0);
    if ((rc = b40c_msbfs_enact(p, warm.data(), nullptr, width, 0, nullptr))) return bail(rc);
    if (s->single_strategy >= 0 &&
        (rc = b40c_bfs_enact_limited(p, s->single_strategy, B40C_ENACT_FUSED, 0, -1, 0, nullptr)))
        return bail(rc);
    // charged by the plan whether or not searches use them
    if ((rc = rt::ensure_hubs(p)) || (rc = rt::ensure_unvisited_lists(p))) return bail(rc);
    if (cudaStreamSynchronize(s->streams[0]) != cudaSuccess) {
        const cudaError_t e = cudaGetLastError();
        return bail(b40c::fail((int)e, "graph warm-up failed: %s", cudaGetErrorString(e)));
    }
    auto *g = new Graph();
    g->p = p;
    g->nodes = nodes;
    g->edges = edges;
    g->width = width;
    g->bytes = rt::device_bytes(p);
    std::lock_guard<std::mutex> lk(s->mu);
    s->used += g->bytes;
    *graph_id = (int32_t)s->graphs.size();
    s->graphs.push_back(g);
    return B40C_SUCCESS;
}

int b40c_server_remove_graph(b40c_server *s, int32_t graph_id)
{
    b40c::clear_error();
    if (!s) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null server");
    std::lock_guard<std::mutex> admin(s->admin);
    b40c_bfs_problem *p = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (graph_id < 0 || graph_id >= (int32_t)s->graphs.size() || !s->graphs[graph_id] ||
            s->graphs[graph_id]->removed)
            return b40c::fail(B40C_ERROR_INVALID_VALUE, "no graph %d in the server", graph_id);
        Graph *g = s->graphs[graph_id];
        if (g->pending || g->busy) return b40c::fail(B40C_ERROR_NOT_READY, "graph %d has queries pending", graph_id);
        g->removed = true;
        s->used -= g->bytes;
        p = g->p;
        g->p = nullptr;
        // the freed bytes widen the other graphs' batches again (oldest graph
        // first, up to max_batch), charged at the new width's plan; the extra
        // label rows are allocated by their next batch
        for (Graph *o : s->graphs) {
            if (!o || o->removed || o->width >= s->max_batch) continue;
            int w = o->width;
            while (w * 2 <= s->max_batch &&
                   rt::planned_bytes(o->nodes, o->edges, w * 2, kQueueSizing) - o->bytes <= s->budget - s->used)
                w *= 2;
            if (w == o->width) continue;
            const int64_t nb = rt::planned_bytes(o->nodes, o->edges, w, kQueueSizing);
            s->used += nb - o->bytes;
            o->bytes = nb;
            o->width = w;
        }
    }
    rt::DeviceGuard guard(s->device);
    return b40c_bfs_problem_destroy(p);
}

int b40c_server_set_graph_policy(b40c_server *s, int32_t graph_id, const b40c_bfs_policy *single,
                                  const b40c_bfs_policy *batch)
{
    b40c::clear_error();
    if (!s) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null server");
    b40c_bfs_policy a{}, b{};
    int rc;
    if (single && (rc = rt::resolve_policy(s->single_strategy < 0 ? B40C_EXPAND_CONTRACT : s->single_strategy, single,
                                           &a)))
        return rc;
    if (batch && (rc = rt::resolve_policy(B40C_EXPAND_CONTRACT, batch, &b))) return rc;
    std::lock_guard<std::mutex> lk(s->mu);
    if (graph_id < 0 || graph_id >= (int32_t)s->graphs.size() || !s->graphs[graph_id] || s->graphs[graph_id]->removed)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "no graph %d in the server", graph_id);
    Graph *g = s->graphs[graph_id];
    g->has_single = single != nullptr;
    g->has_batch = batch != nullptr;
    if (single) g->single = *single;
    if (batch) g->batch = *batch;
    return B40C_SUCCESS;
}

int b40c_server_graph_info(b40c_server *s, int32_t graph_id, int64_t *device_bytes, int32_t *max_batch)
{
    b40c::clear_error();
    if (!s) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (graph_id < 0 || graph_id >= (int32_t)s->graphs.size() || !s->graphs[graph_id] || s->graphs[graph_id]->removed)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "no graph %d in the server", graph_id);
    if (device_bytes) *device_bytes = s->graphs[graph_id]->bytes;
    if (max_batch) *max_batch = s->graphs[graph_id]->width;
    return B40C_SUCCESS;
}

int b40c_server_now_ns(b40c_server *s, int64_t *now_ns)
{
    b40c::clear_error();
    if (!s || !now_ns) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null argument");
    *now_ns = s->now();
    return B40C_SUCCESS;
}

int b40c_server_submit(b40c_server *s, int32_t graph_id, int32_t source, int32_t depth_limit, int32_t *h_labels,
                       int64_t arrival_ns, int64_t *ticket)
{
    b40c::clear_error();
    if (!s) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null server");
    int64_t t;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        int rc = check_query(s, graph_id, source);
        if (rc) return rc;
        t = enqueue(s, graph_id, source, depth_limit, h_labels, arrival_ns);
    }
    s->cv_work.notify_all();
    if (ticket) *ticket = t;
    return B40C_SUCCESS;
}

int b40c_server_submit_many(b40c_server *s, int64_t count, const int32_t *graph_ids, const int32_t *sources,
                            const int32_t *depth_limits, const int64_t *arrival_ns, int64_t *tickets)
{
    b40c::clear_error();
    if (!s || count < 0 || (count > 0 && (!graph_ids || !sources)))
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "bad arguments");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (int64_t i = 0; i < count; i++) {
            int rc = check_query(s, graph_ids[i], sources[i]);
            if (rc) return rc;
        }
        for (int64_t i = 0; i < count; i++) {
            const int64_t t = enqueue(s, graph_ids[i], sources[i], depth_limits ? depth_limits[i] : -1, nullptr,
                                      arrival_ns ? arrival_ns[i] : -1);
            if (tickets) tickets[i] = t;
        }
    }
    s->cv_work.notify_all();
    return B40C_SUCCESS;
}

int b40c_server_result_get(b40c_server *s, int64_t ticket, b40c_server_result *out)
{
    b40c::clear_error();
    if (!s || !out) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    if (ticket < 0 || ticket >= (int64_t)s->results.size())
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "no ticket %lld", (long long)ticket);
    *out = s->results[ticket];
    return B40C_SUCCESS;
}

int b40c_server_wait(b40c_server *s, int64_t ticket, b40c_server_result *out)
{
    b40c::clear_error();
    if (!s) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    if (ticket < 0 || ticket >= (int64_t)s->results.size())
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "no ticket %lld", (long long)ticket);
    s->cv_done.wait(lk, [s, ticket] { return s->results[ticket].status != B40C_ERROR_NOT_READY; });
    if (out) *out = s->results[ticket];
    return B40C_SUCCESS;
}

int b40c_server_results(b40c_server *s, int64_t first, int64_t count, b40c_server_result *out)
{
    b40c::clear_error();
    if (!s || !out || first < 0 || count < 0) return b40c::fail(B40C_ERROR_INVALID_VALUE, "bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    if (first + count > (int64_t)s->results.size())
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "tickets past the last submitted");
    std::copy(s->results.begin() + first, s->results.begin() + first + count, out);
    return B40C_SUCCESS;
}

int b40c_server_counters_get(b40c_server *s, b40c_server_counters *out)
{
    b40c::clear_error();
    if (!s || !out) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    b40c_server_counters c{};
    c.submitted = s->submitted;
    c.completed = s->completed;
    c.failed = s->failed;
    c.batches = s->batches;
    c.batched_queries = s->batched_queries;
    c.single_queries = s->single_queries;
    c.joined_queries = s->joined_queries;
    c.memory_used_bytes = s->used;
    c.memory_budget_bytes = s->budget;
    for (Graph *g : s->graphs)
        if (g && !g->removed) c.graphs++;
    *out = c;
    return B40C_SUCCESS;
}

}  // extern "C"
