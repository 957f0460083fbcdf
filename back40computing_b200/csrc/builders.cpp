// Native graph builders behind the C ABI (b40c_build_*).
//
// Topology follows the reference builders (b40c/graph/builder/*.cuh); the
// random ones draw from a counter-based generator (splitmix64, Vigna 2015)
// keyed by (seed, edge index) instead of libc rand(), so a graph is a pure
// function of its seed, independent of thread count, and large graphs build
// in parallel.  CSR conversion is the reference's stable by-row ordering
// (CsrGraph::FromCoo, csr_graph.cuh:109-152) done as a parallel two-level
// stable counting sort.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "b40c_bfs.h"
#include "errors.h"

namespace {

inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// One independent splitmix64 stream per (seed, key).
struct Stream {
    uint64_t x;
    Stream(uint64_t seed, uint64_t key) : x(mix64(seed * 0xD1B54A32D192ED03ull + key + 1)) {}
    uint64_t next()
    {
        x += 0x9E3779B97F4A7C15ull;
        return mix64(x);
    }
    // uniform double in [0, 1) with 53 random bits
    double uniform() { return double(next() >> 11) * (1.0 / 9007199254740992.0); }
    // uniform integer in [0, n)
    uint64_t below(uint64_t n) { return (uint64_t)(((__uint128_t)next() * n) >> 64); }
};

int num_threads()
{
    const char *env = getenv("B40C_BUILD_THREADS");
    int t = env ? atoi(env) : 0;
    if (t <= 0) t = (int)std::thread::hardware_concurrency();
    if (t <= 0) t = 1;
    return std::min(t, 64);
}

template <typename F>
void parallel_for(int64_t n, F f)
{
    int t = num_threads();
    if (n < 65536 || t == 1) {
        f(0, n, 0);
        return;
    }
    t = (int)std::min<int64_t>(t, n / 16384 + 1);
    std::vector<std::thread> pool;
    for (int i = 0; i < t; i++) {
        int64_t b = n * i / t, e = n * (i + 1) / t;
        pool.emplace_back([=] { f(b, e, i); });
    }
    for (auto &th : pool) th.join();
}

bool alloc_csr(b40c_csr *out, int64_t nodes, int64_t edges, int pinned)
{
    out->nodes = nodes;
    out->edges = edges;
    out->pinned = pinned ? 1 : 0;
    out->row_offsets = nullptr;
    out->column_indices = nullptr;
    size_t rb = sizeof(int32_t) * (size_t)(nodes + 1), cb = sizeof(int32_t) * (size_t)std::max<int64_t>(edges, 1);
    if (pinned) {
        if (cudaHostAlloc((void **)&out->row_offsets, rb, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess ||
            cudaHostAlloc((void **)&out->column_indices, cb, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            b40c_graph_free(out);
            return false;
        }
    } else {
        out->row_offsets = (int32_t *)malloc(rb);
        out->column_indices = (int32_t *)malloc(cb);
        if (!out->row_offsets || !out->column_indices) {
            b40c_graph_free(out);
            return false;
        }
    }
    return true;
}

// Stable by-row CSR of a COO list (the ordering of CsrGraph::FromCoo):
// pass 1 buckets edges by the high bits of their row stably (per-thread
// contiguous blocks with a bucket histogram each), pass 2 counting-sorts each
// bucket by row, buckets in parallel.
int coo_to_csr(const int32_t *rows, const int32_t *cols, int64_t nodes, int64_t edges, int pinned,
               b40c_csr *out)
{
    if (!alloc_csr(out, nodes, edges, pinned))
        return b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "graph allocation failed (%lld vertices, %lld edges)",
                          (long long)nodes, (long long)edges);
    int shift = 0;
    while (((nodes - 1) >> shift) >= 4096) shift++;
    const int64_t nbuckets = ((nodes - 1) >> shift) + 1;
    const int T = std::max(1, std::min(num_threads(), (int)(edges / 65536) + 1));
    std::vector<int64_t> hist((size_t)T * nbuckets, 0);
    auto block = [&](int t, int64_t &b, int64_t &e) {
        b = edges * t / T;
        e = edges * (t + 1) / T;
    };
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < T; t++)
            pool.emplace_back([&, t] {
                int64_t b, e;
                block(t, b, e);
                int64_t *h = &hist[(size_t)t * nbuckets];
                for (int64_t i = b; i < e; i++) h[rows[i] >> shift]++;
            });
        for (auto &th : pool) th.join();
    }
    // exclusive prefix in (bucket, thread) order
    std::vector<int64_t> bucket_start(nbuckets + 1, 0);
    int64_t run = 0;
    for (int64_t k = 0; k < nbuckets; k++) {
        bucket_start[k] = run;
        for (int t = 0; t < T; t++) {
            int64_t c = hist[(size_t)t * nbuckets + k];
            hist[(size_t)t * nbuckets + k] = run;
            run += c;
        }
    }
    bucket_start[nbuckets] = run;
    std::vector<int32_t> trow((size_t)edges), tcol((size_t)edges);
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < T; t++)
            pool.emplace_back([&, t] {
                int64_t b, e;
                block(t, b, e);
                int64_t *h = &hist[(size_t)t * nbuckets];
                for (int64_t i = b; i < e; i++) {
                    int64_t k = rows[i] >> shift;
                    int64_t p = h[k]++;
                    trow[p] = rows[i];
                    tcol[p] = cols[i];
                }
            });
        for (auto &th : pool) th.join();
    }
    int32_t *ro = out->row_offsets;
    int32_t *ci = out->column_indices;
    std::atomic<int64_t> next_bucket(0);
    auto worker = [&] {
        std::vector<int64_t> cnt((size_t)1 << shift);
        for (;;) {
            int64_t k = next_bucket.fetch_add(1);
            if (k >= nbuckets) break;
            int64_t r0 = k << shift, r1 = std::min<int64_t>(nodes, (k + 1) << shift);
            int64_t s = bucket_start[k], e = bucket_start[k + 1];
            std::fill(cnt.begin(), cnt.begin() + (r1 - r0), 0);
            for (int64_t i = s; i < e; i++) cnt[trow[i] - r0]++;
            int64_t pos = s;
            for (int64_t r = r0; r < r1; r++) {
                ro[r] = (int32_t)pos;
                int64_t c = cnt[r - r0];
                cnt[r - r0] = pos;
                pos += c;
            }
            for (int64_t i = s; i < e; i++) ci[cnt[trow[i] - r0]++] = tcol[i];
        }
    };
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < num_threads(); t++) pool.emplace_back(worker);
        for (auto &th : pool) th.join();
    }
    ro[nodes] = (int32_t)edges;
    return B40C_SUCCESS;
}

}  // namespace

extern "C" {

void b40c_graph_free(b40c_csr *g)
{
    if (!g) return;
    if (g->pinned) {
        if (g->row_offsets) cudaFreeHost(g->row_offsets);
        if (g->column_indices) cudaFreeHost(g->column_indices);
    } else {
        free(g->row_offsets);
        free(g->column_indices);
    }
    g->row_offsets = nullptr;
    g->column_indices = nullptr;
    g->nodes = g->edges = 0;
}

int b40c_csr_from_coo(const int32_t *rows, const int32_t *cols, int64_t nodes, int64_t edges, int pinned,
                      b40c_csr *out)
{
    b40c::clear_error();
    if (!rows || !cols || !out || nodes <= 0 || edges < 0 || nodes >= INT32_MAX || edges >= INT32_MAX)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "b40c_csr_from_coo: bad arguments");
    for (int64_t i = 0; i < edges; i++)
        if (rows[i] < 0 || rows[i] >= nodes || cols[i] < 0 || cols[i] >= nodes)
            return b40c::fail(B40C_ERROR_INVALID_VALUE, "b40c_csr_from_coo: edge %lld out of range", (long long)i);
    return coo_to_csr(rows, cols, nodes, edges, pinned, out);
}

// grid2d.cuh:54-114
int b40c_build_grid2d(int32_t width, int pinned, b40c_csr *out)
{
    b40c::clear_error();
    if (!out || width < 1 || (int64_t)width * width * 5 >= INT32_MAX)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "b40c_build_grid2d: invalid width %d", width);
    const int64_t w = width, nodes = w * w;
    // degree of (j, k): 1 (self) + neighbours present
    auto deg = [w](int64_t j, int64_t k) {
        return (int64_t)1 + (k > 0) + (k + 1 < w) + (j > 0) + (j + 1 < w);
    };
    int64_t edges = 0;
    for (int64_t j = 0; j < w; j++)
        for (int64_t k = 0; k < w; k++) edges += deg(j, k);
    if (!alloc_csr(out, nodes, edges, pinned)) return b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "grid2d allocation failed");
    // row offsets in closed form per grid row so rows can be filled in parallel
    std::vector<int64_t> row_base(w + 1, 0);
    for (int64_t j = 0; j < w; j++) {
        int64_t s = 0;
        for (int64_t k = 0; k < w; k++) s += deg(j, k);
        row_base[j + 1] = row_base[j] + s;
    }
    int32_t *ro = out->row_offsets, *ci = out->column_indices;
    parallel_for(w, [&](int64_t jb, int64_t je, int) {
        for (int64_t j = jb; j < je; j++) {
            int64_t total = row_base[j];
            for (int64_t k = 0; k < w; k++) {
                int64_t me = j * w + k;
                ro[me] = (int32_t)total;
                if (k - 1 >= 0) ci[total++] = (int32_t)(me - 1);
                if (k + 1 < w) ci[total++] = (int32_t)(me + 1);
                if (j - 1 >= 0) ci[total++] = (int32_t)(me - w);
                if (j + 1 < w) ci[total++] = (int32_t)(me + w);
                ci[total++] = (int32_t)me;
            }
        }
    });
    ro[nodes] = (int32_t)edges;
    return B40C_SUCCESS;
}

// grid3d.cuh:54-129
int b40c_build_grid3d(int32_t width, int pinned, b40c_csr *out)
{
    b40c::clear_error();
    if (!out || width < 1 || (int64_t)width * width * width * 7 >= INT32_MAX)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "b40c_build_grid3d: invalid width %d", width);
    const int64_t w = width, nodes = w * w * w;
    auto deg = [w](int64_t i, int64_t j, int64_t k) {
        return (int64_t)1 + (k > 0) + (k + 1 < w) + (j > 0) + (j + 1 < w) + (i > 0) + (i + 1 < w);
    };
    std::vector<int64_t> plane_base(w + 1, 0);
    for (int64_t i = 0; i < w; i++) {
        int64_t s = 0;
        for (int64_t j = 0; j < w; j++)
            for (int64_t k = 0; k < w; k++) s += deg(i, j, k);
        plane_base[i + 1] = plane_base[i] + s;
    }
    const int64_t edges = plane_base[w];
    if (!alloc_csr(out, nodes, edges, pinned)) return b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "grid3d allocation failed");
    int32_t *ro = out->row_offsets, *ci = out->column_indices;
    parallel_for(w, [&](int64_t ib, int64_t ie, int) {
        for (int64_t i = ib; i < ie; i++) {
            int64_t total = plane_base[i];
            for (int64_t j = 0; j < w; j++)
                for (int64_t k = 0; k < w; k++) {
                    int64_t me = i * w * w + j * w + k;
                    ro[me] = (int32_t)total;
                    if (k - 1 >= 0) ci[total++] = (int32_t)(me - 1);
                    if (k + 1 < w) ci[total++] = (int32_t)(me + 1);
                    if (j - 1 >= 0) ci[total++] = (int32_t)(me - w);
                    if (j + 1 < w) ci[total++] = (int32_t)(me + w);
                    if (i - 1 >= 0) ci[total++] = (int32_t)(me - w * w);
                    if (i + 1 < w) ci[total++] = (int32_t)(me + w * w);
                    ci[total++] = (int32_t)me;
                }
        }
    });
    ro[nodes] = (int32_t)edges;
    return B40C_SUCCESS;
}

// rmat.cuh:128-206 (ChoosePartition :56-81, VaryParams :83-116).  Each edge
// draws from its own stream; per level: one uniform for the quadrant choice,
// then the noise step -- four sign flips and four uniforms in [0,1) -- that
// perturbs a, b, c, d by up to 5% and renormalises.
int b40c_build_rmat(int64_t nodes, int64_t edges, int undirected, double a0, double b0, double c0,
                    uint64_t seed, int permute, int pinned, b40c_csr *out)
{
    b40c::clear_error();
    if (!out || nodes < 2 || (nodes & (nodes - 1)) != 0 || edges < 0 || a0 < 0 || b0 < 0 || c0 < 0 ||
        a0 + b0 + c0 > 1.0 || (undirected ? 2 * edges : edges) >= INT32_MAX || nodes >= INT32_MAX)
        return b40c::fail(B40C_ERROR_INVALID_VALUE,
                          "b40c_build_rmat: nodes must be a power of two >= 2 and edges < 2^31 (got %lld, %lld)",
                          (long long)nodes, (long long)edges);
    const int64_t directed = undirected ? 2 * edges : edges;
    std::vector<int32_t> rows((size_t)directed), cols((size_t)directed);
    const double d0 = 1.0 - (a0 + b0 + c0);
    parallel_for(edges, [&](int64_t eb, int64_t ee, int) {
        for (int64_t i = eb; i < ee; i++) {
            Stream rng(seed, (uint64_t)i);
            double a = a0, b = b0, c = c0, d = d0;
            int64_t u = 1, v = 1;
            for (int64_t step = nodes / 2; step >= 1; step /= 2) {
                double p = rng.uniform();
                if (p < a) {
                } else if (a < p && p < a + b) {
                    v += step;
                } else if (a + b < p && p < a + b + c) {
                    u += step;
                } else if (a + b + c < p && p < a + b + c + d) {
                    u += step;
                    v += step;
                }
                uint64_t flips = rng.next();
                uint64_t noise = rng.next();
                double *q[4] = {&a, &b, &c, &d};
                for (int t = 0; t < 4; t++) {
                    double r = double((noise >> (16 * t)) & 0xFFFF) * (1.0 / 65536.0);
                    if ((flips >> t) & 1)
                        *q[t] += *q[t] * 0.05 * r;
                    else
                        *q[t] -= *q[t] * 0.05 * r;
                }
                double s = a + b + c + d;
                a /= s;
                b /= s;
                c /= s;
                d /= s;
            }
            // the walk reaches ids 1..nodes; id `nodes` (only reachable by
            // taking the last quadrant at every level) wraps to 0
            if (u == nodes) u = 0;
            if (v == nodes) v = 0;
            rows[i] = (int32_t)u;
            cols[i] = (int32_t)v;
            if (undirected) {
                rows[edges + i] = (int32_t)v;
                cols[edges + i] = (int32_t)u;
            }
        }
    });
    if (permute) {
        std::vector<int32_t> perm((size_t)nodes);
        for (int64_t i = 0; i < nodes; i++) perm[i] = (int32_t)i;
        Stream rng(seed ^ 0x5bd1e995ull, 0xFFFFFFFFull);
        for (int64_t i = nodes - 1; i > 0; i--) {
            int64_t j = (int64_t)rng.below((uint64_t)i + 1);
            std::swap(perm[i], perm[j]);
        }
        parallel_for(directed, [&](int64_t b, int64_t e, int) {
            for (int64_t i = b; i < e; i++) {
                rows[i] = perm[rows[i]];
                cols[i] = perm[cols[i]];
            }
        });
    }
    return coo_to_csr(rows.data(), cols.data(), nodes, directed, pinned, out);
}

// random.cuh:54-98 (RandomNode, utils.cuh:55-61)
int b40c_build_random(int64_t nodes, int64_t edges, int undirected, uint64_t seed, int pinned, b40c_csr *out)
{
    b40c::clear_error();
    if (!out || nodes < 1 || edges < 0 || (undirected ? 2 * edges : edges) >= INT32_MAX || nodes >= INT32_MAX)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "b40c_build_random: invalid size");
    const int64_t directed = undirected ? 2 * edges : edges;
    std::vector<int32_t> rows((size_t)directed), cols((size_t)directed);
    parallel_for(edges, [&](int64_t b, int64_t e, int) {
        for (int64_t i = b; i < e; i++) {
            Stream rng(seed, (uint64_t)i);
            rows[i] = (int32_t)rng.below((uint64_t)nodes);
            cols[i] = (int32_t)rng.below((uint64_t)nodes);
            if (undirected) {
                rows[edges + i] = cols[i];
                cols[edges + i] = rows[i];
            }
        }
    });
    return coo_to_csr(rows.data(), cols.data(), nodes, directed, pinned, out);
}

// rr.cuh:53-91; with symmetrize, back-edges are appended as in random.cuh:81-86
int b40c_build_rr(int64_t nodes, int32_t degree, int symmetrize, uint64_t seed, int pinned, b40c_csr *out)
{
    b40c::clear_error();
    const int64_t fwd = nodes * (int64_t)degree;
    if (!out || nodes < 1 || degree < 0 || (symmetrize ? 2 * fwd : fwd) >= INT32_MAX || nodes >= INT32_MAX)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "b40c_build_rr: invalid size");
    auto draw = [&](int64_t b, int64_t e, int32_t *dst) {
        for (int64_t u = b; u < e; u++) {
            Stream rng(seed, (uint64_t)u);
            for (int32_t k = 0; k < degree; k++) dst[u * degree + k] = (int32_t)rng.below((uint64_t)nodes);
        }
    };
    if (!symmetrize) {
        if (!alloc_csr(out, nodes, fwd, pinned)) return b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "rr allocation failed");
        parallel_for(nodes, [&](int64_t b, int64_t e, int) {
            draw(b, e, out->column_indices);
            for (int64_t u = b; u < e; u++) out->row_offsets[u] = (int32_t)(u * degree);
        });
        out->row_offsets[nodes] = (int32_t)fwd;
        return B40C_SUCCESS;
    }
    std::vector<int32_t> rows((size_t)(2 * fwd)), cols((size_t)(2 * fwd));
    parallel_for(nodes, [&](int64_t b, int64_t e, int) {
        draw(b, e, cols.data());
        for (int64_t u = b; u < e; u++)
            for (int32_t k = 0; k < degree; k++) {
                int64_t i = u * degree + k;
                rows[i] = (int32_t)u;
                rows[fwd + i] = cols[i];
                cols[fwd + i] = (int32_t)u;
            }
    });
    return coo_to_csr(rows.data(), cols.data(), nodes, 2 * fwd, pinned, out);
}

int b40c_sample_sources(const b40c_csr *g, int32_t count, uint64_t seed, int32_t *out)
{
    b40c::clear_error();
    if (!g || !out || count < 0 || g->nodes <= 0) return b40c::fail(B40C_ERROR_INVALID_VALUE, "b40c_sample_sources: bad arguments");
    int64_t nonzero = 0;
    for (int64_t v = 0; v < g->nodes; v++) nonzero += g->row_offsets[v + 1] > g->row_offsets[v];
    if (nonzero < count) return b40c::fail(B40C_ERROR_INVALID_VALUE, "b40c_sample_sources: only %lld vertices have edges", (long long)nonzero);
    Stream rng(seed, 0xA5A5A5A5ull);
    int32_t got = 0;
    while (got < count) {
        int32_t v = (int32_t)rng.below((uint64_t)g->nodes);
        if (g->row_offsets[v + 1] == g->row_offsets[v]) continue;
        bool dup = false;
        for (int32_t i = 0; i < got; i++) dup |= out[i] == v;
        if (!dup) out[got++] = v;
    }
    return B40C_SUCCESS;
}

int b40c_host_alloc(void **ptr, size_t bytes, int mapped)
{
    b40c::clear_error();
    if (!ptr) return b40c::fail(B40C_ERROR_INVALID_VALUE, "b40c_host_alloc: null ptr");
    cudaError_t e = cudaHostAlloc(ptr, bytes, (mapped ? cudaHostAllocMapped : 0) | cudaHostAllocPortable);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *ptr = nullptr;
        return b40c::fail((int)e, "cudaHostAlloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    return B40C_SUCCESS;
}

int b40c_host_free(void *ptr)
{
    b40c::clear_error();
    if (!ptr) return B40C_SUCCESS;
    cudaError_t e = cudaFreeHost(ptr);
    if (e != cudaSuccess) return b40c::fail((int)e, "cudaFreeHost failed: %s", cudaGetErrorString(e));
    return B40C_SUCCESS;
}

}  // extern "C"
