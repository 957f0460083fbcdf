// Graph file readers behind the C ABI (b40c_read_market / _dimacs / _metis).
//
// Formats and edge order follow the reference readers
// (b40c/graph/builder/market.cuh:49-208, dimacs.cuh:52-283, metis.cuh:51-287):
// 1-based vertex ids, optional back-edges, and the COO list turned into CSR by
// a stable by-row sort (CsrGraph::FromCoo) so each row keeps file order.  Lines
// have no length limit, and ids outside [1, nodes] are reported as errors
// (the reference would index out of bounds).
#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "b40c_bfs.h"
#include "errors.h"

namespace {

struct LineReader {
    FILE *f;
    char *buf = nullptr;
    size_t cap = 0;
    explicit LineReader(FILE *file) : f(file) {}
    LineReader(const LineReader &) = delete;
    LineReader(LineReader &&o) noexcept : f(o.f), buf(o.buf), cap(o.cap) { o.buf = nullptr; }
    ~LineReader() { free(buf); }
    // next line without its newline; false at end of file
    bool next(std::string &line)
    {
        ssize_t n = getline(&buf, &cap, f);
        if (n < 0) return false;
        while (n > 0 && (buf[n - 1] == '\n' || buf[n - 1] == '\r')) n--;
        line.assign(buf, (size_t)n);
        return true;
    }
};

bool blank(const std::string &s)
{
    for (char c : s)
        if (c != ' ' && c != '\t') return false;
    return true;
}

struct File {
    FILE *f = nullptr;
    bool owned = false;
    File() = default;
    File(const File &) = delete;
    ~File()
    {
        if (owned && f) fclose(f);
    }
};

int open_input(const char *path, File &out)
{
    if (!path) {
        out.f = stdin;
        return B40C_SUCCESS;
    }
    out.f = fopen(path, "r");
    out.owned = true;
    if (!out.f) return b40c::fail(B40C_ERROR_INVALID_VALUE, "unable to open %s: %s", path, strerror(errno));
    return B40C_SUCCESS;
}

// Allocates an empty CSR of the given size (pageable or pinned host memory).
int alloc_csr(int64_t nodes, int64_t edges, int pinned, b40c_csr *out)
{
    out->nodes = nodes;
    out->edges = edges;
    out->pinned = pinned ? 1 : 0;
    const size_t rb = sizeof(int32_t) * (size_t)(nodes + 1), cb = sizeof(int32_t) * (size_t)std::max<int64_t>(edges, 1);
    if (pinned) {
        if (cudaMallocHost((void **)&out->row_offsets, rb) != cudaSuccess ||
            cudaMallocHost((void **)&out->column_indices, cb) != cudaSuccess) {
            cudaGetLastError();
            b40c_graph_free(out);
            return b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "pinned graph allocation failed");
        }
    } else {
        out->row_offsets = (int32_t *)malloc(rb);
        out->column_indices = (int32_t *)malloc(cb);
        if (!out->row_offsets || !out->column_indices) {
            b40c_graph_free(out);
            return b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "graph allocation failed");
        }
    }
    return B40C_SUCCESS;
}

bool id_ok(long long id, int64_t nodes) { return id >= 1 && id <= nodes; }

}  // namespace

extern "C" {

// market.cuh:49-160: '%' comment lines, "rows cols nnz" (square), then one
// "a b [value]" line per entry with a the column and b the row (1-based); with
// `undirected` each entry's reverse edge follows it in the COO list.
int b40c_read_market(const char *path, int undirected, int pinned, b40c_csr *out)
{
    b40c::clear_error();
    if (!out) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null out");
    out->row_offsets = out->column_indices = nullptr;
    File in;
    int rc = open_input(path, in);
    if (rc) return rc;
    LineReader rd(in.f);
    std::string line;
    int64_t nodes = -1, edges = 0;
    std::vector<int32_t> rows, cols;
    while (rd.next(line)) {
        if (line.empty() || line[0] == '%' || blank(line)) continue;
        if (nodes < 0) {
            long long nx, ny, ne;
            if (sscanf(line.c_str(), "%lld %lld %lld", &nx, &ny, &ne) != 3 || nx < 1 || ne < 0)
                return b40c::fail(B40C_ERROR_INVALID_VALUE, "MARKET: invalid problem description");
            if (nx != ny) return b40c::fail(B40C_ERROR_INVALID_VALUE, "MARKET: not square (%lld, %lld)", nx, ny);
            if (nx >= INT32_MAX || (undirected ? 2 * ne : ne) >= INT32_MAX)
                return b40c::fail(B40C_ERROR_INVALID_VALUE, "MARKET: graph exceeds 32-bit ids");
            nodes = nx;
            edges = undirected ? 2 * ne : ne;
            rows.reserve((size_t)edges);
            cols.reserve((size_t)edges);
            continue;
        }
        if ((int64_t)rows.size() >= edges)
            return b40c::fail(B40C_ERROR_INVALID_VALUE, "MARKET: more than %lld edges", (long long)edges);
        long long c, r;
        if (sscanf(line.c_str(), "%lld %lld", &c, &r) != 2)
            return b40c::fail(B40C_ERROR_INVALID_VALUE, "MARKET: badly formed edge \"%s\"", line.c_str());
        if (!id_ok(c, nodes) || !id_ok(r, nodes))
            return b40c::fail(B40C_ERROR_INVALID_VALUE, "MARKET: vertex id out of [1, %lld] in \"%s\"",
                              (long long)nodes, line.c_str());
        rows.push_back((int32_t)(r - 1));
        cols.push_back((int32_t)(c - 1));
        if (undirected) {
            rows.push_back((int32_t)(c - 1));
            cols.push_back((int32_t)(r - 1));
        }
    }
    if (nodes < 0) return b40c::fail(B40C_ERROR_INVALID_VALUE, "MARKET: no graph found");
    if ((int64_t)rows.size() != edges)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "MARKET: only %lld/%lld edges read", (long long)rows.size(),
                          (long long)edges);
    return b40c_csr_from_coo(rows.data(), cols.data(), nodes, edges, pinned, out);
}

// dimacs.cuh:52-228: per file, lines up to the "p <type> nodes arcs" line are
// skipped; then every "a u v [w]" line is an arc (1-based).  With `splice` > 0
// the files <path>.0, <path>.1, ... (up to splice of them, stopping at the first
// that does not open) are merged by repeatedly taking the pending arc with the
// smallest row (the lowest file on ties).  With `undirected` an arc's reverse
// edge enters the COO list when the arc is read, ahead of the arc itself.
int b40c_read_dimacs(const char *path, int undirected, int splice, int pinned, b40c_csr *out)
{
    b40c::clear_error();
    if (!out || splice < 0) return b40c::fail(B40C_ERROR_INVALID_VALUE, "bad arguments");
    out->row_offsets = out->column_indices = nullptr;
    std::vector<File> files(splice > 0 ? (size_t)splice : 1);
    size_t nfiles = 0;
    if (splice > 0) {
        if (!path) return b40c::fail(B40C_ERROR_INVALID_VALUE, "DIMACS: splice needs a path");
        for (int i = 0; i < splice; i++) {
            std::string name = std::string(path) + "." + std::to_string(i);
            FILE *f = fopen(name.c_str(), "r");
            if (!f) break;
            files[nfiles].f = f;
            files[nfiles].owned = true;
            nfiles++;
        }
        if (nfiles == 0) return b40c::fail(B40C_ERROR_INVALID_VALUE, "unable to open %s.0", path);
    } else {
        int rc = open_input(path, files[0]);
        if (rc) return rc;
        nfiles = 1;
    }
    std::vector<LineReader> readers;
    readers.reserve(nfiles);
    for (size_t i = 0; i < nfiles; i++) readers.emplace_back(files[i].f);
    std::string line;
    int64_t nodes = 0, arcs = 0;
    for (size_t i = 0; i < nfiles; i++) {
        while (readers[i].next(line)) {
            if (line.empty() || line[0] != 'p') continue;
            char type[256];
            long long n, m;
            if (sscanf(line.c_str(), "p %255s %lld %lld", type, &n, &m) != 3 || n < 1 || m < 0)
                return b40c::fail(B40C_ERROR_INVALID_VALUE, "DIMACS: invalid problem line \"%s\"", line.c_str());
            if (nodes && nodes != n)
                return b40c::fail(B40C_ERROR_INVALID_VALUE, "DIMACS: splice files name different vertex counts");
            nodes = n;
            arcs += m;
            break;
        }
    }
    const int64_t edges = undirected ? 2 * arcs : arcs;
    if (edges == 0) return b40c::fail(B40C_ERROR_INVALID_VALUE, "DIMACS: no graph found");
    if (nodes >= INT32_MAX || edges >= INT32_MAX)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "DIMACS: graph exceeds 32-bit ids");
    std::vector<int32_t> rows, cols;
    rows.reserve((size_t)edges);
    cols.reserve((size_t)edges);
    struct Pending {
        int64_t row = -1, col = 0;
    };
    std::vector<Pending> pend(nfiles);
    for (;;) {
        int smallest = -1;
        for (size_t i = 0; i < nfiles; i++) {
            while (pend[i].row < 0 && readers[i].next(line)) {
                if (line.empty() || line[0] != 'a') continue;
                if ((int64_t)rows.size() >= edges)
                    return b40c::fail(B40C_ERROR_INVALID_VALUE, "DIMACS: more than %lld edges", (long long)edges);
                long long u, v;
                if (sscanf(line.c_str(), "a %lld %lld", &u, &v) != 2)
                    return b40c::fail(B40C_ERROR_INVALID_VALUE, "DIMACS: badly formed arc \"%s\"", line.c_str());
                if (!id_ok(u, nodes) || !id_ok(v, nodes))
                    return b40c::fail(B40C_ERROR_INVALID_VALUE, "DIMACS: vertex id out of [1, %lld] in \"%s\"",
                                      (long long)nodes, line.c_str());
                pend[i].row = u - 1;
                pend[i].col = v - 1;
                if (undirected) {
                    rows.push_back((int32_t)(v - 1));
                    cols.push_back((int32_t)(u - 1));
                }
            }
            if (pend[i].row >= 0 && (smallest < 0 || pend[i].row < pend[smallest].row)) smallest = (int)i;
        }
        if (smallest < 0) break;
        if ((int64_t)rows.size() >= edges)
            return b40c::fail(B40C_ERROR_INVALID_VALUE, "DIMACS: more than %lld edges", (long long)edges);
        rows.push_back((int32_t)pend[smallest].row);
        cols.push_back((int32_t)pend[smallest].col);
        pend[smallest].row = -1;
    }
    if ((int64_t)rows.size() != edges)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "DIMACS: only %lld/%lld edges read", (long long)rows.size(),
                          (long long)edges);
    return b40c_csr_from_coo(rows.data(), cols.data(), nodes, edges, pinned, out);
}

// metis.cuh:51-187: '%' comments; the first data line is "nodes edges [...]";
// then line i (1-based) lists the neighbours of vertex i-1, so the graph is
// read straight into CSR.  `edges` usually counts undirected edges, each listed
// twice: 2 * edges ids are expected, or exactly `edges` ids (the header then
// counted every listed id).  Lines past the last vertex must be empty.
int b40c_read_metis(const char *path, int pinned, b40c_csr *out)
{
    b40c::clear_error();
    if (!out) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null out");
    out->row_offsets = out->column_indices = nullptr;
    File in;
    int rc = open_input(path, in);
    if (rc) return rc;
    LineReader rd(in.f);
    std::string line;
    int64_t nodes = -1, declared = 0, vertex = 0;
    std::vector<int32_t> ro, ci;
    while (rd.next(line)) {
        if (!line.empty() && line[0] == '%') continue;
        if (nodes < 0) {
            if (blank(line)) continue;
            long long n, m;
            if (sscanf(line.c_str(), "%lld %lld", &n, &m) != 2 || n < 1 || m < 0)
                return b40c::fail(B40C_ERROR_INVALID_VALUE, "METIS: invalid header \"%s\"", line.c_str());
            if (n >= INT32_MAX || 2 * m >= INT32_MAX)
                return b40c::fail(B40C_ERROR_INVALID_VALUE, "METIS: graph exceeds 32-bit ids");
            nodes = n;
            declared = m;
            ro.assign((size_t)nodes + 1, 0);
            ci.reserve((size_t)(2 * m));
            continue;
        }
        if (vertex >= nodes) {
            if (blank(line)) continue;
            return b40c::fail(B40C_ERROR_INVALID_VALUE, "METIS: more adjacency lines than %lld vertices",
                              (long long)nodes);
        }
        ro[(size_t)vertex] = (int32_t)ci.size();
        const char *s = line.c_str();
        char *end = nullptr;
        for (;;) {
            while (*s == ' ' || *s == '\t') s++;
            if (!*s) break;
            errno = 0;
            long long id = strtoll(s, &end, 10);
            if (end == s || errno)
                return b40c::fail(B40C_ERROR_INVALID_VALUE, "METIS: invalid entry on line of vertex %lld",
                                  (long long)vertex + 1);
            if (!id_ok(id, nodes))
                return b40c::fail(B40C_ERROR_INVALID_VALUE, "METIS: neighbour %lld out of [1, %lld]", id,
                                  (long long)nodes);
            if ((int64_t)ci.size() >= 2 * declared)
                return b40c::fail(B40C_ERROR_INVALID_VALUE, "METIS: more than %lld edges", (long long)(2 * declared));
            ci.push_back((int32_t)(id - 1));
            s = end;
        }
        vertex++;
    }
    if (nodes < 0) return b40c::fail(B40C_ERROR_INVALID_VALUE, "METIS: no graph found");
    for (int64_t v = vertex; v <= nodes; v++) ro[(size_t)v] = (int32_t)ci.size();
    const int64_t got = (int64_t)ci.size();
    if (got != 2 * declared && got != declared)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "METIS: only %lld/%lld edges read", (long long)got,
                          (long long)(2 * declared));
    rc = alloc_csr(nodes, got, pinned, out);
    if (rc) return rc;
    memcpy(out->row_offsets, ro.data(), sizeof(int32_t) * (size_t)(nodes + 1));
    if (got) memcpy(out->column_indices, ci.data(), sizeof(int32_t) * (size_t)got);
    return B40C_SUCCESS;
}

}  // extern "C"
