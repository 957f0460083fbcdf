// Batched multi-source BFS (up to 64 sources per launch) for sm_100a.
//
// No counterpart in the reference (its BFS searches one source at a time);
// the traversal arithmetic per source is the same as a single-source search:
// labels[s][v] = distance of v from source s (-1 unreached).
//
// Per vertex the search keeps a 64-bit visited mask V[v] (bit s: source s
// reached v) and, for the current and next level, 64-bit frontier masks
// F[cur][v] / F[next][v].  Two level kinds:
//  * push (sparse frontiers): the frontier queue is expanded with the same
//    edge-balanced per-CTA ranges as the single-source kernels, so each
//    adjacency list is read once per level for all sources together; for a
//    gathered edge u -> w:
//        new = F[cur][u] & active & ~V[w]    (active: sources under their depth limit)
//        set = new & ~atomicOr(&V[w], new)   (the bits this edge is first to set)
//        labels[s][w] = level + 1 for s in set
//        if atomicOr(&F[next][w], set) was 0: w joins the next frontier queue;
//  * pull (dense frontiers, symmetric graphs only): every vertex still missing
//    some active source ORs its neighbours' F[cur] masks (no atomics; a warp
//    stores source s's labels of 32 consecutive vertices at once).
// After each level F[cur] is cleared over the level's queue (two grid
// barriers per level).
#pragma once
#include "bfs_kernels.cuh"

namespace b40c {
namespace dev {

struct MsParams {
    unsigned long long *visited;     // V[n]
    unsigned long long *fmask[2];    // F[2][n]
    int32_t *labels;                 // [rows][n], source-major
    int32_t *depth_limit;            // [64]; < 0 unlimited
    int32_t *depth;                  // [64]; search depth of each source (max label + 1)
    int32_t *level_off;              // [64]; level at which each slot's source was seeded
    MsJoin *join;                    // sources joining the running batch (null: none)
    int32_t k;
    int32_t rows;                    // label rows allocated (joined slots must be below)
    int32_t pull_ok;                 // 1: the graph is symmetric, dense levels may pull
};

template <int B>
struct MsSmem {
    int32_t colstart[kChunkMax + 2];
    int32_t rel[kChunkMax + 2];
    unsigned long long fm[kChunkMax + 2];  // frontier mask of run j's vertex
    uint16_t own[kChunkMax];
    int32_t out[kChunkMax];
    int32_t limits[64];
    int32_t off[64];                 // level_off of each slot
    int32_t jn0, jn1;                // join requests taken at this level end: [jn0, jn1)
    unsigned long long used;         // slots in use
    int32_t out_count;
    int32_t flag;
    int32_t q, E;
    unsigned long long active;
    unsigned long long found;        // sources that reached a vertex this level
    unsigned long long scan_warp[B / 32];
    unsigned long long prefix;
};

// Push level: expansion of the CTA's share of the level's frontier queue.
template <int B>
__device__ __forceinline__ void ms_expand_range(const BfsParams &p, const MsParams &m, MsSmem<B> &s, int level,
                                                const VertexFrontier &in, const VertexFrontier &vout,
                                                unsigned long long *qe_out, unsigned long long &found)
{
    const int tid = threadIdx.x, lane = tid & 31;
    const int q = s.q, E = s.E;
    constexpr int PER = kChunkMax / B;
    const unsigned long long *fcur = m.fmask[level & 1];
    unsigned long long *fnext = m.fmask[(level + 1) & 1];
    const long long n = p.nodes;
    int rs, re;
    cta_range(E, blockIdx.x, gridDim.x, rs, re);
    if (rs >= re) return;
    int i_cur = ld_cg(in.cf + rs / kChunkGrain);
    const int chunk = min(max(p.chunk_edges, 256), kChunkMax);
    for (int cs = rs; cs < re; cs += chunk) {
        const int ce = min(cs + chunk, re);
        const int len = ce - cs;
        if (tid == 0) s.out_count = 0;
        int k = 0;
        for (int base = i_cur;; base += B) {
            const int i = base + tid;
            bool inside = false;
            if (i < q) {
                // (degree prefix, row start and vertex in one round trip)
                const int Pi = ld_cg(in.P + i);
                const int ci = ld_cg(in.col + i);
                const int vi = ld_cg(in.v + i);
                if (Pi < ce && i - i_cur <= kChunkMax) {
                    inside = true;
                    const int j = i - i_cur;
                    const int start = max(Pi, cs);
                    s.rel[j] = start - cs;
                    s.colstart[j] = ci + (start - Pi);
                    s.fm[j] = ld_keep64(fcur + vi) & s.active;
                }
            }
            const int c = __syncthreads_count(inside);
            k += c;
            if (c < B) break;
        }
        if (tid == 0) s.rel[k] = len;
        __syncthreads();
        {
            const int x0 = tid * PER;
            if (x0 < len) {
                int lo = 0, hi = k - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (s.rel[mid] <= x0) lo = mid; else hi = mid - 1;
                }
                int j = lo;
                int next = s.rel[j + 1];
#pragma unroll
                for (int t = 0; t < PER; t++) {
                    const int x = x0 + t;
                    if (x < len) {
                        while (x >= next) {
                            j++;
                            next = s.rel[j + 1];
                        }
                        s.own[x] = (uint16_t)j;
                    }
                }
            }
        }
        __syncthreads();
        int w[PER];
        unsigned long long f[PER];
#pragma unroll
        for (int t = 0; t < PER; t++) {
            const int x = t * B + tid;
            w[t] = -1;
            f[t] = 0;
            if (x < len) {
                const int j = s.own[x];
                f[t] = s.fm[j];
                if (f[t]) w[t] = ld_stream(p.column_indices + s.colstart[j] + (x - s.rel[j]));
            }
        }
        i_cur += k - 1;
        __syncthreads();  // run tables consumed: they now collect the sub-round's output
        unsigned long long nw[PER];
#pragma unroll
        for (int t = 0; t < PER; t++) nw[t] = (w[t] >= 0) ? (f[t] & ~ld_keep64(m.visited + w[t])) : 0ull;
        unsigned long long set[PER];
#pragma unroll
        for (int t = 0; t < PER; t++) set[t] = nw[t] ? (nw[t] & ~atomicOr(m.visited + w[t], nw[t])) : 0ull;
        bool first[PER];
#pragma unroll
        for (int t = 0; t < PER; t++) {
            first[t] = false;
            found |= set[t];
            if (set[t]) {
                unsigned long long bits = set[t];
                while (bits) {
                    const int src = __ffsll((long long)bits) - 1;
                    bits &= bits - 1;
                    st_stream(m.labels + (long long)src * n + w[t], level + 1 - s.off[src]);
                }
                first[t] = atomicOr(fnext + w[t], set[t]) == 0ull;
            }
        }
        int r0[PER], r1[PER];
#pragma unroll
        for (int t = 0; t < PER; t++) {
            r0[t] = r1[t] = 0;
            if (first[t]) {
                r0[t] = ld_ro(p.row_offsets + w[t]);
                r1[t] = ld_ro(p.row_offsets + w[t] + 1);
            }
        }
#pragma unroll
        for (int t = 0; t < PER; t++) {
            if (t * B >= len) continue;  // CTA-uniform
            if (set[t]) s.flag = 1;
            const bool push = first[t] && r1[t] > r0[t];
            const unsigned bal = __ballot_sync(0xffffffffu, push);
            if (bal == 0) continue;
            const int leader = __ffs(bal) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&s.out_count, __popc(bal));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (push) {
                const int slot = base + __popc(bal & lanemask_lt());
                s.out[slot] = w[t];
                s.colstart[slot] = r0[t];
                s.rel[slot] = r1[t] - r0[t];
            }
        }
        __syncthreads();
        emit_frontier<B>(p, s, level, vout, qe_out);
        __syncthreads();
    }
}

// Pull level (symmetric graphs): one thread per vertex, eight neighbours per
// step, stopping once every missing source is found; lists longer than
// kPullLongList are searched by the whole warp afterwards.  Only v's own
// thread writes V[v] and F[next][v].
constexpr int kPullLongList = 256;

// One warp's block of 32 consecutive vertices [vb, vb + 32) of a pull level,
// below `re`: every lane takes one vertex, eight neighbours per step, stopping
// once every missing source is found; lists longer than kPullLongList are
// searched by the whole warp afterwards.  Only v's own lane writes V[v] and
// F[next][v]; the labels are stored source by source, one coalesced store per
// warp.  Returns whether the lane's vertex joins the next frontier (it was
// reached and has edges), with its row start and degree.
template <int B>
__device__ __forceinline__ bool ms_pull_block(const BfsParams &p, const MsParams &m, MsSmem<B> &s, int level,
                                              int vb, int re, unsigned long long &found, int &r0_out,
                                              int &deg_out)
{
    const int lane = threadIdx.x & 31;
    constexpr int U = 8;
    const unsigned long long *fcur = m.fmask[level & 1];
    unsigned long long *fnext = m.fmask[(level + 1) & 1];
    const unsigned long long active = s.active;
    const long long n = p.nodes;
    const int v = vb + lane;
    const bool inr = v < re;
    unsigned long long vold = 0, missing = 0;
    int r0 = 0, r1 = 0;
    // vertices without edges are never reached (their labels are set at the end)
    const bool iso = inr && p.iso && ((p.iso[v >> 5] >> (v & 31)) & 1u);
    if (inr && !iso) {
        vold = ld_keep64(m.visited + v);
        missing = active & ~vold;
        if (missing) {
            r0 = ld_ro(p.row_offsets + v);
            r1 = ld_ro(p.row_offsets + v + 1);
        }
    }
    unsigned long long acc = 0;
    if (missing && p.hub2) {
        // the vertex's two highest-degree neighbours first (one coalesced load)
        const int2 h = p.hub2[v];
        if (h.x >= 0) acc |= ld_keep64(fcur + h.x) & missing;
        if (h.y >= 0) acc |= ld_keep64(fcur + h.y) & missing;
        if (acc == missing || r1 - r0 <= 2) missing = 0;  // nothing left to look for
    }
    const bool longlist = missing && (r1 - r0) > kPullLongList;
    if (missing && !longlist) {
        for (int e = r0; e < r1 && acc != missing;) {
            // eight neighbours per step from two 16-byte loads
            int nb[U], q0[4], q1[4];
            e = ld_quad(p.column_indices, p.edges, e, r1, q0);
            e = ld_quad(p.column_indices, p.edges, e, r1, q1);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                nb[k] = q0[k];
                nb[4 + k] = q1[k];
            }
            unsigned long long fm[U];
#pragma unroll
            for (int k = 0; k < U; k++) fm[k] = nb[k] >= 0 ? ld_keep64(fcur + nb[k]) : 0ull;
#pragma unroll
            for (int k = 0; k < U; k++) acc |= fm[k] & missing;
        }
    }
    unsigned lmask = __ballot_sync(0xffffffffu, longlist);
    while (lmask) {
        const int owner = __ffs(lmask) - 1;
        lmask &= lmask - 1;
        const int lr0 = __shfl_sync(0xffffffffu, r0, owner), lr1 = __shfl_sync(0xffffffffu, r1, owner);
        const unsigned long long miss = __shfl_sync(0xffffffffu, missing, owner);
        unsigned long long a = 0;
        for (int eb = lr0; eb < lr1; eb += 32) {
            const int ee = eb + lane;
            if (ee < lr1) a |= ld_keep64(fcur + ld_stream(p.column_indices + ee)) & miss;
            for (int off = 16; off > 0; off >>= 1) a |= __shfl_xor_sync(0xffffffffu, a, off);
            if (a == miss) break;
        }
        if (lane == owner) acc = a;
    }
    found |= acc;
    if (acc) {
        m.visited[v] = vold | acc;
        fnext[v] = acc;
        s.flag = 1;
    }
    // labels, source by source: one coalesced store per warp
    const unsigned long long wor_lo = __reduce_or_sync(0xffffffffu, (unsigned)(acc & 0xffffffffull));
    const unsigned long long wor_hi = __reduce_or_sync(0xffffffffu, (unsigned)(acc >> 32));
    unsigned long long wor = wor_lo | (wor_hi << 32);
    while (wor) {
        const int src = __ffsll((long long)wor) - 1;
        wor &= wor - 1;
        if ((acc >> src) & 1ull) st_stream(m.labels + (long long)src * n + v, level + 1 - s.off[src]);
    }
    r0_out = r0;
    deg_out = r1 - r0;
    return acc && r1 > r0;
}

// Pull level (symmetric graphs) in CTA-wide chunks: each warp takes PER
// blocks of the CTA's chunk; the chunk's discoveries go to the next frontier
// through one emit per chunk.
template <int B>
__device__ __forceinline__ void ms_pull_range(const BfsParams &p, const MsParams &m, MsSmem<B> &s, int level,
                                              const VertexFrontier &vout, unsigned long long *qe_out,
                                              unsigned long long &found)
{
    const int tid = threadIdx.x, lane = tid & 31;
    constexpr int PER = kChunkMax / B;
    int rs, re;
    cta_range(p.nodes, blockIdx.x, gridDim.x, rs, re);
    for (int cs = rs; cs < re; cs += kChunkMax) {
        if (tid == 0) s.out_count = 0;
        __syncthreads();
#pragma unroll 1
        for (int t = 0; t < PER; t++) {
            const int vb = cs + t * B + (tid & ~31);
            if (vb >= re) break;  // warp-uniform
            const int v = vb + lane;
            int r0, deg;
            const bool push = ms_pull_block<B>(p, m, s, level, vb, re, found, r0, deg);
            const unsigned bal = __ballot_sync(0xffffffffu, push);
            if (bal) {
                const int leader = __ffs(bal) - 1;
                int base = 0;
                if (lane == leader) base = atomicAdd(&s.out_count, __popc(bal));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (push) {
                    const int slot = base + __popc(bal & lanemask_lt());
                    s.out[slot] = v;
                    s.colstart[slot] = r0;
                    s.rel[slot] = deg;
                }
            }
        }
        __syncthreads();
        emit_frontier<B>(p, s, level, vout, qe_out);
        __syncthreads();
    }
}

// Pull level warp by warp (policy.warp_contract): blocks of 32 vertices dealt
// warp-major over every warp of the grid (warp_slice0), no CTA barrier; each
// warp's discoveries collect in its slice of the shared tables and go to the
// next frontier in flushes of their own (warp_emit).  A warp whose block holds
// a long scan no longer holds up the rest of its CTA.
template <int B>
__device__ __forceinline__ void ms_pull_range_warp(const BfsParams &p, const MsParams &m, MsSmem<B> &s, int level,
                                                   const VertexFrontier &vout, unsigned long long *qe_out,
                                                   unsigned long long &found)
{
    constexpr int NW = B / 32;
    constexpr int CAP = kChunkMax / NW;  // >= 32: a block's discoveries always fit after a flush
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t *bv = s.out + warp * CAP;
    int32_t *bc = s.colstart + warp * CAP;
    int32_t *bd = s.rel + warp * CAP;
    int count = 0;  // warp-uniform
    const int n = p.nodes;
    const long long stride = (long long)gridDim.x * NW * 32;
    for (long long b64 = (long long)warp_slice0(warp) * 32; b64 < n; b64 += stride) {
        const int vb = (int)b64;
        int r0, deg;
        const bool push = ms_pull_block<B>(p, m, s, level, vb, n, found, r0, deg);
        const unsigned bal = __ballot_sync(0xffffffffu, push);
        if (count + __popc(bal) > CAP) {
            warp_emit(p, bv, bc, bd, count, vout, qe_out);
            __syncwarp();  // the flush has read the output before it is refilled
            count = 0;
        }
        if (push) {
            const int slot = count + __popc(bal & lanemask_lt());
            bv[slot] = vb + lane;
            bc[slot] = r0;
            bd[slot] = deg;
        }
        count += __popc(bal);
    }
    if (count) warp_emit(p, bv, bc, bd, count, vout, qe_out);
}

// Block 0, between the grid barriers that end level `level` (no CTA touches the
// masks or the next frontier then): takes the join requests the host has
// raised since the last level end and seeds each as a source of level + 1 --
// label 0 in its slot's row, its visited bit, its bit in the next frontier
// mask and, if no other source put it there, an entry in the next frontier
// queue (emitted like any discovery, so the level's counters include it).
template <int B>
__device__ __forceinline__ void take_joins(const BfsParams &p, const MsParams &m, MsSmem<B> &s, int level,
                                           const VertexFrontier &vout, unsigned long long *qe_out)
{
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid == 0) {
        const int c = min((int)ld_acquire((const unsigned *)&m.join->count), 64);
        const int t = m.join->taken;  // written by block 0 only
        s.jn0 = t;
        s.jn1 = max(c, t);
        s.out_count = 0;
    }
    __syncthreads();
    const int t0 = s.jn0, t1 = s.jn1;
    if (t1 == t0) return;  // CTA-uniform
    unsigned long long *fnext = m.fmask[(level + 1) & 1];
    const long long n = p.nodes;
    for (int jb = t0; jb < t1; jb += B) {
        const int j = jb + tid;
        bool push = false;
        int v = 0, r0 = 0, r1 = 0;
        if (j < t1) {
            v = ld_cg(&m.join->src[j]);
            const int slot = ld_cg(&m.join->slot[j]);
            if (v >= 0 && v < p.nodes && slot >= 0 && slot < min(m.rows, 64)) {  // checked by the host too
                const unsigned long long bit = 1ull << slot;
                m.depth_limit[slot] = ld_cg(&m.join->limit[j]);
                m.level_off[slot] = level + 1;
                m.depth[slot] = 1;
                m.labels[(long long)slot * n + v] = 0;
                atomicOr(m.visited + v, bit);
                atomicOr(&m.join->used, bit);
                if (atomicOr(fnext + v, bit) == 0ull) {  // not yet in the next frontier
                    r0 = ld_ro(p.row_offsets + v);
                    r1 = ld_ro(p.row_offsets + v + 1);
                    push = r1 > r0;
                }
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, push);
        if (bal) {
            const int leader = __ffs(bal) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&s.out_count, __popc(bal));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (push) {
                const int slot_i = base + __popc(bal & lanemask_lt());
                s.out[slot_i] = v;
                s.colstart[slot_i] = r0;
                s.rel[slot_i] = r1 - r0;
            }
        }
    }
    __syncthreads();
    emit_frontier<B>(p, s, level, vout, qe_out);
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        m.join->taken = t1;
    }
}

// Whole batched search in one persistent cooperative grid.
template <int B>
__global__ void __launch_bounds__(B, 1024 / B) msbfs_kernel(BfsParams p, MsParams m)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MsSmem<B> &s = *reinterpret_cast<MsSmem<B> *>(smem_raw);
    __shared__ int s_ok;
    const int tid = threadIdx.x;
    unsigned generation = 0;
    int max_level_seen = -1;
    DutyClock duty(p);
    for (int level = 0;; level++) {
        const int pass = level;
        // the slots' depth limits and level offsets (sources may have joined at the last level end)
        if (tid < 64) {
            s.limits[tid] = ld_cg(m.depth_limit + tid);
            s.off[tid] = ld_cg(m.level_off + tid);
        }
        if (tid == 0) s.used = m.join ? ld_cg64(&m.join->used) : (m.k >= 64 ? ~0ull : ((1ull << m.k) - 1ull));
        __syncthreads();
        if (tid == 0) {
            const unsigned long long x = ld_cg64(&p.st->qe[pass % 3]);
            s.q = qe_count(x);
            s.E = qe_edges(x);
            s.flag = 0;
            if ((unsigned)s.E > (unsigned)p.edges || (unsigned)s.q > (unsigned)p.vcap) {
                atomicOr(&p.st->error, kErrOverflow);  // never read a frontier past its arrays
                s.q = 0;
            }
            s.found = 0;
            unsigned long long act = 0;
            for (int src = 0; src < 64; src++)
                if (((s.used >> src) & 1ull) && (s.limits[src] < 0 || level - s.off[src] < s.limits[src]))
                    act |= 1ull << src;
            s.active = act;
            if (blockIdx.x == 0) {
                p.st->qe[(pass + 2) % 3] = 0;
                p.st->tile_ctr[(pass + 1) % 3] = 0;
                atomicAdd(&p.st->total_queued, (unsigned long long)s.q);
                if (p.levels && pass < kMaxLevelRecords) {
                    LevelRecord r;
                    r.vertices = s.q;
                    r.edges = s.E;
                    r.bottom_up = 0;
                    r.pass = pass;
                    r.t_ns = globaltimer_ns();
                    p.levels[pass] = r;
                }
            }
        }
        __syncthreads();
        if (s.q == 0 || s.active == 0 || ld_cg(&p.st->error) != 0) break;
        // pull when the frontier's edges are a large share of the graph (symmetric graphs)
        const bool pull = m.pull_ok && (long long)s.E * p.bu_alpha > (long long)p.edges;
        if (tid == 0 && blockIdx.x == 0 && pull && p.levels && pass < kMaxLevelRecords) p.levels[pass].bottom_up = 1;
        unsigned long long found = 0;
        if (pull && p.warp_contract)
            ms_pull_range_warp<B>(p, m, s, level, p.vf[(level + 1) & 1], &p.st->qe[(pass + 1) % 3], found);
        else if (pull)
            ms_pull_range<B>(p, m, s, level, p.vf[(level + 1) & 1], &p.st->qe[(pass + 1) % 3], found);
        else
            ms_expand_range<B>(p, m, s, level, p.vf[level & 1], p.vf[(level + 1) & 1], &p.st->qe[(pass + 1) % 3],
                               found);
        {
            const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)(found & 0xffffffffull));
            const unsigned hi = __reduce_or_sync(0xffffffffu, (unsigned)(found >> 32));
            if ((tid & 31) == 0 && (lo | hi)) atomicOr(&s.found, ((unsigned long long)hi << 32) | lo);
        }
        __syncthreads();
        if (s.flag) max_level_seen = level + 1;
        if (tid == 0) {
            // sources that labelled a vertex level + 1 have search depth >= level + 2
            unsigned long long bits = s.found;
            while (bits) {
                const int src = __ffsll((long long)bits) - 1;
                bits &= bits - 1;
                atomicMax(m.depth + src, level + 2 - s.off[src]);
            }
        }
        if (!duty.barrier(p.st, generation, &s_ok)) break;
        // clear this level's frontier masks (the queue lists every vertex with edges that has one)
        {
            const VertexFrontier in = p.vf[level & 1];
            unsigned long long *fcur = m.fmask[level & 1];
            for (int i = blockIdx.x * B + tid; i < s.q; i += gridDim.x * B) fcur[ld_cg(in.v + i)] = 0ull;
        }
        if (m.join && blockIdx.x == 0) take_joins<B>(p, m, s, level, p.vf[(level + 1) & 1], &p.st->qe[(pass + 1) % 3]);
        if (!duty.barrier(p.st, generation, &s_ok)) break;
    }
    // The (source, vertex) pairs no level reached get label -1 here; every
    // other label was written by the level that reached the pair, so each
    // entry is written once (no fill of the k label rows before the search).
    // The loop above ends after a grid barrier, so every level's writes are done.
    {
        const unsigned long long kmask =
            m.join ? ld_cg64(&m.join->used) : (m.k >= 64 ? ~0ull : ((1ull << m.k) - 1ull));
        const int lane = tid & 31;
        const long long n = p.nodes, warps = (long long)gridDim.x * (B / 32);
        for (long long vb = ((long long)blockIdx.x * (B / 32) + (tid >> 5)) * 32; vb < n; vb += warps * 32) {
            const long long v = vb + lane;
            const unsigned long long miss = v < n ? ~ld_cg64(m.visited + v) & kmask : 0ull;
            const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)(miss & 0xffffffffull));
            const unsigned hi = __reduce_or_sync(0xffffffffu, (unsigned)(miss >> 32));
            unsigned long long wor = ((unsigned long long)hi << 32) | lo;
            while (wor) {
                const int src = __ffsll((long long)wor) - 1;
                wor &= wor - 1;
                if ((miss >> src) & 1ull) st_stream(m.labels + (long long)src * n + v, -1);
            }
        }
    }
    if (tid == 0 && max_level_seen >= 0) atomicMax(&p.st->max_level, max_level_seen);
    duty.finish();
    if (tid == 0 && blockIdx.x == 0) p.st->done = 1;
}

// Batch set-up: masks <- 0 (grid-stride) and the search state.  The label
// rows are not filled: the search writes every entry once (reached pairs by
// their level, the rest at its end).
template <int DUMMY = 0>
__global__ void msbfs_init_kernel(BfsParams p, MsParams m)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (long long v = t0; v < p.nodes; v += stride) {
        m.visited[v] = 0;
        m.fmask[0][v] = 0;
        m.fmask[1][v] = 0;
    }
    if (t0 == 0) {
        SearchState *st = p.st;
        st->tile_ctr[0] = st->tile_ctr[1] = st->tile_ctr[2] = 0;
        st->epoch += 1ull << 24;
        st->cur_level = 0;
        st->barrier = 0;
        st->error = 0;
        st->max_level = 0;
        st->done = 0;
        st->total_queued = 0;
        st->finished = 0;
        st->qe[1] = st->qe[2] = 0;
    }
}

// The batch's sources, passed by value to the seed kernel (no host staging).
struct MsSeed {
    int32_t src[64];               // distinct source vertices
    unsigned long long mask[64];   // combined source mask of each distinct vertex
    int32_t limit[64];             // depth limit of each source slot (< 0 unlimited)
    int32_t n_distinct;
};

// Second set-up step (after the fill): the depth limits, the sources' labels,
// masks and search depths, and the level-0 frontier queue of the distinct
// source vertices; one thread.
template <int DUMMY = 0>
__global__ void msbfs_seed_kernel(BfsParams p, MsParams m, MsSeed seed)
{
    if (threadIdx.x == 0) {
        for (int s = 0; s < 64; s++) {
            m.depth_limit[s] = s < m.k ? seed.limit[s] : 0;
            m.level_off[s] = 0;
            m.depth[s] = 1;
        }
        if (m.join) {
            m.join->count = 0;
            m.join->taken = 0;
            m.join->used = m.k >= 64 ? ~0ull : ((1ull << m.k) - 1ull);
        }
        int g = 0, d = 0;
        for (int i = 0; i < seed.n_distinct; i++) {
            const int v = seed.src[i];
            const unsigned long long mask = seed.mask[i];
            m.visited[v] = mask;
            m.fmask[0][v] = mask;
            for (int s = 0; s < m.k; s++)
                if ((mask >> s) & 1ull) m.labels[(long long)s * p.nodes + v] = 0;
            const int r0 = p.row_offsets[v], deg = p.row_offsets[v + 1] - r0;
            if (deg > 0) {
                p.vf[0].v[g] = v;
                p.vf[0].col[g] = r0;
                p.vf[0].P[g] = d;
                for (int c = (d + kChunkGrain - 1) / kChunkGrain; c * kChunkGrain < d + deg && c < p.cf_cap; c++)
                    p.vf[0].cf[c] = g;
                g++;
                d += deg;
            }
        }
        p.st->qe[0] = pack((unsigned)g, (unsigned)d);
    }
}

}  // namespace dev
}  // namespace b40c
