// BFS kernels for sm_100a.
//
// Reference semantics (b40c/graph/bfs): distances label[src] = 0,
// label[v] = BFS level, unvisited -1 (contract_expand_atomic/cta.cuh:293-297,
// expand_contract_atomic/kernel.cuh:314-318); predecessors label[src] = -2,
// label[v] = a vertex one level up (contract_expand_atomic/kernel.cuh:321-325).
//
// Design (B200-first, not a translation of the reference's CTA code):
//  * visited status is a 1-bit-per-vertex mask in 32-bit words (same memory
//    layout as the reference's byte mask); discovery is an atomicOr
//    test-and-set, so every vertex is labelled and enqueued exactly once and
//    labels never race;
//  * vertex frontiers carry each entry's degree prefix P and a chunk-first
//    index cf, so a level's flattened edge space is cut into equal
//    contiguous ranges, one per CTA (edge-balanced: a hub's adjacency list is
//    spread over many CTAs), walked in sub-rounds of kChunkMax edges;
//  * inside a sub-round, adjacency runs are gathered three ways: CTA-
//    cooperative (the sub-round lies inside one list: one cp.async.bulk
//    copy into shared memory), warp-cooperative (a warp reads 32 consecutive
//    positions of a run, one coalesced segment) and scan-based fine-grained
//    (short runs through a shared-memory position -> owner map);
//  * discovery is issued in overlapped phases (pre-check loads, atomics, CSR
//    rows of the winners) so every thread keeps its memory operations in
//    flight;
//  * frontier slots come from a CTA-wide shuffle scan plus either a
//    decoupled look-back over tile ids or one packed 64-bit atomic per tile,
//    never from per-item atomics;
//  * one kernel body serves per-level launches, CUDA-graph replays and a
//    persistent grid with a bounded software barrier between levels.
#pragma once
#include <cstdint>

#include "bfs_state.h"
#include "device_primitives.cuh"

namespace b40c {
namespace dev {

constexpr int kChunkMax = 2048;   // edges (or edge-frontier items) per sub-round
constexpr int kChunkGrain = 256;  // CTA ranges start at multiples of this; granularity of the cf index
// With a sub-grid threshold (p.subgrid_edges), mid-size top-down levels (more
// edges than a solo level, at most the threshold) of a persistent search run on
// the first kSubgridCtas CTAs, which synchronise among themselves; the rest of
// the grid waits at the grid barrier.
constexpr int kSubgridCtas = 16;

// emit_frontier: output entries whose degree spans more chunks than this have
// their cf runs written by the whole CTA.
constexpr unsigned kCfSerialChunks = 8;

template <int B, bool PRED>
struct ExpandSmem {
    // per-sub-round run tables; after the gather they hold the sub-round's
    // output (colstart = row start, rel = degree of each discovered vertex)
    int32_t colstart[kChunkMax + 2];
    int32_t rel[kChunkMax + 2];
    int32_t vert[PRED ? kChunkMax + 2 : 1];
    alignas(16) uint16_t own[kChunkMax];  // position -> run j owning it
    int32_t out[kChunkMax];   // discovered vertices of the sub-round
    alignas(16) int32_t stage[kChunkMax + 16];  // bulk-staged run (sub-round inside one list)
    uint64_t bar;             // mbarrier of the bulk copy
    int32_t out_count;
    int32_t flag;             // a vertex was labelled by this CTA in the current pass
    int32_t q, E;
    unsigned long long visited_edges;  // degree sum of the vertices visited up to this pass
    int32_t prev_bu;                   // the previous level ran bottom-up
    uint32_t *mask;                    // the visited-mask buffer of this pass (mask or mask_alt)
    int32_t wl_count;                  // bottom-up: still-unvisited vertices of the current chunk (in stage)
    int32_t ul_in;                     // bottom-up list mode: buffer holding this pass's unvisited list, or -1
    int32_t ul_n;                      // entries of that list
    int32_t ul_base;                   // where this chunk's still-unvisited vertices go in the next list
    int32_t solo_stop;                 // the solo phase writes its frontier out (CTA-uniform decision)
    int32_t run_count;                 // expand: runs of a sub-round that spans more than B entries
    uint32_t win_word[B];              // bottom-up windows: the window's visited words, discoveries OR'ed in
    unsigned long long scan_warp[B / 32];
    unsigned long long prefix;
    uint32_t *hist;                    // history cull table (dynamic shared memory past this struct), or null
    struct BuPrefetch *pf;             // bottom-up chunk prefetch buffer (dynamic shared memory), or null
    unsigned pf_phase;                 // parity of its mbarrier's next completion
    uint16_t *wmap;                    // warp-autonomous levels: each warp's position -> entry map, or null
    int32_t *wcol;                     // and its entry -> column index table (kWarpSlice entries per warp)
};

// The first bottom-up level of a run walks its CTA's vertex ids in chunks of
// kChunkMax.  With p.bu_prefetch, the next chunk's visited words, row offsets
// and hub pairs are staged into shared memory by bulk copies (cp.async.bulk,
// one mbarrier) while the current chunk's lists are scanned, so a chunk starts
// from shared memory instead of two dependent round trips to L2/HBM.  Entries
// a 16-byte copy cannot cover (the ragged end of the vertex range) are read
// from global memory.
struct alignas(16) BuPrefetch {
    int32_t rows[kChunkMax + 4];  // row_offsets[cs .. cs + nr)
    int2 hub[kChunkMax];          // hub2[cs .. cs + nh)
    uint32_t words[kChunkMax / 32];
    uint64_t bar;
    int32_t nr, nh, nw;           // entries staged (the rest: global loads)
};
constexpr size_t kBuPrefetchBytes = (sizeof(BuPrefetch) + 15) & ~size_t(15);

// History culling (the reference's HistoryCull, two_phase/contract_atomic/
// cta.cuh:276-297, as a B200 shared-memory filter): each CTA keeps a
// direct-mapped table of 2^p.hist_log vertex ids it has sent to the visited
// test in this launch.  Every id in it is visited (its first test set the
// bit, or found it set), so a gathered neighbour found in the table is
// dropped without touching the visited mask in L2; a collision only
// overwrites an entry (less filtering, never a wrong drop).  The table lives
// past ExpandSmem in dynamic shared memory and is cleared when a launch starts.
constexpr uint32_t kHistEmpty = 0xffffffffu;
__device__ __forceinline__ unsigned hist_slot(int v, int log2) { return ((unsigned)v * 2654435761u) >> (32 - log2); }

// Positions per slice of a warp-autonomous level (one cf chunk), and the
// shared memory of a warp's tables for it (position -> entry map, entry ->
// column index).
constexpr int kWarpSlice = kChunkGrain;
constexpr size_t kWarpTableBytes = kWarpSlice * (sizeof(uint16_t) + sizeof(int32_t));

// Dynamic shared memory past ExpandSmem: the history table (when on), then
// the bottom-up prefetch buffer (when on), then (CTAs of more than 256
// threads) the warp-autonomous levels' tables; the caller's barrier
// publishes them.
template <int B, bool PRED>
__device__ __forceinline__ void hist_init(const BfsParams &p, ExpandSmem<B, PRED> &s, unsigned char *smem_raw)
{
    size_t off = (sizeof(ExpandSmem<B, PRED>) + 15) & ~size_t(15);
    s.hist = nullptr;
    s.pf = nullptr;
    s.pf_phase = 0;
    if (p.hist_log > 0) {
        uint32_t *h = reinterpret_cast<uint32_t *>(smem_raw + off);
        for (int i = threadIdx.x; i < (1 << p.hist_log); i += B) h[i] = kHistEmpty;
        s.hist = h;
        off += sizeof(uint32_t) << p.hist_log;
    }
    if (p.bu_prefetch) {
        s.pf = reinterpret_cast<BuPrefetch *>(smem_raw + off);
        if (threadIdx.x == 0) mbar_init(&s.pf->bar, 1);
        off += kBuPrefetchBytes;
    }
    // the warp-autonomous levels' tables: in the sub-round arrays they leave
    // unused for CTAs of up to 256 threads, past the rest for larger CTAs
    // (kWarpTableBytes per warp; the host sizes the launch the same way)
    if (B <= 256) {
        s.wmap = s.own;
        s.wcol = s.stage;
    } else if (p.warp_contract) {
        s.wmap = reinterpret_cast<uint16_t *>(smem_raw + off);
        s.wcol = reinterpret_cast<int32_t *>(smem_raw + off + (B / 32) * kWarpSlice * sizeof(uint16_t));
    } else {
        s.wmap = nullptr;
        s.wcol = nullptr;
    }
}

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Instrumented searches: thread 0 records when its CTA reached `phase` of pass
// `pass` (first work chunk of the level only for phases < kPhaseArrive).
__device__ __forceinline__ void stamp(const BfsParams &p, int pass, int phase)
{
    if (p.arrive && threadIdx.x == 0 && pass < kMaxArrivePasses && blockIdx.x < kMaxArriveCtas)
        p.arrive[((size_t)pass * kMaxArriveCtas + blockIdx.x) * kPhaseStamps + phase] = globaltimer_ns();
}

// The same after a CTA barrier (so the stamp marks the slowest warp), only in
// instrumented searches; `when` and p.arrive are CTA-uniform.
__device__ __forceinline__ void stamp_synced(const BfsParams &p, int pass, int phase, bool when)
{
    if (when && p.arrive) {
        __syncthreads();
        stamp(p, pass, phase);
    }
}

// Test-only (p.late_start_ns): every CTA but CTA 0 waits that long before it
// reads its start state, like a CTA the hardware schedules late.  The wait is
// on the global timer, with an iteration cap as well.
__device__ __forceinline__ void late_start(const BfsParams &p)
{
    if (p.late_start_ns && blockIdx.x != 0) {
        if (threadIdx.x == 0) {
            const unsigned long long t0 = globaltimer_ns();
            for (unsigned i = 0; i < (p.late_start_ns >> 8) + 1024 && globaltimer_ns() - t0 < p.late_start_ns; i++)
                __nanosleep(256);
        }
        __syncthreads();
    }
}

// Packed (count, degree) pair: count in the high 32 bits.
__device__ __forceinline__ unsigned long long pack(unsigned cnt, unsigned deg)
{
    return ((unsigned long long)cnt << 32) | deg;
}

// CTA-wide exclusive scan of one 64-bit value per thread; returns the
// exclusive prefix and writes the CTA total to *total (all threads).
template <int B>
__device__ __forceinline__ unsigned long long cta_exclusive_scan(unsigned long long x, unsigned long long *warp_buf,
                                                                 unsigned long long *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long incl = x;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        unsigned long long y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += y;
    }
    if (lane == 31) warp_buf[warp] = incl;
    __syncthreads();
    unsigned long long wpre = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < B / 32; w++) {
        unsigned long long t = warp_buf[w];
        if (w < warp) wpre += t;
        tot += t;
    }
    __syncthreads();
    *total = tot;
    return wpre + incl - x;
}

// Optional warp culling: among lanes holding the same vertex only the lowest stays valid.
__device__ __forceinline__ bool warp_cull(bool valid, int v)
{
    const int lane = threadIdx.x & 31;
    unsigned peers = __match_any_sync(0xffffffffu, valid ? v : -2 - lane);
    return valid && (__ffs(peers) - 1 == lane);
}

// Discovery of up to U gathered neighbours per thread, in overlapped phases
// (visited-word pre-checks, then atomic test-and-sets, then the CSR rows of
// the winners) so each thread keeps all of its memory operations in flight.
// A winner is labelled and, when it has edges, appended to the sub-round's
// output (s.out = vertex, s.colstart = row start, s.rel = degree; the run
// tables are consumed by then).  With LEAVES (vertex-frontier searches) the
// winners without edges, which never enter a frontier, are added to the
// search's total_queued: the reference's expand-contract queues every
// discovered vertex (expand_contract_atomic/cta.cuh:432-466).  All threads of
// the CTA call it with CTA-uniform `active`.
template <int B, bool PRED, int U, bool LISTS = false, bool LEAVES = false>
__device__ __forceinline__ void discover_batch(const BfsParams &p, ExpandSmem<B, PRED> &s, const int (&v)[U],
                                               const int (&u)[U], const bool (&valid)[U], const bool (&active)[U],
                                               int label_value, bool precheck = true)
{
    bool go[U];
    unsigned word[U];
    precheck = precheck && p.precheck && !(LISTS && s.ul_in >= 0);
    uint32_t *hist = s.hist;
#pragma unroll
    for (int t = 0; t < U; t++) {
        go[t] = valid[t];
        if (active[t] && p.warp_cull) go[t] = warp_cull(go[t], v[t]);
        if (hist && go[t]) {
            const unsigned h = hist_slot(v[t], p.hist_log);
            if (hist[h] == (uint32_t)v[t])
                go[t] = false;  // already sent to the visited test by this CTA: visited
            else
                hist[h] = (uint32_t)v[t];
        }
        word[t] = 0;
        if (go[t] && precheck) word[t] = p.precheck == 2 ? ld_cg(s.mask + (v[t] >> 5)) : ld_mask(s.mask + (v[t] >> 5));
    }
    bool found[U];
    if (LISTS && s.ul_in >= 0) {
        // after a bottom-up list-mode level the visited mask is not kept: the
        // labels decide (a distance search's unreached vertices hold -1)
#pragma unroll
        for (int t = 0; t < U; t++) {
            found[t] = false;
            if (go[t] && ld_cg(p.labels + v[t]) == -1) found[t] = atomicCAS(p.labels + v[t], -1, label_value) == -1;
        }
    } else {
#pragma unroll
        for (int t = 0; t < U; t++) {
            const unsigned bit = 1u << (v[t] & 31);
            found[t] = false;
            if (go[t] && !(word[t] & bit)) found[t] = !(atomicOr(s.mask + (v[t] >> 5), bit) & bit);
        }
    }
    int r0[U], r1[U];
#pragma unroll
    for (int t = 0; t < U; t++) {
        r0[t] = r1[t] = 0;
        if (found[t]) {
            p.labels[v[t]] = PRED ? u[t] : label_value;
            r0[t] = ld_ro(p.row_offsets + v[t]);
            r1[t] = ld_ro(p.row_offsets + v[t] + 1);
        }
    }
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int t = 0; t < U; t++) {
        if (!active[t]) continue;
        if (found[t]) s.flag = 1;  // benign race: every writer stores 1
        const bool push = found[t] && r1[t] > r0[t];
        if (LEAVES) {
            const unsigned leaf = __ballot_sync(0xffffffffu, found[t] && !push);
            if (leaf && lane == __ffs(leaf) - 1) atomicAdd(&p.st->total_queued, (unsigned long long)__popc(leaf));
        }
        const unsigned bal = __ballot_sync(0xffffffffu, push);
        if (bal == 0) continue;
        const int leader = __ffs(bal) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&s.out_count, __popc(bal));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (push) {
            const int slot = base + __popc(bal & lanemask_lt());
            s.out[slot] = v[t];
            s.colstart[slot] = r0[t];
            s.rel[slot] = r1[t] - r0[t];
        }
    }
}

// Turns the sub-round's output entries (s.out / s.colstart / s.rel over
// [0, s.out_count): vertex, row start, degree > 0) into entries of the vertex
// frontier `vout`.  A CTA scan of (count, degree) pairs gives each entry its
// offset inside the tile; the tile's base comes from a decoupled look-back
// over tile ids (taken once the tile's aggregate is known, so no tile ever
// waits for another tile's gather) or, with alloc_lookback = 0, from one
// packed 64-bit atomicAdd on the pass's output counter (always with
// lookback = false).  Each entry gets its slot, its degree prefix P and its
// kChunkGrain boundaries in vout.cf.  The pass total accumulates in *qe_out.
// A tile whose output ends past `skip_above` edges of the pass total only
// counts: the caller passes the edge total beyond which the next level is
// certain to run bottom-up (which never reads the frontier).  All threads must
// call it.
template <int B, typename Smem>
__device__ __forceinline__ void emit_frontier(const BfsParams &p, Smem &s, int pass, const VertexFrontier &vout,
                                              unsigned long long *qe_out, bool lookback = true,
                                              unsigned long long skip_above = ~0ull)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int cnt = s.out_count;
    constexpr int PER = kChunkMax / B;
    const int per = (cnt + B - 1) / B;
    const int jb = min(tid * per, cnt), je = min(jb + per, cnt);
    unsigned my_deg = 0;
#pragma unroll
    for (int t = 0; t < PER; t++)
        if (jb + t < je) my_deg += (unsigned)s.rel[jb + t];
    unsigned long long tot;
    const unsigned long long excl = cta_exclusive_scan<B>(pack((unsigned)(je - jb), my_deg), s.scan_warp, &tot);
    if (tot == 0) return;  // CTA-uniform: nothing to allocate
    if (warp == 0) {
        unsigned long long prefix = 0;
        if (!p.alloc_lookback || !lookback) {
            if (lane == 0) prefix = atomicAdd(qe_out, tot);
        } else {
            const unsigned long long epoch = p.st->epoch + (unsigned long long)pass;
            int tile = 0;
            if (lane == 0) tile = (int)atomicAdd(&p.st->tile_ctr[pass % 3], 1u);
            tile = __shfl_sync(0xffffffffu, tile, 0);
            if (tile >= p.max_chunks) {
                if (lane == 0) atomicOr(&p.st->error, kErrOverflow);
                prefix = ~0ull;
            } else if (tile == 0) {
                if (lane == 0) lookback_publish(&p.slots[0], epoch, kFlagInclusive, tot);
            } else {
                if (lane == 0) lookback_publish(&p.slots[tile], epoch, kFlagAggregate, tot);
                prefix = lookback_exclusive(p.slots, (unsigned)tile, epoch, &p.st->error, p.spin_limit);
                if (lane == 0 && prefix != ~0ull) lookback_publish(&p.slots[tile], epoch, kFlagInclusive, prefix + tot);
            }
            if (lane == 0 && prefix != ~0ull) atomicAdd(qe_out, tot);  // pass totals
        }
        if (lane == 0) s.prefix = prefix;
    }
    __syncthreads();
    const unsigned long long prefix = s.prefix;
    if (prefix == ~0ull) return;
    const unsigned g0 = (unsigned)(prefix >> 32), d0 = (unsigned)(prefix & 0xffffffffu);
    if ((unsigned long long)d0 + (tot & 0xffffffffull) > skip_above) {
        // counted above; the entries themselves are never read
        if (tid == 0 && (unsigned long long)g0 + (tot >> 32) > (unsigned long long)p.vcap)
            atomicOr(&p.st->error, kErrOverflow);
        return;
    }
    unsigned g = g0 + (unsigned)(excl >> 32);
    unsigned d = d0 + (unsigned)(excl & 0xffffffffu);
    bool long_run = false;
    for (int j = jb; j < je; j++) {
        const unsigned deg = (unsigned)s.rel[j];
        if ((int)g < p.vcap) {
            vout.v[g] = s.out[j];
            vout.col[g] = s.colstart[j];
            vout.P[g] = (int)d;
            // cf[c] = g for the chunks c starting inside [d, d + deg); long runs
            // (high-degree vertices) are left to the whole CTA below
            const unsigned c0 = (d + kChunkGrain - 1) / kChunkGrain, c1 = (d + deg + kChunkGrain - 1) / kChunkGrain;
            if (c1 - c0 > kCfSerialChunks) {
                long_run = true;
            } else {
                for (unsigned c = c0; c < c1; c++) {
                    if (c >= (unsigned)p.cf_cap) {  // a level's edges exceed the graph's: never past the end
                        atomicOr(&p.st->error, kErrOverflow);
                        break;
                    }
                    vout.cf[c] = (int)g;
                }
            }
        } else {
            atomicOr(&p.st->error, kErrOverflow);
        }
        s.colstart[j] = (int)(d - d0);  // tile-relative degree prefix, for the pass below
        g++;
        d += deg;
    }
    if (!__syncthreads_or(long_run)) return;  // CTA-uniform
    // the long runs: each thread takes a contiguous stretch of the tile's
    // chunks, finds the owner of its first chunk by binary search and walks on;
    // owners spanning more than kCfSerialChunks chunks are written here
    const unsigned tdeg = (unsigned)(tot & 0xffffffffu);
    const unsigned c0 = (d0 + kChunkGrain - 1) / kChunkGrain, c1 = (d0 + tdeg + kChunkGrain - 1) / kChunkGrain;
    if (tid == 0 && c1 > (unsigned)p.cf_cap) atomicOr(&p.st->error, kErrOverflow);
    const unsigned c_end = min(c1, (unsigned)p.cf_cap);
    const unsigned stretch = (c_end > c0 ? c_end - c0 : 0u) / B + 1;
    const unsigned cb = c0 + tid * stretch, ce = min(cb + stretch, c_end);
    if (cb < ce) {
        const int x0 = (int)(cb * kChunkGrain - d0);  // in [0, tdeg)
        int lo = 0, hi = cnt - 1;                     // last entry whose prefix is <= x0
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s.colstart[mid] <= x0) lo = mid; else hi = mid - 1;
        }
        int j = lo;
        int next = j + 1 < cnt ? s.colstart[j + 1] : INT_MAX;
        bool long_j = false;
        int j_known = -1;
        for (unsigned c = cb; c < ce; c++) {
            const int x = (int)(c * kChunkGrain - d0);
            while (x >= next) {
                j++;
                next = j + 1 < cnt ? s.colstart[j + 1] : INT_MAX;
            }
            if (j != j_known) {
                const unsigned ed = d0 + (unsigned)s.colstart[j], edeg = (unsigned)s.rel[j];
                long_j = (ed + edeg + kChunkGrain - 1) / kChunkGrain - (ed + kChunkGrain - 1) / kChunkGrain >
                         kCfSerialChunks;
                j_known = j;
            }
            if (long_j && (int)(g0 + j) < p.vcap) vout.cf[c] = (int)(g0 + j);
        }
    }
}

// Share `part` of `parts` of n items: [rs, re), with rs and re multiples of
// kChunkGrain except re = n for the last share.
__device__ __forceinline__ void cta_range(int n, int part, int parts, int &rs, int &re)
{
    const long long b = part, G = parts;
    rs = (int)((long long)n * b / G / kChunkGrain * kChunkGrain);
    re = (b == G - 1) ? n : (int)((long long)n * (b + 1) / G / kChunkGrain * kChunkGrain);
}

// ------------------------------------------------------------------------------------
// Edge-balanced expansion of the CTA's range of a vertex frontier's flattened
// edge space, in sub-rounds of kChunkMax positions.
//   FUSED_CULL = true  : expand-contract (EC): every gathered neighbour goes
//                        through discovery; discoveries become the next
//                        vertex frontier (one emit per sub-round).
//   FUSED_CULL = false : two-phase expand: neighbours are written to the edge
//                        frontier at their flattened edge position.
// ------------------------------------------------------------------------------------
template <int B, bool PRED, bool FUSED_CULL, bool LISTS = false>
__device__ __forceinline__ void expand_range(const BfsParams &p, const VertexFrontier &in, ExpandSmem<B, PRED> &s,
                                             int level, int pass, const VertexFrontier &vout,
                                             const EdgeFrontier &eout, unsigned long long *qe_out,
                                             unsigned &bar_phase, int part, int parts, bool defer_emit = false,
                                             unsigned long long skip_above = ~0ull)
{
    const int tid = threadIdx.x;
    const int q = s.q, E = s.E;
    constexpr int PER = kChunkMax / B;  // sub-round positions per thread
    int rs, re;
    cta_range(E, part, parts, rs, re);
    if (rs >= re) return;
    int i_cur = ld_cg(in.cf + rs / kChunkGrain);  // entry owning position rs
    if (FUSED_CULL) stamp(p, pass, 0);
    // sub-round length: policy.chunk_edges (a solo level kept in shared memory is one full sub-round)
    const int chunk = defer_emit ? kChunkMax : min(max(p.chunk_edges, 256), kChunkMax);
    for (int cs = rs; cs < re; cs += chunk) {
        const int ce = min(cs + chunk, re);
        const int len = ce - cs;
        const bool first = FUSED_CULL && cs == rs;
        // ---- load the runs of entries i_cur.. that start before ce ----------------
        if (tid == 0) {
            s.out_count = 0;
            s.run_count = B;
        }
        int k;
        {
            // (an entry's degree prefix, row start and vertex are loaded together:
            // one round trip, not two)
            const int i = i_cur + tid;
            bool inside = false;
            if (i < q) {
                const int Pi = ld_cg(in.P + i);
                const int ci = ld_cg(in.col + i);
                const int vi = PRED ? ld_cg(in.v + i) : 0;
                if (Pi < ce) {
                    inside = true;
                    const int start = max(Pi, cs);
                    s.rel[tid] = start - cs;
                    s.colstart[tid] = ci + (start - Pi);
                    if (PRED) s.vert[tid] = vi;
                }
            }
            k = __syncthreads_count(inside);
        }
        if (k == B) {
            // the sub-round spans more than B entries (short lists): the rest, at
            // most kChunkMax + 1 - B (every entry has an edge), are loaded at once
            // rather than B at a time; the entries inside form a prefix
            constexpr int R = (kChunkMax + B) / B - 1;
            int Pr[R];
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int i = i_cur + (r + 1) * B + tid;
                Pr[r] = (i < q && i - i_cur <= kChunkMax) ? ld_cg(in.P + i) : INT_MAX;
            }
            int last = 0;
#pragma unroll
            for (int r = 0; r < R; r++) {
                if (Pr[r] < ce) {
                    const int i = i_cur + (r + 1) * B + tid;
                    const int j = (r + 1) * B + tid;
                    const int start = max(Pr[r], cs);
                    s.rel[j] = start - cs;
                    s.colstart[j] = ld_cg(in.col + i) + (start - Pr[r]);
                    if (PRED) s.vert[j] = ld_cg(in.v + i);
                    last = j + 1;
                }
            }
            if (last) atomicMax(&s.run_count, last);
            __syncthreads();
            k = s.run_count;
        }
        if (tid == 0) s.rel[k] = len;
        if (first) stamp(p, pass, 1);
        const int j_last = k - 1;  // its run may continue into the next sub-round

        // ---- CTA-cooperative gather: a sub-round inside one adjacency list is
        // staged into shared memory with one bulk copy of its 16-byte aligned
        // body (aligned by address, so any 4-byte aligned column array works) --
        const bool single = p.bulk_ok && (k == 1) && (len >= p.cta_thresh);
        int b0 = 0, b1 = 0;
        bool staged = true;  // false: this thread's wait for the bulk copy ran out
        if (single) {
            const int c0 = s.colstart[0];
            // column index i sits at a 16-byte boundary when (i + mis) % 4 == 0
            const int mis = (int)((reinterpret_cast<uintptr_t>(p.column_indices) >> 2) & 3u);
            b0 = ((c0 + mis + 3) & ~3) - mis;
            b1 = ((c0 + len + mis) & ~3) - mis;
            if (b1 > b0) {
                if (tid == 0) {
                    fence_proxy_async_smem();
                    mbar_arrive_expect_tx(&s.bar, (unsigned)(b1 - b0) * 4u);
                    bulk_g2s(s.stage, p.column_indices + b0, (unsigned)(b1 - b0) * 4u, &s.bar);
                }
                unsigned spins = 0;
                while (!mbar_try_wait(&s.bar, bar_phase)) {
                    if (++spins > p.spin_limit) {
                        staged = false;
                        break;
                    }
                }
            }
        } else {
            // ---- owner map: thread t resolves positions [t*PER, t*PER + PER)
            // (binary search for the first, then a walk over run starts) -----------
            __syncthreads();
            const int x0 = tid * PER;
            if (x0 < len) {
                int lo = 0, hi = k - 1;  // last j with rel[j] <= x0
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
        if (!__syncthreads_and(staged)) {
            // the copy did not land in time: report it, give the copy still in
            // flight one more bounded wait (so it cannot land in shared memory
            // the CTA reuses) and stop; every caller reads the error word next
            if (tid == 0) {
                atomicOr(&p.st->error, kErrBulk);
                unsigned spins = 0;
                while (!mbar_try_wait(&s.bar, bar_phase) && ++spins <= p.spin_limit) __nanosleep(256);
            }
            __syncthreads();
            return;
        }
        if (single && b1 > b0) bar_phase ^= 1u;

        if (first) stamp(p, pass, 2);
        // ---- gather: thread t takes positions t, t + B, ...: a warp reads 32
        // consecutive positions (one coalesced segment of any run >= 32 long) ------
        int v[PER], u[PER];
        bool valid[PER], active[PER];
#pragma unroll
        for (int t = 0; t < PER; t++) {
            const int x = t * B + tid;
            active[t] = t * B < len;  // CTA-uniform
            valid[t] = x < len;
            v[t] = -1;
            u[t] = -1;
            if (valid[t]) {
                const int j = single ? 0 : s.own[x];
                const int c = s.colstart[j] + (x - s.rel[j]);
                v[t] = (c >= b0 && c < b1) ? s.stage[c - b0] : ld_stream(p.column_indices + c);
                if (PRED) u[t] = s.vert[j];
            }
        }
        i_cur += j_last;
        if (!FUSED_CULL) {
#pragma unroll
            for (int t = 0; t < PER; t++) {
                if (valid[t]) {
                    eout.v[cs + t * B + tid] = v[t];
                    if (PRED) eout.pred[cs + t * B + tid] = u[t];
                }
            }
            __syncthreads();  // run tables and stage free for the next sub-round
            continue;
        }
        __syncthreads();  // run tables consumed: they now collect the sub-round's output
        if (first) stamp(p, pass, 3);
        discover_batch<B, PRED, PER, LISTS, true>(p, s, v, u, valid, active, level + 1);
        __syncthreads();
        if (first) stamp(p, pass, 4);
        if (defer_emit) return;  // single sub-round (the caller checked): the output stays in s.out / colstart / rel
        emit_frontier<B>(p, s, pass, vout, qe_out, true, skip_above);
        __syncthreads();
        if (first) stamp(p, pass, 5);
    }
}

// Solo levels (CTA 0 alone, one sub-round each) can pass their frontier from
// one level to the next in shared memory.  A level's discoveries sit in
// s.out / colstart / rel (n entries: vertex, row start, degree); the next
// level turns them in place into its run tables (rel = degree prefix with
// rel[n] = E, colstart = row start, vert = vertex) and runs from there, with
// no frontier, counter or chunk-index traffic.  solo_level_smem runs such a
// level: owner map, gather, discovery (atomic test-and-set without the
// visited-word pre-check), output back in s.out / colstart / rel.
template <int B, bool PRED, bool LISTS>
__device__ __forceinline__ void solo_level_smem(const BfsParams &p, ExpandSmem<B, PRED> &s, int level, int n, int E)
{
    const int tid = threadIdx.x;
    constexpr int PER = kChunkMax / B;
    {
        const int x0 = tid * PER;
        if (x0 < E) {
            int lo = 0, hi = n - 1;  // last j with rel[j] <= x0
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (s.rel[mid] <= x0) lo = mid; else hi = mid - 1;
            }
            int j = lo;
            int next = s.rel[j + 1];
#pragma unroll
            for (int t = 0; t < PER; t++) {
                const int x = x0 + t;
                if (x < E) {
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
    int v[PER], u[PER];
    bool valid[PER], active[PER];
#pragma unroll
    for (int t = 0; t < PER; t++) {
        const int x = t * B + tid;
        active[t] = t * B < E;
        valid[t] = x < E;
        v[t] = -1;
        u[t] = -1;
        if (valid[t]) {
            const int j = s.own[x];
            v[t] = ld_stream(p.column_indices + s.colstart[j] + (x - s.rel[j]));
            if (PRED) u[t] = s.vert[j];
        }
    }
    __syncthreads();  // run tables consumed: they now collect the level's output
    discover_batch<B, PRED, PER, LISTS, true>(p, s, v, u, valid, active, level + 1, false);
    __syncthreads();
}

// Contraction of the CTA's range of an edge frontier (q items), in sub-rounds
// of kChunkMax items: each item's visited bit is test-and-set; a first visit
// labels the vertex with the current level (or its predecessor) and the
// vertices with edges become the vertex frontier vf[0].
template <int B, bool PRED>
__device__ __forceinline__ void contract_range(const BfsParams &p, ExpandSmem<B, PRED> &s, const EdgeFrontier &in,
                                               int level, int pass, unsigned long long *qe_out)
{
    const int tid = threadIdx.x;
    const int q = s.q;
    constexpr int PER = kChunkMax / B;
    int rs, re;
    cta_range(q, blockIdx.x, gridDim.x, rs, re);
    const int chunk = min(max(p.chunk_edges, 256), kChunkMax);
    for (int cs = rs; cs < re; cs += chunk) {
        const int ce = min(cs + chunk, re);
        if (tid == 0) s.out_count = 0;
        int v[PER], u[PER];
        bool valid[PER], active[PER];
#pragma unroll
        for (int t = 0; t < PER; t++) {
            const int i = cs + t * B + tid;
            active[t] = cs + t * B < ce;
            valid[t] = i < ce;
            v[t] = valid[t] ? ld_cg(in.v + i) : -1;
            u[t] = (PRED && valid[t]) ? ld_cg(in.pred + i) : -1;
        }
        __syncthreads();
        discover_batch<B, PRED, PER>(p, s, v, u, valid, active, level);
        __syncthreads();
        emit_frontier<B>(p, s, pass, p.vf[0], qe_out);
        __syncthreads();
    }
}

// One warp's output (bv = vertex, bc = row start, bd = degree, `count`
// entries in the warp's own slice of the shared tables) appended to the
// vertex frontier: a warp scan of (count, degree) pairs, one packed 64-bit
// atomicAdd on the pass counter for the slots and the degree prefix, then the
// entries, their degree prefixes P and their kChunkGrain boundaries in cf
// (runs over more than kCfSerialChunks chunks written by the whole warp).
// bc is overwritten with each entry's flush-relative degree prefix.  A flush
// whose output ends past `skip_above` edges of the pass total only counts
// (see emit_frontier).  All 32 lanes call it with the same count.
__device__ __forceinline__ void warp_emit(const BfsParams &p, const int32_t *bv, int32_t *bc, const int32_t *bd,
                                          int count, const VertexFrontier &vout, unsigned long long *qe_out,
                                          unsigned long long skip_above = ~0ull)
{
    const int lane = threadIdx.x & 31;
    __syncwarp();
    const int per = (count + 31) >> 5;
    const int jb = min(lane * per, count), je = min(jb + per, count);
    unsigned my_deg = 0;
    for (int j = jb; j < je; j++) my_deg += (unsigned)bd[j];
    const unsigned long long x = pack((unsigned)(je - jb), my_deg);
    unsigned long long incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const unsigned long long tot = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long prefix = 0;
    if (lane == 0) prefix = atomicAdd(qe_out, tot);
    prefix = __shfl_sync(0xffffffffu, prefix, 0);
    const unsigned long long excl = incl - x;
    const unsigned g0 = (unsigned)(prefix >> 32), d0 = (unsigned)(prefix & 0xffffffffu);
    if ((unsigned long long)d0 + (tot & 0xffffffffull) > skip_above) {
        // counted above; the entries themselves are never read (the next level
        // is certain to run bottom-up, as in emit_frontier)
        if (lane == 0 && (unsigned long long)g0 + (tot >> 32) > (unsigned long long)p.vcap)
            atomicOr(&p.st->error, kErrOverflow);
        return;
    }
    unsigned g = g0 + (unsigned)(excl >> 32);
    unsigned d = d0 + (unsigned)(excl & 0xffffffffu);
    bool long_run = false;
    for (int j = jb; j < je; j++) {
        const unsigned deg = (unsigned)bd[j];
        if ((int)g < p.vcap) {
            vout.v[g] = bv[j];
            vout.col[g] = bc[j];
            vout.P[g] = (int)d;
            const unsigned c0 = (d + kChunkGrain - 1) / kChunkGrain, c1 = (d + deg + kChunkGrain - 1) / kChunkGrain;
            if (c1 - c0 > kCfSerialChunks) {
                long_run = true;
            } else {
                for (unsigned c = c0; c < c1; c++) {
                    if (c >= (unsigned)p.cf_cap) {  // a level's edges exceed the graph's: never past the end
                        atomicOr(&p.st->error, kErrOverflow);
                        break;
                    }
                    vout.cf[c] = (int)g;
                }
            }
        } else {
            atomicOr(&p.st->error, kErrOverflow);
        }
        bc[j] = (int)(d - d0);
        g++;
        d += deg;
    }
    unsigned lanes = __ballot_sync(0xffffffffu, long_run);
    if (!lanes) return;
    __syncwarp();  // bc holds the flush-relative prefixes
    // entries spanning many chunks (high-degree vertices): the whole warp
    // writes each one's run of cf, 32 chunks per step
    while (lanes) {
        const int L = __ffs(lanes) - 1;
        lanes &= lanes - 1;
        const int lb = min(L * per, count), le = min(lb + per, count);
        for (int j = lb; j < le; j++) {
            const unsigned ed = d0 + (unsigned)bc[j], deg = (unsigned)bd[j];
            const unsigned c0 = (ed + kChunkGrain - 1) / kChunkGrain, c1 = (ed + deg + kChunkGrain - 1) / kChunkGrain;
            if (c1 - c0 <= kCfSerialChunks || (int)(g0 + j) >= p.vcap) continue;
            if (lane == 0 && c1 > (unsigned)p.cf_cap) atomicOr(&p.st->error, kErrOverflow);
            const unsigned c_end = min(c1, (unsigned)p.cf_cap);
            for (unsigned c = c0 + lane; c < c_end; c += 32) vout.cf[c] = (int)(g0 + j);
        }
    }
}

// Warp-autonomous passes are taken by levels with at least a full sub-round
// of work per CTA: in smaller ones (the first levels from a hub, which
// discover most of what they touch) a warp would flush its output after
// nearly every slice, and the CTA-wide sub-rounds measured 3x faster there.
__device__ __forceinline__ bool warp_sized(int items) { return items >= (int)gridDim.x * kChunkMax; }

// Warp-autonomous passes deal their slices over every warp of the grid,
// warp-major (slice k goes to warp k / gridDim of CTA k % gridDim, then
// every gridDim * NW slices on), so a small level spreads over all SMs and a
// large one is balanced to a slice.  First slice of warp `warp` of this CTA.
__device__ __forceinline__ int warp_slice0(int warp) { return warp * (int)gridDim.x + (int)blockIdx.x; }

// Visited test of one warp's batch of PER neighbours per lane (pre-check
// loads, atomic test-and-set, the CSR rows of the winners; each winner is
// labelled), then the winners with edges appended to the warp's output
// (bv / bc / bd, `count` entries of at most `cap`, flushed to the vertex
// frontier first when the batch could overrun it).  With LEAVES the winners
// without edges are added to total_queued (vertex-frontier strategies queue
// every discovered vertex, expand_contract_atomic/cta.cuh:432-466).  Returns
// whether this lane labelled a vertex.  All 32 lanes call it.
template <int PER, bool PRED, bool LEAVES, int CAP>
__device__ __forceinline__ bool warp_discover(const BfsParams &p, uint32_t *mask, const int (&v)[PER],
                                             const int (&u)[PER], const bool (&go)[PER], int label_value,
                                             int32_t *bv, int32_t *bc, int32_t *bd, int &count,
                                             const VertexFrontier &vout, unsigned long long *qe_out,
                                             unsigned long long skip_above = ~0ull)
{
    const int lane = threadIdx.x & 31;
    const int pre = p.precheck;
    unsigned word[PER];
#pragma unroll
    for (int t = 0; t < PER; t++) {
        word[t] = 0;
        if (go[t] && pre) word[t] = pre == 2 ? ld_cg(mask + (v[t] >> 5)) : ld_mask(mask + (v[t] >> 5));
    }
    bool found[PER];
#pragma unroll
    for (int t = 0; t < PER; t++) {
        const unsigned bit = 1u << (v[t] & 31);
        found[t] = go[t] && !(word[t] & bit) && !(atomicOr(mask + (v[t] >> 5), bit) & bit);
    }
    bool any = false;
    int r0[PER], deg[PER];
#pragma unroll
    for (int t = 0; t < PER; t++) {
        r0[t] = deg[t] = 0;
        if (found[t]) {
            p.labels[v[t]] = PRED ? u[t] : label_value;
            r0[t] = ld_ro(p.row_offsets + v[t]);
            deg[t] = ld_ro(p.row_offsets + v[t] + 1);
            any = true;
        }
    }
    unsigned leaves = 0;
#pragma unroll
    for (int t = 0; t < PER; t++) {
        deg[t] -= r0[t];  // 0 for the lanes that found nothing
        if (LEAVES) leaves += __popc(__ballot_sync(0xffffffffu, found[t] && deg[t] == 0));
    }
    if (LEAVES && leaves && lane == 0) atomicAdd(&p.st->total_queued, (unsigned long long)leaves);
    // append, flushing first when the winners could overrun the output; a batch
    // larger than the output (CTAs of more than 256 threads test 256 neighbours
    // into 128 entries) is appended in halves
    constexpr int HALF = PER * 32 > CAP ? PER / 2 : PER;
    static_assert(HALF * 32 <= CAP && PER % HALF == 0, "a half batch's winners fit the warp's output");
#pragma unroll
    for (int h0 = 0; h0 < PER; h0 += HALF) {
        int n_new = 0;
#pragma unroll
        for (int t = h0; t < h0 + HALF; t++) n_new += __popc(__ballot_sync(0xffffffffu, deg[t] > 0));
        if (count + n_new > CAP) {
            warp_emit(p, bv, bc, bd, count, vout, qe_out, skip_above);
            __syncwarp();  // the flush has read the output before it is refilled
            count = 0;
        }
#pragma unroll
        for (int t = h0; t < h0 + HALF; t++) {
            const unsigned bal = __ballot_sync(0xffffffffu, deg[t] > 0);
            if (deg[t] > 0) {
                const int slot = count + __popc(bal & lanemask_lt());
                bv[slot] = v[t];
                bc[slot] = r0[t];
                bd[slot] = deg[t];
            }
            count += __popc(bal);
        }
    }
    return any;
}

// Warp-autonomous contraction of the CTA's share of an edge frontier
// (policy.warp_contract): each warp takes its slices of 256 items
// (warp_slice0) and runs the visited test on each with no CTA barrier;
// winners with edges collect in the warp's slice of the shared tables and go
// to the vertex frontier in flushes of their own (warp_emit).  A warp never
// waits for the slowest load of another warp, and the frontier slots cost one
// atomic per flush.  Same labels and frontier contents as contract_range (the
// reference's contraction, contract_expand_atomic/cta.cuh:213-304); the
// entries' order differs.
template <int B, bool PRED>
__device__ __forceinline__ void contract_range_warp(const BfsParams &p, ExpandSmem<B, PRED> &s,
                                                    const EdgeFrontier &in, int level, const VertexFrontier &vout,
                                                    unsigned long long *qe_out)
{
    // eight items per lane whatever the CTA size: with 512-thread CTAs a warp's
    // output holds half a slice, and warp_discover appends the winners in halves
    constexpr int PER = 8;
    constexpr int NW = B / 32;
    constexpr int S = 32 * PER;           // items per slice
    constexpr int CAP = kChunkMax / NW;   // entries of a warp's output
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t *bv = s.out + warp * CAP;
    int32_t *bc = s.colstart + warp * CAP;
    int32_t *bd = s.rel + warp * CAP;
    const int re = s.q;
    int count = 0;  // warp-uniform
    bool any = false;
    const long long stride = (long long)gridDim.x * NW * S;
    for (long long b64 = (long long)warp_slice0(warp) * S; b64 < re; b64 += stride) {
        const int base = (int)b64;
        int v[PER], u[PER];
        bool go[PER];
#pragma unroll
        for (int t = 0; t < PER; t++) {
            const int i = base + t * 32 + lane;
            go[t] = i < re;
            v[t] = go[t] ? ld_cg(in.v + i) : -1;
            u[t] = (PRED && go[t]) ? ld_cg(in.pred + i) : -1;
        }
        any |= warp_discover<PER, PRED, false, CAP>(p, s.mask, v, u, go, level, bv, bc, bd, count, vout, qe_out);
    }
    if (count) warp_emit(p, bv, bc, bd, count, vout, qe_out);
    if (__any_sync(0xffffffffu, any) && lane == 0) s.flag = 1;  // benign race: every writer stores 1
}

// One warp's tables for the slice [x0, x0 + len) of a vertex frontier's
// flattened edge space (x0 a chunk start): the entries overlapping the slice,
// loaded 32 per round trip starting from the chunk index's owner of x0, each
// marking its first slice position in `own` (cleared first), which a warp
// max-scan then fills: position r belongs to the largest mark at or before r
// (the entries start in increasing order).  tcol[k] + r is the column index
// of slice position r in entry k's list; tver[k] is entry k's vertex.  All
// 32 lanes call it, after every lane has finished reading the tables.
template <bool PRED>
__device__ __forceinline__ void warp_slice_map(const VertexFrontier &in, int q, int x0, int len, uint16_t *own,
                                               int32_t *tcol, int32_t *tver)
{
    const int lane = threadIdx.x & 31;
    reinterpret_cast<uint4 *>(own)[lane] = make_uint4(0u, 0u, 0u, 0u);
    __syncwarp();
    const int i0 = ld_cg(in.cf + x0 / kChunkGrain);  // owns position x0 (a chunk start)
    int n = 0;
    for (int i = i0;; i += 32) {
        const int j = i + lane;
        int Pj = INT_MAX;
        int cj = 0, vj = -1;
        if (j < q) {
            Pj = ld_cg(in.P + j);
            cj = ld_cg(in.col + j);
            if (PRED) vj = ld_cg(in.v + j);
        }
        const bool inside = Pj < x0 + len;  // the inside lanes form a prefix (P increases)
        const unsigned in_mask = __ballot_sync(0xffffffffu, inside);
        const int k = n + lane;
        if (inside && k < kWarpSlice) {
            const int start = max(Pj, x0) - x0;
            own[start] = (uint16_t)k;
            tcol[k] = cj + (max(Pj, x0) - Pj) - start;  // + slice position = column index
            if (PRED) tver[k] = vj;
        }
        n += __popc(in_mask);
        if (in_mask != 0xffffffffu || i + 32 >= q) break;
    }
    __syncwarp();
    static_assert(kWarpSlice == 256, "a lane's share of the map is one 16-byte word");
    uint4 w = reinterpret_cast<uint4 *>(own)[lane];
    unsigned e[8] = {w.x & 0xffffu, w.x >> 16, w.y & 0xffffu, w.y >> 16, w.z & 0xffffu, w.z >> 16, w.w & 0xffffu, w.w >> 16};
#pragma unroll
    for (int t = 1; t < 8; t++) e[t] = max(e[t], e[t - 1]);
    unsigned incl = e[7];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl = max(incl, y);
    }
    unsigned before = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) before = 0;
#pragma unroll
    for (int t = 0; t < 8; t++) e[t] = max(e[t], before);
    w.x = e[0] | (e[1] << 16);
    w.y = e[2] | (e[3] << 16);
    w.z = e[4] | (e[5] << 16);
    w.w = e[6] | (e[7] << 16);
    reinterpret_cast<uint4 *>(own)[lane] = w;
    __syncwarp();
}

// Lane positions (h * PB + t) * 32 + lane, t < PB, of a slice of `len`
// positions: the gathered neighbour (a coalesced read along a run) and its
// predecessor, from the warp's tables.
template <int PB, bool PRED>
__device__ __forceinline__ void warp_slice_gather(const BfsParams &p, int h, int len, const uint16_t *own,
                                                  const int32_t *tcol, const int32_t *tver, int (&v)[PB],
                                                  int (&u)[PB], bool (&go)[PB])
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int t = 0; t < PB; t++) {
        const int r = (h * PB + t) * 32 + lane;
        go[t] = r < len;
        v[t] = -1;
        u[t] = -1;
        if (go[t]) {
            const int k = own[r];
            v[t] = ld_stream(p.column_indices + tcol[k] + r);
            if (PRED) u[t] = tver[k];
        }
    }
}

// Warp-autonomous top-down level (policy.warp_contract; levels with a full
// sub-round per CTA): each warp takes its kWarpSlice-position slices
// (warp_slice0) of the frontier's flattened edge space, builds its tables
// for a slice (warp_slice_map), gathers kWarpSlice / 32 positions per lane
// (a warp reads 32 consecutive positions of a run, one coalesced segment)
// and runs the visited test (warp_discover) with no CTA barrier (batch sizes
// below).  (Building the next slice's tables and issuing its loads before
// testing the current slice measured slower: 908 -> 968 us per R-MAT 22
// search; the second slice's registers spill.)  Same labels and frontier
// contents as expand_range (the reference's expand-contract,
// expand_contract_atomic/cta.cuh:82-789); the entries' order differs.
// `skip_above` as in emit_frontier (direction-optimizing searches).
// With CULL = false (the expand pass of the edge-frontier strategies) the
// gathered neighbours (and their predecessors) are written to the edge
// frontier `eout` at their flattened positions instead: the reference's
// two-phase expansion (two_phase/expand_atomic/cta.cuh:215-423).
// Predecessor searches with CTAs of more than 256 threads keep the CTA-wide
// sub-rounds (the entries' vertices would need a third table).
template <int B, bool PRED, bool CULL = true, bool WHOLE = false>
__device__ __forceinline__ void expand_range_warp(const BfsParams &p, const VertexFrontier &in,
                                                  ExpandSmem<B, PRED> &s, int level, const VertexFrontier &vout,
                                                  unsigned long long *qe_out, const EdgeFrontier *eout = nullptr,
                                                  unsigned long long skip_above = ~0ull)
{
    static_assert(B <= 256 || !PRED, "predecessor tables exist for CTAs of up to 256 threads only");
    constexpr int NW = B / 32;
    constexpr int PW = kWarpSlice / 32;    // positions per lane per slice
    constexpr int CAP = kChunkMax / NW;    // a warp's output entries
    // positions per lane per batch: with CTAs of more than 256 threads a warp's
    // output holds half a slice, so the slice goes in two halves, except with
    // WHOLE (top-down-only searches), which test the whole slice at once and
    // append its winners in halves: expand-contract 888 -> 852 us per R-MAT 22
    // search, while direction-optimizing searches and the edge strategies'
    // copy pass measured 1-4% slower that way
    constexpr int PB = (CULL && WHOLE) || CAP / 32 >= PW ? PW : CAP / 32;
    static_assert(PW % PB == 0, "a slice splits into whole batches");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t *bv = s.out + warp * CAP;
    int32_t *bc = s.colstart + warp * CAP;
    int32_t *bd = s.rel + warp * CAP;
    uint16_t *own = s.wmap + warp * kWarpSlice;  // slice position -> table entry
    int32_t *tcol = s.wcol + warp * kWarpSlice;  // table entry -> column index of slice position 0
    int32_t *tver = PRED ? s.vert + warp * kWarpSlice : nullptr;
    const int q = s.q, re = s.E;
    int count = 0;  // warp-uniform
    bool any = false;
    const long long stride = (long long)gridDim.x * NW * kWarpSlice;
    for (long long x64 = (long long)warp_slice0(warp) * kWarpSlice; x64 < re; x64 += stride) {
        const int x0 = (int)x64;
        const int len = min(kWarpSlice, re - x0);
        warp_slice_map<PRED>(in, q, x0, len, own, tcol, tver);
#pragma unroll
        for (int h = 0; h < PW / PB; h++) {
            int v[PB], u[PB];
            bool go[PB];
            warp_slice_gather<PB, PRED>(p, h, len, own, tcol, tver, v, u, go);
            if constexpr (CULL) {
                any |= warp_discover<PB, PRED, true, CAP>(p, s.mask, v, u, go, level + 1, bv, bc, bd, count,
                                                     vout, qe_out, skip_above);
            } else {
#pragma unroll
                for (int t = 0; t < PB; t++) {
                    if (go[t]) {
                        const int r = (h * PB + t) * 32 + lane;
                        eout->v[x0 + r] = v[t];
                        if (PRED) eout->pred[x0 + r] = u[t];
                    }
                }
            }
        }
        __syncwarp();  // the slice's tables are free for the next slice
    }
    if constexpr (CULL) {
        if (count) warp_emit(p, bv, bc, bd, count, vout, qe_out, skip_above);
        if (__any_sync(0xffffffffu, any) && lane == 0) s.flag = 1;  // benign race: every writer stores 1
    }
}

// ------------------------------------------------------------------------------------
// Bottom-up step (direction-optimizing levels, undirected graphs only)
// ------------------------------------------------------------------------------------

// Level `level` run bottom-up over the CTA's share of vertex ids: every
// unvisited vertex with edges looks for a neighbour whose visited bit is set
// in the snapshot taken at the start of the level; on an undirected graph
// such a neighbour is exactly one level up, so the vertex is labelled
// level + 1 (or that neighbour, the first one in CSR order).  The visited set
// is read from the pass's mask buffer (s.mask, unchanged during the level)
// and written, old bits | discoveries, to every word of the other buffer,
// which the next pass reads; discoveries also go, through emit_frontier, into
// the next vertex frontier.
// A warp handles blocks of 32 consecutive vertices (one visited-mask word);
// each thread first issues, for all of its PER vertices at once, the
// vertices' own visited words, their rows and their first kBottomUpProbe
// neighbours' visited bits; vertices still without a parent then scan on
// (short lists one lane each, four neighbours at a time; long lists by the
// whole warp, 32 neighbours at a time).
constexpr int kBottomUpProbe = 2;

// Visited-before-this-level tests of a batch of neighbours: the level-start
// mask snapshot (bit test), or in list mode the distance labels (a label in
// [0, level] was written before this level; this level writes level + 1).
template <bool LABELS>
__device__ __forceinline__ unsigned probe_load(const uint32_t *mask, const int32_t *labels, int u)
{
    return LABELS ? (unsigned)ld_cg(labels + u) : ld_mask(mask + (u >> 5));
}
template <bool LABELS>
__device__ __forceinline__ bool probe_hit(unsigned x, int u, int level)
{
    return LABELS ? ((int)x >= 0 && (int)x <= level) : (((x >> (u & 31)) & 1u) != 0);
}

// Bottom-up continuation, one lane per vertex (list-mode levels; range levels
// use bottom_up_queue): each lane scans its own list
// on (K neighbours already probed at its start; lists of at most MIN_LEN are
// finished), four neighbours at a time; lists longer than p.bu_long
// are searched by the whole warp, 32 neighbours at a time.
template <int PER, int K, int MIN_LEN, bool LABELS>
__device__ __forceinline__ void bottom_up_lanes(const BfsParams &p, const uint32_t *mask, int level,
                                                const bool (&todo)[PER], const int (&r0)[PER], const int (&r1)[PER],
                                                int (&parent)[PER])
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int t = 0; t < PER; t++) {
        const bool more = todo[t] && parent[t] < 0 && r1[t] - r0[t] > MIN_LEN;
        if (!__any_sync(0xffffffffu, more)) continue;
        const bool longlist = more && (r1[t] - r0[t]) > p.bu_long;
        bool scan = more && !longlist;
        int e = r0[t] + K;
        while (__any_sync(0xffffffffu, scan)) {
            if (scan) {
                int nb[4];
                unsigned w[4];
#pragma unroll
                for (int k = 0; k < 4; k++) nb[k] = (e + k < r1[t]) ? ld_stream(p.column_indices + e + k) : -1;
#pragma unroll
                for (int k = 0; k < 4; k++) w[k] = nb[k] >= 0 ? probe_load<LABELS>(mask, p.labels, nb[k]) : 0u;
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (parent[t] < 0 && nb[k] >= 0 && probe_hit<LABELS>(w[k], nb[k], level)) parent[t] = nb[k];
                e += 4;
                if (parent[t] >= 0 || e >= r1[t]) scan = false;
            }
        }
        unsigned lmask = __ballot_sync(0xffffffffu, longlist);
        while (lmask) {
            const int owner = __ffs(lmask) - 1;
            lmask &= lmask - 1;
            const int lr0 = __shfl_sync(0xffffffffu, r0[t], owner) + K;
            const int lr1 = __shfl_sync(0xffffffffu, r1[t], owner);
            int found_u = -1;
            for (int eb = lr0; eb < lr1; eb += 32) {
                const int ee = eb + lane;
                const int nb = ee < lr1 ? ld_stream(p.column_indices + ee) : -1;
                const bool hit = nb >= 0 && probe_hit<LABELS>(probe_load<LABELS>(mask, p.labels, nb), nb, level);
                const unsigned hb = __ballot_sync(0xffffffffu, hit);
                if (hb) {
                    found_u = __shfl_sync(0xffffffffu, nb, __ffs(hb) - 1);
                    break;
                }
            }
            if (lane == owner) parent[t] = found_u;
        }
    }
}

// Bottom-up continuation with the warp's pending lists in a queue: the lists
// (slot t, lane) still without a parent after the first probes, of length in
// (MIN_LEN, p.bu_long], are listed in the warp's region of q_lo / q_hi
// (next position, end; 32 * PER entries per warp) and handed out to lanes as
// they become free, so a warp keeps 32 scans in flight until its queue is
// empty instead of waiting for the longest list of each slot in turn; each
// step reads four neighbours and their visited words.  The parent found for
// entry i lands in q_par[i] and goes back to its slot.  Longer lists are then
// searched by the whole warp, 32 neighbours at a time.  The queue arrays are
// shared memory the caller does not use until after a CTA barrier.
template <int PER, int K, int MIN_LEN>
__device__ __forceinline__ void bottom_up_queue(const BfsParams &p, const uint32_t *mask, const bool (&todo)[PER],
                                                const int (&r0)[PER], const int (&r1)[PER], int (&parent)[PER],
                                                int32_t *q_lo, int32_t *q_hi, int32_t *q_par)
{
    const int lane = threadIdx.x & 31;
    const int wbase = (threadIdx.x >> 5) * 32 * PER;
    q_lo += wbase;
    q_hi += wbase;
    q_par += wbase;
    int n = 0;
#pragma unroll
    for (int t = 0; t < PER; t++) {
        const int len = r1[t] - r0[t];
        const bool pend = todo[t] && parent[t] < 0 && len > MIN_LEN && len <= p.bu_long;
        const unsigned bal = __ballot_sync(0xffffffffu, pend);
        if (pend) {
            const int i = n + __popc(bal & lanemask_lt());
            q_lo[i] = r0[t] + K;
            q_hi[i] = r1[t];
            q_par[i] = -1;
        }
        n += __popc(bal);
    }
    __syncwarp();
    int cur = -1, e = 0, hi = 0, handed = 0;
    for (;;) {
        const bool idle = cur < 0;
        const unsigned ib = __ballot_sync(0xffffffffu, idle);
        if (idle) {
            const int i = handed + __popc(ib & lanemask_lt());
            if (i < n) {
                cur = i;
                e = q_lo[i];
                hi = q_hi[i];
            }
        }
        handed += __popc(ib);
        if (!__any_sync(0xffffffffu, cur >= 0)) break;
        if (cur >= 0) {
            int nb[4];
            unsigned w[4];
            e = ld_quad(p.column_indices, p.edges, e, hi, nb);  // one 16-byte load per step
#pragma unroll
            for (int k = 0; k < 4; k++) w[k] = nb[k] >= 0 ? ld_mask(mask + (nb[k] >> 5)) : 0u;
            int found = -1;
#pragma unroll
            for (int k = 3; k >= 0; k--)
                if (nb[k] >= 0 && ((w[k] >> (nb[k] & 31)) & 1u)) found = nb[k];
            if (found >= 0) q_par[cur] = found;
            if (found >= 0 || e >= hi) cur = -1;
        }
    }
    __syncwarp();
    n = 0;
#pragma unroll
    for (int t = 0; t < PER; t++) {
        const int len = r1[t] - r0[t];
        const bool pend = todo[t] && parent[t] < 0 && len > MIN_LEN && len <= p.bu_long;
        const unsigned bal = __ballot_sync(0xffffffffu, pend);
        if (pend) parent[t] = q_par[n + __popc(bal & lanemask_lt())];
        n += __popc(bal);
    }
    // long lists: the whole warp, one list at a time
#pragma unroll
    for (int t = 0; t < PER; t++) {
        const bool longlist = todo[t] && parent[t] < 0 && r1[t] - r0[t] > p.bu_long;
        unsigned lmask = __ballot_sync(0xffffffffu, longlist);
        while (lmask) {
            const int owner = __ffs(lmask) - 1;
            lmask &= lmask - 1;
            const int lr0 = __shfl_sync(0xffffffffu, r0[t], owner) + K;
            const int lr1 = __shfl_sync(0xffffffffu, r1[t], owner);
            int found_u = -1;
            for (int eb = lr0; eb < lr1; eb += 32) {
                const int ee = eb + lane;
                const int nb = ee < lr1 ? ld_stream(p.column_indices + ee) : -1;
                const bool hit = nb >= 0 && ((ld_mask(mask + (nb >> 5)) >> (nb & 31)) & 1u);
                const unsigned hb = __ballot_sync(0xffffffffu, hit);
                if (hb) {
                    found_u = __shfl_sync(0xffffffffu, nb, __ffs(hb) - 1);
                    break;
                }
            }
            if (lane == owner) parent[t] = found_u;
        }
    }
}

// Still-unvisited vertices of a bottom-up chunk, collected in s.stage (free
// during bottom-up levels) and then appended to the next unvisited list with
// one atomic per chunk.  Called by whole warps.
template <typename Smem>
__device__ __forceinline__ void append_unvisited(Smem &s, bool keep, int v)
{
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    if (bal == 0) return;
    const int lane = threadIdx.x & 31, leader = __ffs(bal) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&s.wl_count, __popc(bal));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (keep) s.stage[base + __popc(bal & lanemask_lt())] = v;
}

template <int B, typename Smem>
__device__ __forceinline__ void write_unvisited(const BfsParams &p, Smem &s, int32_t *list, unsigned *ctr)
{
    __syncthreads();
    const int n = s.wl_count;
    if (n == 0) return;  // CTA-uniform
    if (threadIdx.x == 0) s.ul_base = (int)atomicAdd(ctr, (unsigned)n);
    __syncthreads();
    const int base = s.ul_base;
    for (int j = threadIdx.x; j < n; j += B)
        if (base + j < p.nodes) list[base + j] = s.stage[j];
}

// Thread 0: stages chunk [cs, cs + kChunkMax) of [.., re) into the prefetch
// buffer (the buffer's previous contents must be consumed, and a CTA barrier
// passed, before the call).  Every source is 16-byte aligned (cudaMalloc'd
// arrays, cs a multiple of 32); sizes are rounded down to whole 16 bytes.
__device__ __forceinline__ void bu_prefetch_issue(const BfsParams &p, BuPrefetch &f, const uint32_t *mask, int cs,
                                                  int re)
{
    const int nv = min(kChunkMax, re - cs);
    const int nr = (nv + 1) & ~3;                                  // of the nv + 1 row offsets
    const int nh = p.hub2 ? (nv & ~1) : 0;                         // hub pairs (8 bytes each)
    const int nw = (((nv + 31) >> 5) & ~3);                        // visited words
    f.nr = nr;
    f.nh = nh;
    f.nw = nw;
    const unsigned bytes = 4u * nr + 8u * nh + 4u * nw;
    if (bytes == 0) return;  // the consumer sees nothing staged and waits for nothing
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&f.bar, bytes);
    if (nr) bulk_g2s(f.rows, p.row_offsets + cs, 4u * nr, &f.bar);
    if (nh) bulk_g2s(f.hub, p.hub2 + cs, 8u * nh, &f.bar);
    if (nw) bulk_g2s(f.words, mask + (cs >> 5), 4u * nw, &f.bar);
}

//
// With `defer` (CTA-uniform) the discoveries are only counted: each thread
// sums (1 << 32 | degree) over its discoveries and the CTA adds its total to
// *qe_out once; materialize_frontier builds the vertex frontier from the two
// mask buffers if a top-down level follows.
template <int B, bool PRED, bool LISTS>
__device__ __forceinline__ void bottom_up_range(const BfsParams &p, ExpandSmem<B, PRED> &s, int level, int pass,
                                                const VertexFrontier &vout, unsigned long long *qe_out, bool defer)
{
    const int tid = threadIdx.x, lane = tid & 31;
    constexpr int PER = kChunkMax / B;
    constexpr int K = kBottomUpProbe;
    const uint32_t *mask = s.mask;
    uint32_t *mask_out = (s.mask == p.mask) ? p.mask_alt : p.mask;
    int rs, re;
    cta_range(p.nodes, blockIdx.x, gridDim.x, rs, re);
    unsigned long long found_acc = 0;  // defer: this thread's (count << 32 | degree) of discoveries
    BuPrefetch *pf = s.pf;             // CTA-uniform
    if (pf && tid == 0 && rs < re) bu_prefetch_issue(p, *pf, mask, rs, re);
    for (int cs = rs; cs < re; cs += kChunkMax) {
        const bool first = cs == rs;
        if (tid == 0) {
            s.out_count = 0;
            s.wl_count = 0;
        }
        __syncthreads();  // the counters are reset before any warp appends
        if (first) stamp(p, pass, 0);
        bool staged = false;
        const unsigned ph = s.pf_phase;  // (thread 0 flips it below, after every thread has read it)
        if (pf) {
            // this chunk's words, rows and hub pairs, staged during the last chunk
            staged = true;
            if (pf->nr + pf->nh + pf->nw > 0) {
                unsigned spins = 0;
                while (!mbar_try_wait(&pf->bar, ph)) {
                    if (++spins > p.spin_limit) {
                        staged = false;
                        break;
                    }
                }
            }
            if (!__syncthreads_and(staged)) {
                // the copy did not land in time: report it, one more bounded wait for
                // the copy in flight, and leave the level (every caller reads the error word)
                if (tid == 0) {
                    atomicOr(&p.st->error, kErrBulk);
                    unsigned spins = 0;
                    while (!mbar_try_wait(&pf->bar, ph) && ++spins <= p.spin_limit) __nanosleep(256);
                }
                __syncthreads();
                return;
            }
        }
        const int pnr = pf ? pf->nr : 0, pnh = pf ? pf->nh : 0, pnw = pf ? pf->nw : 0;
        // ---- own visited words (the snapshot is read coherently: ld.cg) ----------
        unsigned word[PER];
#pragma unroll
        for (int t = 0; t < PER; t++) {
            const int vb = cs + t * B + (tid & ~31);
            const int wi = (vb - cs) >> 5;
            word[t] = vb < re ? (wi < pnw ? pf->words[wi] : ld_cg(mask + (vb >> 5))) : 0xffffffffu;
        }
        int r0[PER], r1[PER];
        bool todo[PER];
        int2 hubv[PER];
#pragma unroll
        for (int t = 0; t < PER; t++) {
            const int v = cs + t * B + tid, j = v - cs;
            todo[t] = v < re && !((word[t] >> lane) & 1u);
            r0[t] = r1[t] = 0;
            hubv[t] = make_int2(-1, -1);
            if (todo[t]) {
                r0[t] = j < pnr ? pf->rows[j] : ld_ro(p.row_offsets + v);
                r1[t] = j + 1 < pnr ? pf->rows[j + 1] : ld_ro(p.row_offsets + v + 1);
                if (pf && p.hub2) hubv[t] = j < pnh ? pf->hub[j] : p.hub2[v];
            }
        }
        if (pf) {
            // the buffer is consumed: stage the next chunk while this one is scanned
            __syncthreads();
            if (tid == 0) {
                if (pnr + pnh + pnw > 0) s.pf_phase = ph ^ 1u;
                if (cs + kChunkMax < re) bu_prefetch_issue(p, *pf, mask, cs + kChunkMax, re);
            }
        }
        stamp_synced(p, pass, 1, first);
        // ---- first K neighbours of every candidate -----------------------------------
        int parent[PER];
        {
            int nb[PER][K];
            static_assert(K == 2, "the hub pair supplies two probes");
#pragma unroll
            for (int t = 0; t < PER; t++) {
                todo[t] = todo[t] && r1[t] > r0[t];
                if (p.hub2) {
                    // the vertex's two highest-degree neighbours (one coalesced 8-byte load,
                    // or staged with the chunk)
                    int2 h = hubv[t];
                    if (!pf && todo[t]) h = p.hub2[cs + t * B + tid];
                    if (!todo[t]) h = make_int2(-1, -1);
                    nb[t][0] = h.x;
                    nb[t][1] = h.y;
                } else {
#pragma unroll
                    for (int k = 0; k < K; k++)
                        nb[t][k] = (todo[t] && r0[t] + k < r1[t]) ? ld_stream(p.column_indices + r0[t] + k) : -1;
                }
            }
            unsigned w[PER][K];
#pragma unroll
            for (int t = 0; t < PER; t++)
#pragma unroll
                for (int k = 0; k < K; k++) w[t][k] = nb[t][k] >= 0 ? ld_mask(mask + (nb[t][k] >> 5)) : 0u;
#pragma unroll
            for (int t = 0; t < PER; t++) {
                parent[t] = -1;
#pragma unroll
                for (int k = K - 1; k >= 0; k--)
                    if (nb[t][k] >= 0 && ((w[t][k] >> (nb[t][k] & 31)) & 1u)) parent[t] = nb[t][k];
            }
        }
        stamp_synced(p, pass, 2, first);
        // ---- continue the scan for candidates still without a parent ---------------
        if (LISTS) {
            if (p.hub2)  // the pair came from anywhere in the list: longer lists are scanned from the start
                bottom_up_lanes<PER, 0, K, false>(p, mask, level, todo, r0, r1, parent);
            else
                bottom_up_lanes<PER, K, K, false>(p, mask, level, todo, r0, r1, parent);
        } else {
            // (s.colstart / s.rel / s.out are free until the discoveries are appended)
            if (p.hub2)
                bottom_up_queue<PER, 0, K>(p, mask, todo, r0, r1, parent, s.colstart, s.rel, s.out);
            else
                bottom_up_queue<PER, K, K>(p, mask, todo, r0, r1, parent, s.colstart, s.rel, s.out);
            if (!defer) __syncthreads();  // every warp's queue is done before the appends
        }
        stamp_synced(p, pass, 3, first);
        // ---- label, mark and append the discoveries --------------------------------
#pragma unroll
        for (int t = 0; t < PER; t++) {
            const int vb = cs + t * B + (tid & ~31);
            if (vb >= re) continue;  // warp-uniform
            const int v = vb + lane;
            const bool found = parent[t] >= 0;
            const unsigned fb = __ballot_sync(0xffffffffu, found);
            if (lane == 0) mask_out[vb >> 5] = word[t] | fb;  // this warp owns the whole word
            if (LISTS && p.ul[0]) append_unvisited(s, todo[t] && !found, v);
            if (fb == 0) continue;
            if (found) {
                p.labels[v] = PRED ? parent[t] : level + 1;
                s.flag = 1;
            }
            if (defer) {
                if (found) found_acc += pack(1u, (unsigned)(r1[t] - r0[t]));
                continue;
            }
            const int leader = __ffs(fb) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&s.out_count, __popc(fb));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (found) {
                const int slot = base + __popc(fb & lanemask_lt());
                s.out[slot] = v;
                s.colstart[slot] = r0[t];
                s.rel[slot] = r1[t] - r0[t];
            }
        }
        if (defer) {
            if (first) stamp(p, pass, 4);
            continue;
        }
        __syncthreads();
        if (first) stamp(p, pass, 4);
        emit_frontier<B>(p, s, pass, vout, qe_out);
        if (LISTS && p.ul[0]) write_unvisited<B>(p, s, p.ul[0], &p.st->ul_count[(pass + 1) % 3]);
        __syncthreads();
        if (first) stamp(p, pass, 5);
    }
    if (defer) {
        unsigned long long tot;
        cta_exclusive_scan<B>(found_acc, s.scan_warp, &tot);
        if (tid == 0 && tot != 0) atomicAdd(qe_out, tot);
    }
}

// The first bottom-up level of a run, when it only counts its discoveries
// (fused searches, not list mode), warp by warp (policy.warp_bottom_up): each
// warp takes blocks of 32 * PER vertex ids dealt over every warp of the grid
// (warp_slice0) and handles them with no CTA barrier -- the blocks' visited
// words, rows and hub pairs in one round trip (rows and pairs of visited
// vertices too: at a first bottom-up level nearly every vertex is
// unvisited), the hub probes, the per-warp queue of lists still to scan
// (bottom_up_queue), then the block's words of the other mask buffer, the
// labels and the count of discoveries and their edges.  The CTA adds its
// count to the pass counter once, at the end.  Same labels and visited words
// as bottom_up_range.  (Later bottom-up levels, where most vertices are
// visited, keep the compacted windows: warp by warp they measured slower.)
template <int B, bool PRED>
__device__ __forceinline__ void bottom_up_range_warp(const BfsParams &p, ExpandSmem<B, PRED> &s, int level,
                                                     unsigned long long *qe_out)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int PER = kChunkMax / B;
    constexpr int NW = B / 32;
    constexpr int K = kBottomUpProbe;
    static_assert(K == 2, "the hub pair supplies two probes");
    constexpr int S = 32 * PER;  // vertices per warp block
    const uint32_t *mask = s.mask;
    uint32_t *mask_out = (s.mask == p.mask) ? p.mask_alt : p.mask;
    const int n = p.nodes;
    unsigned long long found_acc = 0;  // (count << 32 | degree) of this lane's discoveries
    bool any = false;
    const long long stride = (long long)gridDim.x * NW * S;
    for (long long c64 = (long long)warp_slice0(warp) * S; c64 < n; c64 += stride) {
        const int cs = (int)c64;
        unsigned word[PER];
        int r0[PER], r1[PER];
        int2 hubv[PER];
#pragma unroll
        for (int t = 0; t < PER; t++) {
            const int vb = cs + t * 32, v = vb + lane;
            word[t] = vb < n ? ld_cg(mask + (vb >> 5)) : 0xffffffffu;
            r0[t] = r1[t] = 0;
            hubv[t] = make_int2(-1, -1);
            if (v < n) {
                r0[t] = ld_ro(p.row_offsets + v);
                r1[t] = ld_ro(p.row_offsets + v + 1);
                if (p.hub2) hubv[t] = p.hub2[v];
            }
        }
        bool todo[PER];
        int parent[PER];
        {
            int nb[PER][K];
#pragma unroll
            for (int t = 0; t < PER; t++) {
                const int v = cs + t * 32 + lane;
                todo[t] = v < n && !((word[t] >> lane) & 1u) && r1[t] > r0[t];
                if (p.hub2) {
                    nb[t][0] = todo[t] ? hubv[t].x : -1;
                    nb[t][1] = todo[t] ? hubv[t].y : -1;
                } else {
#pragma unroll
                    for (int k = 0; k < K; k++)
                        nb[t][k] = (todo[t] && r0[t] + k < r1[t]) ? ld_stream(p.column_indices + r0[t] + k) : -1;
                }
            }
            unsigned w[PER][K];
#pragma unroll
            for (int t = 0; t < PER; t++)
#pragma unroll
                for (int k = 0; k < K; k++) w[t][k] = nb[t][k] >= 0 ? ld_mask(mask + (nb[t][k] >> 5)) : 0u;
#pragma unroll
            for (int t = 0; t < PER; t++) {
                parent[t] = -1;
#pragma unroll
                for (int k = K - 1; k >= 0; k--)
                    if (nb[t][k] >= 0 && ((w[t][k] >> (nb[t][k] & 31)) & 1u)) parent[t] = nb[t][k];
            }
        }
        // (s.colstart / s.rel / s.out: each warp's own part is its queue)
        if (p.hub2)
            bottom_up_queue<PER, 0, K>(p, mask, todo, r0, r1, parent, s.colstart, s.rel, s.out);
        else
            bottom_up_queue<PER, K, K>(p, mask, todo, r0, r1, parent, s.colstart, s.rel, s.out);
#pragma unroll
        for (int t = 0; t < PER; t++) {
            const int vb = cs + t * 32;
            if (vb >= n) continue;  // warp-uniform
            const int v = vb + lane;
            const bool found = parent[t] >= 0;
            const unsigned fb = __ballot_sync(0xffffffffu, found);
            if (lane == 0) mask_out[vb >> 5] = word[t] | fb;  // this warp owns the whole word
            if (found) {
                p.labels[v] = PRED ? parent[t] : level + 1;
                found_acc += pack(1u, (unsigned)(r1[t] - r0[t]));
                any = true;
            }
        }
    }
    if (__any_sync(0xffffffffu, any) && lane == 0) s.flag = 1;  // benign race: every writer stores 1
    unsigned long long tot;
    cta_exclusive_scan<B>(found_acc, s.scan_warp, &tot);
    if (tid == 0 && tot != 0) atomicAdd(qe_out, tot);
}

// Writes the vertex ids of the set bits of `bits` (the word of vertices
// v0..v0+31) whose positions, counted from `pos` in bit order, fall in
// [lo, lo + n), to list[position - lo].
__device__ __forceinline__ void scatter_bits(unsigned bits, int v0, int pos, int lo, int n, int32_t *list)
{
    const int c = __popc(bits);
    int k = min(c, max(0, lo - pos));
    const int k1 = min(c, lo + n - pos);
    if (k >= k1) return;
    for (int i = 0; i < k; i++) bits &= bits - 1;
    for (; k < k1; k++) {
        list[pos + k - lo] = v0 + __ffs(bits) - 1;
        bits &= bits - 1;
    }
}

// Level `level` bottom-up over the CTA's range of vertex ids, in windows of
// 32 * B ids (one visited word per thread).  The window's unvisited vertices
// (clear bits of the level-start snapshot) are numbered by a CTA scan and
// handled in batches of up to kChunkMax from a shared-memory list, so only
// unvisited vertices take lanes and a mostly visited window costs one batch.
// A batch: rows and hub pairs (independent loads, issued together), the
// pair's probes, the queued per-lane (per-warp for long lists) scan of the rest,
// then labels; a discovery sets its bit in the window's shared copy of the
// words (s.win_word), written whole to the other mask buffer when the window
// ends.  With `defer` (CTA-uniform) discoveries are only counted (one packed
// atomic per CTA; materialize_frontier builds the frontier when a top-down
// level follows), else each batch's discoveries are emitted.
template <int B, bool PRED>
__device__ __forceinline__ void bottom_up_windows(const BfsParams &p, ExpandSmem<B, PRED> &s, int level, int pass,
                                                  const VertexFrontier &vout, unsigned long long *qe_out, bool defer)
{
    const int tid = threadIdx.x, lane = tid & 31;
    constexpr int PER = kChunkMax / B;
    constexpr int K = kBottomUpProbe;
    static_assert(K == 2, "the hub pair supplies two probes");
    const uint32_t *mask = s.mask;
    uint32_t *mask_out = (s.mask == p.mask) ? p.mask_alt : p.mask;
    int rs, re;
    cta_range(p.nodes, blockIdx.x, gridDim.x, rs, re);  // rs is a multiple of kChunkGrain (so of 32)
    unsigned long long found_acc = 0;  // defer: this thread's (count << 32 | degree) of discoveries
    bool first = true;
    for (int wb = rs; wb < re; wb += 32 * B) {
        const int v0 = wb + 32 * tid;  // first vertex of this thread's word
        unsigned w = 0xffffffffu;
        if (v0 < re) w = ld_cg(mask + (v0 >> 5));
        unsigned unv = v0 < re ? ~w : 0u;
        if (v0 < re && re - v0 < 32) unv &= (1u << (re - v0)) - 1u;
        s.win_word[tid] = w;
        unsigned long long total;
        const int pos = (int)cta_exclusive_scan<B>((unsigned long long)__popc(unv), s.scan_warp, &total);
        const int U = (int)total;  // the scan's closing barrier also publishes win_word
        for (int lo = 0; lo < U; lo += kChunkMax) {
            const int n = min(U - lo, kChunkMax);
            if (tid == 0) s.out_count = 0;
            scatter_bits(unv, v0, pos, lo, n, s.stage);
            __syncthreads();
            if (first) stamp(p, pass, 0);
            int r0[PER], r1[PER], parent[PER];
            bool todo[PER];
            int nb[PER][K];
#pragma unroll
            for (int t = 0; t < PER; t++) {
                const int j = t * B + tid;
                todo[t] = j < n;
                r0[t] = r1[t] = 0;
                nb[t][0] = nb[t][1] = -1;
                if (todo[t]) {
                    const int v = s.stage[j];  // read again at the end (not kept in registers)
                    r0[t] = ld_ro(p.row_offsets + v);
                    r1[t] = ld_ro(p.row_offsets + v + 1);
                    if (p.hub2) {
                        // the vertex's two highest-degree neighbours (one 8-byte load)
                        const int2 h = p.hub2[v];
                        nb[t][0] = h.x;
                        nb[t][1] = h.y;
                    }
                }
            }
            stamp_synced(p, pass, 1, first);
#pragma unroll
            for (int t = 0; t < PER; t++) {
                todo[t] = todo[t] && r1[t] > r0[t];
                if (!p.hub2) {
#pragma unroll
                    for (int k = 0; k < K; k++)
                        nb[t][k] = (todo[t] && r0[t] + k < r1[t]) ? ld_stream(p.column_indices + r0[t] + k) : -1;
                } else if (!todo[t]) {
                    nb[t][0] = nb[t][1] = -1;
                }
            }
            {
                unsigned pw[PER][K];
#pragma unroll
                for (int t = 0; t < PER; t++)
#pragma unroll
                    for (int k = 0; k < K; k++) pw[t][k] = nb[t][k] >= 0 ? ld_mask(mask + (nb[t][k] >> 5)) : 0u;
#pragma unroll
                for (int t = 0; t < PER; t++) {
                    parent[t] = -1;
#pragma unroll
                    for (int k = K - 1; k >= 0; k--)
                        if (nb[t][k] >= 0 && ((pw[t][k] >> (nb[t][k] & 31)) & 1u)) parent[t] = nb[t][k];
                }
            }
            stamp_synced(p, pass, 2, first);
            // the pair came from anywhere in the list: longer lists are scanned from the
            // start (s.colstart / s.rel / s.out are free until the discoveries are appended)
            if (p.hub2)
                bottom_up_queue<PER, 0, K>(p, mask, todo, r0, r1, parent, s.colstart, s.rel, s.out);
            else
                bottom_up_queue<PER, K, K>(p, mask, todo, r0, r1, parent, s.colstart, s.rel, s.out);
            if (!defer) __syncthreads();  // every warp's queue is done before the appends
            stamp_synced(p, pass, 3, first);
#pragma unroll
            for (int t = 0; t < PER; t++) {
                if (t * B >= n) break;  // CTA-uniform
                const bool found = todo[t] && parent[t] >= 0;
                const int v = found ? s.stage[t * B + tid] : 0;
                {
                    // the list is sorted, so a warp's discoveries share few words: one
                    // shared atomic per word, with the bits OR-reduced over its lanes
                    const int wi = (v - wb) >> 5;
                    const unsigned grp = __match_any_sync(0xffffffffu, found ? wi : -1 - lane);
                    const unsigned bits = __reduce_or_sync(grp, found ? 1u << (v & 31) : 0u);
                    if (found && lane == __ffs(grp) - 1) atomicOr(&s.win_word[wi], bits);
                }
                if (found) {
                    p.labels[v] = PRED ? parent[t] : level + 1;
                    s.flag = 1;
                }
                if (defer) {
                    if (found) found_acc += pack(1u, (unsigned)(r1[t] - r0[t]));
                    continue;
                }
                const unsigned fb = __ballot_sync(0xffffffffu, found);
                if (fb == 0) continue;
                const int leader = __ffs(fb) - 1;
                int base = 0;
                if (lane == leader) base = atomicAdd(&s.out_count, __popc(fb));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (found) {
                    const int slot = base + __popc(fb & lanemask_lt());
                    s.out[slot] = v;
                    s.colstart[slot] = r0[t];
                    s.rel[slot] = r1[t] - r0[t];
                }
            }
            __syncthreads();  // the list is consumed; the batch's output and bits are complete
            if (first) stamp(p, pass, 4);
            if (!defer) {
                emit_frontier<B>(p, s, pass, vout, qe_out);
                __syncthreads();
            }
            if (first) stamp(p, pass, 5);
            first = false;
        }
        if (v0 < re) mask_out[v0 >> 5] = s.win_word[tid];  // every word of the range, old bits | discoveries
    }
    if (defer) {
        unsigned long long tot;
        cta_exclusive_scan<B>(found_acc, s.scan_warp, &tot);
        if (tid == 0 && tot != 0) atomicAdd(qe_out, tot);
    }
}

// The vertex frontier of a bottom-up level that only counted its
// discoveries: the vertices set in this pass's mask buffer and clear in the
// other one (that level's input), emitted into `vout` like any level output,
// slots from one packed atomic per batch on st->mat_ctr.  Every CTA takes its
// range of vertex ids in windows of 32 * B (one word pair per thread); all
// threads call it.
template <int B, bool PRED>
__device__ __forceinline__ void materialize_frontier(const BfsParams &p, ExpandSmem<B, PRED> &s,
                                                     const VertexFrontier &vout)
{
    const int tid = threadIdx.x;
    constexpr int PER = kChunkMax / B;
    const uint32_t *cur = s.mask;
    const uint32_t *prev = (s.mask == p.mask) ? p.mask_alt : p.mask;
    int rs, re;
    cta_range(p.nodes, blockIdx.x, gridDim.x, rs, re);
    for (int wb = rs; wb < re; wb += 32 * B) {
        const int v0 = wb + 32 * tid;
        unsigned fresh = 0u;
        if (v0 < re) fresh = ld_cg(cur + (v0 >> 5)) & ~ld_cg(prev + (v0 >> 5));
        if (v0 < re && re - v0 < 32) fresh &= (1u << (re - v0)) - 1u;
        unsigned long long total;
        const int pos = (int)cta_exclusive_scan<B>((unsigned long long)__popc(fresh), s.scan_warp, &total);
        const int U = (int)total;
        for (int lo = 0; lo < U; lo += kChunkMax) {
            const int n = min(U - lo, kChunkMax);
            scatter_bits(fresh, v0, pos, lo, n, s.out);
            __syncthreads();
#pragma unroll
            for (int t = 0; t < PER; t++) {
                const int j = t * B + tid;
                if (j < n) {
                    const int v = s.out[j];
                    const int a = ld_ro(p.row_offsets + v), b = ld_ro(p.row_offsets + v + 1);
                    s.colstart[j] = a;
                    s.rel[j] = b - a;  // > 0: a bottom-up level only discovers vertices with edges
                }
            }
            if (tid == 0) s.out_count = n;
            __syncthreads();
            emit_frontier<B>(p, s, 0, vout, &p.st->mat_ctr, false);
            __syncthreads();
        }
    }
}

// Bottom-up list mode (distance searches, a bottom-up level right after the
// first one, or later): instead of every vertex id, the CTA's share of the
// list of vertices still unvisited after the last bottom-up level (entries
// found meanwhile by top-down levels are skipped by their label).  A
// neighbour counts as visited when its distance label was written before this
// level (in [0, level]; this level writes level + 1), so the visited mask is
// neither read nor written: after the first list-mode level it is given up for
// the rest of the search (top-down levels then claim vertices on the labels).
// The vertices still without a parent form the next list.
template <int B, bool PRED>
__device__ __forceinline__ void bottom_up_list(const BfsParams &p, ExpandSmem<B, PRED> &s, int level, int pass,
                                               const VertexFrontier &vout, unsigned long long *qe_out)
{
    const int tid = threadIdx.x, lane = tid & 31;
    constexpr int PER = kChunkMax / B;
    constexpr int K = kBottomUpProbe;
    const int32_t *in = p.ul[s.ul_in];
    int32_t *outl = p.ul[s.ul_in ^ 1];
    unsigned *ctr = &p.st->ul_count[(pass + 1) % 3];
    int rs, re;
    cta_range(s.ul_n, blockIdx.x, gridDim.x, rs, re);
    for (int cs = rs; cs < re; cs += kChunkMax) {
        if (tid == 0) {
            s.out_count = 0;
            s.wl_count = 0;
        }
        __syncthreads();
        int v[PER], r0[PER], r1[PER];
        bool todo[PER];
#pragma unroll
        for (int t = 0; t < PER; t++) {
            const int i = cs + t * B + tid;
            v[t] = i < re ? ld_cg(in + i) : -1;
        }
#pragma unroll
        for (int t = 0; t < PER; t++) todo[t] = v[t] >= 0 && ld_cg(p.labels + v[t]) == -1;
#pragma unroll
        for (int t = 0; t < PER; t++) {
            r0[t] = r1[t] = 0;
            if (todo[t]) {
                r0[t] = ld_ro(p.row_offsets + v[t]);
                r1[t] = ld_ro(p.row_offsets + v[t] + 1);
            }
        }
        int parent[PER];
        {
            int nb[PER][K];
#pragma unroll
            for (int t = 0; t < PER; t++) {
                if (p.hub2) {
                    int2 h = make_int2(-1, -1);
                    if (todo[t]) h = p.hub2[v[t]];
                    nb[t][0] = h.x;
                    nb[t][1] = h.y;
                } else {
#pragma unroll
                    for (int k = 0; k < K; k++)
                        nb[t][k] = (todo[t] && r0[t] + k < r1[t]) ? ld_stream(p.column_indices + r0[t] + k) : -1;
                }
            }
            unsigned w[PER][K];
#pragma unroll
            for (int t = 0; t < PER; t++)
#pragma unroll
                for (int k = 0; k < K; k++) w[t][k] = nb[t][k] >= 0 ? probe_load<true>(nullptr, p.labels, nb[t][k]) : 0u;
#pragma unroll
            for (int t = 0; t < PER; t++) {
                parent[t] = -1;
#pragma unroll
                for (int k = K - 1; k >= 0; k--)
                    if (nb[t][k] >= 0 && probe_hit<true>(w[t][k], nb[t][k], level)) parent[t] = nb[t][k];
            }
        }
        if (p.hub2)
            bottom_up_lanes<PER, 0, K, true>(p, nullptr, level, todo, r0, r1, parent);
        else
            bottom_up_lanes<PER, K, K, true>(p, nullptr, level, todo, r0, r1, parent);
#pragma unroll
        for (int t = 0; t < PER; t++) {
            if (t * B >= re - cs) continue;  // CTA-uniform
            const bool found = parent[t] >= 0;
            append_unvisited(s, todo[t] && !found, v[t]);
            const unsigned fb = __ballot_sync(0xffffffffu, found);
            if (fb == 0) continue;
            if (found) {
                p.labels[v[t]] = level + 1;
                s.flag = 1;
            }
            const int leader = __ffs(fb) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&s.out_count, __popc(fb));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (found) {
                const int slot = base + __popc(fb & lanemask_lt());
                s.out[slot] = v[t];
                s.colstart[slot] = r0[t];
                s.rel[slot] = r1[t] - r0[t];
            }
        }
        __syncthreads();
        emit_frontier<B>(p, s, pass, vout, qe_out);
        write_unvisited<B>(p, s, outl, ctr);
        __syncthreads();
    }
}

// Direction of a level from the frontier's size (Beamer, Asanovic and
// Patterson, SC'12 heuristic): top-down -> bottom-up when the frontier's
// edges exceed the unvisited edges / alpha, bottom-up -> top-down when the
// frontier falls under n / beta vertices.
__device__ __forceinline__ bool choose_bottom_up(const BfsParams &p, bool was_bottom_up, int q, int E,
                                                 unsigned long long visited_edges)
{
    if (!p.direction_opt) return false;
    const long long unvisited_edges = (long long)p.edges - (long long)visited_edges;
    if (!was_bottom_up) return (long long)E * p.bu_alpha > unvisited_edges;
    return (long long)q * p.bu_beta >= (long long)p.nodes;
}

// ------------------------------------------------------------------------------------
// Level drivers
// ------------------------------------------------------------------------------------


__device__ __forceinline__ unsigned long long ld_cg64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.global.cg.u64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}

// Per-CTA busy time (lifetime minus grid-barrier waits), accumulated into
// p.duty when the search is instrumented: avg duty = busy / lifetime.
struct DutyClock {
    const BfsParams &p;
    unsigned long long t0 = 0, waited = 0;
    __device__ explicit DutyClock(const BfsParams &params) : p(params)
    {
        if (p.duty && threadIdx.x == 0) t0 = globaltimer_ns();
    }
    __device__ bool barrier(SearchState *st, unsigned &generation, int *s_flag)
    {
        unsigned long long a = 0;
        if (p.duty && threadIdx.x == 0) a = globaltimer_ns();
        const bool ok = grid_barrier(&st->barrier, generation, &st->error, s_flag, 0, p.spin_limit);
        if (p.duty && threadIdx.x == 0) waited += globaltimer_ns() - a;
        return ok;
    }
    __device__ void finish()
    {
        if (p.duty && threadIdx.x == 0) {
            const unsigned long long t1 = globaltimer_ns(), life = t1 - t0;
            atomicAdd(&p.duty[0], life - min(waited, life));
            atomicAdd(&p.duty[1], life);
            atomicMax(&p.duty[2], t1);
        }
    }
};

// Epilogue of every non-persistent launch: the last CTA to finish advances
// the level (unless `stop`: the launch found nothing to do -- an empty
// frontier or an error -- or overflowed) and decides whether the search
// continues; inside a captured graph it sets the WHILE node's condition, so
// a launch must never end without coming here or the loop would not stop.
__device__ __forceinline__ void finish_launch(const BfsParams &p, int level, int next_pass, bool limit_hit,
                                              bool stop = false)
{
    if (threadIdx.x != 0) return;
    __threadfence();
    const unsigned t = atomicAdd(&p.st->finished, 1u);
    if (t == gridDim.x - 1) {
        __threadfence();
        p.st->finished = 0;
        if (!stop) p.st->cur_level = level + 1;
        // a search has at most one level per vertex, plus the final empty
        // contraction of the edge strategies: past that a replayed loop is
        // stopped whatever the counters say
        if (level > p.nodes) {
            atomicOr(&p.st->error, kErrLevels);
            stop = true;
        }
        const int qn = stop ? 0 : qe_count(ld_cg64(&p.st->qe[next_pass % 3]));
        const bool done = stop || (qn == 0) || limit_hit || (ld_cg(&p.st->error) != 0);
        if (done) p.st->done = 1;
        if (p.cond_handle) cudaGraphSetConditional((cudaGraphConditionalHandle)p.cond_handle, done ? 0u : 1u);
    }
}

// Start of pass `pass`: loads its input size into shared memory and lets
// block 0 clear the counters two passes ahead.
template <int B, bool PRED>
__device__ __forceinline__ void begin_pass(const BfsParams &p, ExpandSmem<B, PRED> &s, int pass, bool count_queue)
{
    if (threadIdx.x == 0) {
        const unsigned long long x = ld_cg64(&p.st->qe[pass % 3]);
        s.q = qe_count(x);
        s.E = qe_edges(x);
        s.flag = 0;
        if ((unsigned)s.E > (unsigned)p.edges || (unsigned)s.q > (unsigned)max(p.vcap, p.ecap)) {
            // counters past the graph's size: stop before any frontier read
            atomicOr(&p.st->error, kErrOverflow);
            s.q = 0;
        }
        if (blockIdx.x == 0) {
            p.st->qe[(pass + 2) % 3] = 0;
            p.st->tile_ctr[(pass + 1) % 3] = 0;
            // (the reference counts the queues after the source's: kernel_runtime_stats
            // aggregates from iteration 1 on, contract_expand_atomic/kernel.cuh:333-345)
            if (count_queue && pass > 0) atomicAdd(&p.st->total_queued, (unsigned long long)s.q);
        }
        s.visited_edges = ld_cg64(&p.st->visited_edges[pass % 3]) + (unsigned long long)s.E;
        s.prev_bu = ld_cg(&p.st->dir[pass % 3]);
        s.mask = ld_cg(&p.st->mask_sel[pass % 3]) ? p.mask_alt : p.mask;
        s.ul_in = -1;
        s.ul_n = 0;
        if (p.ul[0]) {
            s.ul_in = ld_cg(&p.st->ul_sel[pass % 3]);
            s.ul_n = (int)ld_cg(&p.st->ul_count[pass % 3]);
            if (s.ul_n > p.nodes || s.ul_in > 1) {  // never read past a list
                atomicOr(&p.st->error, kErrOverflow);
                s.q = 0;
            }
            if (blockIdx.x == 0) p.st->ul_count[(pass + 2) % 3] = 0;
        }
        if (p.levels && blockIdx.x == 0 && pass < kMaxLevelRecords) {
            LevelRecord r;
            r.vertices = s.q;
            r.edges = s.E;
            r.bottom_up = 0;
            r.pass = pass;
            r.t_ns = globaltimer_ns();
            p.levels[pass] = r;
        }
    }
    __syncthreads();
}

// Direction bookkeeping of pass `pass` (block 0): the visited-edge total,
// whether the level ran bottom-up and which mask buffer the next pass reads
// (a bottom-up level writes the other one).
__device__ __forceinline__ void record_direction(const BfsParams &p, unsigned long long visited_edges, int pass,
                                                 bool bu, const uint32_t *pass_mask, int ul_in, int ul_n,
                                                 bool deferred = false)
{
    p.st->visited_edges[(pass + 1) % 3] = visited_edges;
    p.st->dir[(pass + 1) % 3] = bu ? (deferred ? 2 : 1) : 0;
    if (deferred) p.st->mat_ctr = 0;
    p.st->mask_sel[(pass + 1) % 3] = (pass_mask == p.mask) == bu ? 1 : 0;
    if (p.ul[0]) {
        // a bottom-up level writes the next list (range mode into buffer 0,
        // list mode into the other buffer); a top-down level carries it on
        p.st->ul_sel[(pass + 1) % 3] = bu ? (ul_in < 0 ? 0 : ul_in ^ 1) : ul_in;
        if (!bu) p.st->ul_count[(pass + 1) % 3] = (uint32_t)ul_n;
    }
    if (bu && p.levels && pass < kMaxLevelRecords) p.levels[pass].bottom_up = 1;
}

// A phase of levels run by part of the grid (CTA 0 alone, or the first
// kSubgridCtas CTAs) starts at a pass whose state slots (qe[pass % 3] and the
// direction slots) every CTA reads in begin_pass; the CTAs outside the phase
// then wait at the grid barrier.  Block 0 reuses those slots two passes on, so
// before its second level it waits (thread 0, bounded) until the `outside` CTAs
// have arrived at that barrier, which they do right after their read -- a late
// CTA (one launched last, at kernel start) must not read a cleared slot.
template <int B, bool PRED>
__device__ __forceinline__ void outside_arrived(const BfsParams &p, ExpandSmem<B, PRED> &s, unsigned generation,
                                                unsigned outside)
{
    if (threadIdx.x == 0) wait_outside_arrivals(&p.st->barrier, generation, outside, &p.st->error, p.spin_limit);
    __syncthreads();
}

constexpr int kSoloLevelCap = 4096;  // small levels CTA 0 runs alone before the grid resynchronises
// bottom-up levels emit their frontier (rather than count it) once the unvisited
// edges are under 1 / kDeferMinShare of the graph's
constexpr unsigned long long kDeferMinShare = 512;

// Expand-contract (vertex frontiers): one level per pass.  With
// direction_opt, levels with a large frontier run bottom-up.  In a
// persistent launch, a run of levels whose frontiers have at most
// p.small_edges edges is processed by CTA 0 alone, separated by CTA-level
// barriers only, while the other CTAs wait at the grid barrier; while those
// levels fit one sub-round their frontier stays in shared memory.
// BU = false builds a top-down-only variant (plain expand-contract searches):
// without the bottom-up code the kernel needs fewer registers.
template <int B, bool PRED, bool LISTS, bool SUBGRID = false, bool BU = true>
__global__ void __launch_bounds__(B, 1024 / B) ec_kernel(BfsParams p)
{
    // top-down levels with at least a full sub-round per CTA run warp by warp
    // (expand_range_warp) when the policy asks for it (not in list mode, nor
    // predecessor searches with CTAs of more than 256 threads)
    const auto warp_levels = [](const BfsParams &q, int E) {
        return !LISTS && (B <= 256 || !PRED) && q.warp_contract != 0 && warp_sized(E);
    };
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ExpandSmem<B, PRED> &s = *reinterpret_cast<ExpandSmem<B, PRED> *>(smem_raw);
    __shared__ int s_ok;
    const int tid = threadIdx.x;
    if (tid == 0) mbar_init(&s.bar, 1);
    hist_init<B, PRED>(p, s, smem_raw);
    unsigned bar_phase = 0, generation = 0;
    int max_level_seen = -1;
    late_start(p);
    int level = ld_cg(&p.st->cur_level);
    bool limit_hit = false, worked = false;
    int solo_phase = 0;  // small-frontier phases so far (the same count in every CTA)
    int sub_phase = 0;   // sub-grid phases so far (the same count in every CTA)
    unsigned sub_generation = 0;  // barriers of sub-grid phases this CTA took part in
    DutyClock duty(p);
    __syncthreads();
    for (int iter = 0; iter < p.max_levels; iter++, level++) {
        int pass = level;
        begin_pass<B, PRED>(p, s, pass, true);
        if (s.q == 0 || ld_cg(&p.st->error) != 0) break;
        const int dl = p.st->depth_limit;
        if (dl >= 0 && level >= dl) {
            limit_hit = true;
            break;
        }
        if (BU && s.prev_bu == 2 &&
            ((p.persistent && s.E <= p.small_edges) || !choose_bottom_up(p, true, s.q, s.E, s.visited_edges))) {
            // the previous level ran bottom-up and only counted its discoveries:
            // this top-down level (or solo phase) reads them as a vertex frontier
            materialize_frontier<B, PRED>(p, s, p.vf[level & 1]);
            if (!duty.barrier(p.st, generation, &s_ok)) break;
            if (tid == 0 && ld_cg64(&p.st->mat_ctr) != ld_cg64(&p.st->qe[pass % 3]))
                atomicOr(&p.st->error, kErrFrontier);
        }
        if (p.persistent && s.E <= p.small_edges) {
            // ---- small frontiers: CTA 0 alone, level after level ----------------------
            const int solo_pass = pass;  // (instrumented searches stamp the arrivals under it)
            if (blockIdx.x == 0) {
                int smem_n = -1;  // >= 0: this level's frontier is the run tables in shared memory (entries)
                for (int solo = 0;; solo++) {
                    if (tid == 0) record_direction(p, s.visited_edges, pass, false, s.mask, s.ul_in, s.ul_n);
                    const bool one_round = s.E > 0 && s.E <= kChunkMax;  // CTA-uniform
                    if (smem_n >= 0)
                        solo_level_smem<B, PRED, LISTS>(p, s, level, smem_n, s.E);
                    else
                        expand_range<B, PRED, true, LISTS>(p, p.vf[level & 1], s, level, pass,
                                                           p.vf[(level + 1) & 1], p.ef[0],
                                                           &p.st->qe[(pass + 1) % 3], bar_phase, 0, 1, one_round);
                    __syncthreads();
                    if (s.flag) max_level_seen = level + 1;
                    level++;
                    pass = level;
                    if (one_round) {
                        // the discoveries are still in s.out / colstart / rel: stay in
                        // shared memory while the next level is one sub-round too
                        constexpr int PER = kChunkMax / B;
                        const int n = s.out_count;
                        int deg[PER];
                        unsigned long long sum = 0;
#pragma unroll
                        for (int k = 0; k < PER; k++) {
                            const int j = tid * PER + k;
                            deg[k] = j < n ? s.rel[j] : 0;
                            sum += (unsigned long long)deg[k];
                        }
                        unsigned long long En;
                        unsigned long long run = cta_exclusive_scan<B>(sum, s.scan_warp, &En);
                        // (a frontier larger than the queue goes out too, so the overflow is reported)
                        if (tid == 0)
                            s.solo_stop = n == 0 || n > p.vcap ||
                                          En > (unsigned long long)min(p.small_edges, kChunkMax) ||
                                          (dl >= 0 && level >= dl) || solo + 1 >= kSoloLevelCap ||
                                          ld_cg(&p.st->error) != 0;
                        __syncthreads();
                        if (!s.solo_stop && solo == 0) outside_arrived(p, s, generation, gridDim.x - 1);
                        if (!s.solo_stop) {
#pragma unroll
                            for (int k = 0; k < PER; k++) {
                                const int j = tid * PER + k;
                                if (j < n) {
                                    s.rel[j] = (int)run;
                                    if (PRED) s.vert[j] = s.out[j];
                                }
                                run += (unsigned long long)deg[k];
                            }
                            if (tid == 0) {
                                // begin_pass without the frontier counters
                                s.rel[n] = (int)En;
                                s.q = n;
                                s.E = (int)En;
                                s.flag = 0;
                                s.out_count = 0;
                                s.visited_edges += En;
                                p.st->qe[(pass + 2) % 3] = 0;
                                p.st->tile_ctr[(pass + 1) % 3] = 0;
                                atomicAdd(&p.st->total_queued, (unsigned long long)n);
                                if (p.ul[0]) p.st->ul_count[(pass + 2) % 3] = 0;
                                if (p.levels && pass < kMaxLevelRecords) {
                                    LevelRecord r;
                                    r.vertices = n;
                                    r.edges = (int)En;
                                    r.bottom_up = 0;
                                    r.pass = pass;
                                    r.t_ns = globaltimer_ns();
                                    p.levels[pass] = r;
                                }
                            }
                            smem_n = n;
                            __syncthreads();
                            continue;
                        }
                        // leaving shared memory: the discoveries become the frontier of `pass`
                        emit_frontier<B>(p, s, pass - 1, p.vf[level & 1], &p.st->qe[pass % 3]);
                        __syncthreads();
                        smem_n = -1;
                        // the phase ends here unless only the one-sub-round limit stopped it
                        // (the frontier's size is known: no read of the counter it went to)
                        if (n == 0 || En > (unsigned long long)p.small_edges || (dl >= 0 && level >= dl) ||
                            solo + 1 >= kSoloLevelCap)
                            break;
                    }
                    if (tid == 0) {
                        const unsigned long long x = ld_cg64(&p.st->qe[pass % 3]);
                        s.q = qe_count(x);
                        s.E = qe_edges(x);
                    }
                    __syncthreads();
                    const bool stop = s.q == 0 || s.E > p.small_edges || (dl >= 0 && level >= dl) ||
                                      solo + 1 >= kSoloLevelCap || ld_cg(&p.st->error) != 0;
                    if (stop) break;
                    if (solo == 0) outside_arrived(p, s, generation, gridDim.x - 1);
                    begin_pass<B, PRED>(p, s, pass, true);
                }
                if (tid == 0) p.st->solo_resume[solo_phase & 1] = level;
            }
            worked = true;
            stamp(p, solo_pass, kPhaseArrive);
            if (!duty.barrier(p.st, generation, &s_ok)) break;
            // not st->cur_level: CTA 0 may already have moved it on by the time a slow CTA reads
            level = ld_cg(&p.st->solo_resume[solo_phase & 1]) - 1;  // the loop increment brings it back
            solo_phase++;
            continue;
        }
        // (a kernel variant of its own: the code would cost the other paths registers)
        if (SUBGRID && p.persistent && p.subgrid_edges > 0 && s.E <= p.subgrid_edges &&
            (int)gridDim.x >= 4 * kSubgridCtas &&
            !(BU && choose_bottom_up(p, s.prev_bu != 0, s.q, s.E, s.visited_edges))) {
            // ---- mid-size top-down levels: the first kSubgridCtas CTAs, level after
            // level, with a barrier of their own; the others wait at the grid barrier
            if ((int)blockIdx.x < kSubgridCtas) {
                for (int sub = 0;; sub++) {
                    if (tid == 0 && blockIdx.x == 0)
                        record_direction(p, s.visited_edges, pass, false, s.mask, s.ul_in, s.ul_n);
                    expand_range<B, PRED, true, LISTS>(p, p.vf[level & 1], s, level, pass, p.vf[(level + 1) & 1],
                                                       p.ef[0], &p.st->qe[(pass + 1) % 3], bar_phase, blockIdx.x,
                                                       kSubgridCtas);
                    __syncthreads();
                    if (s.flag) max_level_seen = level + 1;
                    // (a wait that expires sets the error word: the test below then
                    // ends the phase in every CTA of it)
                    grid_barrier(&p.st->sub_barrier, sub_generation, &p.st->error, &s_ok, kSubgridCtas,
                                 p.spin_limit);
                    level++;
                    pass = level;
                    if (sub == 0 && blockIdx.x == 0) outside_arrived(p, s, generation, gridDim.x - kSubgridCtas);
                    // the level's frontier is counted once, by the pass that processes it
                    begin_pass<B, PRED>(p, s, pass, false);
                    if (tid == 0)
                        s.solo_stop = s.q == 0 || s.E > p.subgrid_edges || s.E <= p.small_edges ||
                                      (dl >= 0 && level >= dl) || sub + 1 >= kSoloLevelCap ||
                                      ld_cg(&p.st->error) != 0 ||
                                      (BU && choose_bottom_up(p, s.prev_bu != 0, s.q, s.E, s.visited_edges));
                    __syncthreads();
                    if (s.solo_stop) break;
                    if (tid == 0 && blockIdx.x == 0) atomicAdd(&p.st->total_queued, (unsigned long long)s.q);
                }
                if (tid == 0 && blockIdx.x == 0) p.st->sub_resume[sub_phase & 1] = level;
            }
            worked = true;
            if (!duty.barrier(p.st, generation, &s_ok)) break;
            level = ld_cg(&p.st->sub_resume[sub_phase & 1]) - 1;  // the loop increment brings it back
            sub_phase++;
            continue;
        }
        const bool bu = BU && choose_bottom_up(p, s.prev_bu != 0, s.q, s.E, s.visited_edges);
        // a bottom-up level counts its discoveries instead of emitting them, unless
        // the edges still unvisited (a bound on the next frontier's) are so few that
        // emitting them costs less than building the frontier from the masks later
        const unsigned long long unvisited =
            (unsigned long long)p.edges - min((unsigned long long)p.edges, s.visited_edges);
        const bool defer = !LISTS && bu && p.bu_defer && p.persistent &&
                           unvisited * kDeferMinShare > (unsigned long long)p.edges;
        if (tid == 0 && blockIdx.x == 0)
            record_direction(p, s.visited_edges, pass, bu, s.mask, s.ul_in, s.ul_n, defer);
        if (LISTS && bu && s.ul_in >= 0)
            bottom_up_list<B, PRED>(p, s, level, pass, p.vf[(level + 1) & 1], &p.st->qe[(pass + 1) % 3]);
        else if (bu && !LISTS && s.prev_bu == 0 && defer && p.warp_bu)
            // the first bottom-up level of a run, counting only: warp by warp
            bottom_up_range_warp<B, PRED>(p, s, level, &p.st->qe[(pass + 1) % 3]);
        else if (bu && (LISTS || s.prev_bu == 0))
            // the first bottom-up level of a run: most vertices are unvisited, so the
            // chunks of vertex ids are walked directly
            bottom_up_range<B, PRED, LISTS>(p, s, level, pass, p.vf[(level + 1) & 1], &p.st->qe[(pass + 1) % 3],
                                            defer);
        else if (bu)
            // later bottom-up levels: the unvisited vertices of each window, compacted
            bottom_up_windows<B, PRED>(p, s, level, pass, p.vf[(level + 1) & 1], &p.st->qe[(pass + 1) % 3], defer);
        else if (!BU && warp_levels(p, s.E))
        {
            if constexpr (!BU && !LISTS && (B <= 256 || !PRED))
                expand_range_warp<B, PRED, true, true>(p, p.vf[level & 1], s, level, p.vf[(level + 1) & 1],
                                                       &p.st->qe[(pass + 1) % 3]);
        }
        else
        {
            // direction-optimizing: once this level's output passes E* edges, where
            // E* * (alpha + 1) > the edges unvisited after this level's input, the
            // next level runs bottom-up whatever the rest adds (the switch test is
            // E * alpha > m - visited - E), so later tiles need not write entries.
            // E* is at least the solo-phase threshold: a next level that small runs
            // top-down on CTA 0 before any switch test.
            unsigned long long skip_above = ~0ull;
            if (BU && p.direction_opt && !LISTS) {
                const unsigned long long un =
                    (unsigned long long)p.edges - min((unsigned long long)p.edges, s.visited_edges);
                skip_above = max(un / (unsigned long long)(p.bu_alpha + 1),
                                 (unsigned long long)max(p.small_edges, 0));
            }
            if (BU && warp_levels(p, s.E)) {
                if constexpr (BU && !LISTS && (B <= 256 || !PRED))
                    expand_range_warp<B, PRED>(p, p.vf[level & 1], s, level, p.vf[(level + 1) & 1],
                                               &p.st->qe[(pass + 1) % 3], nullptr, skip_above);
            } else {
                expand_range<B, PRED, true, LISTS>(p, p.vf[level & 1], s, level, pass, p.vf[(level + 1) & 1],
                                                   p.ef[0], &p.st->qe[(pass + 1) % 3], bar_phase, blockIdx.x,
                                                   gridDim.x, false, skip_above);
            }
        }
        __syncthreads();
        worked = true;
        if (s.flag) max_level_seen = level + 1;
        if (!p.persistent) break;
        stamp(p, pass, kPhaseArrive);
        if ((int)blockIdx.x == p.skip_arrival_cta)
            return;  // test-only: never arrives, so the others' bounded waits must run out
        if (!duty.barrier(p.st, generation, &s_ok)) break;
        // only after the barrier: a CTA that starts late reads cur_level as its
        // first level, so it must not move on before every CTA has arrived once
        if (tid == 0 && blockIdx.x == 0) p.st->cur_level = level + 1;
    }
    if (tid == 0 && max_level_seen >= 0) atomicMax(&p.st->max_level, max_level_seen);
    duty.finish();
    if (p.persistent) {
        if (tid == 0 && blockIdx.x == 0) {
            p.st->cur_level = level;
            p.st->done = 1;
        }
    } else {
        // a launch that broke out before its level (empty frontier, error) stops the search
        finish_launch(p, level, level + 1, limit_hit, !(worked || limit_hit));
    }
}

// Edge strategies: per level, contract the edge frontier into vf[0] (pass
// 2L), then expand vf[0] into the next edge frontier at flattened edge
// positions (pass 2L+1).  phase_mask selects the phases of a non-persistent
// launch; a persistent launch runs both with a grid barrier after each.
// With `hybrid`, a persistent launch returns when the edge frontier exceeds
// gridDim * saturation items (SATURATION_QUIT, enactor_hybrid.cuh:571).
template <int B, bool PRED>
__global__ void __launch_bounds__(B, 1024 / B) edge_kernel(BfsParams p)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ExpandSmem<B, PRED> &s = *reinterpret_cast<ExpandSmem<B, PRED> *>(smem_raw);
    __shared__ int s_ok;
    const int tid = threadIdx.x;
    if (tid == 0) mbar_init(&s.bar, 1);
    hist_init<B, PRED>(p, s, smem_raw);
    unsigned bar_phase = 0, generation = 0;
    int max_level_seen = -1;
    late_start(p);
    int level = ld_cg(&p.st->cur_level);
    bool limit_hit = false, saturated = false, completed_level = false;
    DutyClock duty(p);
    __syncthreads();
    for (int iter = 0; iter < p.max_levels; iter++, level++) {
        const int in_idx = p.edge_pingpong ? (level & 1) : 0;
        const int out_idx = p.edge_pingpong ? ((level + 1) & 1) : 0;
        if (p.phase_mask & 1) {
            const int pass = 2 * level;
            begin_pass<B, PRED>(p, s, pass, false);
            if (ld_cg(&p.st->error) != 0 || s.q == 0) break;
            if (p.hybrid && p.persistent && s.q > (int)gridDim.x * p.saturation) {
                saturated = true;  // the two-phase launches take this pass over (and count it)
                break;
            }
            if (tid == 0 && blockIdx.x == 0 && pass > 0) atomicAdd(&p.st->total_queued, (unsigned long long)s.q);
            if (p.warp_contract && warp_sized(s.q))
                contract_range_warp<B, PRED>(p, s, p.ef[in_idx], level, p.vf[0], &p.st->qe[(pass + 1) % 3]);
            else
                contract_range<B, PRED>(p, s, p.ef[in_idx], level, pass, &p.st->qe[(pass + 1) % 3]);
            __syncthreads();
            if (s.flag) max_level_seen = max(max_level_seen, level);
            if (p.persistent) {
                if ((int)blockIdx.x == p.skip_arrival_cta)
                    return;  // test-only: never arrives, so the others' bounded waits must run out
                if (!duty.barrier(p.st, generation, &s_ok)) break;
            }
        }
        const int dl = p.st->depth_limit;
        if (dl >= 0 && level >= dl) {
            limit_hit = true;
            break;
        }
        if (p.phase_mask & 2) {
            const int pass = 2 * level + 1;
            begin_pass<B, PRED>(p, s, pass, false);
            const int q = s.q, E = s.E;
            if (E > p.ecap) {
                if (tid == 0) atomicOr(&p.st->error, kErrOverflow);
                break;
            }
            if (tid == 0 && blockIdx.x == 0) p.st->qe[(pass + 1) % 3] = pack((unsigned)(q == 0 ? 0 : E), 0u);
            if (q > 0) {
                if ((B <= 256 || !PRED) && p.warp_contract && warp_sized(E)) {
                    if constexpr (B <= 256 || !PRED)
                        expand_range_warp<B, PRED, false>(p, p.vf[0], s, level, p.vf[1], nullptr, &p.ef[out_idx]);
                } else {
                    expand_range<B, PRED, false>(p, p.vf[0], s, level, pass, p.vf[1], p.ef[out_idx], nullptr,
                                                 bar_phase, blockIdx.x, gridDim.x);
                }
            }
            __syncthreads();
            completed_level = true;
            if (p.persistent) {
                if (!duty.barrier(p.st, generation, &s_ok)) break;
                // after the barrier, as in ec_kernel: late-starting CTAs read cur_level
                if (tid == 0 && blockIdx.x == 0) p.st->cur_level = level + 1;
            }
        }
        if (!p.persistent) break;
    }
    if (tid == 0 && max_level_seen >= 0) atomicMax(&p.st->max_level, max_level_seen);
    duty.finish();
    if (p.persistent) {
        if (tid == 0 && blockIdx.x == 0) {
            p.st->cur_level = level;
            if (saturated)
                p.st->saturated = 1;
            else
                p.st->done = 1;
        }
    } else if (completed_level || limit_hit) {
        finish_launch(p, level, 2 * (level + 1), limit_hit);
    } else if (p.phase_mask & 2) {
        // an expand launch that broke out (overflow, error) stops the search; a
        // contract-only launch leaves the level's epilogue to its expand launch
        finish_launch(p, level, 2 * (level + 1), false, true);
    }
}

// Sets up a search: the source's label, visited bit and the level-0
// frontier, plus the search state.  With FULL it first initialises every
// label to -1 and the visited mask to 0 (what CsrProblem::Reset does,
// csr_problem.cuh:723-745), for searches not preceded by a reset and for
// captured graphs.  The source is read from the state so a captured graph
// replays with whatever source was uploaded last.
template <bool PRED, bool VERTEX_FRONTIER, bool FULL>
__global__ void init_kernel(BfsParams p)
{
    const int src = p.src_by_value ? p.src_arg : p.st->src;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int src_label = PRED ? -2 : 0;
    if (FULL) {
        // 16-byte stores when the labels array is 16-byte aligned (a caller's
        // array given to the allocation-free search may not be); the source's
        // label is set by the thread that stores its vector
        const long long n4 = (reinterpret_cast<uintptr_t>(p.labels) & 15) == 0 ? p.nodes / 4 : 0;
        int4 *labels4 = reinterpret_cast<int4 *>(p.labels);
        for (long long i = t0; i < n4; i += stride) {
            int4 x = make_int4(-1, -1, -1, -1);
            if (VERTEX_FRONTIER && (src >> 2) == i) {
                const int r = src & 3;
                x.x = r == 0 ? src_label : -1;
                x.y = r == 1 ? src_label : -1;
                x.z = r == 2 ? src_label : -1;
                x.w = r == 3 ? src_label : -1;
            }
            labels4[i] = x;
        }
        for (long long i = 4 * n4 + t0; i < p.nodes; i += stride)
            p.labels[i] = (VERTEX_FRONTIER && i == src) ? src_label : -1;
        for (long long w = t0; w < p.mask_words; w += stride) {
            // edgeless vertices start visited; the source's bit is set for a vertex
            // frontier and clear for an edge frontier (whose contraction labels it)
            uint32_t m = p.iso ? p.iso[w] : 0u;
            if (w == (src >> 5)) m = VERTEX_FRONTIER ? (m | (1u << (src & 31))) : (m & ~(1u << (src & 31)));
            p.mask[w] = m;
        }
    } else if (t0 == 0) {
        // after a reset (labels -1, mask = the edgeless bits)
        if (VERTEX_FRONTIER) {
            p.labels[src] = src_label;
            p.mask[src >> 5] |= 1u << (src & 31);
        } else {
            p.mask[src >> 5] &= ~(1u << (src & 31));
        }
    }
    if (t0 == 0) {
        SearchState *st = p.st;
        if (p.src_by_value) {
            st->src = p.src_arg;
            st->depth_limit = p.depth_arg;
        }
        const int r0 = p.row_offsets[src], r1 = p.row_offsets[src + 1];
        st->tile_ctr[0] = st->tile_ctr[1] = st->tile_ctr[2] = 0;
        st->cur_level = 0;
        st->epoch += 1ull << 24;
        st->barrier = 0;
        st->sub_barrier = 0;
        st->error = 0;
        st->max_level = 0;
        st->done = 0;
        st->saturated = 0;
        st->total_queued = 0;
        st->finished = 0;
        st->qe[1] = st->qe[2] = 0;
        st->dir[0] = st->dir[1] = st->dir[2] = 0;
        st->mask_sel[0] = st->mask_sel[1] = st->mask_sel[2] = 0;
        st->ul_sel[0] = st->ul_sel[1] = st->ul_sel[2] = -1;
        st->ul_count[0] = st->ul_count[1] = st->ul_count[2] = 0;
        st->visited_edges[0] = st->visited_edges[1] = st->visited_edges[2] = 0;
        if (VERTEX_FRONTIER) {
            const int deg = r1 - r0;
            st->qe[0] = deg > 0 ? pack(1u, (unsigned)deg) : 0ull;
            p.vf[0].v[0] = src;
            p.vf[0].col[0] = r0;
            p.vf[0].P[0] = 0;
        } else {
            // edge frontier: the source is the only item; its predecessor is -2
            st->qe[0] = pack(1u, 0u);
            p.ef[0].v[0] = src;
            if (PRED) p.ef[0].pred[0] = -2;
        }
    }
    if (VERTEX_FRONTIER) {
        // the source owns every chunk of the level-0 frontier (a hub source has many)
        const int deg = p.row_offsets[src + 1] - p.row_offsets[src];
        const long long chunks = min((long long)(deg + kChunkGrain - 1) / kChunkGrain, (long long)p.cf_cap);
        for (long long c = t0; c < chunks; c += stride) p.vf[0].cf[c] = 0;
    }
}

}  // namespace dev
}  // namespace b40c
