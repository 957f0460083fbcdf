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
//  * vertex frontiers carry each entry's degree prefix P, so the next level
//    splits its flattened edge space into equal chunks (edge-balanced): a
//    hub's adjacency list is spread over many CTAs;
//  * inside a chunk, adjacency runs are gathered three ways: CTA-cooperative
//    (runs >= cta_thresh, bulk-copied into shared memory with cp.async.bulk),
//    warp-cooperative (runs >= warp_thresh), and scan-based fine-grained
//    (shorter runs, through a shared-memory slot -> owner map);
//  * queue slots come from a CTA-wide shuffle scan and a decoupled look-back
//    over chunk ids (one 64-bit (count, degree-sum) pair per chunk), never
//    from per-item atomics;
//  * one kernel body serves per-level launches, CUDA-graph replays and a
//    persistent grid with a bounded software barrier between levels.
#pragma once
#include <cstdint>

#include "bfs_state.h"
#include "device_primitives.cuh"

namespace b40c {
namespace dev {

constexpr int kChunkMax = 2048;  // edges (EC) or items (CE/contract) per chunk, maximum
constexpr int kMaxCtaRuns = 8;   // CTA-gathered runs per chunk (cta_thresh >= kChunkMax / 8)

// ------------------------------------------------------------------------------------
// Shared-memory layout of the edge-balanced expansion (EC and 2P expand)
// ------------------------------------------------------------------------------------
template <int B, bool PRED>
struct ExpandSmem {
    int32_t colstart[kChunkMax + 1];  // column index where vertex j's in-chunk run starts
    int32_t rel[kChunkMax + 2];       // run start relative to the chunk start (k + 1 entries)
    uint16_t foff[kChunkMax + 1];     // first fine slot of a fine-gathered run
    int32_t vert[PRED ? kChunkMax + 1 : 1];
    uint16_t fmap[kChunkMax];         // fine slot -> vertex j
    int32_t out[kChunkMax];           // discovered vertices of this chunk
    alignas(16) int32_t stage[kChunkMax + 16];  // bulk-staged CTA runs
    uint64_t bar;                     // mbarrier for the bulk copies
    int32_t probe[257];               // per-level cache of P at 256 evenly spaced entries
    int32_t warp_runs[kChunkMax / 32 + 1];
    int32_t cta_runs[kMaxCtaRuns];
    int32_t cta_stage_off[kMaxCtaRuns];
    int32_t n_warp_runs, n_cta_runs, n_fine, out_count;
    int32_t i0, k, chunk, flag;
    int32_t q, E, level, C, nchunks;
    unsigned long long scan_warp[B / 32];
    unsigned long long prefix;
    int32_t sfound;
};

// Packed (count, degree) pair helpers: count in the high 32 bits.
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

// Test-and-set of v's visited bit; on discovery writes the label.
template <bool PRED>
__device__ __forceinline__ bool discover(const BfsParams &p, int v, int u, int new_level, bool precheck)
{
    uint32_t *w = p.mask + (v >> 5);
    const uint32_t bit = 1u << (v & 31);
    if (precheck && (ld_mask(w) & bit)) return false;
    uint32_t old = atomicOr(w, bit);
    if (old & bit) return false;
    p.labels[v] = PRED ? u : new_level;
    return true;
}

// Warp-aggregated append of `v` (when `found`) to the chunk's output list.
__device__ __forceinline__ void push_out(bool found, int v, int32_t *out, int32_t *out_count)
{
    const unsigned bal = __ballot_sync(0xffffffffu, found);
    if (bal == 0) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(bal) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(out_count, __popc(bal));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (found) out[base + __popc(bal & lanemask_lt())] = v;
}

// Optional warp culling: among lanes holding the same vertex only the lowest stays valid.
__device__ __forceinline__ bool warp_cull(bool valid, int v)
{
    const int lane = threadIdx.x & 31;
    unsigned peers = __match_any_sync(0xffffffffu, valid ? v : -2 - lane);
    return valid && (__ffs(peers) - 1 == lane);
}

// Finds i0 = the last frontier entry with P[i0] <= x (P strictly increasing,
// P[0] = 0).  CTA-wide 256-ary search; the first round uses the per-level
// probe cache.  All threads must call; returns the same value in all threads.
template <int B, bool PRED>
__device__ __forceinline__ int locate(const int32_t *P, int q, int x, ExpandSmem<B, PRED> &s)
{
    // probe[t] = P[min(t * stride, q)] for t in [0, 256]
    const int stride0 = (q + 256) / 256;  // ceil((q+1)/256)
    int lo, hi;
    // binary-search the cached probes (257 entries, warp-uniform smem reads)
    {
        int a = 0, b = 256;  // probe[a] <= x (probe[0] = P[0] = 0)
        while (a < b) {
            int mid = (a + b + 1) >> 1;
            if (s.probe[mid] <= x) a = mid; else b = mid - 1;
        }
        lo = min(a * stride0, q);
        hi = min(lo + stride0 - 1, q);  // answer in [lo, hi]
    }
    while (hi - lo > 0) {
        const int span = hi - lo;
        if (span < B) {
            int idx = lo + 1 + (int)threadIdx.x;
            bool le = (idx <= hi) && (ld_cg(P + idx) <= x);
            int c = __syncthreads_count(le);
            return lo + c;
        }
        const int stride = (span + B - 1) / B;
        int idx = lo + ((int)threadIdx.x + 1) * stride;
        bool le = (idx <= hi) && (ld_cg(P + min(idx, q)) <= x);
        int c = __syncthreads_count(le);
        lo = lo + c * stride;
        hi = min(lo + stride - 1, hi);
        if (lo > hi) lo = hi;
    }
    return lo;
}

// Turns the chunk's discovered vertices (s.out[0, s.out_count)) into entries
// of the vertex frontier `vout`: reads each one's CSR row, drops degree-0
// vertices, allocates slots with a CTA scan plus a decoupled look-back over
// chunk ids, and writes (v, col, P).  The last chunk publishes the totals to
// *q_out / *e_out and closes P.  All threads must call it.
template <int B, bool PRED>
__device__ __forceinline__ void emit_frontier(const BfsParams &p, ExpandSmem<B, PRED> &s, int level, int phase,
                                              const VertexFrontier &vout, int32_t *q_out, int32_t *e_out,
                                              bool &any_discovered)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int chunk = s.chunk;
    const int cnt = s.out_count;
    if (cnt > 0) any_discovered = true;
    constexpr int PER = kChunkMax / B;
    const int per = (cnt + B - 1) / B;
    const int jb = min(tid * per, cnt), je = min(jb + per, cnt);
    int rv[PER], rc[PER], rd[PER];
    unsigned my_cnt = 0, my_deg = 0;
#pragma unroll
    for (int t = 0; t < PER; t++) {
        rd[t] = 0;
        rv[t] = -1;
        rc[t] = 0;
        if (jb + t < je) {
            const int v = s.out[jb + t];
            const int r0 = ld_ro(p.row_offsets + v);
            const int r1 = ld_ro(p.row_offsets + v + 1);
            rv[t] = v;
            rc[t] = r0;
            rd[t] = r1 - r0;
            if (rd[t] > 0) {
                my_cnt++;
                my_deg += (unsigned)rd[t];
            }
        }
    }
    unsigned long long tot;
    const unsigned long long excl = cta_exclusive_scan<B>(pack(my_cnt, my_deg), s.scan_warp, &tot);
    const unsigned long long epoch = p.st->epoch + 4ull * (unsigned long long)level + (unsigned)phase;
    if (warp == 0) {
        unsigned long long prefix = 0;
        if (chunk == 0) {
            if (lane == 0) lookback_publish(&p.slots[0], epoch, kFlagInclusive, tot);
        } else {
            if (lane == 0) lookback_publish(&p.slots[chunk], epoch, kFlagAggregate, tot);
            prefix = lookback_exclusive(p.slots, (unsigned)chunk, epoch, &p.st->error);
            if (lane == 0 && prefix != ~0ull) lookback_publish(&p.slots[chunk], epoch, kFlagInclusive, prefix + tot);
        }
        if (lane == 0) {
            s.prefix = prefix;
            if (prefix != ~0ull && chunk == s.nchunks - 1) {
                const unsigned long long all = prefix + tot;
                const int qn = (int)(all >> 32);
                const int en = (int)(all & 0xffffffffu);
                if (qn > p.vcap) {
                    atomicOr(&p.st->error, kErrOverflow);
                } else {
                    *q_out = qn;
                    *e_out = en;
                    vout.P[qn] = en;
                }
            }
        }
    }
    __syncthreads();
    const unsigned long long prefix = s.prefix;
    if (prefix == ~0ull) return;
    unsigned g = (unsigned)(prefix >> 32) + (unsigned)(excl >> 32);
    unsigned d = (unsigned)(prefix & 0xffffffffu) + (unsigned)(excl & 0xffffffffu);
#pragma unroll
    for (int t = 0; t < PER; t++) {
        if (rd[t] > 0) {
            if ((int)g < p.vcap) {
                vout.v[g] = rv[t];
                vout.col[g] = rc[t];
                vout.P[g] = (int)d;
            } else {
                atomicOr(&p.st->error, kErrOverflow);
            }
            g++;
            d += (unsigned)rd[t];
        }
    }
}

// ------------------------------------------------------------------------------------
// Edge-balanced expansion of one chunk of a vertex frontier.
//   FUSED_CULL = true  : expand-contract (EC): every gathered neighbour goes
//                        through discover(); discoveries become the next
//                        vertex frontier (look-back allocated).
//   FUSED_CULL = false : two-phase expand: neighbours are written to the edge
//                        frontier at their flattened edge position (no allocation).
// ------------------------------------------------------------------------------------
template <int B, bool PRED, bool FUSED_CULL>
__device__ __forceinline__ void expand_chunk(const BfsParams &p, const VertexFrontier &in, ExpandSmem<B, PRED> &s,
                                             int level, const VertexFrontier &vout, const EdgeFrontier &eout,
                                             unsigned &bar_phase, bool &any_discovered)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = B / 32;
    const int q = s.q, E = s.E, C = s.C, chunk = s.chunk;
    const int cs = chunk * C;
    const int ce = min(cs + C, E);
    const int new_level = level + 1;

    // ---- locate the chunk's vertices and load their runs ---------------------------
    const int i0 = locate<B, PRED>(in.P, q, cs, s);
    if (tid == 0) {
        s.n_warp_runs = 0;
        s.n_cta_runs = 0;
        s.out_count = 0;
    }
    // load tiles of entries from i0 until P >= ce
    int k = 0;
    for (int base = i0;; base += B) {
        const int i = base + tid;
        bool inside = false;
        if (i < q) {
            const int Pi = ld_cg(in.P + i);
            if (Pi < ce && i - i0 < kChunkMax) {
                inside = true;
                const int j = i - i0;
                const int start = max(Pi, cs);
                s.rel[j] = start - cs;
                s.colstart[j] = ld_cg(in.col + i) + (start - Pi);
                if (PRED) s.vert[j] = ld_cg(in.v + i);
            }
        }
        const int c = __syncthreads_count(inside);
        k += c;
        if (c < B) break;
    }
    if (tid == 0) {
        s.rel[k] = ce - cs;
        s.k = k;
    }
    __syncthreads();

    // ---- classify runs ---------------------------------------------------------------
    // thread-per-vertex; fine runs get disjoint slot ranges (warp scan + one
    // shared atomic per warp), warp and CTA runs are listed
    if (tid == 0) s.n_fine = 0;
    __syncthreads();
    for (int jb = 0; jb < k; jb += B) {
        const int j = jb + tid;
        int r = 0;
        bool fine = false;
        if (j < k) {
            r = s.rel[j + 1] - s.rel[j];
            if (r >= p.cta_thresh) {
                const int slot = atomicAdd(&s.n_cta_runs, 1);
                if (slot < kMaxCtaRuns) s.cta_runs[slot] = j;
            } else if (r >= p.warp_thresh) {
                s.warp_runs[atomicAdd(&s.n_warp_runs, 1)] = j;
            } else {
                fine = true;
            }
        }
        int len = fine ? r : 0;
        int incl = len;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += y;
        }
        int wbase = 0;
        if (lane == 31 && incl > 0) wbase = atomicAdd(&s.n_fine, incl);
        wbase = __shfl_sync(0xffffffffu, wbase, 31);
        if (fine) {
            const int off = wbase + incl - len;
            s.foff[j] = (uint16_t)off;
            for (int x = 0; x < len; x++) s.fmap[off + x] = (uint16_t)j;
        }
    }
    __syncthreads();

    // ---- CTA runs: stage the aligned body of each with one bulk copy -------------------
    const int n_cta = min(s.n_cta_runs, kMaxCtaRuns);
    bool bulk_issued = false;
    if (n_cta > 0) {
        if (tid == 0) {
            unsigned total_bytes = 0;
            int soff = 0;
            for (int r = 0; r < n_cta; r++) {
                const int j = s.cta_runs[r];
                const int c0 = s.colstart[j], len = s.rel[j + 1] - s.rel[j];
                const int b0 = (c0 + 3) & ~3, b1 = (c0 + len) & ~3;
                s.cta_stage_off[r] = soff;
                if (b1 > b0) {
                    total_bytes += (unsigned)(b1 - b0) * 4u;
                    soff += b1 - b0;
                }
            }
            if (total_bytes > 0) {
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&s.bar, total_bytes);
                for (int r = 0; r < n_cta; r++) {
                    const int j = s.cta_runs[r];
                    const int c0 = s.colstart[j], len = s.rel[j + 1] - s.rel[j];
                    const int b0 = (c0 + 3) & ~3, b1 = (c0 + len) & ~3;
                    if (b1 > b0)
                        bulk_g2s(&s.stage[s.cta_stage_off[r]], p.column_indices + b0, (unsigned)(b1 - b0) * 4u, &s.bar);
                }
                s.flag = 1;
            } else {
                s.flag = 0;
            }
        }
        __syncthreads();
        bulk_issued = s.flag != 0;
    }

    // visit one gathered neighbour (all lanes of the warp call it together)
    auto visit = [&](bool valid, int v, int u, int epos) {
        if (FUSED_CULL) {
            if (p.warp_cull) valid = warp_cull(valid, v);
            bool found = valid && discover<PRED>(p, v, u, new_level, p.precheck);
            push_out(found, v, s.out, &s.out_count);
        } else {
            if (valid) {
                eout.v[epos] = v;
                if (PRED) eout.pred[epos] = u;
            }
        }
    };

    // ---- fine-grained gather (scan-based) ---------------------------------------------
    {
        const int F = s.n_fine;
        constexpr int U = 4;
        for (int base = 0; base < F; base += B * U) {
            int v[U], u[U], epos[U];
            bool valid[U];
#pragma unroll
            for (int t = 0; t < U; t++) {
                const int slot = base + t * B + tid;
                valid[t] = slot < F;
                v[t] = -1;
                u[t] = -1;
                epos[t] = 0;
                if (valid[t]) {
                    const int j = s.fmap[slot];
                    const int x = slot - (int)s.foff[j];
                    v[t] = ld_stream(p.column_indices + s.colstart[j] + x);
                    if (PRED) u[t] = s.vert[j];
                    epos[t] = cs + s.rel[j] + x;
                }
            }
#pragma unroll
            for (int t = 0; t < U; t++) visit(valid[t], v[t], u[t], epos[t]);
        }
    }

    // ---- warp-cooperative gather -------------------------------------------------------
    {
        const int nwr = s.n_warp_runs;
        for (int r = warp; r < nwr; r += NW) {
            const int j = s.warp_runs[r];
            const int c0 = s.colstart[j], len = s.rel[j + 1] - s.rel[j];
            const int u = PRED ? s.vert[j] : -1;
            const int eb = cs + s.rel[j];
            constexpr int U = 4;
            for (int x0 = 0; x0 < len; x0 += 32 * U) {
                int v[U];
                bool valid[U];
#pragma unroll
                for (int t = 0; t < U; t++) {
                    const int x = x0 + t * 32 + lane;
                    valid[t] = x < len;
                    v[t] = valid[t] ? ld_stream(p.column_indices + c0 + x) : -1;
                }
#pragma unroll
                for (int t = 0; t < U; t++) visit(valid[t], v[t], u, eb + x0 + t * 32 + lane);
            }
        }
    }

    // ---- CTA-cooperative gather from the staged runs -----------------------------------
    if (n_cta > 0) {
        bool staged_ok = true;
        if (bulk_issued) {
            unsigned spins = 0;
            while (!mbar_try_wait(&s.bar, bar_phase)) {
                if (++spins > kSpinLimit) {
                    atomicOr(&p.st->error, kErrBulk);
                    staged_ok = false;
                    break;
                }
            }
            bar_phase ^= 1u;
        }
        // an expired wait leaves the staged words undefined: gather nothing from them
        for (int r = 0; r < (staged_ok ? n_cta : 0); r++) {
            const int j = s.cta_runs[r];
            const int c0 = s.colstart[j], len = s.rel[j + 1] - s.rel[j];
            const int b0 = (c0 + 3) & ~3, b1 = (c0 + len) & ~3;
            const int soff = s.cta_stage_off[r];
            const int u = PRED ? s.vert[j] : -1;
            const int eb = cs + s.rel[j];
            constexpr int U = 4;
            for (int x0 = 0; x0 < len; x0 += B * U) {
                int v[U];
                bool valid[U];
#pragma unroll
                for (int t = 0; t < U; t++) {
                    const int x = x0 + t * B + tid;
                    valid[t] = x < len;
                    v[t] = -1;
                    if (valid[t]) {
                        const int c = c0 + x;
                        v[t] = (c >= b0 && c < b1) ? s.stage[soff + (c - b0)] : ld_stream(p.column_indices + c);
                    }
                }
#pragma unroll
                for (int t = 0; t < U; t++) visit(valid[t], v[t], u, eb + x0 + t * B + tid);
            }
        }
    }
    __syncthreads();  // out[] complete; stage and lists free for the next chunk

    if (!FUSED_CULL) return;

    emit_frontier<B, PRED>(p, s, level, 0, vout, &p.st->q_len[(level + 1) & 1], &p.st->e_len[(level + 1) & 1],
                           any_discovered);
}

// ------------------------------------------------------------------------------------
// Level drivers
// ------------------------------------------------------------------------------------

// Chunk size for a level: enough chunks for every CTA, at most kChunkMax
__device__ __forceinline__ int level_chunk(int E, int c_max)
{
    int c = (E + (int)gridDim.x - 1) / (int)gridDim.x;
    c = (c + 31) & ~31;
    c = max(c, 256);
    return min(c, c_max);
}

// Shared epilogue of a non-persistent launch: the last CTA to finish
// advances the level and decides whether the search continues.
__device__ __forceinline__ void finish_launch(const BfsParams &p, int level, int q_next, bool limit_hit)
{
    if (threadIdx.x != 0) return;
    __threadfence();
    const unsigned t = atomicAdd(&p.st->finished, 1u);
    if (t == gridDim.x - 1) {
        __threadfence();
        p.st->finished = 0;
        p.st->cur_level = level + 1;
        const int qn = ld_cg(&p.st->q_len[(level + 1) & 1]);
        const bool done = (qn == 0) || limit_hit || (ld_cg(&p.st->error) != 0);
        if (done) p.st->done = 1;
        if (p.cond_handle) cudaGraphSetConditional((cudaGraphConditionalHandle)p.cond_handle, done ? 0u : 1u);
    }
    (void)q_next;
}

// Expand-contract (vertex frontier): one level per iteration of the loop.
template <int B, bool PRED>
__global__ void __launch_bounds__(B, 4) ec_kernel(BfsParams p)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ExpandSmem<B, PRED> &s = *reinterpret_cast<ExpandSmem<B, PRED> *>(smem_raw);
    __shared__ int s_ok;
    const int tid = threadIdx.x;
    if (tid == 0) mbar_init(&s.bar, 1);
    unsigned bar_phase = 0, generation = 0;
    bool any = false;
    int max_level_seen = -1;
    int level = ld_cg(&p.st->cur_level);
    bool limit_hit = false;
    __syncthreads();
    for (int iter = 0; iter < p.max_levels; iter++, level++) {
        if (tid == 0) {
            s.q = ld_cg(&p.st->q_len[level & 1]);
            s.E = ld_cg(&p.st->e_len[level & 1]);
            s.level = level;
            if (blockIdx.x == 0) p.st->chunk_ctr[(level + 1) % 3] = 0;
        }
        __syncthreads();
        const int q = s.q, E = s.E;
        const int dl = p.st->depth_limit;
        if (q == 0 || ld_cg(&p.st->error) != 0) break;
        if (dl >= 0 && level >= dl) {
            limit_hit = true;
            if (tid == 0 && blockIdx.x == 0) p.st->q_len[(level + 1) & 1] = 0;
            break;
        }
        const VertexFrontier in = p.vf[level & 1];
        const VertexFrontier out = p.vf[(level + 1) & 1];
        // per-level probe cache of P
        {
            const int stride0 = (q + 256) / 256;
            for (int t = tid; t <= 256; t += B) s.probe[t] = ld_cg(in.P + min(t * stride0, q));
        }
        if (tid == 0) {
            s.C = level_chunk(E, p.chunk_edges);
            s.nchunks = (E + s.C - 1) / s.C;
            if (s.nchunks > p.max_chunks) {
                atomicOr(&p.st->error, kErrOverflow);
                s.nchunks = 0;
            }
            if (blockIdx.x == 0) atomicAdd(&p.st->total_queued, (unsigned long long)q);
        }
        __syncthreads();
        any = false;
        while (true) {
            if (tid == 0) s.chunk = (int)atomicAdd(&p.st->chunk_ctr[level % 3], 1u);
            __syncthreads();
            if (s.chunk >= s.nchunks) break;
            expand_chunk<B, PRED, true>(p, in, s, level, out, p.ef[0], bar_phase, any);
            __syncthreads();
        }
        if (any) max_level_seen = level + 1;
        if (!p.persistent) break;
        if (tid == 0 && blockIdx.x == 0) p.st->cur_level = level + 1;
        if ((int)blockIdx.x == p.skip_arrival_cta) {
            if (tid == 0) atomicOr(&p.st->error, kErrInjected);
            return;  // never arrives: the others' bounded waits must expire
        }
        if (!grid_barrier(&p.st->barrier, generation, &p.st->error, &s_ok)) break;
    }
    if (tid == 0 && max_level_seen >= 0) atomicMax(&p.st->max_level, max_level_seen);
    if (p.persistent) {
        if (tid == 0 && blockIdx.x == 0) {
            p.st->cur_level = level;
            p.st->done = 1;
        }
    } else {
        finish_launch(p, level, 0, limit_hit);
    }
}


// ------------------------------------------------------------------------------------
// Edge-frontier strategies (contract-expand, two-phase, hybrid)
// ------------------------------------------------------------------------------------

// Contraction of one chunk of an edge frontier: each item's visited bit is
// test-and-set; a first visit labels the vertex with the current level (or
// its predecessor) and the survivors become the vertex frontier vf[0].
template <int B, bool PRED>
__device__ __forceinline__ void contract_chunk(const BfsParams &p, ExpandSmem<B, PRED> &s, const EdgeFrontier &in,
                                               int level, bool &any_discovered)
{
    const int tid = threadIdx.x;
    const int C = s.C, chunk = s.chunk, q = s.q;
    const int cs = chunk * C, ce = min(cs + C, q);
    if (tid == 0) s.out_count = 0;
    __syncthreads();
    constexpr int U = 4;
    for (int base = cs; base < ce; base += B * U) {
        int v[U], u[U];
        bool valid[U];
#pragma unroll
        for (int t = 0; t < U; t++) {
            const int i = base + t * B + tid;
            valid[t] = i < ce;
            v[t] = valid[t] ? ld_cg(in.v + i) : -1;
            u[t] = (PRED && valid[t]) ? ld_cg(in.pred + i) : -1;
        }
#pragma unroll
        for (int t = 0; t < U; t++) {
            bool ok = valid[t];
            if (p.warp_cull) ok = warp_cull(ok, v[t]);
            const bool found = ok && discover<PRED>(p, v[t], u[t], level, p.precheck);
            push_out(found, v[t], s.out, &s.out_count);
        }
    }
    __syncthreads();
    emit_frontier<B, PRED>(p, s, level, 1, p.vf[0], &p.st->vq_len, &p.st->ve_len, any_discovered);
}

// Per level: contract the edge frontier into vf[0], then expand vf[0] into
// the next edge frontier (flattened edge positions, no allocation needed).
// phase_mask selects the phases of a non-persistent launch; a persistent
// launch runs both with a grid barrier after each.  With `hybrid`, a
// persistent launch returns when the edge frontier exceeds
// gridDim * saturation items (SATURATION_QUIT, enactor_hybrid.cuh:571).
template <int B, bool PRED>
__global__ void __launch_bounds__(B, 4) edge_kernel(BfsParams p)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ExpandSmem<B, PRED> &s = *reinterpret_cast<ExpandSmem<B, PRED> *>(smem_raw);
    __shared__ int s_ok;
    const int tid = threadIdx.x;
    if (tid == 0) mbar_init(&s.bar, 1);
    unsigned bar_phase = 0, generation = 0;
    int max_level_seen = -1;
    int level = ld_cg(&p.st->cur_level);
    bool limit_hit = false, saturated = false, completed_level = false, failed = false;
    __syncthreads();
    for (int iter = 0; iter < p.max_levels; iter++, level++) {
        const int in_idx = p.edge_pingpong ? (level & 1) : 0;
        const int out_idx = p.edge_pingpong ? ((level + 1) & 1) : 0;
        if (p.phase_mask & 1) {
            const int pass = 2 * level;
            if (tid == 0) {
                s.q = ld_cg(&p.st->q_len[level & 1]);
                if (blockIdx.x == 0) p.st->chunk_ctr[(pass + 1) % 3] = 0;
            }
            __syncthreads();
            const int q = s.q;
            if (ld_cg(&p.st->error) != 0) {
                failed = true;
                break;
            }
            if (q == 0) {
                if (tid == 0 && blockIdx.x == 0) p.st->vq_len = p.st->ve_len = 0;
                break;
            }
            if (p.hybrid && p.persistent && q > (int)gridDim.x * p.saturation) {
                saturated = true;
                break;
            }
            if (tid == 0) {
                s.C = level_chunk(q, p.chunk_edges);
                s.nchunks = (q + s.C - 1) / s.C;
                if (s.nchunks > p.max_chunks) {
                    atomicOr(&p.st->error, kErrOverflow);
                    s.nchunks = 0;
                }
                if (blockIdx.x == 0) atomicAdd(&p.st->total_queued, (unsigned long long)q);
            }
            __syncthreads();
            bool any = false;
            while (true) {
                if (tid == 0) s.chunk = (int)atomicAdd(&p.st->chunk_ctr[pass % 3], 1u);
                __syncthreads();
                if (s.chunk >= s.nchunks) break;
                contract_chunk<B, PRED>(p, s, p.ef[in_idx], level, any);
                __syncthreads();
            }
            if (any) max_level_seen = max(max_level_seen, level);
            if (p.persistent) {
                if ((int)blockIdx.x == p.skip_arrival_cta) {
                    if (tid == 0) atomicOr(&p.st->error, kErrInjected);
                    return;
                }
                if (!grid_barrier(&p.st->barrier, generation, &p.st->error, &s_ok)) {
                    failed = true;
                    break;
                }
            }
        }
        const int dl = p.st->depth_limit;
        if (dl >= 0 && level >= dl) {
            limit_hit = true;
            if (tid == 0 && blockIdx.x == 0) p.st->q_len[(level + 1) & 1] = 0;
            break;
        }
        if (p.phase_mask & 2) {
            const int pass = 2 * level + 1;
            if (tid == 0) {
                s.q = ld_cg(&p.st->vq_len);
                s.E = ld_cg(&p.st->ve_len);
                if (blockIdx.x == 0) p.st->chunk_ctr[(pass + 1) % 3] = 0;
            }
            __syncthreads();
            const int q = s.q, E = s.E;
            if (E > p.ecap) {
                if (tid == 0) atomicOr(&p.st->error, kErrOverflow);
                failed = true;
                break;
            }
            if (tid == 0 && blockIdx.x == 0) p.st->q_len[(level + 1) & 1] = q == 0 ? 0 : E;
            if (q > 0) {
                const int stride0 = (q + 256) / 256;
                for (int t = tid; t <= 256; t += B) s.probe[t] = ld_cg(p.vf[0].P + min(t * stride0, q));
                if (tid == 0) {
                    s.C = level_chunk(E, p.chunk_edges);
                    s.nchunks = (E + s.C - 1) / s.C;
                    if (s.nchunks > p.max_chunks) {
                        atomicOr(&p.st->error, kErrOverflow);
                        s.nchunks = 0;
                    }
                }
                __syncthreads();
                bool unused = false;
                while (true) {
                    if (tid == 0) s.chunk = (int)atomicAdd(&p.st->chunk_ctr[pass % 3], 1u);
                    __syncthreads();
                    if (s.chunk >= s.nchunks) break;
                    expand_chunk<B, PRED, false>(p, p.vf[0], s, level, p.vf[1], p.ef[out_idx], bar_phase, unused);
                    __syncthreads();
                }
            }
            completed_level = true;
            if (p.persistent) {
                if (tid == 0 && blockIdx.x == 0) p.st->cur_level = level + 1;
                if (!grid_barrier(&p.st->barrier, generation, &p.st->error, &s_ok)) {
                    failed = true;
                    break;
                }
            }
        }
        if (!p.persistent) break;
    }
    if (tid == 0 && max_level_seen >= 0) atomicMax(&p.st->max_level, max_level_seen);
    if (p.persistent) {
        if (tid == 0 && blockIdx.x == 0) {
            p.st->cur_level = level;
            if (saturated)
                p.st->saturated = 1;
            else
                p.st->done = 1;
        }
    } else if (completed_level || limit_hit) {
        finish_launch(p, level, 0, limit_hit);
    }
    (void)failed;
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
    const int src = p.st->src;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int src_label = PRED ? -2 : 0;
    if (FULL) {
        for (long long i = t0; i < p.nodes; i += stride) p.labels[i] = (VERTEX_FRONTIER && i == src) ? src_label : -1;
        for (long long w = t0; w < p.mask_words; w += stride)
            p.mask[w] = (VERTEX_FRONTIER && w == (src >> 5)) ? (1u << (src & 31)) : 0u;
    } else if (VERTEX_FRONTIER && t0 == 0) {
        p.labels[src] = src_label;
        p.mask[src >> 5] = 1u << (src & 31);
    }
    if (t0 == 0) {
        SearchState *st = p.st;
        const int r0 = p.row_offsets[src], r1 = p.row_offsets[src + 1];
        st->chunk_ctr[0] = st->chunk_ctr[1] = st->chunk_ctr[2] = 0;
        st->cur_level = 0;
        st->epoch += 1ull << 24;
        st->barrier = 0;
        st->error = 0;
        st->max_level = 0;
        st->done = 0;
        st->saturated = 0;
        st->total_queued = 0;
        st->finished = 0;
        st->q_len[1] = st->e_len[1] = 0;
        if (VERTEX_FRONTIER) {
            const int deg = r1 - r0;
            st->q_len[0] = deg > 0 ? 1 : 0;
            st->e_len[0] = deg;
            p.vf[0].v[0] = src;
            p.vf[0].col[0] = r0;
            p.vf[0].P[0] = 0;
            p.vf[0].P[1] = deg;
        } else {
            // edge frontier: the source is the only item; its predecessor is -2
            st->q_len[0] = 1;
            st->e_len[0] = 0;
            p.ef[0].v[0] = src;
            if (PRED) p.ef[0].pred[0] = -2;
        }
    }
}

}  // namespace dev
}  // namespace b40c
