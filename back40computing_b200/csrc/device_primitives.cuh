// Device-side building blocks for the BFS kernels (sm_100a):
// cache-qualified loads, the bounded software grid barrier, bulk-copy
// (cp.async.bulk) staging with an mbarrier, and the decoupled look-back used
// to allocate frontier-queue slots.
//
// Every spin in this file is bounded: after kSpinLimit polls the waiter sets
// an error bit in the search state and gives up, so a missing arrival can
// never hang the GPU (the reference's GlobalBarrier::Sync spins forever,
// util/global_barrier.cuh:99-121).
#pragma once
#include <cstdint>

namespace b40c {
namespace dev {

constexpr unsigned kErrOverflow = 1u;       // a frontier queue would overflow
constexpr unsigned kErrBarrier = 2u;        // grid barrier wait expired
constexpr unsigned kErrLookback = 4u;       // look-back wait expired
constexpr unsigned kErrBulk = 8u;           // bulk-copy wait expired
constexpr unsigned kErrLevels = 32u;        // more levels than vertices: a captured loop was stopped
constexpr unsigned kErrFrontier = 64u;      // a deferred bottom-up frontier did not match its counted size
constexpr unsigned kSpinLimit = 1u << 22;   // polls before a wait gives up (~1-2 s with backoff)

// ---- L2 residency -------------------------------------------------------------
// Column indices are read once per search (a stream larger than L2); they are
// loaded with an evict-first L2 policy so that what levels and searches read
// again -- visited masks, the batched search's frontier and visited masks,
// row offsets, hub pairs, labels -- stays in L2.  The batched search's random
// mask gathers are marked evict-last.  B40C_L2_HINTS=0 builds without hints.
#ifndef B40C_L2_HINTS
#define B40C_L2_HINTS 1
#endif
__device__ __forceinline__ uint64_t l2_evict_first()
{
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ uint64_t l2_evict_last()
{
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// ---- loads / stores ----------------------------------------------------------
__device__ __forceinline__ int ld_cg(const int *p)
{
    int v;
    asm volatile("ld.global.cg.s32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ unsigned ld_cg(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
// streaming read-only load (column indices: read once per search)
__device__ __forceinline__ int ld_stream(const int *p)
{
    int v;
#if B40C_L2_HINTS
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(l2_evict_first()));
#else
    asm volatile("ld.global.nc.L1::no_allocate.s32 %0, [%1];" : "=r"(v) : "l"(p));
#endif
    return v;
}
__device__ __forceinline__ int4 ld_stream4(const int4 *p)
{
    int4 v;
#if B40C_L2_HINTS
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p), "l"(l2_evict_first()));
#else
    asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
#endif
    return v;
}
// coherent (L2) 64-bit load of data read again and again (the batched search's
// frontier and visited masks): evict-last in L2
__device__ __forceinline__ unsigned long long ld_keep64(const unsigned long long *p)
{
    unsigned long long v;
#if B40C_L2_HINTS
    asm volatile("ld.global.cg.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(l2_evict_last()));
#else
    asm volatile("ld.global.cg.u64 %0, [%1];" : "=l"(v) : "l"(p));
#endif
    return v;
}
// store of data written once and not read again by the search (batch labels)
__device__ __forceinline__ void st_stream(int *p, int v)
{
#if B40C_L2_HINTS
    asm volatile("st.global.L1::no_allocate.L2::cache_hint.s32 [%0], %1, %2;" ::"l"(p), "r"(v), "l"(l2_evict_first())
                 : "memory");
#else
    *p = v;
#endif
}
// Column indices [e, hi) of one list, four positions per call from one
// 16-byte load: the load covers the aligned quad holding e (aligned by
// address, so any 4-byte aligned array works; positions outside [e, hi) come
// back as -1); where the quad would leave the array [0, m) the positions are
// read one by one.  Returns the next position to read.
__device__ __forceinline__ int ld_quad(const int32_t *ci, int m, int e, int hi, int (&nb)[4])
{
    if (e >= hi) {
        nb[0] = nb[1] = nb[2] = nb[3] = -1;
        return e;
    }
    const int mis = (int)((reinterpret_cast<uintptr_t>(ci) >> 2) & 3u);
    const int ea = ((e + mis) & ~3) - mis;
    if (ea >= 0 && ea + 4 <= m) {
        const int4 x = ld_stream4(reinterpret_cast<const int4 *>(ci + ea));
        nb[0] = (ea >= e && ea < hi) ? x.x : -1;
        nb[1] = (ea + 1 >= e && ea + 1 < hi) ? x.y : -1;
        nb[2] = (ea + 2 >= e && ea + 2 < hi) ? x.z : -1;
        nb[3] = (ea + 3 >= e && ea + 3 < hi) ? x.w : -1;
        return ea + 4;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) nb[k] = (e + k < hi) ? ld_stream(ci + e + k) : -1;
    return e + 4;
}
// read-only load through L1 (row offsets)
__device__ __forceinline__ int ld_ro(const int *p) { return __ldg(p); }
// visited-word pre-check: weak load that may hit a stale L1 line; a stale
// line can only show fewer bits set (bits only ever go 0 -> 1), so it never
// drops an undiscovered vertex -- the atomic test-and-set decides.
__device__ __forceinline__ unsigned ld_mask(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.global.ca.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---- bounded grid barrier ------------------------------------------------------
// Monotone arrival counter: the g-th barrier of a launch completes when the
// counter reaches g * gridDim.x; waiters poll the counter itself (one round
// trip less than a separate release flag).  The counter sits on its own cache
// line, away from the frontier counters' atomics.  It is zeroed before each
// persistent launch.  Requires every CTA to be resident (cooperative launch).
// Returns false when the wait expired or an error was seen while waiting; an
// error reported just before the barrier completed is left to the callers'
// next read of the error word (every caller reads it before its next step, the
// same value in every CTA), which saves a round trip per barrier.
// `count` CTAs take part (the whole grid unless given: a sub-grid barrier has
// its own counter).  `spin_limit` polls bound the wait (kSpinLimit in
// production; tests pass a short limit to make a wait run out quickly).
__device__ __forceinline__ bool grid_barrier(unsigned long long *counter, unsigned &generation, unsigned *error_word,
                                             int *s_flag, unsigned count = 0, unsigned spin_limit = kSpinLimit)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        generation++;
        const unsigned long long target = (unsigned long long)generation * (count ? count : gridDim.x);
        __threadfence();
        atomicAdd(counter, 1ull);
        unsigned spins = 0;
        int ok = 1;
        while (ld_acquire(counter) < target) {
            if (++spins > spin_limit) {
                atomicOr(error_word, kErrBarrier);
                ok = 0;
                break;
            }
            if ((spins & 7) == 0 && ld_cg(error_word) != 0) {
                ok = 0;
                break;
            }
            __nanosleep(spins < 64 ? 32 : 256);
        }
        __threadfence();
        *s_flag = ok;
    }
    __syncthreads();
    return *s_flag != 0;
}

// For a CTA that runs levels while `outside` other CTAs of the grid wait at the
// next grid barrier (generation `generation` + 1): called by thread 0 before the
// CTA first overwrites state those CTAs read at the start of the pass.  They
// arrive right after that read, so once the counter shows their `outside`
// arrivals (the barrier's own count starts at generation * gridDim.x: no CTA
// can pass it while this one has not arrived) the state is free.  Bounded like
// grid_barrier; returns false with kErrBarrier set when the wait expired, or
// when another error was seen.
__device__ __forceinline__ bool wait_outside_arrivals(const unsigned long long *counter, unsigned generation,
                                                      unsigned outside, unsigned *error_word,
                                                      unsigned spin_limit = kSpinLimit)
{
    const unsigned long long target = (unsigned long long)generation * gridDim.x + outside;
    unsigned spins = 0;
    while (ld_acquire(counter) < target) {
        if (++spins > spin_limit) {
            atomicOr(error_word, kErrBarrier);
            return false;
        }
        if ((spins & 7) == 0 && ld_cg(error_word) != 0) return false;
        __nanosleep(spins < 64 ? 32 : 256);
    }
    return true;
}

// ---- mbarrier + bulk copy (cp.async.bulk, global -> this CTA's shared) ----------
__device__ __forceinline__ unsigned smem_addr(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// Copies `bytes` (multiple of 16; both addresses 16-byte aligned) into shared memory.
__device__ __forceinline__ void bulk_g2s(void *smem_dst, const void *gmem_src, unsigned bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---- decoupled look-back ---------------------------------------------------------
// One slot per work chunk of a level.  `status` = epoch << 2 | flag, where flag
// 1 = aggregate published, 2 = inclusive prefix published; the epoch is
// unique per (search, level), so slots never need clearing between levels.
// Values are (count << 32 | degree_sum) pairs that add component-wise.
struct alignas(32) LookbackSlot {
    unsigned long long status;
    unsigned long long aggregate;
    unsigned long long inclusive;
    unsigned long long pad;
};
constexpr unsigned long long kFlagAggregate = 1ull;
constexpr unsigned long long kFlagInclusive = 2ull;

__device__ __forceinline__ void lookback_publish(LookbackSlot *slot, unsigned long long epoch,
                                                 unsigned long long flag, unsigned long long value)
{
    if (flag == kFlagAggregate)
        st_relaxed(&slot->aggregate, value);
    else
        st_relaxed(&slot->inclusive, value);
    st_release(&slot->status, (epoch << 2) | flag);
}

// Called by one full warp.  Returns the exclusive prefix of chunk `chunk`
// (sum of the values of chunks 0..chunk-1); chunk 0 must not call it.  On
// a wait that expires it sets kErrLookback and returns ~0ull.
__device__ __forceinline__ unsigned long long lookback_exclusive(LookbackSlot *slots, unsigned chunk,
                                                                 unsigned long long epoch, unsigned *error_word,
                                                                 unsigned spin_limit = kSpinLimit)
{
    const unsigned lane = threadIdx.x & 31;
    unsigned long long prefix = 0;
    long long window_end = (long long)chunk - 1;  // nearest predecessor
    unsigned spins = 0;
    while (true) {
        long long j = window_end - lane;
        unsigned long long flag = kFlagInclusive, value = 0;
        if (j >= 0) {
            // wait until this lane's slot carries a flag of the current epoch
            while (true) {
                unsigned long long st = ld_acquire(&slots[j].status);
                if ((st >> 2) == epoch && (st & 3ull) != 0) {
                    flag = st & 3ull;
                    value = (flag == kFlagInclusive) ? ld_relaxed(&slots[j].inclusive)
                                                     : ld_relaxed(&slots[j].aggregate);
                    break;
                }
                if (++spins > spin_limit) {
                    atomicOr(error_word, kErrLookback);
                    flag = kFlagInclusive;
                    value = ~0ull;
                    break;
                }
                __nanosleep(spins < 32 ? 20 : 200);
            }
        }
        unsigned incl = __ballot_sync(0xffffffffu, flag == kFlagInclusive);
        unsigned bad = __ballot_sync(0xffffffffu, value == ~0ull);
        if (bad) return ~0ull;
        // only lanes up to (and including) the nearest inclusive slot count
        int stop = incl ? (__ffs(incl) - 1) : 31;
        unsigned long long contrib = ((int)lane <= stop) ? value : 0ull;
        for (int off = 16; off > 0; off >>= 1) contrib += __shfl_down_sync(0xffffffffu, contrib, off);
        contrib = __shfl_sync(0xffffffffu, contrib, 0);
        prefix += contrib;
        if (incl) return prefix;
        window_end -= 32;
    }
}

}  // namespace dev
}  // namespace b40c
