// Edge-frontier enactors: contract-expand (two O(m) edge frontiers), two-phase
// (one O(n) vertex and one O(m) edge frontier) and hybrid (fused
// contract-expand while the frontier is small, two-phase launches while it is
// saturated; EnactorHybrid::EnactSearch, enactor_hybrid.cuh:279-551).
#include "launch_common.cuh"

namespace b40c {
namespace rt {

namespace {

template <int B, bool PRED>
int enact_edge_t(b40c_bfs_problem *p, int strategy, int mode, int32_t src, int max_grid, const b40c_bfs_policy &pol,
                 int32_t depth_limit)
{
    int rc;
    const bool pingpong = strategy == B40C_CONTRACT_EXPAND || strategy == B40C_HYBRID;
    const int64_t ecap = cap_of(p->queue_sizing, p->edges), vcap = cap_of(p->queue_sizing, p->nodes);
    if ((rc = ensure_ef(p, 0, ecap))) return rc;
    if (pingpong && (rc = ensure_ef(p, 1, ecap))) return rc;
    if ((rc = ensure_vf(p, 0, vcap))) return rc;
    if ((rc = ensure_slots(p))) return rc;
    BfsParams k = make_params(p, pol);
    // hybrid's hand-off: saturation_quit queue items per 256 threads of the grid,
    // so the frontier size at which it leaves the fused kernel does not move
    // with the CTA size (the grid of 512-thread CTAs has half as many)
    k.saturation = (int32_t)std::max<int64_t>(1, (int64_t)pol.saturation_quit * B / 256);
    k.edge_pingpong = pingpong ? 1 : 0;
    k.vcap = (int32_t)p->vcap[0];
    k.ecap = (int32_t)(pingpong ? std::min(p->ecap[0], p->ecap[1]) : p->ecap[0]);
    const void *kern = (const void *)dev::edge_kernel<B, PRED>;
    const size_t smem = kernel_smem<dev::ExpandSmem<B, PRED>>(pol);
    int grid = 0;
    if ((rc = persistent_grid(p, kern, pol, max_grid, smem, &grid))) return rc;
    if ((rc = begin_enact(p, src, depth_limit))) return rc;
    if ((rc = begin_instrumented(p))) return rc;

    BfsParams kc = k, kx = k;  // one-phase launches: contract, expand
    kc.phase_mask = 1;
    kx.phase_mask = 2;
    kc.max_levels = kx.max_levels = 1;

    if (mode == B40C_ENACT_GRAPH) {
        if ((rc = mark_search_start(p))) return rc;
        KernelNode init{init_kernel_ptr<PRED>(false, true), dim3(init_grid(p, true)), dim3(kThreads), 0, k};
        KernelNode body[2] = {{kern, dim3(grid), dim3(B), smem, kc}, {kern, dim3(grid), dim3(B), smem, kx}};
        if ((rc = run_graph(p, strategy, init, body, 2))) return rc;
        return finish_timing(p);
    }
    if ((rc = upload_source(p))) return rc;
    if ((rc = launch_init<PRED>(p, k, false, p->needs_init))) return rc;
    if ((rc = mark_search_start(p))) return rc;

    // one level as two launches (contract, expand); returns with the state read back
    auto two_phase_level = [&]() -> int {
        int r;
        if ((r = launch_plain(p, kern, grid, B, smem, kc, "contract launch"))) return r;
        if ((r = launch_plain(p, kern, grid, B, smem, kx, "expand launch"))) return r;
        return read_state(p);
    };

    if (strategy == B40C_HYBRID && mode == B40C_ENACT_FUSED) {
        BfsParams kf = k;
        kf.persistent = 1;
        kf.phase_mask = 3;
        kf.hybrid = 1;
        kf.max_levels = INT32_MAX;
        kf.skip_arrival_cta = injected_skip_cta();
        kf.late_start_ns = injected_late_start_ns();
        const int threshold = grid * k.saturation;
        while (true) {
            CUDA_TRY(cudaMemsetAsync(&p->st->barrier, 0, sizeof(unsigned long long), p->stream), "barrier reset");
            CUDA_TRY(cudaMemsetAsync(&p->st->saturated, 0, sizeof(int32_t), p->stream), "flag reset");
            if ((rc = launch_cooperative(p, kern, grid, B, smem, kf, "cooperative launch of the contract-expand kernel")))
                return rc;
            if ((rc = read_state(p))) return rc;
            if (p->h_st->error || p->h_st->done || !p->h_st->saturated) break;
            // saturated: two-phase levels until the frontier falls back under the threshold
            bool finished = false;
            while (true) {
                if ((rc = two_phase_level())) return rc;
                const SearchState &h = *p->h_st;
                if (h.error || h.done || qe_count(h.qe[(2 * h.cur_level) % 3]) == 0) {
                    finished = true;
                    break;
                }
                if (qe_count(h.qe[(2 * h.cur_level) % 3]) <= threshold) break;
            }
            if (finished) break;
        }
    } else if (mode == B40C_ENACT_FUSED) {
        BfsParams kf = k;
        kf.persistent = 1;
        kf.phase_mask = 3;
        kf.max_levels = INT32_MAX;
        kf.skip_arrival_cta = injected_skip_cta();
        kf.late_start_ns = injected_late_start_ns();
        if ((rc = launch_cooperative(p, kern, grid, B, smem, kf, "cooperative launch of the contract-expand kernel")))
            return rc;
    } else if (mode == B40C_ENACT_ITERATIVE) {
        if ((rc = read_state(p))) return rc;
        while (!(p->h_st->error || p->h_st->done || qe_count(p->h_st->qe[(2 * p->h_st->cur_level) % 3]) == 0))
            if ((rc = two_phase_level())) return rc;
    } else {
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "unknown enact mode %d", mode);
    }
    return finish_timing(p);
}

}  // namespace

int enact_edge(b40c_bfs_problem *p, int strategy, int mode, int32_t src, int max_grid, const b40c_bfs_policy &pol,
               int32_t depth_limit)
{
#define B40C_EDGE(B)                                                                      \
    (p->mark_pred ? enact_edge_t<B, true>(p, strategy, mode, src, max_grid, pol, depth_limit) \
                  : enact_edge_t<B, false>(p, strategy, mode, src, max_grid, pol, depth_limit))
    switch (pol.threads) {
    case 128: return B40C_EDGE(128);
    case 512: return B40C_EDGE(512);
    default: return B40C_EDGE(256);
    }
#undef B40C_EDGE
}

}  // namespace rt
}  // namespace b40c
