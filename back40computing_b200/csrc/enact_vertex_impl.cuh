// The expand-contract enactor's body for one CTA size (included by the
// per-size translation units enact_vertex_<B>.cu, so the kernel variants of
// each size compile in parallel).
#pragma once
#include "launch_common.cuh"

namespace b40c {
namespace rt {

template <int B, bool PRED>
int enact_ec_t(b40c_bfs_problem *p, int mode, int32_t src, int max_grid, const b40c_bfs_policy &pol,
               int32_t depth_limit, bool direction_opt)
{
    int rc;
    if ((rc = ensure_vf(p, 0, cap_of(p->queue_sizing, p->nodes)))) return rc;
    if ((rc = ensure_vf(p, 1, cap_of(p->queue_sizing, p->nodes)))) return rc;
    if ((rc = ensure_slots(p))) return rc;
    if (direction_opt && pol.bottom_up_hub_probes > 0 && (rc = ensure_hubs(p))) return rc;
    const bool lists = direction_opt && !PRED && pol.bottom_up_list > 0;
    if (lists && (rc = ensure_unvisited_lists(p))) return rc;
    BfsParams k = make_params(p, pol);
    k.direction_opt = direction_opt ? 1 : 0;
    if (!direction_opt) k.hub2 = nullptr;
    if (lists) {
        // distance searches: bottom-up levels after the first one scan the unvisited list
        k.ul[0] = p->d_ul[0];
        k.ul[1] = p->d_ul[1];
    }
    // distance searches with unvisited lists run the kernel variant that
    // carries list mode; the others keep the leaner code
    const bool lists_kernel = direction_opt && !PRED && pol.bottom_up_list > 0;
    // fused searches with a sub-grid threshold run the variant that carries the
    // sub-grid phase (not combined with list mode)
    const bool subgrid_kernel = !lists_kernel && mode == B40C_ENACT_FUSED && pol.subgrid_frontier_edges > 0;
    // plain expand-contract searches (and directed graphs) never go bottom-up:
    // they run the top-down-only variants; list mode and the sub-grid phase are
    // built for 256-thread CTAs only
    const void *kern = nullptr;
    if (lists_kernel || subgrid_kernel) {
        if constexpr (B == 256) {
            kern = lists_kernel    ? (const void *)dev::ec_kernel<256, false, true>
                   : direction_opt ? (const void *)dev::ec_kernel<256, PRED, false, true>
                                   : (const void *)dev::ec_kernel<256, PRED, false, true, false>;
        } else {
            return b40c::fail(B40C_ERROR_INVALID_VALUE,
                              "policy.threads %d: bottom-up list mode and the sub-grid phase need 256", B);
        }
    } else {
        kern = direction_opt ? (const void *)dev::ec_kernel<B, PRED, false>
                             : (const void *)dev::ec_kernel<B, PRED, false, false, false>;
    }
    const size_t smem = kernel_smem<dev::ExpandSmem<B, PRED>>(pol);
    int grid = 0;
    if ((rc = persistent_grid(p, kern, pol, max_grid, smem, &grid))) return rc;
    if ((rc = begin_enact(p, src, depth_limit))) return rc;
    if ((rc = begin_instrumented(p))) return rc;
    if (mode == B40C_ENACT_GRAPH) {
        if ((rc = mark_search_start(p))) return rc;
        KernelNode init{init_kernel_ptr<PRED>(true, true), dim3(init_grid(p, true)), dim3(kThreads), 0, k};
        KernelNode body[1] = {{kern, dim3(grid), dim3(B), smem, k}};
        const int slot = direction_opt ? B40C_HYBRID + 1 : B40C_EXPAND_CONTRACT;
        if ((rc = run_graph(p, slot, init, body, 1))) return rc;
        return finish_timing(p);
    }
    // the source and depth limit travel as kernel arguments of the init kernel
    // (no host-to-device copy in the search's stream)
    k.src_by_value = 1;
    k.src_arg = src;
    k.depth_arg = depth_limit;
    if ((rc = launch_init<PRED>(p, k, true, p->needs_init))) return rc;
    if ((rc = mark_search_start(p))) return rc;
    if (mode == B40C_ENACT_FUSED) {
        k.persistent = 1;
        k.max_levels = INT32_MAX;
        k.skip_arrival_cta = injected_skip_cta();
        k.late_start_ns = injected_late_start_ns();
        if ((rc = launch_cooperative(p, kern, grid, B, smem, k, "cooperative launch of the expand-contract kernel")))
            return rc;
    } else if (mode == B40C_ENACT_ITERATIVE) {
        // one launch per level; the host reads the next frontier's size
        for (int level = 0;; level++) {
            if ((rc = read_state(p))) return rc;
            if (p->h_st->error || p->h_st->done) break;
            const int q = qe_count(p->h_st->qe[level % 3]), E = qe_edges(p->h_st->qe[level % 3]);
            if (q == 0) break;
            int g = std::max(1, std::min(grid, (E + dev::kChunkGrain - 1) / dev::kChunkGrain));
            if (direction_opt) g = grid;  // a bottom-up level spans every vertex
            if ((rc = launch_plain(p, kern, g, B, smem, k, "expand-contract level launch"))) return rc;
        }
    } else {
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "unknown enact mode %d", mode);
    }
    return finish_timing(p);
}

// One CTA size's entry, instantiated in enact_vertex_<B>.cu.
template <int B>
int enact_vertex_b(b40c_bfs_problem *p, int mode, int32_t src, int max_grid, const b40c_bfs_policy &pol,
                   int32_t depth_limit, bool direction_optimizing)
{
    return p->mark_pred ? enact_ec_t<B, true>(p, mode, src, max_grid, pol, depth_limit, direction_optimizing)
                        : enact_ec_t<B, false>(p, mode, src, max_grid, pol, depth_limit, direction_optimizing);
}

}  // namespace rt
}  // namespace b40c
