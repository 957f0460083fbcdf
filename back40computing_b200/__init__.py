"""B200-native single-GPU BFS (the b40c/graph/bfs path) behind a C ABI.

The compute path is libb40c_bfs.so (sm_100a kernels + host runtime, built
in-tree by ``python -m back40computing_b200.build``).  This package holds
the Python mirror of the reference interface used by tests, the benchmark
and the query server; it has no CPU fallback.
"""
from . import _native
from ._native import B40cError, device_count
from .graph import (CsrGraph, BuildGrid2dGraph, BuildGrid3dGraph, BuildRmatGraph, BuildRandomGraph,
                    BuildRandomRegularishGraph, BuildMarketGraph, BuildDimacsGraph, BuildMetisGraph, sample_sources)
from .bfs import (CsrProblem, EnactorExpandContract, EnactorContractExpand, EnactorTwoPhase, EnactorHybrid,
                  EnactorDirectionOptimizing, search, default_policy, VERTEX_FRONTIERS, EDGE_FRONTIERS, MIXED_FRONTIERS, EXPAND_CONTRACT,
                  CONTRACT_EXPAND, TWO_PHASE, HYBRID, DIRECTION_OPTIMIZING)

__all__ = [
    "B40cError", "device_count", "CsrGraph", "BuildGrid2dGraph", "BuildGrid3dGraph", "BuildRmatGraph",
    "BuildRandomGraph", "BuildRandomRegularishGraph", "BuildMarketGraph", "BuildDimacsGraph", "BuildMetisGraph",
    "sample_sources", "CsrProblem", "EnactorExpandContract",
    "EnactorContractExpand", "EnactorTwoPhase", "EnactorHybrid", "search", "default_policy",
]
