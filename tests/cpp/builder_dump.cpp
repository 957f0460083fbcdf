// Builds one graph with the C++ builder headers after srand(seed) and writes
// it as int64 nodes, int64 edges, int32 row_offsets[nodes + 1],
// int32 column_indices[edges] to the output file.
//   builder_dump <out> <seed> <grid2d W | grid3d W | rmat N M U | random N M U | rr N D |
//                              market FILE U | dimacs FILE U SPLICE | metis FILE>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>

#include <b40c/graph/builder/grid2d.cuh>
#include <b40c/graph/builder/grid3d.cuh>
#include <b40c/graph/builder/random.cuh>
#include <b40c/graph/builder/rmat.cuh>
#include <b40c/graph/builder/rr.cuh>
#include <b40c/graph/builder/market.cuh>
#include <b40c/graph/builder/dimacs.cuh>
#include <b40c/graph/builder/metis.cuh>

using namespace b40c::graph;

int main(int argc, char **argv)
{
    if (argc < 5) return 2;
    srand((unsigned)atoi(argv[2]));
    std::string t = argv[3];
    CsrGraph<int, int, int> g;
    int rc = -1;
    if (t == "grid2d") rc = builder::BuildGrid2dGraph<false>(atoi(argv[4]), g);
    else if (t == "grid3d") rc = builder::BuildGrid3dGraph<false>(atoi(argv[4]), g);
    else if (t == "rmat" && argc > 6) rc = builder::BuildRmatGraph<false>(atoi(argv[4]), atoi(argv[5]), g, atoi(argv[6]) != 0, 0.57, 0.19, 0.19);
    else if (t == "random" && argc > 6) rc = builder::BuildRandomGraph<false>(atoi(argv[4]), atoi(argv[5]), g, atoi(argv[6]) != 0);
    else if (t == "rr" && argc > 5) rc = builder::BuildRandomRegularishGraph<false>(atoi(argv[4]), atoi(argv[5]), g);
    else if (t == "market" && argc > 5) rc = builder::BuildMarketGraph<false>(argv[4], g, atoi(argv[5]) != 0);
    else if (t == "dimacs" && argc > 6) rc = builder::BuildDimacsGraph<false>(argv[4], g, atoi(argv[5]) != 0, atoi(argv[6]));
    else if (t == "metis") rc = builder::BuildMetisGraph<false>(argv[4], g);
    if (rc) return 1;
    FILE *f = fopen(argv[1], "wb");
    if (!f) return 1;
    long long n = g.nodes, m = g.edges;
    fwrite(&n, 8, 1, f);
    fwrite(&m, 8, 1, f);
    fwrite(g.row_offsets, 4, (size_t)n + 1, f);
    fwrite(g.column_indices, 4, (size_t)m, f);
    fclose(f);
    return 0;
}
