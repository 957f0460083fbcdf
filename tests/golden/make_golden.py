"""Generates the golden BFS fixtures from the reference's own code.

Runs in a container where the reference tree is mounted: the graphs come from
the reference's builders (grid2d/grid3d/rmat/random/rr, libc rand() seeded
with srand(seed) as its driver does) and the labels and search depth from its
SimpleReferenceBfs (test/bfs/test_bfs.cu:503-578), both compiled from the
reference sources by oracle/build_ref.sh.  Output: tests/golden/bfs_golden.npz.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

CASES = [
    # name, builder, args, sources
    ("grid2d_16", "grid2d", (16,), [0, 8 * 16 + 8, 255]),
    ("grid2d_1", "grid2d", (1,), [0]),
    ("grid3d_8", "grid3d", (8,), [0, 4 * 64 + 4 * 8 + 4]),
    ("rmat_s10_ef8_u", "rmat", (1024, 8192, 1, 0.57, 0.19, 0.19, 0), None),
    ("rmat_s9_ef4_d", "rmat", (512, 2048, 0, 0.45, 0.15, 0.15, 1), None),
    ("random_1000_u", "random", (1000, 4000, 1, 2), None),
    ("rr_800_4", "rr", (800, 4, 3), None),
]


def main():
    out = {}
    rng = np.random.default_rng(0)
    for name, kind, args, srcs in CASES:
        ro, ci = oracle.ref_build(kind, *args)
        deg = np.diff(ro)
        if srcs is None:
            nz = np.flatnonzero(deg > 0)
            srcs = [int(x) for x in rng.choice(nz, size=3, replace=False)]
        out[name + "/row_offsets"] = ro
        out[name + "/column_indices"] = ci
        out[name + "/sources"] = np.array(srcs, dtype=np.int32)
        for k, s in enumerate(srcs):
            labels, depth, _ = oracle.ref_bfs(ro, ci, s)
            out[f"{name}/labels{k}"] = labels
            out[f"{name}/depth{k}"] = np.array(depth, dtype=np.int64)
        print(f"{name}: {ro.size - 1} vertices, {ci.size} edges, sources {srcs}")
    path = os.path.join(ROOT, "tests", "golden", "bfs_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
