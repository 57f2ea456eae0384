"""Generates tests/golden/hashgrid_small.npz from the reference's own
SpatialHashGrid<float, uint32_t> (src/sparse_data_structures.h), compiled
into oracle/_ref/libref_hashgrid.so by oracle/Makefile (make ref).

Three seeded cases: points and queries uniform in the domain plus a few
outside it on every side (below min, above max), several radii, cell counts
that are and are not powers of two (Morton codes past total_cells wrap, so
some cells share a bucket).  Run from the repository root:
    python tests/golden/make_hashgrid_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import hashgrid as H  # noqa: E402

CASES = [  # cell size, domain min, domain max, n, nq, radius
    (0.05, (-0.5, -0.25, 0.0), (0.7, 0.55, 0.8), 3000, 300, 0.06),
    (0.0625, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 2500, 200, 0.0),
    (0.1, (-1.0, 0.2, -0.3), (0.35, 1.0, 0.9), 1500, 150, 0.25),
]


def main():
    assert H.reference_available(), "build oracle/_ref first (make -C oracle ref)"
    rng = np.random.default_rng(2024)
    out = {}
    for k, (cs, mn, mx, n, nq, r) in enumerate(CASES):
        mn, mx = np.array(mn, np.float32), np.array(mx, np.float32)
        ext = mx - mn
        p = (mn + rng.random((n, 3)) * ext).astype(np.float32)
        q = (mn + rng.random((nq, 3)) * ext).astype(np.float32)
        p[:20] = (mn - 0.3 * ext + rng.random((20, 3)) * 1.6 * ext).astype(np.float32)  # some outside
        q[:10] = (mn - 0.3 * ext + rng.random((10, 3)) * 1.6 * ext).astype(np.float32)
        counts, starts, idx, offs, lists = H.reference_build_and_query(p, q, r, cs, mn, mx)
        for name, a in (("p", p), ("q", q), ("counts", counts), ("starts", starts), ("indices", idx),
                        ("offsets", offs), ("lists", lists)):
            out[f"c{k}_{name}"] = a
        out[f"c{k}_param"] = np.array([cs, *mn, *mx, r], np.float32)
    np.savez_compressed(os.path.join(HERE, "hashgrid_small.npz"), **out)
    print("wrote hashgrid_small.npz", {k: v.shape for k, v in out.items() if k.endswith("lists")})


if __name__ == "__main__":
    main()
