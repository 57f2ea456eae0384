"""Generate the committed golden fixtures of tests/golden/.

ref_cpu_small  -- the reference's OWN CPU solver (physgrad::mpm::MPMSolver<
                  float,64>, src/material_point_method.h:430-676) built from
                  its sources by oracle/Makefile into oracle/_ref; seeded
                  inputs and its outputs after 30 steps.  Needs the reference
                  tree, so it runs only where that tree exists.
mls_small      -- the FP64 oracle's MLS step (three materials, sticky walls);
                  a regression fixture (the reference has no MLS physics).
sort_small     -- keys and the stable permutation of a CPU stable sort.

Run:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as O  # noqa: E402


def save(name, meta, **arrs):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
    with open(os.path.join(HERE, name + ".json"), "w") as f:
        json.dump(meta, f, indent=1)


def ref_cpu_small():
    rng = np.random.default_rng(2024)
    N, n, steps = 1024, (16, 16, 16), 30
    dx = np.float32(1 / 16)
    x = rng.uniform(0.3, 0.7, (N, 3)).astype(np.float32)
    v = rng.normal(0, 0.2, (N, 3)).astype(np.float32)
    vol = np.full(N, dx ** 3 / 8, np.float32)
    m = (1000 * vol).astype(np.float32)
    dt, g = np.float32(1e-3), (0.0, np.float32(-9.8), 0.0)
    r = O.ref_run(x, v, m, vol, n, dx, dt, g, steps, want_grid=True)
    meta = {"source": "reference MPMSolver<float,64> via oracle/_ref/libref_mpm.so", "n": list(n), "dx": float(dx),
            "dt": float(dt), "gravity": [float(a) for a in g], "steps": steps, "seed": 2024}
    save("ref_cpu_small", meta, x0=x, v0=v, m=m, vol=vol, x=r["x"], v=r["v"], grid_m=r["grid_m"], grid_v=r["grid_v"])


def mls_small():
    rng = np.random.default_rng(99)
    N, n, steps, dx = 512, (16, 16, 16), 20, 1 / 16
    x = rng.uniform(0.35, 0.65, (N, 3)).astype(np.float32)
    v = rng.normal(0, 0.2, (N, 3)).astype(np.float32)
    mat = (np.arange(N) % 3).astype(np.int32)
    V0 = np.full(N, (dx / 2) ** 3)
    st = dict(x=x.astype(np.float64), v=v.astype(np.float64), C=np.zeros((N, 9)),
              F=np.tile(np.eye(3).ravel(), (N, 1)), m=1000 * V0, V0=V0, mat=mat)
    mats = [(O.FIXED_COROTATED, 1e4, 0.3), (O.NEO_HOOKEAN, 3e4, 0.25), (O.EOS_FLUID, 1e4, 0.0)]
    sc = O.make_scene(n, dx, 1e-3, physics=O.MLS, boundary=O.BC_STICKY, bthick=3)
    o = O.run(sc, O.make_materials(mats), st, steps, prec=64)
    meta = {"source": "FP64 oracle (oracle/oracle.cpp), MLS physics", "n": list(n), "dx": dx, "dt": 1e-3,
            "gravity": [0.0, -9.8, 0.0], "boundary": "sticky", "bthick": 3, "steps": steps, "materials": mats,
            "seed": 99}
    save("mls_small", meta, x0=x, v0=v, mat=mat, x=o["x"], v=o["v"], C=o["C"], F=o["F"])


def sort_small():
    rng = np.random.default_rng(5)
    keys = np.concatenate([rng.integers(0, 1 << 12, 3000), np.repeat(rng.integers(0, 64, 40), 25)]).astype(np.uint32)
    ok, ov = O.stable_sort(keys)
    save("sort_small", {"source": "std::stable_sort via oracle_stable_sort", "key_bits": 12}, keys=keys,
         sorted_keys=ok, order=ov)


if __name__ == "__main__":
    O.build(with_ref=True)
    if O.ref_available():
        ref_cpu_small()
    mls_small()
    sort_small()
    print("fixtures written to", HERE)
