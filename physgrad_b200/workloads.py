"""Seeded synthetic inputs for the benchmark configurations of the MLS-MPM step.

Every generator returns plain numpy arrays (float32, upload order) so the
same inputs feed the CUDA path and the CPU oracle.  Unstated values are
fixed here and recorded in the returned ``meta``: density 1000, initial
particle volume (dx/2)^3, gravity (0, -9.8, 0), walls 3 nodes thick.
"""
from __future__ import annotations

import math

import numpy as np

from . import _capi as C
from .solver import MaterialParameters, Scene, createElasticMaterial, createFluidMaterial, ConstitutiveModel

RHO = 1000.0
G = (0.0, -9.8, 0.0)


def _state(x, v=None, dx=1 / 64, mat=None):
    n = x.shape[0]
    V0 = np.full(n, (dx / 2) ** 3, np.float32)
    return {
        "x": np.ascontiguousarray(x, np.float32),
        "v": np.zeros((n, 3), np.float32) if v is None else np.ascontiguousarray(v, np.float32),
        "C": np.zeros((n, 3, 3), np.float32),
        "F": np.tile(np.eye(3, dtype=np.float32), (n, 1, 1)),
        "m": (RHO * V0).astype(np.float32),
        "V0": V0,
        "mat": None if mat is None else np.ascontiguousarray(mat, np.int32),
    }


def elastic_cube(n_particles=32768, n=64, steps=200, seed=0, E=1e4, nu=0.3, dt=1e-4, lo=0.3, hi=0.6,
                 v_sigma=0.0, model=ConstitutiveModel.FIXED_COROTATED, boundary=C.BC_STICKY,
                 physics=C.PHYSICS_MLS):
    """Config 1 (defaults) and config 3 (n_particles=262144, v_sigma=0.1, 256 steps)."""
    rng = np.random.default_rng(seed)
    dx = 1.0 / n
    x = rng.uniform(lo, hi, (n_particles, 3)).astype(np.float32)
    v = rng.normal(0.0, v_sigma, (n_particles, 3)).astype(np.float32) if v_sigma > 0 else None
    scene = Scene((n, n, n), dx, dt, G, (0.0, 0.0, 0.0), physics, boundary, 3)
    mats = [createElasticMaterial(RHO, E, nu, model)]
    meta = {"workload": "elastic_cube", "grid": n, "n_particles": n_particles, "steps": steps, "seed": seed, "E": E,
            "nu": nu, "dt": dt, "rho": RHO, "V0": "(dx/2)^3", "gravity": G, "walls": "sticky 3 nodes"}
    return [scene], [n_particles], mats, _state(x, v, dx), meta


def config1(seed=0):
    return elastic_cube(seed=seed)


def config3(seed=0, n_particles=262144, steps=256):
    return elastic_cube(n_particles=n_particles, n=64, steps=steps, seed=seed, v_sigma=0.1)


def two_material_drop(n_particles=2097152, n=128, seed=0, steps=1000, dt=5e-5):
    """Config 2: neo-Hookean block + EOS fluid column, slip walls."""
    rng = np.random.default_rng(seed)
    dx = 1.0 / n
    h = n_particles // 2
    xa = rng.uniform(0.2, 0.5, (h, 3))
    xb = np.stack([rng.uniform(0.55, 0.85, n_particles - h), rng.uniform(0.05, 0.6, n_particles - h),
                   rng.uniform(0.2, 0.8, n_particles - h)], 1)
    x = np.concatenate([xa, xb], 0).astype(np.float32)
    mat = np.concatenate([np.zeros(h, np.int32), np.ones(n_particles - h, np.int32)])
    scene = Scene((n, n, n), dx, dt, G, (0.0, 0.0, 0.0), C.PHYSICS_MLS, C.BC_SLIP, 3)
    mats = [createElasticMaterial(RHO, 5e4, 0.3, ConstitutiveModel.NEO_HOOKEAN), createFluidMaterial(RHO, 0.0, 1e4)]
    meta = {"workload": "two_material_drop", "grid": n, "n_particles": n_particles, "steps": steps, "seed": seed,
            "dt": dt, "rho": RHO, "V0": "(dx/2)^3", "gravity": G, "walls": "slip 3 nodes",
            "materials": "neo-Hookean E=5e4 nu=0.3 / EOS fluid K=1e4"}
    return [scene], [n_particles], mats, _state(x, None, dx, mat), meta


def config2(seed=0, n_particles=2097152):
    return two_material_drop(n_particles=n_particles, seed=seed)


def _grid_for_count(c, grids):
    if grids == "small":
        return 32 if c < 16384 else (64 if c < 131072 else 128)
    return 64 if c < 131072 else 128


def batched_scenes(n_scenes=64, lo=4096, hi=262144, seed=0, steps=500, dt=1e-4, grids="small", E_range=(5e3, 5e4),
                   v_sigma=0.0):
    """Config 4 (defaults) / config 5 (32 scenes, [16384, 524288], 64-128^3).

    Counts are floor(exp(U(ln lo, ln hi))); grid by count: < 16384 -> 32^3,
    < 131072 -> 64^3, else 128^3 (config 5: < 131072 -> 64^3 else 128^3);
    each scene a seeded-uniform cube [0.3, 0.6]^3 with its own E."""
    rng = np.random.default_rng(seed)
    counts = np.floor(np.exp(rng.uniform(math.log(lo), math.log(hi), n_scenes))).astype(np.int64)
    Es = rng.uniform(E_range[0], E_range[1], n_scenes)
    scenes, mats, xs, vs, V0s, mids = [], [], [], [], [], []
    for s in range(n_scenes):
        c = int(counts[s])
        n = _grid_for_count(c, grids)
        dx = 1.0 / n
        scenes.append(Scene((n, n, n), dx, dt, G, (0.0, 0.0, 0.0), C.PHYSICS_MLS, C.BC_STICKY, 3))
        mats.append(createElasticMaterial(RHO, float(Es[s]), 0.3))
        xs.append(rng.uniform(0.3, 0.6, (c, 3)).astype(np.float32))
        vs.append(rng.normal(0.0, v_sigma, (c, 3)).astype(np.float32) if v_sigma > 0 else np.zeros((c, 3), np.float32))
        V0s.append(np.full(c, (dx / 2) ** 3, np.float32))
        mids.append(np.full(c, s, np.int32))
    x = np.concatenate(xs, 0)
    V0 = np.concatenate(V0s, 0)
    N = x.shape[0]
    st = {"x": x, "v": np.concatenate(vs, 0), "C": np.zeros((N, 3, 3), np.float32),
          "F": np.tile(np.eye(3, dtype=np.float32), (N, 1, 1)), "m": (RHO * V0).astype(np.float32), "V0": V0,
          "mat": np.concatenate(mids, 0)}
    meta = {"workload": "batched_scenes", "n_scenes": n_scenes, "counts": counts.tolist(), "total": int(N),
            "grids": [int(s.n[0]) for s in scenes], "E": Es.tolist(), "steps": steps, "seed": seed, "dt": dt}
    return scenes, counts.tolist(), mats, st, meta


def config4(seed=0):
    return batched_scenes(seed=seed)


def config5(seed=0, steps=128):
    return batched_scenes(n_scenes=32, lo=16384, hi=524288, seed=seed, steps=steps, grids="large", v_sigma=0.1)


def oracle_inputs(scenes, mats, st):
    """Arguments for the CPU oracle (one scene): scene fields and materials."""
    s = scenes[0]
    return {"n": tuple(int(a) for a in s.n), "dx": s.dx, "dt": s.dt, "gravity": tuple(s.gravity),
            "origin": tuple(s.origin), "physics": s.physics, "boundary": s.boundary, "bthick": s.boundary_thickness,
            "materials": [(int(m.model), float(m.youngs_modulus), float(m.poisson_ratio)) for m in mats]}
