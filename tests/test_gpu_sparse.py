"""Sparse MPM grids (pgmpm_create_ex with sparse_grid = 1).

Only the 4^3 tiles particles reach are stored, in a pool found through a
hash of the tile coordinates.  Checks:
  * the sparse grid gives the dense grid's result (same kernels, other tile
    order: FP32 rounding only) and the FP64 oracle's, with the bounds of
    tests/test_gpu_forward.py, and the same downloaded grid;
  * a nominal 2048^3 domain (dense: 275 GB of grid) runs in a few MB of tile
    pool and matches a dense 64^3 grid placed over the particles (node
    positions identical) and the FP64 oracle;
  * a pool too small for the particles is reported (PGMPM_FLAG_TILE_POOL),
    and the sparse solver refuses what it does not build.
"""
import numpy as np
import pytest

from test_gpu_forward import _assert_mls, _oracle_scene, _oracle_state, _sim

pytestmark = pytest.mark.gpu


def _sparse(gpu, scenes, counts, mats, st, tiles=0):
    sim = gpu.Simulator(scenes, counts, mats, sparse_tiles=tiles)
    sim.upload(st["x"], st["v"], st["C"].reshape(-1, 9), st["F"].reshape(-1, 9), st["m"], st["V0"], st.get("mat"))
    return sim


def _omats(oracle, mats):
    return oracle.make_materials([(int(m.model), float(m.youngs_modulus), float(m.poisson_ratio)) for m in mats])


@pytest.mark.parametrize("tiles", [0, 3000])
def test_sparse_grid_matches_dense_and_fp64(gpu, oracle, tiles):
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.two_material_drop(n_particles=60000, n=64, seed=51)
    steps = 30
    sp = _sparse(gpu, scenes, counts, mats, st, tiles)
    sp.step(steps)
    out = sp.download()
    assert sp.status() == 0
    de = _sim(gpu, scenes, counts, mats, st)
    de.step(steps)
    ref_d = de.download()
    dx = np.abs(out["x"] - ref_d["x"]).max()
    dv = np.abs(out["v"] - ref_d["v"]).max()
    print(f"sparse vs dense ({tiles} tiles asked): |dx| {dx:.2e} |dv| {dv:.2e}")
    assert dx <= 1e-6 and dv <= 1e-4 * (np.abs(ref_d["v"]).max() + 1e-3)
    ref = oracle.run(_oracle_scene(oracle, scenes[0]), _omats(oracle, mats), _oracle_state(st), steps, prec=64)
    _assert_mls(out, ref, "sparse two-material drop")
    m_s, v_s = sp.grid(0)
    m_d, v_d = de.grid(0)
    assert np.abs(m_s - m_d).max() <= 1e-5 * m_d.max()
    assert np.abs(v_s - v_d).max() <= 1e-4 * np.abs(v_d).max() + 1e-6
    assert np.count_nonzero(m_s) == np.count_nonzero(m_d)


def test_sparse_grid_on_a_2048_cubed_domain(gpu, oracle):
    """262,144 particles (about 4 per cell) in a 40-cell cube of a 2048^3
    domain: the tile pool holds what they touch, not the domain."""
    import torch

    from physgrad_b200 import _capi as C
    from physgrad_b200.solver import Scene, createElasticMaterial

    n, N, steps, dt = 2048, 262144, 10, 2.5e-5
    dx = 1.0 / n
    rng = np.random.default_rng(52)
    lo = 0.5
    x = rng.uniform(lo, lo + 40 * dx, (N, 3)).astype(np.float32)
    v = rng.normal(0.0, 0.1, (N, 3)).astype(np.float32)
    V0 = np.full(N, (dx / 2) ** 3, np.float32)
    st = {"x": x, "v": v, "C": np.zeros((N, 3, 3), np.float32), "F": np.tile(np.eye(3, dtype=np.float32), (N, 1, 1)),
          "m": (1000 * V0).astype(np.float32), "V0": V0, "mat": None}
    mats = [createElasticMaterial(1000.0, 1e4, 0.3)]
    big = Scene((n, n, n), dx, dt, (0.0, -9.8, 0.0), (0.0, 0.0, 0.0), C.PHYSICS_MLS, C.BC_NONE, 0)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    sp = _sparse(gpu, [big], [N], mats, st)
    sp.step(steps)
    torch.cuda.synchronize()
    used = free0 - torch.cuda.mem_get_info()[0]
    out = sp.download()
    assert sp.status() == 0
    dense_grid_bytes = 32 * (n ** 3)
    print(f"2048^3 sparse: device memory used {used / 2 ** 20:.1f} MiB (a dense grid would be "
          f"{dense_grid_bytes / 2 ** 30:.0f} GiB), active nodes {sp.metrics()['active_nodes']}")
    assert used < 2 ** 30
    # a dense 64^3 grid over the particles: origin 12 cells below them, so its
    # nodes sit exactly on the big grid's nodes
    org = (lo - 12 * dx,) * 3
    small = Scene((64, 64, 64), dx, dt, (0.0, -9.8, 0.0), org, C.PHYSICS_MLS, C.BC_NONE, 0)
    de = _sim(gpu, [small], [N], mats, st)
    de.step(steps)
    ref_d = de.download()
    ex = np.abs(out["x"] - ref_d["x"]).max()
    print(f"2048^3 sparse vs 64^3 dense: |dx| {ex:.2e}")
    assert ex <= 1e-6
    ref = oracle.run(_oracle_scene(oracle, small), _omats(oracle, mats), _oracle_state(st), steps, prec=64)
    _assert_mls(out, ref, "2048^3 sparse vs FP64")


def test_sparse_pool_overflow_is_reported(gpu):
    from physgrad_b200 import _capi as C
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.elastic_cube(n_particles=20000, n=64, v_sigma=0.1, seed=53)
    sp = _sparse(gpu, scenes, counts, mats, st, tiles=4)  # a pool of 8 slots for ~200 tiles
    sp.step(3)
    assert sp.status() & C.FLAG_TILE_POOL


def test_sparse_solver_refuses_what_it_does_not_build(gpu):
    from physgrad_b200 import PGMPMError
    from physgrad_b200 import _capi as C
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.elastic_cube(n_particles=4096, n=32, v_sigma=0.1, seed=54)
    sp = _sparse(gpu, scenes, counts, mats, st)
    for call in (lambda: sp.set_variants(p2g_variant=5), lambda: sp.set_variants(g2p_variant=0),
                 lambda: sp.set_step_sort(C.SORT_RADIX), lambda: sp.forward_checkpointed(4, 2)):
        with pytest.raises(PGMPMError) as e:
            call()
        assert e.value.code == C.PGMPM_ERR_UNSUPPORTED
    sp.step(2)
    assert sp.status() == 0
