"""The CPU oracle, pinned before it is trusted (CPU only)."""
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _load_golden(name):
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        meta = json.load(f)
    arrs = np.load(os.path.join(GOLDEN, name + ".npz"))
    return meta, arrs


def test_ref_compat_matches_reference_golden(oracle):
    """Oracle REF_COMPAT (float) is bit-identical to the reference's own CPU
    solver (src/material_point_method.h:479-666) on the committed fixture."""
    meta, g = _load_golden("ref_cpu_small")
    n = tuple(meta["n"])
    sc = oracle.make_scene(n, np.float32(meta["dx"]), np.float32(meta["dt"]),
                           gravity=tuple(np.float32(a) for a in meta["gravity"]), physics=oracle.REF_COMPAT,
                           boundary=oracle.BC_NONE)
    mats = oracle.make_materials([(0, 1e4, 0.3)])
    N = g["x0"].shape[0]
    st = dict(x=g["x0"].astype(np.float64), v=g["v0"].astype(np.float64), C=np.zeros((N, 9)),
              F=np.tile(np.eye(3).ravel(), (N, 1)), m=g["m"].astype(np.float64), V0=g["vol"].astype(np.float64))
    out = oracle.run(sc, mats, st, meta["steps"], prec=32, want_grid=True)
    assert np.array_equal(out["x"].astype(np.float32), g["x"])
    assert np.array_equal(out["v"].astype(np.float32), g["v"])
    assert np.array_equal(out["grid_m"].astype(np.float32), g["grid_m"])
    assert np.array_equal(out["grid_v"].astype(np.float32), g["grid_v"])


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                    "libref_mpm.so")), reason="reference build absent")
def test_ref_compat_matches_reference_live(oracle):
    """Same pin, live against oracle/_ref on config-1 geometry (20 steps)."""
    rng = np.random.default_rng(7)
    N, n, dx = 32768, (64, 64, 64), np.float32(1 / 64)
    x = rng.uniform(0.3, 0.6, (N, 3)).astype(np.float32)
    v = rng.normal(0, 0.05, (N, 3)).astype(np.float32)
    vol = np.full(N, dx ** 3 / 8, np.float32)
    m = (1000 * vol).astype(np.float32)
    r = oracle.ref_run(x, v, m, vol, n, dx, np.float32(1e-4), (0, np.float32(-9.8), 0), 20)
    sc = oracle.make_scene(n, dx, np.float32(1e-4), gravity=(0, np.float32(-9.8), 0), physics=oracle.REF_COMPAT,
                           boundary=oracle.BC_NONE)
    st = dict(x=x.astype(np.float64), v=v.astype(np.float64), C=np.zeros((N, 9)),
              F=np.tile(np.eye(3).ravel(), (N, 1)), m=m.astype(np.float64), V0=vol.astype(np.float64))
    o = oracle.run(sc, oracle.make_materials([(0, 1e4, 0.3)]), st, 20, prec=32)
    assert np.array_equal(o["x"].astype(np.float32), r["x"])
    assert np.array_equal(o["v"].astype(np.float32), r["v"])


def test_stable_sort_and_keys(oracle):
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 50, 5000).astype(np.uint32)
    ok, ov = oracle.stable_sort(keys)
    ref = np.argsort(keys, kind="stable")
    assert np.array_equal(ov, ref.astype(np.uint32))
    assert np.array_equal(ok, keys[ref])
    # keys: stencil origin floor(u - 0.5) clamped, tile-major
    sc = oracle.make_scene((16, 16, 16), 1 / 16, 1e-4)
    x = np.array([[0.5, 0.5, 0.5], [0.0, 0.0, 0.0], [0.99, 0.99, 0.99], [0.2, 0.3, 0.4]], np.float32)
    k = oracle.keys(sc, x)
    def key(s):
        ct = ((16 - 3) >> 2) + 1
        t = ((s[2] >> 2) * ct + (s[1] >> 2)) * ct + (s[0] >> 2)
        return t * 64 + (s[2] & 3) * 16 + (s[1] & 3) * 4 + (s[0] & 3)
    exp = []
    for p in x:
        s = [int(min(max(np.floor(np.float32(np.float32(a) / np.float32(1 / 16)) - np.float32(0.5)), 0), 13)) for a in p]
        exp.append(key(s))
    assert k.tolist() == exp


def _small_state(rng, N, dx, spread=0.05):
    x = rng.uniform(0.35, 0.6, (N, 3))
    return dict(x=x, v=rng.normal(0, 0.3, (N, 3)), C=rng.normal(0, 0.5, (N, 9)),
                F=np.tile(np.eye(3).ravel(), (N, 1)) + rng.normal(0, spread, (N, 9)),
                m=np.full(N, 1000 * (dx / 2) ** 3), V0=np.full(N, (dx / 2) ** 3), mat=(np.arange(N) % 3).astype(np.int32))


@pytest.mark.parametrize("bc", [1, 2, 3])
def test_oracle_adjoint_matches_central_differences(oracle, bc):
    """FP64 oracle adjoint vs central FD, three materials, each wall type."""
    rng = np.random.default_rng(11 + bc)
    N, dx, steps = 200, 1 / 16, 3
    st = _small_state(rng, N, dx)
    sc = oracle.make_scene((16, 16, 16), dx, 2e-3, physics=oracle.MLS, boundary=bc, bthick=3)
    mlist = [(oracle.FIXED_COROTATED, 1e4, 0.3), (oracle.NEO_HOOKEAN, 3e4, 0.25), (oracle.EOS_FLUID, 1e4, 0.0)]
    mats = oracle.make_materials(mlist)
    tgt = np.array([0.5, 0.3, 0.5])

    def loss(s, mt=mats):
        o = oracle.run(sc, mt, s, steps, prec=64)
        return ((o["x"].mean(0) - tgt) ** 2).sum() + 0.1 * (o["v"] ** 2).sum() + 0.01 * (o["F"] ** 2).sum()

    o = oracle.run(sc, mats, st, steps, prec=64)
    g = oracle.adjoint(sc, mats, st, steps, dict(x=np.tile(2 * (o["x"].mean(0) - tgt) / N, (N, 1)), v=0.2 * o["v"],
                                                 F=0.02 * o["F"].reshape(N, 9)))
    eps = 1e-6
    num, ana = [], []
    for key, cols in (("x", 3), ("v", 3), ("C", 9), ("F", 9)):
        for _ in range(4):
            i, j = rng.integers(N), rng.integers(cols)
            sp = {k: (a.copy() if isinstance(a, np.ndarray) else a) for k, a in st.items()}
            sm = {k: (a.copy() if isinstance(a, np.ndarray) else a) for k, a in st.items()}
            sp[key] = sp[key].reshape(N, cols)
            sm[key] = sm[key].reshape(N, cols)
            sp[key][i, j] += eps
            sm[key][i, j] -= eps
            num.append((loss(sp) - loss(sm)) / (2 * eps))
            ana.append(g[key].reshape(N, -1)[i, j])
    for mi in range(3):
        hi = [(a, b + (1e-2 if k == mi else 0), c) for k, (a, b, c) in enumerate(mlist)]
        lo = [(a, b - (1e-2 if k == mi else 0), c) for k, (a, b, c) in enumerate(mlist)]
        num.append((loss(st, oracle.make_materials(hi)) - loss(st, oracle.make_materials(lo))) / 2e-2)
        ana.append(g["E"][mi])
    num, ana = np.array(num), np.array(ana)
    # relative to the largest gradient entry of the set (tolerance 1e-4)
    assert np.abs(num - ana).max() <= 1e-4 * np.abs(num).max() + 1e-10


@pytest.mark.parametrize("bc", [1, 2, 3])
def test_oracle_adjoint_at_walls_on_ragged_grid(oracle, bc):
    """FP64 oracle adjoint vs central FD on a 14 x 9 x 17 grid with an
    origin and off-axis gravity, particles spread through the wall layers
    (most stencils touch a wall node), each wall type."""
    rng = np.random.default_rng(70 + bc)
    n, dx, org, steps = (14, 9, 17), 1 / 16, (0.2, -0.1, 0.05), 3
    N = 200
    o_ = np.asarray(org)
    st = dict(x=rng.uniform(o_ + dx, o_ + (np.asarray(n) - 2.0) * dx, (N, 3)), v=rng.normal(0, 0.3, (N, 3)),
              C=rng.normal(0, 0.5, (N, 9)), F=np.tile(np.eye(3).ravel(), (N, 1)) + rng.normal(0, 0.05, (N, 9)),
              m=np.full(N, 1000 * (dx / 2) ** 3), V0=np.full(N, (dx / 2) ** 3), mat=(np.arange(N) % 3).astype(np.int32))
    s = np.floor((st["x"] - o_) / dx - 0.5).astype(int)
    assert ((s < 3) | (s + 2 >= np.asarray(n) - 3)).any(1).sum() > N // 2
    sc = oracle.make_scene(n, dx, 2e-3, gravity=(0.4, -9.8, 0.0), origin=org, physics=oracle.MLS, boundary=bc,
                           bthick=3)
    mlist = [(oracle.FIXED_COROTATED, 1e4, 0.3), (oracle.NEO_HOOKEAN, 3e4, 0.25), (oracle.EOS_FLUID, 1e4, 0.0)]
    mats = oracle.make_materials(mlist)
    tgt = np.array([0.5, 0.3, 0.5])

    def loss(s_, mt=mats):
        o = oracle.run(sc, mt, s_, steps, prec=64)
        return ((o["x"].mean(0) - tgt) ** 2).sum() + 0.1 * (o["v"] ** 2).sum() + 0.01 * (o["F"] ** 2).sum()

    o = oracle.run(sc, mats, st, steps, prec=64)
    g = oracle.adjoint(sc, mats, st, steps, dict(x=np.tile(2 * (o["x"].mean(0) - tgt) / N, (N, 1)), v=0.2 * o["v"],
                                                 F=0.02 * o["F"].reshape(N, 9)))
    eps = 1e-6
    num, ana = [], []
    for key, cols in (("x", 3), ("v", 3), ("C", 9), ("F", 9)):
        for _ in range(6):
            i, j = rng.integers(N), rng.integers(cols)
            sp = {k: (a.copy() if isinstance(a, np.ndarray) else a) for k, a in st.items()}
            sm = {k: (a.copy() if isinstance(a, np.ndarray) else a) for k, a in st.items()}
            sp[key] = sp[key].reshape(N, cols)
            sm[key] = sm[key].reshape(N, cols)
            sp[key][i, j] += eps
            sm[key][i, j] -= eps
            num.append((loss(sp) - loss(sm)) / (2 * eps))
            ana.append(g[key].reshape(N, -1)[i, j])
    for mi in range(3):
        hi = [(a, b + (1e-2 if k == mi else 0), c) for k, (a, b, c) in enumerate(mlist)]
        lo = [(a, b - (1e-2 if k == mi else 0), c) for k, (a, b, c) in enumerate(mlist)]
        num.append((loss(st, oracle.make_materials(hi)) - loss(st, oracle.make_materials(lo))) / 2e-2)
        ana.append(g["E"][mi])
    num, ana = np.array(num), np.array(ana)
    assert np.abs(num - ana).max() <= 1e-4 * np.abs(num).max() + 1e-10


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                    "libref_mpm.so")), reason="reference build absent")
def test_ref_compat_matches_reference_on_ragged_grid(oracle):
    """The REF_COMPAT pin on a grid that is not whole 4^3 tiles: 30 x 21 x 37
    nodes, a non-zero origin and off-axis gravity, particles up to the
    outermost nodes (30 steps, particles and both grid arrays)."""
    rng = np.random.default_rng(11)
    n, dx = (30, 21, 37), np.float32(1 / 32)
    org = (np.float32(-0.25), np.float32(0.125), np.float32(0.3))
    grav = (np.float32(0.5), np.float32(-9.8), np.float32(1.5))
    N = 6000
    x = rng.uniform(np.array(org, np.float32) + 2 * dx, np.array(org, np.float32) + (np.array(n) - 3) * dx,
                    (N, 3)).astype(np.float32)
    v = rng.normal(0, 0.5, (N, 3)).astype(np.float32)
    vol = np.full(N, dx ** 3 / 8, np.float32)
    m = (1000 * vol).astype(np.float32)
    r = oracle.ref_run(x, v, m, vol, n, dx, np.float32(1e-3), grav, 30, origin=org, want_grid=True)
    sc = oracle.make_scene(n, dx, np.float32(1e-3), gravity=grav, origin=org, physics=oracle.REF_COMPAT,
                           boundary=oracle.BC_NONE)
    st = dict(x=x.astype(np.float64), v=v.astype(np.float64), C=np.zeros((N, 9)),
              F=np.tile(np.eye(3).ravel(), (N, 1)), m=m.astype(np.float64), V0=vol.astype(np.float64))
    o = oracle.run(sc, oracle.make_materials([(0, 1e4, 0.3)]), st, 30, prec=32, want_grid=True)
    assert np.abs(r["x"] - x).max() > dx / 4  # the particles moved
    assert np.array_equal(o["x"].astype(np.float32), r["x"])
    assert np.array_equal(o["v"].astype(np.float32), r["v"])
    assert np.array_equal(o["grid_m"].astype(np.float32), r["grid_m"])
    assert np.array_equal(o["grid_v"].astype(np.float32), r["grid_v"])


def test_oracle_fp32_mirror_close_to_fp64(oracle):
    rng = np.random.default_rng(5)
    N, dx = 1000, 1 / 32
    st = _small_state(rng, N, dx, spread=0.02)
    st["mat"] = np.zeros(N, np.int32)
    sc = oracle.make_scene((32, 32, 32), dx, 1e-4)
    mats = oracle.make_materials([(oracle.FIXED_COROTATED, 1e4, 0.3)])
    a = oracle.run(sc, mats, st, 10, prec=64)
    b = oracle.run(sc, mats, st, 10, prec=32)
    assert np.abs(a["x"] - b["x"]).max() < 1e-6
    assert np.abs(a["F"] - b["F"]).max() < 1e-5


def test_oracle_plastic_and_viscous_models(oracle):
    """ELASTOPLASTIC (model 3: neo-Hookean + von Mises cap) with an unreachable
    yield stress is the neo-Hookean run bit for bit, and with a low one it
    differs; a FLUID viscosity of 0 is the inviscid run bit for bit, and a
    positive one changes it."""
    rng = np.random.default_rng(5)
    n, N = 16, 600
    dx = 1.0 / n
    st = _small_state(rng, N, dx, spread=0.08)
    st["mat"] = np.zeros(N, np.int32)
    sc = oracle.make_scene((n, n, n), dx, 1e-4, gravity=(0, -9.8, 0), boundary=1, bthick=2)
    run = lambda mats: oracle.run(sc, oracle.make_materials(mats), st, 20, prec=64)
    nh = run([(1, 1e4, 0.3)])
    same = run([(3, 1e4, 0.3, 1e30)])
    capped = run([(3, 1e4, 0.3, 10.0)])
    for k in ("x", "v", "C", "F"):
        assert np.array_equal(nh[k], same[k]), k
    assert np.abs(capped["x"] - nh["x"]).max() > 1e-9 and np.isfinite(capped["x"]).all()
    eos = run([(2, 1e4, 0.0)])
    eos0 = run([(2, 1e4, 0.0, 0.0, 0.0)])
    visc = run([(2, 1e4, 0.0, 0.0, 5.0)])
    for k in ("x", "v", "C", "F"):
        assert np.array_equal(eos[k], eos0[k]), k
    assert np.abs(visc["v"] - eos["v"]).max() > 1e-6 and np.isfinite(visc["v"]).all()


def _hashgrid_case(g, k):
    prm = g[f"c{k}_param"]
    return float(prm[0]), prm[1:4], prm[4:7], float(prm[7])


def test_hashgrid_oracle_matches_reference_golden():
    """oracle/hashgrid.py (restated SpatialHashGrid, src/sparse_data_structures.h)
    reproduces the reference class's table and getNeighbors lists bit for bit
    on the committed fixture, points and queries outside the domain included."""
    from oracle import hashgrid as H

    g = np.load(os.path.join(GOLDEN, "hashgrid_small.npz"))
    for k in range(3):
        cs, mn, mx, r = _hashgrid_case(g, k)
        c, s, ix, ids = H.build(g[f"c{k}_p"], cs, mn, mx)
        assert np.array_equal(c, g[f"c{k}_counts"]) and np.array_equal(s, g[f"c{k}_starts"])
        assert np.array_equal(ix, g[f"c{k}_indices"])
        o, l = H.neighbors(g[f"c{k}_q"], r, cs, mn, mx, c, s, ix)
        assert np.array_equal(o, g[f"c{k}_offsets"]) and np.array_equal(l, g[f"c{k}_lists"])


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                    "libref_hashgrid.so")), reason="reference build absent")
def test_hashgrid_oracle_matches_reference_live():
    """The same pin on seeded random cases, live against oracle/_ref."""
    from oracle import hashgrid as H

    rng = np.random.default_rng(7)
    for _ in range(5):
        n, cs = int(rng.integers(1, 2000)), float(rng.choice([0.04, 0.07, 0.1]))
        mn = rng.uniform(-1, 0, 3).astype(np.float32)
        mx = (mn + rng.uniform(0.4, 1.2, 3)).astype(np.float32)
        p = (mn + rng.random((n, 3)) * (mx - mn)).astype(np.float32)
        q = (mn - 0.1 + rng.random((40, 3)) * (mx - mn + 0.2)).astype(np.float32)
        r = float(rng.choice([0.0, 0.05, 0.15]))
        c, s, ix, _ = H.build(p, cs, mn, mx)
        o, l = H.neighbors(q, r, cs, mn, mx, c, s, ix)
        rc, rs, rix, ro, rl = H.reference_build_and_query(p, q, r, cs, mn, mx)
        for a, b in ((c, rc), (s, rs), (ix, rix), (o, ro), (l, rl)):
            assert np.array_equal(a, b)


# ------------------------------------------------------------------ consumers
def _coupling_inputs(seed, n_sph=400, n_mpm=900):
    rng = np.random.default_rng(seed)
    return (rng.uniform(0.3, 0.7, (n_sph, 3)).astype(np.float32), rng.normal(0, 0.5, (n_sph, 3)).astype(np.float32),
            rng.uniform(0.3, 0.7, (n_mpm, 3)).astype(np.float32), rng.normal(0, 0.5, (n_mpm, 3)).astype(np.float32))


@pytest.mark.parametrize("two_way,radius", [(True, 0.05), (False, 0.08), (True, 0.15)])
def test_sph_coupling_restatement_equals_reference_class(oracle, two_way, radius):
    """The oracle's SPH-MPM contact coupling equals the reference's own
    SPHMPMCouplingSystem (src/sph_mpm_coupling.h:453-575, built from its
    sources into oracle/_ref) bit for bit: forces, pair count, energy."""
    if not oracle.ref_coupling_available():
        pytest.skip("oracle/_ref not built")
    sx, sv, mx, mv = _coupling_inputs(7 + int(radius * 100))
    kw = dict(stiffness=2e4, damping=50.0, friction=0.4, radius=radius, two_way=two_way)
    a = oracle.sph_coupling(sx, sv, mx, mv, **kw)
    b = oracle.ref_sph_coupling(sx, sv, mx, mv, **kw)
    assert a["n_pairs"] == b["n_pairs"] > 0
    assert np.array_equal(a["sph_force"], b["sph_force"])
    assert np.array_equal(a["mpm_force"], b["mpm_force"])
    assert a["energy"] == b["energy"]
    if not two_way:
        assert not np.any(a["sph_force"])


def test_kinetic_energy_restatement_matches_reference_monitor(oracle):
    """The oracle's kinetic energy per material against the reference's
    FSISimulationManager energy monitor (src/fsi_coupling.h:837-858) on a
    fluid set and a solid set (float sums there: 1e-6 relative)."""
    if not oracle.ref_fsi_available():
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(3)
    vf, vs = rng.normal(0, 1, (5000, 3)), rng.normal(0, 2, (3000, 3))
    mf, ms = rng.uniform(0.5, 1.5, 5000), rng.uniform(1, 3, 3000)
    v = np.concatenate([vf, vs]).astype(np.float32).astype(np.float64)
    m = np.concatenate([mf, ms]).astype(np.float32).astype(np.float64)
    mat = np.concatenate([np.zeros(5000, np.int32), np.ones(3000, np.int32)])
    ours = oracle.kinetic_energy(v, m, mat, 2)
    ref = oracle.ref_fsi_energy(vf, mf, vs, ms)
    assert abs(ours.sum() - ref) <= 1e-6 * ref


@pytest.mark.parametrize("case", ["plastic", "viscous"])
def test_oracle_adjoint_of_plastic_and_viscous_models(oracle, case):
    """FP64 oracle adjoint vs central FD for the ELASTOPLASTIC model (the
    von Mises cap active on most particles: a low yield stress and stretched
    F) and the viscous EOS fluid (tau += J mu_v (C + C^T)), with an elastic
    material beside it; every field and dL/dE."""
    rng = np.random.default_rng(90 + (case == "viscous"))
    N, dx, steps = 200, 1 / 16, 3
    st = _small_state(rng, N, dx)
    st["F"] = (np.tile(np.eye(3).ravel(), (N, 1)) + rng.normal(0, 0.08, (N, 9)))
    sc = oracle.make_scene((16, 16, 16), dx, 2e-3, physics=oracle.MLS, boundary=1, bthick=3)
    if case == "plastic":
        mlist = [(3, 2e4, 0.3, 150.0), (oracle.FIXED_COROTATED, 1e4, 0.3), (3, 1e4, 0.25, 1e9)]
    else:
        mlist = [(oracle.EOS_FLUID, 1e4, 0.0, 0.0, 30.0), (oracle.NEO_HOOKEAN, 3e4, 0.25),
                 (oracle.EOS_FLUID, 2e4, 0.0, 0.0, 5.0)]
    mats = oracle.make_materials(mlist)
    tgt = np.array([0.5, 0.3, 0.5])

    def loss(s, mt=mats):
        o = oracle.run(sc, mt, s, steps, prec=64)
        return ((o["x"].mean(0) - tgt) ** 2).sum() + 0.1 * (o["v"] ** 2).sum() + 0.01 * (o["F"] ** 2).sum()

    o = oracle.run(sc, mats, st, steps, prec=64)
    g = oracle.adjoint(sc, mats, st, steps, dict(x=np.tile(2 * (o["x"].mean(0) - tgt) / N, (N, 1)), v=0.2 * o["v"],
                                                 F=0.02 * o["F"].reshape(N, 9)))
    eps = 1e-6
    num, ana = [], []
    for key, cols in (("x", 3), ("v", 3), ("C", 9), ("F", 9)):
        for _ in range(5):
            i, j = rng.integers(N), rng.integers(cols)
            sp = {k: (a.copy() if isinstance(a, np.ndarray) else a) for k, a in st.items()}
            sm = {k: (a.copy() if isinstance(a, np.ndarray) else a) for k, a in st.items()}
            sp[key] = sp[key].reshape(N, cols)
            sm[key] = sm[key].reshape(N, cols)
            sp[key][i, j] += eps
            sm[key][i, j] -= eps
            num.append((loss(sp) - loss(sm)) / (2 * eps))
            ana.append(g[key].reshape(N, -1)[i, j])
    for mi in range(3):
        hi = [tuple(b + (1e-2 if (k == mi and q == 1) else 0) for q, b in enumerate(m)) for k, m in enumerate(mlist)]
        lo = [tuple(b - (1e-2 if (k == mi and q == 1) else 0) for q, b in enumerate(m)) for k, m in enumerate(mlist)]
        num.append((loss(st, oracle.make_materials(hi)) - loss(st, oracle.make_materials(lo))) / 2e-2)
        ana.append(g["E"][mi])
    num, ana = np.array(num), np.array(ana)
    assert np.abs(num - ana).max() <= 1e-4 * np.abs(num).max() + 1e-10
