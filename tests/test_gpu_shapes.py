"""GPU parity on grids that are not whole 4^3 tiles: anisotropic node counts
(30 x 21 x 37 and smaller), non-zero origins and off-axis gravity, with
particles spread up to the walls.  The grid is stored in 4^3-node tiles, so
these shapes exercise the padded tail of the last tile on every axis, the
stencil-origin clamp at n - 3 and the wall tests near both ends.

Tolerances are those of the cubic-grid tests:
  * MLS vs the FP64 oracle: positions max abs err <= 2e-5, velocities
    <= 1e-3 * max|v| + 1e-5, F <= 2e-4 absolute;
  * REF_COMPAT vs the float oracle of the reference path (bit-identical to
    the reference's own solver on this shape, tests/test_oracle.py):
    positions <= 2e-6 absolute, velocities <= 1e-4 * max|v|;
  * batched vs single scenes: x <= 1e-6, v <= 1e-4 * max|v|, F <= 1e-5;
  * the last step's grid vs the FP64 oracle: total mass <= 1e-5 relative,
    nodal mass <= 1e-4 * max m, nodal momentum <= 2e-4 * max |m v|;
  * adjoint vs the FP64 oracle adjoint: <= 2e-3 * max|oracle| per field.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RAGGED = dict(n=(30, 21, 37), dx=1.0 / 32, origin=(-0.25, 0.125, 0.3), gravity=(0.5, -9.8, 1.5))


def _state(rng, N, n, dx, origin, margin=1.5, v_sigma=1.0, n_mats=3):
    """Uniform particles over the whole grid interior, `margin` cells from
    the outermost nodes, so that particles sit inside the walls."""
    o = np.asarray(origin, np.float64)
    lo = o + margin * dx
    hi = o + (np.asarray(n) - 1 - margin) * dx
    V0 = np.full(N, (dx / 2) ** 3, np.float32)
    return dict(x=rng.uniform(lo, hi, (N, 3)).astype(np.float32),
                v=rng.normal(0, v_sigma, (N, 3)).astype(np.float32),
                C=np.zeros((N, 9), np.float32), F=np.tile(np.eye(3, dtype=np.float32).ravel(), (N, 1)),
                m=(1000 * V0).astype(np.float32), V0=V0, mat=(np.arange(N) % n_mats).astype(np.int32))


def _mats(pg, oracle):
    gpu = [pg.createElasticMaterial(1000, 1e4, 0.3), pg.createElasticMaterial(1000, 3e4, 0.25, 1),
           pg.createFluidMaterial(1000, 0.0, 1e4)]
    orc = [(oracle.FIXED_COROTATED, 1e4, 0.3), (oracle.NEO_HOOKEAN, 3e4, 0.25), (oracle.EOS_FLUID, 1e4, 0.0)]
    return gpu, orc


def _upload(pg, scenes, counts, mats, st):
    sim = pg.Simulator(scenes, counts, mats)
    sim.upload(st["x"], st["v"], st["C"], st["F"], st["m"], st["V0"], st["mat"])
    return sim


def _ostate(st):
    d = {k: st[k].astype(np.float64) for k in ("x", "v", "C", "F", "m", "V0")}
    d["mat"] = st["mat"]
    return d


@pytest.mark.parametrize("bc,bthick,p2g_variant,sort", [(1, 3, 4, "bins"), (2, 3, 4, "bins"), (3, 2, 4, "bins"),
                                                        (1, 3, 5, "bins"), (2, 3, 5, "bins"), (3, 2, 5, "bins"),
                                                        (1, 3, 2, "bins"), (3, 2, 2, "bins"), (2, 3, 3, "radix")])
def test_mls_ragged_grid_vs_fp64_oracle(gpu, oracle, bc, bthick, p2g_variant, sort):
    from physgrad_b200 import _capi as C

    rng = np.random.default_rng(100 + 10 * bc + p2g_variant)
    N, dt, steps = 6000, 5e-4, 30
    st = _state(rng, N, RAGGED["n"], RAGGED["dx"], RAGGED["origin"])
    mats, omats = _mats(gpu, oracle)
    scene = gpu.Scene(RAGGED["n"], RAGGED["dx"], dt, RAGGED["gravity"], RAGGED["origin"], C.PHYSICS_MLS, bc, bthick)
    sim = _upload(gpu, [scene], [N], mats, st)
    sim.set_variants(p2g_variant=p2g_variant)
    if sort == "radix":
        sim.set_step_sort(C.SORT_RADIX)
    sim.step(steps)
    assert sim.status() == 0
    out = sim.download()
    m, v = sim.grid(0)
    osc = oracle.make_scene(RAGGED["n"], RAGGED["dx"], dt, gravity=RAGGED["gravity"], origin=RAGGED["origin"],
                            physics=oracle.MLS, boundary=bc, bthick=bthick)
    ref = oracle.run(osc, oracle.make_materials(omats), _ostate(st), steps, prec=64, want_grid=True)
    ex = np.abs(out["x"] - ref["x"]).max()
    ev = np.abs(out["v"] - ref["v"]).max()
    vmax = np.abs(ref["v"]).max()
    eF = np.abs(out["F"].reshape(N, 9) - ref["F"].reshape(N, 9)).max()
    print(f"bc{bc} variant {p2g_variant} {sort}: |dx| {ex:.2e} |dv| {ev:.2e} (vmax {vmax:.2e}) |dF| {eF:.2e}")
    assert ex <= 2e-5, ex
    assert ev <= 1e-3 * vmax + 1e-5, (ev, vmax)
    assert eF <= 2e-4, eF
    # The last step's grid in the reference layout (k * nx * ny + j * nx + i).
    # Nodal momenta rather than velocities: v = p / m at the cloud's edge
    # nodes (m ~ 1e-12) amplifies rounding.  After 30 steps the FP32 oracle
    # differs from FP64 by ~1e-5 relative in both, hence the 1e-4 / 2e-4 bounds.
    assert m.shape[0] == np.prod(RAGGED["n"])
    assert abs(m.astype(np.float64).sum() - st["m"].astype(np.float64).sum()) <= 1e-5 * st["m"].sum()
    assert np.abs(m - ref["grid_m"]).max() <= 1e-4 * ref["grid_m"].max()
    p_ref = ref["grid_m"][:, None] * ref["grid_v"]
    assert np.abs(m[:, None] * v - p_ref).max() <= 2e-4 * np.abs(p_ref).max()


def test_ref_compat_ragged_grid_vs_oracle(gpu, oracle):
    """The reference's PIC path (src/material_point_method.h:479-666) on the
    ragged grid with an origin, including particles whose 3-node stencil
    leaves the grid at the low and high ends."""
    from physgrad_b200 import _capi as C

    rng = np.random.default_rng(21)
    N, dt, steps = 6000, 1e-3, 30
    dx = np.float32(RAGGED["dx"])
    org = tuple(np.float32(a) for a in RAGGED["origin"])
    grav = tuple(np.float32(a) for a in RAGGED["gravity"])
    st = _state(rng, N, RAGGED["n"], float(dx), org, margin=0.2, v_sigma=0.5, n_mats=1)
    st["V0"] = np.full(N, dx ** 3 / 8, np.float32)
    st["m"] = (1000 * st["V0"]).astype(np.float32)
    scene = gpu.Scene(RAGGED["n"], float(dx), dt, grav, org, C.PHYSICS_REF_COMPAT, C.BC_NONE, 0)
    sim = _upload(gpu, [scene], [N], [gpu.createElasticMaterial(1000, 1e4, 0.3)], st)
    sim.step(steps)
    out = sim.download()
    osc = oracle.make_scene(RAGGED["n"], dx, np.float32(dt), gravity=grav, origin=org, physics=oracle.REF_COMPAT,
                            boundary=oracle.BC_NONE)
    ref = oracle.run(osc, oracle.make_materials([(0, 1e4, 0.3)]), _ostate(st), steps, prec=32)
    ex = np.abs(out["x"] - ref["x"]).max()
    ev = np.abs(out["v"] - ref["v"]).max() / np.abs(ref["v"]).max()
    print(f"REF_COMPAT ragged: |dx| {ex:.2e} rel |dv| {ev:.2e}")
    assert ex <= 2e-6 and ev <= 1e-4, (ex, ev)


@pytest.mark.parametrize("p2g_variant", [2, 4, 5])
def test_ragged_scenes_batched_equal_single(gpu, oracle, p2g_variant):
    """Three scenes of different ragged shapes, origins and walls in one
    batched solver give each scene's single-scene result."""
    from physgrad_b200 import _capi as C

    specs = [((30, 21, 37), 1.0 / 32, (-0.25, 0.125, 0.3), C.BC_STICKY, 3, 2500),
             ((9, 13, 6), 1.0 / 8, (1.0, -2.0, 0.5), C.BC_SLIP, 1, 700),
             ((41, 17, 23), 1.0 / 40, (0.0, 0.0, -1.0), C.BC_SEPARATE, 2, 3100)]
    rng = np.random.default_rng(31)
    mats_all, _ = _mats(gpu, oracle)
    scenes, counts, parts = [], [], []
    for n, dx, org, bc, bt, N in specs:
        scenes.append(gpu.Scene(n, dx, 5e-4, (0.3, -9.8, -0.7), org, C.PHYSICS_MLS, bc, bt))
        counts.append(N)
        parts.append(_state(rng, N, n, dx, org, margin=bt + 0.5))
    st = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
    sim = _upload(gpu, scenes, counts, mats_all, st)
    sim.set_variants(p2g_variant=p2g_variant)
    sim.step(20)
    assert sim.status() == 0
    out = sim.download()
    off = 0
    for s, N in enumerate(counts):
        sl = slice(off, off + N)
        one = _upload(gpu, [scenes[s]], [N], mats_all, parts[s])
        one.set_variants(p2g_variant=p2g_variant)
        one.step(20)
        o1 = one.download()
        assert np.abs(out["x"][sl] - o1["x"]).max() <= 1e-6, s
        assert np.abs(out["v"][sl] - o1["v"]).max() <= 1e-4 * (np.abs(o1["v"]).max() + 1e-3), s
        assert np.abs(out["F"][sl] - o1["F"]).max() <= 1e-5, s
        m_b, v_b = sim.grid(s)
        m_1, v_1 = one.grid(0)
        assert m_b.shape[0] == np.prod(specs[s][0])
        assert np.abs(m_b - m_1).max() <= 1e-5 * m_1.max(), s
        off += N


@pytest.mark.parametrize("bc,k", [(2, 2), (3, 3)])
def test_adjoint_ragged_grid_vs_fp64_oracle(gpu, oracle, bc, k):
    """Checkpointed forward + backward on a ragged grid with an origin,
    particles spread through the wall layers, against the FP64 oracle
    adjoint (dL/d of x0, v0, C0, F0 and E)."""
    from physgrad_b200 import _capi as C

    rng = np.random.default_rng(50 + bc)
    n, dx, org, dt, steps = (18, 13, 21), 1.0 / 16, (0.2, -0.1, 0.05), 1e-3, 6
    N = 1500
    st = _state(rng, N, n, dx, org, margin=1.0, v_sigma=0.3)  # stencils reach into the wall layers
    st["C"] = rng.normal(0, 0.5, (N, 9)).astype(np.float32)
    st["F"] = (np.tile(np.eye(3).ravel(), (N, 1)) + rng.normal(0, 0.03, (N, 9))).astype(np.float32)
    mats, omats = _mats(gpu, oracle)
    scene = gpu.Scene(n, dx, dt, (0.4, -9.8, 0.0), org, C.PHYSICS_MLS, bc, 3)
    sim = _upload(gpu, [scene], [N], mats, st)
    sim.forward_checkpointed(steps, k)
    out = sim.download()
    go = {"x": np.tile(2 * (out["x"].mean(0) - np.array([0.7, 0.3, 0.6])) / N, (N, 1)).astype(np.float32),
          "v": (0.2 * out["v"]).astype(np.float32), "F": (0.02 * out["F"].reshape(N, 9)).astype(np.float32),
          "C": (0.01 * out["C"].reshape(N, 9)).astype(np.float32)}
    g = sim.backward(go)
    osc = oracle.make_scene(n, dx, dt, gravity=(0.4, -9.8, 0.0), origin=org, physics=oracle.MLS, boundary=bc,
                            bthick=3)
    ref = oracle.adjoint(osc, oracle.make_materials(omats), _ostate(st), steps,
                         {k_: v_.astype(np.float64) for k_, v_ in go.items()})
    for key in ("x", "v", "C", "F", "E"):
        a = np.asarray(g[key]).reshape(-1)
        b = np.asarray(ref[key]).reshape(-1)
        err = np.abs(a - b).max() / np.abs(b).max()
        print(f"ragged bc{bc} k{k} d/d{key}: rel err {err:.2e} (max |ref| {np.abs(b).max():.3e})")
        assert err <= 2e-3, (key, err)
