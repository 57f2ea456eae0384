"""GPU adjoint (pgmpm_forward_checkpointed / pgmpm_backward) against the FP64
oracle adjoint and against central finite differences of the GPU forward.

Tolerances:
  * vs the FP64 oracle adjoint: per field, max |gpu - oracle| <= 2e-3 *
    max |oracle| (FP32 forward replay and atomics vs FP64);
  * vs central FD of the GPU FP32 forward along structured directions (the
    per-coordinate FD of a COM loss is below FP32 resolution, so the
    directions sum many coordinates): relative error <= 1e-3 for v0 and E.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(rng, N, n, spread=0.03, lo=0.35, hi=0.6):
    dx = 1.0 / n
    V0 = np.full(N, (dx / 2) ** 3, np.float32)
    return dict(x=rng.uniform(lo, hi, (N, 3)).astype(np.float32), v=rng.normal(0, 0.3, (N, 3)).astype(np.float32),
                C=rng.normal(0, 0.5, (N, 9)).astype(np.float32),
                F=(np.tile(np.eye(3).ravel(), (N, 1)) + rng.normal(0, spread, (N, 9))).astype(np.float32),
                m=(1000 * V0).astype(np.float32), V0=V0, mat=(np.arange(N) % 3).astype(np.int32))


@pytest.mark.parametrize("bc,k", [(1, 2), (2, 3), (3, 1), (1, 6)])
def test_adjoint_matches_fp64_oracle(gpu, oracle, bc, k):
    rng = np.random.default_rng(40 + bc + k)
    N, n, steps, dt = 1500, 16, 6, 1e-3
    st = _case(rng, N, n)
    mats_o = [(oracle.FIXED_COROTATED, 1e4, 0.3), (oracle.NEO_HOOKEAN, 3e4, 0.25), (oracle.EOS_FLUID, 1e4, 0.0)]
    mats = [gpu.createElasticMaterial(1000, 1e4, 0.3), gpu.createElasticMaterial(1000, 3e4, 0.25, 1),
            gpu.createFluidMaterial(1000, 0.0, 1e4)]
    scene = gpu.Scene((n, n, n), 1.0 / n, dt, (0, -9.8, 0), (0, 0, 0), 0, bc, 3)
    sim = gpu.Simulator([scene], [N], mats)
    sim.upload(st["x"], st["v"], st["C"], st["F"], st["m"], st["V0"], st["mat"])
    sim.forward_checkpointed(steps, k)
    out = sim.download()
    tgt = np.array([0.5, 0.3, 0.5])
    go = {"x": np.tile(2 * (out["x"].mean(0) - tgt) / N, (N, 1)).astype(np.float32),
          "v": (0.2 * out["v"]).astype(np.float32), "F": (0.02 * out["F"].reshape(N, 9)).astype(np.float32),
          "C": (0.01 * out["C"].reshape(N, 9)).astype(np.float32)}
    g = sim.backward(go)
    osc = oracle.make_scene((n, n, n), 1.0 / n, dt, physics=oracle.MLS, boundary=bc, bthick=3)
    ost = {k_: st[k_].astype(np.float64) for k_ in ("x", "v", "C", "F", "m", "V0")}
    ost["mat"] = st["mat"]
    ref = oracle.adjoint(osc, oracle.make_materials(mats_o), ost, steps, {k_: v.astype(np.float64) for k_, v in go.items()})
    for key in ("x", "v", "C", "F", "E"):
        a = np.asarray(g[key]).reshape(-1)
        b = np.asarray(ref[key]).reshape(-1)
        err = np.abs(a - b).max() / np.abs(b).max()
        print(f"bc{bc} k{k} d/d{key}: rel err {err:.2e} (max |ref| {np.abs(b).max():.3e})")
        assert err <= 2e-3, (key, err)


@pytest.mark.parametrize("case,k", [("plastic", 2), ("viscous", 3)])
def test_plastic_and_viscous_adjoint_matches_fp64_oracle(gpu, oracle, case, k):
    """The adjoint of the ELASTOPLASTIC model (von Mises cap active on most
    particles: stretched F, a low yield stress) and of the viscous EOS fluid
    (tau += J mu_v (C + C^T)) against the FP64 oracle's adjoint, which
    matches FP64 central differences (tests/test_oracle.py)."""
    rng = np.random.default_rng(80 + k)
    N, n, steps, dt = 1500, 16, 6, 1e-3
    st = _case(rng, N, n, spread=0.08)
    MT, CM = gpu.MaterialType, gpu.ConstitutiveModel
    if case == "plastic":
        mats_o = [(3, 2e4, 0.3, 150.0), (oracle.FIXED_COROTATED, 1e4, 0.3), (3, 1e4, 0.25, 1e9)]
        mats = [gpu.MaterialParameters(1000, 2e4, 0.3, MT.ELASTOPLASTIC, CM.NEO_HOOKEAN, yield_stress=150.0),
                gpu.createElasticMaterial(1000, 1e4, 0.3),
                gpu.MaterialParameters(1000, 1e4, 0.25, MT.ELASTOPLASTIC, CM.NEO_HOOKEAN, yield_stress=1e9)]
    else:
        mats_o = [(oracle.EOS_FLUID, 1e4, 0.0, 0.0, 30.0), (oracle.NEO_HOOKEAN, 3e4, 0.25),
                  (oracle.EOS_FLUID, 2e4, 0.0, 0.0, 5.0)]
        mats = [gpu.createFluidMaterial(1000, 30.0, 1e4), gpu.createElasticMaterial(1000, 3e4, 0.25, 1),
                gpu.createFluidMaterial(1000, 5.0, 2e4)]
    scene = gpu.Scene((n, n, n), 1.0 / n, dt, (0, -9.8, 0), (0, 0, 0), 0, 1, 3)
    sim = gpu.Simulator([scene], [N], mats)
    sim.upload(st["x"], st["v"], st["C"], st["F"], st["m"], st["V0"], st["mat"])
    sim.forward_checkpointed(steps, k)
    out = sim.download()
    tgt = np.array([0.5, 0.3, 0.5])
    go = {"x": np.tile(2 * (out["x"].mean(0) - tgt) / N, (N, 1)).astype(np.float32),
          "v": (0.2 * out["v"]).astype(np.float32), "F": (0.02 * out["F"].reshape(N, 9)).astype(np.float32),
          "C": (0.01 * out["C"].reshape(N, 9)).astype(np.float32)}
    g = sim.backward(go)
    assert sim.status() == 0
    osc = oracle.make_scene((n, n, n), 1.0 / n, dt, physics=oracle.MLS, boundary=1, bthick=3)
    ost = {k_: st[k_].astype(np.float64) for k_ in ("x", "v", "C", "F", "m", "V0")}
    ost["mat"] = st["mat"]
    ref = oracle.adjoint(osc, oracle.make_materials(mats_o), ost, steps,
                         {k_: v.astype(np.float64) for k_, v in go.items()})
    for key in ("x", "v", "C", "F", "E"):
        a = np.asarray(g[key]).reshape(-1)
        b = np.asarray(ref[key]).reshape(-1)
        err = np.abs(a - b).max() / np.abs(b).max()
        print(f"{case} d/d{key}: rel err {err:.2e} (max |ref| {np.abs(b).max():.3e})")
        assert err <= 2e-3, (key, err)


def test_adjoint_scatter_variants_agree(gpu):
    """The G2P-reverse scatter runs on the P2G kernel variant in use; the
    (cell, z-slice), thread-per-cell and balanced-run (variant 4) scatters
    give the same gradients."""
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.two_material_drop(n_particles=20000, n=32, seed=4)
    N = counts[0]
    res = []
    for variant in (0, 2, 4):
        sim = gpu.Simulator(scenes, counts, mats)
        sim.set_variants(p2g_variant=variant)
        sim.upload(st["x"], st["v"], None, None, st["m"], st["V0"], st["mat"])
        sim.forward_checkpointed(10, 5)
        out = sim.download()
        res.append(sim.backward({"x": (out["x"] - 0.5).astype(np.float32) / N, "v": out["v"] / N}))
    for other in res[1:]:
        for key in ("x", "v", "C", "F", "E"):
            a, b = np.asarray(res[0][key]).ravel(), np.asarray(other[key]).ravel()
            assert np.abs(a - b).max() <= 1e-4 * np.abs(a).max() + 1e-12, key


def test_checkpoint_interval_does_not_change_gradients(gpu):
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.elastic_cube(n_particles=8192, n=32, v_sigma=0.2, seed=21)
    N = counts[0]
    res = []
    for k in (1, 4, 16):
        sim = gpu.Simulator(scenes, counts, mats)
        sim.upload(st["x"], st["v"], None, None, st["m"], st["V0"])
        sim.forward_checkpointed(16, k)
        out = sim.download()
        g = sim.backward({"x": np.tile(2 * (out["x"].mean(0) - np.array([0.5, 0.3, 0.5])) / N, (N, 1)).astype(np.float32)})
        res.append(g)
    for g in res[1:]:
        for key in ("x", "v", "F", "E"):
            a, b = np.asarray(g[key]).ravel(), np.asarray(res[0][key]).ravel()
            assert np.abs(a - b).max() <= 1e-3 * np.abs(b).max() + 1e-12, key


@pytest.mark.parametrize("steps,k", [(40, 6), (32, 8), (12, 8), (5, 16)])
def test_overlapped_and_sequential_backward_agree(gpu, steps, k):
    """With the bin sort the forward leaves its last two segments in the two
    tape sets, and the backward replays segment s - 1 into the free set on a
    side stream while segment s is reversed; with the radix step sort each
    segment is replayed and reversed in turn.  Both give the same gradients:
    segments of uneven length (40 = 6 x 6 + 4), of equal length, two segments
    (no replay at all) and a single segment."""
    from physgrad_b200 import _capi as C
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.two_material_drop(n_particles=20000, n=32, seed=23)
    N = counts[0]
    res = []
    for sort in (C.SORT_BINS, C.SORT_RADIX):
        sim = gpu.Simulator(scenes, counts, mats)
        sim.set_step_sort(sort)
        sim.upload(st["x"], st["v"], None, None, st["m"], st["V0"], st["mat"])
        sim.forward_checkpointed(steps, k)
        out = sim.download()
        res.append(sim.backward({"x": (out["x"] - 0.5).astype(np.float32) / N, "v": out["v"] / N}))
        assert sim.status() == 0
    for key in ("x", "v", "C", "F", "E"):
        a, b = np.asarray(res[0][key]).ravel(), np.asarray(res[1][key]).ravel()
        assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max() + 1e-12, key


def _com_loss_and_grads(gpu, scenes, counts, mats, st, steps, k, E=None, v0=None, want_grad=True, loss_kind="com",
                        F0=None):
    """loss "com": ||COM(x_T) - (0.5, 0.3, 0.5)||^2 (the differentiable
    configuration's loss); "spread": mean ||x_T - (0.5, 0.3, 0.5)||^2."""
    import torch

    from physgrad_b200.autograd import simulate

    N = int(sum(counts))
    sim = gpu.Simulator(scenes, counts, mats)
    dev = torch.device("cuda")
    x0 = torch.tensor(st["x"], device=dev)
    v0t = torch.tensor(st["v"] if v0 is None else v0, device=dev, requires_grad=want_grad)
    Et = torch.tensor([m.youngs_modulus for m in mats] if E is None else E, dtype=torch.float32, device=dev,
                      requires_grad=want_grad)
    m = torch.tensor(st["m"], device=dev)
    V0 = torch.tensor(st["V0"], device=dev)
    mat = torch.tensor(st["mat"], device=dev) if st.get("mat") is not None else None
    F0t = None if F0 is None else torch.tensor(F0, device=dev)
    x, v, C, F = simulate(sim, x0, v0t, Et, m, V0, steps, k, mat=mat, F0=F0t)
    tgt = torch.tensor([0.5, 0.3, 0.5], device=dev, dtype=torch.float64)
    if loss_kind == "com":
        loss = ((x.double().mean(0) - tgt) ** 2).sum()
    else:
        loss = ((x.double() - tgt) ** 2).sum(1).mean()
    if not want_grad:
        return float(loss)
    loss.backward()
    return float(loss.detach()), v0t.grad.cpu().numpy(), Et.grad.cpu().numpy()


def test_autograd_function_vs_central_differences(gpu):
    """Config-3 shapes at reduced size: COM loss, gradients w.r.t. v0 and E."""
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.elastic_cube(n_particles=32768, n=64, v_sigma=0.1, seed=3)
    steps, k = 64, 16
    L, gv0, gE = _com_loss_and_grads(gpu, scenes, counts, mats, st, steps, k)
    # direction 1: uniform shift of v0 in y (sum of all dL/dv0_y)
    for d_dir in ("y", "rand"):
        rng = np.random.default_rng(5)
        d = np.zeros_like(st["v"])
        if d_dir == "y":
            d[:, 1] = 1.0
        else:
            d = rng.choice([-1.0, 1.0], size=st["v"].shape).astype(np.float32) * (rng.random(st["v"].shape) < 0.5)
            d += np.array([0.3, 0.6, -0.2], np.float32)
        eps = 1e-3
        Lp = _com_loss_and_grads(gpu, scenes, counts, mats, st, steps, k, v0=st["v"] + eps * d, want_grad=False)
        Lm = _com_loss_and_grads(gpu, scenes, counts, mats, st, steps, k, v0=st["v"] - eps * d, want_grad=False)
        fd = (Lp - Lm) / (2 * eps)
        ad = float((gv0 * d).sum())
        print(f"v0 direction {d_dir}: FD {fd:.6e} adjoint {ad:.6e} rel {abs(fd - ad) / abs(fd):.2e}")
        assert abs(fd - ad) <= 1e-3 * abs(fd), (fd, ad)
    # The COM loss does not depend on E: the transfers conserve momentum, so
    # internal stress cannot move the centre of mass (no wall contact here).
    assert abs(gE[0]) <= 1e-12
    # dL/dE on a loss that does depend on it: a pre-stretched cube, spread loss
    N = counts[0]
    F0 = np.tile(np.diag([1.04, 0.97, 1.0]).astype(np.float32), (N, 1, 1))
    kw = dict(loss_kind="spread", F0=F0)
    _, _, gE2 = _com_loss_and_grads(gpu, scenes, counts, mats, st, steps, k, **kw)
    E0 = mats[0].youngs_modulus
    hE = 1e-2 * E0
    Lp = _com_loss_and_grads(gpu, scenes, counts, mats, st, steps, k, E=[E0 + hE], want_grad=False, **kw)
    Lm = _com_loss_and_grads(gpu, scenes, counts, mats, st, steps, k, E=[E0 - hE], want_grad=False, **kw)
    fd = (Lp - Lm) / (2 * hE)
    print(f"E (spread loss, stretched cube): FD {fd:.6e} adjoint {gE2[0]:.6e} rel {abs(fd - gE2[0]) / abs(fd):.2e}")
    assert abs(fd - gE2[0]) <= 1e-2 * abs(fd), (fd, gE2[0])


def test_batched_adjoint_equals_single_scenes(gpu):
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.batched_scenes(n_scenes=3, lo=2000, hi=8000, seed=8, v_sigma=0.2)
    N = int(sum(counts))
    sim = gpu.Simulator(scenes, counts, mats)
    sim.upload(st["x"], st["v"], None, None, st["m"], st["V0"], st["mat"])
    sim.forward_checkpointed(8, 4)
    out = sim.download()
    go = {"x": (out["x"] - 0.5).astype(np.float32) / N}
    gb = sim.backward(go)
    off = 0
    for s, c in enumerate(counts):
        sl = slice(off, off + c)
        one = gpu.Simulator([scenes[s]], [c], [mats[s]])
        one.upload(st["x"][sl], st["v"][sl], None, None, st["m"][sl], st["V0"][sl])
        one.forward_checkpointed(8, 4)
        g1 = one.backward({"x": go["x"][sl]})
        assert np.abs(gb["v"][sl] - g1["v"]).max() <= 1e-3 * np.abs(g1["v"]).max()
        assert abs(gb["E"][s] - g1["E"][0]) <= 1e-3 * abs(g1["E"][0]) + 1e-12
        off += c


def test_checkpointed_forward_leaves_the_stepped_state(gpu):
    """forward_checkpointed runs its last segment in the tape and hands the
    state back: the live state, the grid and later steps match plain
    stepping (to FP32 summation-order tolerance: atomic order differs)."""
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.two_material_drop(n_particles=30000, n=32, seed=5)
    outs = []
    for mode in ("plain", "checkpointed"):
        sim = gpu.Simulator(scenes, counts, mats)
        sim.upload(st["x"], st["v"], None, None, st["m"], st["V0"], st["mat"])
        if mode == "plain":
            sim.step(13)
        else:
            sim.forward_checkpointed(13, 5)  # segments of 5, 5, 3: the last runs in the tape
        grid = sim.grid(0)
        mid = sim.download()
        sim.step(4)  # stepping continues from the handed-back state
        outs.append((mid, grid, sim.download(), sim.metrics()["total_steps"]))
        assert sim.status() == 0
        sim.close()
    (m0, g0, e0, n0), (m1, g1, e1, n1) = outs
    assert n0 == n1 == 17
    for key in ("x", "v", "C", "F"):
        for a, b in ((m0, m1), (e0, e1)):
            err = np.abs(a[key] - b[key]).max() / max(np.abs(a[key]).max(), 1e-30)
            assert err < 1e-4, (key, err)
    (gm0, gv0), (gm1, gv1) = g0, g1
    assert np.abs(gm0 - gm1).max() <= 1e-4 * np.abs(gm0).max()
    assert np.abs(gv0 - gv1).max() <= 1e-3 * (np.abs(gv0).max() + 1e-6)


def test_recording_invalidated_by_scene_or_material_change(gpu):
    """pgmpm_backward differentiates the recording of the last
    pgmpm_forward_checkpointed; after pgmpm_set_scene_params or
    pgmpm_set_materials its replay would run other physics, so it fails with
    PGMPM_ERR_STATE until the forward is run again."""
    from physgrad_b200 import _capi as C

    rng = np.random.default_rng(61)
    N, n = 400, 16
    st = _case(rng, N, n)
    mats = [gpu.createElasticMaterial(1000, 1e4, 0.3), gpu.createElasticMaterial(1000, 3e4, 0.25, 1),
            gpu.createFluidMaterial(1000, 0.0, 1e4)]
    sim = gpu.Simulator([gpu.Scene((n, n, n), 1.0 / n, 1e-3, (0, -9.8, 0), (0, 0, 0), 0, 1, 3)], [N], mats)
    sim.upload(st["x"], st["v"], st["C"], st["F"], st["m"], st["V0"], st["mat"])
    go = {"x": np.full((N, 3), 1.0 / N, np.float32)}
    sim.forward_checkpointed(4, 2)
    g0 = sim.backward(go)
    sim.set_scene_params(0, dt=5e-4)
    with pytest.raises(C.PGMPMError) as ei:
        sim.backward(go)
    assert ei.value.code == C.PGMPM_ERR_STATE
    sim.set_scene_params(0, dt=1e-3)
    sim.upload(st["x"], st["v"], st["C"], st["F"], st["m"], st["V0"], st["mat"])
    sim.forward_checkpointed(4, 2)
    g1 = sim.backward(go)
    assert np.abs(g1["v"] - g0["v"]).max() <= 1e-5 * np.abs(g0["v"]).max()
    sim.set_materials(mats)
    with pytest.raises(C.PGMPMError) as ei:
        sim.backward(go)
    assert ei.value.code == C.PGMPM_ERR_STATE


def test_tape_steps_report_error_flags(gpu):
    """A particle leaving the grid inside the segment the forward runs in the
    tape still raises PGMPM_FLAG_ESCAPE on the solver."""
    from physgrad_b200 import _capi as C

    s = gpu.Scene((16, 16, 16), 1 / 16, 1e-3, boundary=C.BC_NONE)
    mats = [gpu.createElasticMaterial(1000, 1e4, 0.3)]
    sim = gpu.Simulator([s], [2], mats)
    x = np.array([[0.5, 0.5, 0.5], [0.5, 0.5, 0.5]], np.float32)
    v = np.array([[0, 0, 0], [0, 0, 300.0]], np.float32)
    sim.upload(x, v, None, None, np.full(2, 1e-3, np.float32), np.full(2, 1e-6, np.float32))
    sim.forward_checkpointed(30, 30)  # one segment: every step runs in the tape
    assert sim.status() & C.FLAG_ESCAPE


# ------------------------------------------- launch_mpm_timestep_backward
def _ref_step_case(rng, N, res):
    """Particles whose fractional cell coordinate is in [0.1, 0.9]: the
    reference's floor-based 3-node stencil jumps where a coordinate crosses a
    cell boundary, so central differences need room on both sides."""
    cells = rng.integers(6, res - 6, (N, 3))
    x = ((cells + rng.uniform(0.1, 0.9, (N, 3))) / res).astype(np.float32)
    v = rng.normal(0, 0.5, (N, 3)).astype(np.float32)
    m = (rng.uniform(0.5, 1.5, N) * 1e-3).astype(np.float32)
    return x, v, m


def _ref_loss(oracle, x, v, m, g, res, dt, steps, sx, sv):
    """sum(sx . x') + sum(sv . v') after `steps` REF steps, FP64 oracle."""
    N = x.shape[0]
    sc = oracle.make_scene((res, res, res), 1.0 / res, dt, gravity=tuple(g), physics=oracle.REF_COMPAT,
                           boundary=oracle.BC_NONE)
    st = dict(x=x, v=v, C=np.zeros((N, 9)), F=np.tile(np.eye(3).ravel(), (N, 1)), m=m, V0=np.full(N, 1e-6))
    o = oracle.run(sc, oracle.make_materials([(0, 1e4, 0.3)]), st, steps, prec=64)
    return float((sx * o["x"]).sum() + (sv * o["v"]).sum())


def _fd_check(oracle, rng, x, v, m, g, res, dt, steps, sx, sv, grads, n_samples=6):
    """Central differences (FP64, eps 1e-6) of _ref_loss at sampled entries
    of x, v, m and every entry of g against the given gradients; per input,
    max error <= 1e-3 * max |difference quotient|."""
    base = dict(x=x.astype(np.float64), v=v.astype(np.float64), m=m.astype(np.float64), g=g.astype(np.float64))
    eps = 1e-6
    for key in ("x", "v", "m", "g"):
        arr = base[key]
        idx = [tuple(rng.integers(0, s) for s in arr.shape) for _ in range(n_samples)] if key != "g" else \
            [(0,), (1,), (2,)]
        num, ana = [], []
        for i in idx:
            hi = {k: a.copy() for k, a in base.items()}
            lo = {k: a.copy() for k, a in base.items()}
            hi[key][i] += eps
            lo[key][i] -= eps
            f = lambda d: _ref_loss(oracle, d["x"], d["v"], d["m"], d["g"], res, dt, steps, sx, sv)
            num.append((f(hi) - f(lo)) / (2 * eps))
            ana.append(float(grads[key][i]))
        num, ana = np.array(num), np.array(ana)
        print(f"d/d{key}: max |fd - adjoint| {np.abs(num - ana).max():.2e} of max |fd| {np.abs(num).max():.2e}")
        assert np.abs(num - ana).max() <= 1e-3 * np.abs(num).max() + 1e-12, (key, num, ana)


def test_launch_mpm_timestep_backward_vs_central_differences(gpu, oracle):
    """launch_mpm_timestep_backward (src/pytorch_autograd.cu:384-402 shape):
    the reverse of the REF_COMPAT step launch_mpm_timestep_forward runs,
    against central differences of the FP64 oracle's REF step for positions,
    velocities, masses and gravity.  Also: the forward output matches the
    float oracle, and a backward without a matching forward is an error."""
    import torch
    from physgrad_b200 import _capi as C

    L = C.lib()
    rng = np.random.default_rng(71)
    N, res, dt = 3000, 32, 2e-3
    x, v, m = _ref_step_case(rng, N, res)
    g = np.array([0.3, -9.8, 0.5], np.float32)
    sx = rng.normal(0, 1, (N, 3))
    sv = rng.normal(0, 1, (N, 3))
    dev = torch.device("cuda:0")
    t = lambda a: torch.tensor(a, dtype=torch.float32, device=dev)
    tx, tv, tm, tg = t(x), t(v), t(m), t(g)
    L.pgmpm_clear_error()
    L.launch_mpm_timestep_forward(tx.data_ptr(), tv.data_ptr(), tm.data_ptr(), N, res, dt, tg.data_ptr(), None)
    torch.cuda.synchronize()
    assert L.pgmpm_last_error() == b""
    sc = oracle.make_scene((res, res, res), np.float32(1.0 / res), np.float32(dt), gravity=tuple(g),
                           physics=oracle.REF_COMPAT, boundary=oracle.BC_NONE)
    st = dict(x=x.astype(np.float64), v=v.astype(np.float64), C=np.zeros((N, 9)),
              F=np.tile(np.eye(3).ravel(), (N, 1)), m=m.astype(np.float64), V0=np.full(N, 1e-6))
    fwd = oracle.run(sc, oracle.make_materials([(0, 1e4, 0.3)]), st, 1, prec=32)
    assert np.abs(tx.cpu().numpy() - fwd["x"]).max() <= 1e-6
    assert np.abs(tv.cpu().numpy() - fwd["v"]).max() <= 1e-4 * np.abs(fwd["v"]).max()
    gix, giv, gim, gg = torch.empty_like(tx), torch.empty_like(tv), torch.empty_like(tm), torch.zeros_like(tg)
    # every tensor whose pointer crosses the C-ABI stays referenced until the
    # kernels are done (a temporary's block would be handed to the next one)
    tsx, tsv, tx0, tv0 = t(sx), t(sv), t(x), t(v)
    L.launch_mpm_timestep_backward(tsx.data_ptr(), tsv.data_ptr(), gix.data_ptr(), giv.data_ptr(), gim.data_ptr(),
                                   gg.data_ptr(), tx0.data_ptr(), tv0.data_ptr(), N, res, dt, None)
    torch.cuda.synchronize()
    assert L.pgmpm_last_error() == b""
    grads = {"x": gix.cpu().numpy(), "v": giv.cpu().numpy(), "m": gim.cpu().numpy(), "g": gg.cpu().numpy()}
    _fd_check(oracle, rng, x, v, m, g, res, dt, 1, sx, sv, grads)
    L.launch_mpm_timestep_backward(tsx.data_ptr(), tsv.data_ptr(), gix.data_ptr(), giv.data_ptr(), gim.data_ptr(),
                                   gg.data_ptr(), tx0.data_ptr(), tv0.data_ptr(), N, res + 4, dt, None)
    torch.cuda.synchronize()
    assert b"no launch_mpm_timestep_forward call" in L.pgmpm_last_error()


def test_mpm_timestep_function_rollout_vs_central_differences(gpu, oracle):
    """physgrad_b200.autograd.MPMTimestep chained over 3 steps by torch
    autograd: gradients of sum(sx . x3) + sum(sv . v3) with respect to the
    initial positions, velocities, masses and gravity against central
    differences of the FP64 oracle's 3-step REF run."""
    import torch
    from physgrad_b200.autograd import MPMTimestep

    rng = np.random.default_rng(72)
    N, res, dt, steps = 2000, 32, 2e-3, 3
    x, v, m = _ref_step_case(rng, N, res)
    g = np.array([0.0, -9.8, 1.0], np.float32)
    sx = rng.normal(0, 1, (N, 3))
    sv = rng.normal(0, 1, (N, 3))
    dev = torch.device("cuda:0")
    leaf = lambda a: torch.tensor(a, dtype=torch.float32, device=dev, requires_grad=True)
    tx, tv, tm, tg = leaf(x), leaf(v), leaf(m), leaf(g)
    xs, vs = tx, tv
    for _ in range(steps):
        xs, vs = MPMTimestep.apply(xs, vs, tm, tg, res, dt)
    loss = (torch.tensor(sx, dtype=torch.float32, device=dev) * xs).sum() + \
        (torch.tensor(sv, dtype=torch.float32, device=dev) * vs).sum()
    loss.backward()
    grads = {"x": tx.grad.cpu().numpy(), "v": tv.grad.cpu().numpy(), "m": tm.grad.cpu().numpy(),
             "g": tg.grad.cpu().numpy()}
    _fd_check(oracle, rng, x, v, m, g, res, dt, steps, sx, sv, grads)


def test_reference_adjoint_returns_zeros_where_ours_matches_fd(gpu, oracle):
    """The reference's own MPM adjoint on the inputs of
    test_adjoint_matches_fp64_oracle (x, v, m of its seeded case; C = 0, F = I,
    the reference's starting state): DifferentiableMPMSystem<float> records an
    empty backward (src/differentiable_mpm.h:871-876), so computeGradients()
    returns zeros for every particle.  Our adjoint of the centre-of-mass loss
    on the same inputs is non-zero and matches FP64 central differences
    (eps 1e-3) at 8 seeded v0 coordinates to 1e-3 relative."""
    if not oracle.ref_diff_available():
        pytest.skip("oracle/_ref not built")
    bc, k = 1, 2
    rng = np.random.default_rng(40 + bc + k)
    N, n, steps, dt = 1500, 16, 6, 1e-3
    st = _case(rng, N, n)
    ref = oracle.ref_diff_run(st["x"], st["v"], st["m"], (n, n, n), 1.0 / n, dt, steps)
    assert np.abs(ref["x"] - st["x"]).max() > 0.0  # the reference did step the particles
    mats = [gpu.createElasticMaterial(1000, 1e4, 0.3)]
    scene = gpu.Scene((n, n, n), 1.0 / n, dt, (0, -9.8, 0), (0, 0, 0), 0, bc, 3)
    sim = gpu.Simulator([scene], [N], mats)
    sim.upload(st["x"], st["v"], None, None, st["m"], st["V0"])
    sim.forward_checkpointed(steps, k)
    x = sim.download()["x"].astype(np.float64)
    tgt = np.array([0.5, 0.3, 0.5])
    g = sim.backward({"x": np.tile(2.0 * (x.mean(0) - tgt) / N, (N, 1)).astype(np.float32)})
    osc = oracle.make_scene((n, n, n), 1.0 / n, dt, physics=oracle.MLS, boundary=bc, bthick=3)
    ost = {"x": st["x"].astype(np.float64), "v": st["v"].astype(np.float64), "C": np.zeros((N, 9)),
           "F": np.tile(np.eye(3).ravel(), (N, 1)), "m": st["m"].astype(np.float64), "V0": st["V0"].astype(np.float64)}
    coords = [(int(p), int(a)) for p, a in zip(rng.choice(N, 8, replace=False), rng.integers(0, 3, 8))]
    fd = oracle.fd_v0_com(osc, oracle.make_materials([(oracle.FIXED_COROTATED, 1e4, 0.3)]), ost, steps, coords,
                          eps=1e-3, target=tgt)
    ours = np.array([g["v"][p, c] for p, c in coords])
    theirs = np.array([ref["grad_v"][p, c] for p, c in coords])
    for (p, c), a, b, f in zip(coords, ours, theirs, fd):
        print(f"dL/dv0[{p},{c}]: ours {a:+.6e}  reference {b:+.1e}  FP64 central difference {f:+.6e}")
    assert not np.any(ref["grad_v"]) and not np.any(ref["grad_x"])
    assert np.abs(ours).min() > 0.0
    assert (np.abs(ours - fd) <= 1e-3 * np.abs(fd)).all(), (ours, fd)


def test_backward_twice_on_one_recording_gives_the_same_gradients(gpu):
    """A second backward over the same recording replays every segment
    (including the one the forward left in the tape, which the first
    backward overwrote) and must return the same non-zero gradients: the
    reverse scatter takes its work from the cursor the replayed step's grid
    update leaves at zero."""
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.two_material_drop(n_particles=20000, n=32, seed=31)
    N = counts[0]
    sim = gpu.Simulator(scenes, counts, mats)
    sim.upload(st["x"], st["v"], None, None, st["m"], st["V0"], st["mat"])
    sim.forward_checkpointed(24, 8)
    out = sim.download()
    go = {"x": (out["x"] - 0.5).astype(np.float32) / N, "v": out["v"] / N}
    g1 = sim.backward(go)
    g2 = sim.backward(go)
    for key in ("x", "v", "C", "F", "E"):
        a, b = np.asarray(g1[key]).ravel(), np.asarray(g2[key]).ravel()
        assert np.abs(a).max() > 0.0, key
        assert np.abs(a - b).max() <= 1e-4 * np.abs(a).max(), key


def test_two_rollouts_on_one_simulator_refuse_a_stale_backward(gpu):
    """MPMSimulate keeps the Simulator in its context; the Simulator holds one
    recording.  Two rollouts on one Simulator in one graph: the first
    rollout's backward would see the second's recording, so it raises."""
    import torch

    from physgrad_b200 import PGMPMError
    from physgrad_b200.autograd import simulate
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.elastic_cube(n_particles=4096, n=32, v_sigma=0.1, seed=33)
    sim = gpu.Simulator(scenes, counts, mats)
    dev = torch.device("cuda")
    x0 = torch.tensor(st["x"], device=dev)
    m, V0 = torch.tensor(st["m"], device=dev), torch.tensor(st["V0"], device=dev)
    E = torch.tensor([1e4], device=dev, requires_grad=True)
    va = torch.tensor(st["v"], device=dev, requires_grad=True)
    vb = torch.tensor(st["v"] * 0.5, device=dev, requires_grad=True)
    xa = simulate(sim, x0, va, E, m, V0, 8, 4)[0]
    xb = simulate(sim, x0, vb, E, m, V0, 8, 4)[0]
    with pytest.raises(PGMPMError, match="another forward"):
        (xa.sum() + xb.sum()).backward()
    # one Simulator per rollout works
    sim2 = gpu.Simulator(scenes, counts, mats)
    va.grad = None
    xa = simulate(sim, x0, va, E, m, V0, 8, 4)[0]
    xb = simulate(sim2, x0, vb, E, m, V0, 8, 4)[0]
    (xa.sum() + xb.sum()).backward()
    assert va.grad is not None and vb.grad is not None


def _grads(gpu, scenes, counts, mats, st, steps, k, record, between=None):
    """Gradients of a COM-and-velocity loss with the sort recording in mode
    `record`; with a recording also a second backward over it.  between(sim)
    runs after the forward."""
    sim = gpu.Simulator(scenes, counts, mats)
    sim.set_sort_record(record)
    sim.upload(st["x"], st["v"], None, None, st["m"], st["V0"], st.get("mat"))
    sim.forward_checkpointed(steps, k)
    out = sim.download()
    N = int(sum(counts))
    go = {"x": (out["x"] - 0.5).astype(np.float32) / N, "v": (out["v"] / N).astype(np.float32)}
    if between is not None:
        between(sim)
    g = sim.backward(go)
    g2 = sim.backward(go) if record else None
    return g, g2, sim.replay_resorts()


def test_recorded_sorts_give_the_gradients_of_sorting_replays(gpu):
    """With the bin sort, pgmpm_forward_checkpointed records every step's sort
    and the backward's replays keep it.  The gradients equal those of replays
    that sort every step (recording off) to FP32 rounding, and a second
    backward over the same recording gives them again."""
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.two_material_drop(n_particles=20000, n=32, seed=31)
    ga, ga2, _ = _grads(gpu, scenes, counts, mats, st, 40, 8, True)
    gb, _, _ = _grads(gpu, scenes, counts, mats, st, 40, 8, False)
    for key in ("x", "v", "C", "F", "E"):
        a, a2, b = (np.asarray(g[key]).ravel() for g in (ga, ga2, gb))
        scale = np.abs(b).max()
        print(f"d/d{key}: recorded vs sorting replays {np.abs(a - b).max() / scale:.2e}, "
              f"second backward {np.abs(a2 - a).max() / scale:.2e}")
        assert scale > 0.0, key
        assert np.abs(a - b).max() <= 1e-4 * scale, key
        assert np.abs(a2 - a).max() <= 1e-4 * scale, key


def test_replayed_steps_that_sort_again_give_the_same_gradients(gpu):
    """The conditional sort of a replayed step: with the recording in mode 2
    every replayed step after a segment's first runs it (counted by
    pgmpm_get_replay_resorts), and the gradients equal those of replays that
    sort every step.  (In mode 1 a step runs it only after a G2P put a
    particle in another cell than the forward did, which rounding makes
    rare.)"""
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.config3(n_particles=65536, steps=64)
    ga, ga2, resorts = _grads(gpu, scenes, counts, mats, st, 64, 16, 2)
    gb, _, none = _grads(gpu, scenes, counts, mats, st, 64, 16, 0)
    # two backwards; each replays 2 of the 4 segments the first time and all
    # 4 the second (the forward's tape is overwritten), 15 steps each
    print(f"replayed steps that sorted again: {resorts}")
    assert none == 0
    assert resorts == (2 + 4) * 15
    for key in ("x", "v", "C", "F", "E"):
        a, a2, b = (np.asarray(g[key]).ravel() for g in (ga, ga2, gb))
        scale = np.abs(b).max()
        print(f"d/d{key}: re-sorting replays vs sorting replays {np.abs(a - b).max() / scale:.2e}")
        assert scale > 0.0, key
        assert np.abs(a - b).max() <= 1e-4 * scale, key
        assert np.abs(a2 - b).max() <= 1e-4 * scale, key


@pytest.mark.parametrize("change", ["radix_sort", "fused_kernel"])
def test_backward_after_a_sort_or_kernel_change_replays_every_segment(gpu, change):
    """A recorded forward, then the step sort switched to the radix sort or
    P2G to the fused kernel: the backward cannot keep the recorded sorts
    (the radix path does not index them, the fused steps sort their own), so
    it replays every segment, the ones the forward left on the tape too, with
    their own sorts.  The gradients equal those of an unrecorded run."""
    from physgrad_b200 import _capi as C
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.two_material_drop(n_particles=20000, n=32, seed=31)
    act = {"radix_sort": lambda s: s.set_step_sort(C.SORT_RADIX),
           "fused_kernel": lambda s: s.set_variants(p2g_variant=5)}[change]
    ga, ga2, _ = _grads(gpu, scenes, counts, mats, st, 40, 8, 1, between=act)
    gb, _, _ = _grads(gpu, scenes, counts, mats, st, 40, 8, 0)
    for key in ("x", "v", "C", "F", "E"):
        a, a2, b = (np.asarray(g[key]).ravel() for g in (ga, ga2, gb))
        scale = np.abs(b).max()
        print(f"{change} d/d{key}: {np.abs(a - b).max() / scale:.2e}, second backward {np.abs(a2 - b).max() / scale:.2e}")
        assert np.abs(a - b).max() <= 1e-4 * scale, key
        assert np.abs(a2 - b).max() <= 1e-4 * scale, key
