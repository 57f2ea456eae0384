"""Parity at the full sizes of the benchmarked configurations.

The bench line is measured on the two-material drop (2,097,152 particles on
a 128^3 grid) and the differentiable elastic cube (262,144 particles, 64^3,
256 steps); these tests check the CUDA path on exactly those inputs
(physgrad_b200.workloads, the same seeds bench.py uses) against the FP64 CPU
oracle, with the bounds of tests/test_gpu_forward.py:
  * MLS positions: max |dx| <= 2e-5 (domain of size 1, so also relative);
  * velocities: max |dv| <= 1e-3 max |v| + 1e-5;  F: max |dF| <= 2e-4;
  * REF_COMPAT against the reference's own CPU solver: max |err| / max |ref|
    <= 1e-4 on positions and velocities;
  * the adjoint against the FP64 oracle adjoint: max |err| <= 2e-3 max |ref|
    per field, and <= 1e-3 relative at each of 64 seeded v0 coordinates;
  * the adjoint against FP64 central differences (eps = 1e-3, 64 seeded v0
    coordinates): <= 1e-3 relative per coordinate.
Each test prints its errors (pytest -s).
"""
import numpy as np
import pytest

from test_gpu_forward import _assert_mls, _oracle_scene, _oracle_state, _sim

pytestmark = pytest.mark.gpu

TARGET = np.array([0.5, 0.3, 0.5])


def _omats(oracle, mats):
    return oracle.make_materials([(int(m.model), float(m.youngs_modulus), float(m.poisson_ratio)) for m in mats])


def test_two_material_drop_full_size_vs_fp64(gpu, oracle):
    """The benchmarked workload itself: 2,097,152 particles (neo-Hookean block
    and EOS fluid column), 128^3, slip walls, dt 5e-5, 20 steps in one call
    (the step graphs a multi-step call runs, as in the bench)."""
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, meta = W.config2()
    assert counts == [2097152] and tuple(scenes[0].n) == (128, 128, 128)
    steps = 20
    sim = _sim(gpu, scenes, counts, mats, st)
    sim.step(steps)
    out = sim.download()
    assert sim.status() == 0
    ref = oracle.run(_oracle_scene(oracle, scenes[0]), _omats(oracle, mats), _oracle_state(st), steps, prec=64)
    _assert_mls(out, ref, f"two-material drop full size ({counts[0]} particles, 128^3, {steps} steps)")


def test_elastic_cube_full_size_vs_fp64(gpu, oracle):
    """The differentiable configuration's forward: 262,144 particles (about
    37 per cell), 64^3, v0 ~ N(0, 0.1^2), fixed-corotated, 256 steps."""
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, meta = W.config3()
    assert counts == [262144] and meta["steps"] == 256
    sim = _sim(gpu, scenes, counts, mats, st)
    sim.step(meta["steps"])
    out = sim.download()
    assert sim.status() == 0
    ref = oracle.run(_oracle_scene(oracle, scenes[0]), _omats(oracle, mats), _oracle_state(st), meta["steps"],
                     prec=64)
    _assert_mls(out, ref, f"elastic cube full size ({counts[0]} particles, 64^3, {meta['steps']} steps)")


def test_ref_compat_full_size_vs_reference(gpu, oracle):
    """REF_COMPAT physics on the two-material drop's 2,097,152 positions on
    the 128^3 grid against the reference's own MPMSolver<float,64>::step
    (src/material_point_method.h:479-500) built from its sources."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.config2()
    n = tuple(int(a) for a in scenes[0].n)
    dx = np.float32(scenes[0].dx)
    steps, dt, g = 5, np.float32(5e-5), (0.0, np.float32(-9.8), 0.0)
    r = oracle.ref_run(st["x"], st["v"], st["m"], st["V0"], n, dx, dt, g, steps)
    s = gpu.RefCompatSolver(n, dx, (0, 0, 0), gpu.RefCompatSolver.SimulationParams(dt, (0.0, -9.8, 0.0)))
    s.addParticles(st["x"], st["v"], st["m"], st["V0"])
    s.step(steps)
    out = s.getParticles()
    ex = np.abs(out["x"] - r["x"]).max() / np.abs(r["x"]).max()
    ev = np.abs(out["v"] - r["v"]).max() / np.abs(r["v"]).max()
    print(f"REF_COMPAT full size ({st['x'].shape[0]} particles, 128^3, {steps} steps): rel err x {ex:.3e} v {ev:.3e}")
    assert ex <= 1e-4 and ev <= 1e-4, (ex, ev)


def _gpu_com_adjoint(gpu, scenes, counts, mats, st, steps, k):
    """Checkpointed forward and backward of the COM loss through the C-ABI;
    returns (loss, dL/dv0 [N,3], dL/dE)."""
    N = int(sum(counts))
    sim = gpu.Simulator(scenes, counts, mats)
    sim.upload(st["x"], st["v"], None, None, st["m"], st["V0"])
    sim.forward_checkpointed(steps, k)
    x = sim.download()["x"].astype(np.float64)
    com = x.mean(0)
    g = sim.backward({"x": np.tile(2.0 * (com - TARGET) / N, (N, 1)).astype(np.float32)})
    assert sim.status() == 0
    return float(((com - TARGET) ** 2).sum()), np.asarray(g["v"], np.float64), np.asarray(g["E"], np.float64)


def _seeded_coords(N, count=64, seed=2024):
    rng = np.random.default_rng(seed)
    return [(int(p), int(a)) for p, a in zip(rng.choice(N, count, replace=False), rng.integers(0, 3, count))]


def test_elastic_cube_full_size_adjoint_vs_fp64_oracle_adjoint(gpu, oracle):
    """The differentiable configuration at full size (262,144 particles, 256
    steps, checkpoints every 16): the GPU adjoint of the COM loss against the
    FP64 oracle's adjoint on the same inputs, every coordinate of dL/dv0 and
    the 64 seeded coordinates the finite-difference check uses."""
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, meta = W.config3()
    N, steps = counts[0], meta["steps"]
    L, gv, gE = _gpu_com_adjoint(gpu, scenes, counts, mats, st, steps, 16)
    osc = _oracle_scene(oracle, scenes[0])
    ost = _oracle_state(st)
    xT = oracle.run(osc, _omats(oracle, mats), ost, steps, prec=64)["x"]
    com = xT.mean(0)
    ref = oracle.adjoint(osc, _omats(oracle, mats), ost, steps, {"x": np.tile(2.0 * (com - TARGET) / N, (N, 1))})
    err = np.abs(gv - ref["v"]).max() / np.abs(ref["v"]).max()
    coords = _seeded_coords(N)
    a = np.array([gv[p, c] for p, c in coords])
    b = np.array([ref["v"][p, c] for p, c in coords])
    rel = np.abs(a - b) / np.abs(b)
    print(f"elastic cube full size adjoint: loss {L:.6e} (FP64 {((com - TARGET) ** 2).sum():.6e}); dL/dv0 max rel "
          f"err {err:.2e} (max |ref| {np.abs(ref['v']).max():.3e}); 64 coordinates max rel {rel.max():.2e}; "
          f"dL/dE {gE[0]:.3e} (FP64 {ref['E'][0]:.3e})")
    assert err <= 2e-3, err
    assert rel.max() <= 1e-3, rel.max()


def test_elastic_cube_fd_64_coordinates(gpu, oracle):
    """The finite-difference check of the differentiable configuration: eps =
    1e-3 on 64 seeded v0 coordinates, central differences of the COM loss
    computed in FP64 by the oracle (one coordinate's loss change is ~1e-9 of
    the loss, below FP32 resolution).  128 FP64 rollouts at 262,144 particles
    and 256 steps do not fit a test's time, so the scene keeps the
    configuration's density, material, velocities and checkpoint interval on
    32,768 particles and 64 steps (4 checkpointed segments)."""
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.elastic_cube(n_particles=32768, n=64, v_sigma=0.1, seed=7, lo=0.3, hi=0.45)
    N, steps = counts[0], 64
    L, gv, _ = _gpu_com_adjoint(gpu, scenes, counts, mats, st, steps, 16)
    coords = _seeded_coords(N)
    fd = oracle.fd_v0_com(_oracle_scene(oracle, scenes[0]), _omats(oracle, mats), _oracle_state(st), steps, coords,
                          eps=1e-3, target=TARGET)
    ad = np.array([gv[p, c] for p, c in coords])
    rel = np.abs(ad - fd) / np.abs(fd)
    print(f"64-coordinate FD (eps 1e-3, FP64): max rel err {rel.max():.2e}, median {np.median(rel):.2e}; "
          f"|dL/dv0| {np.abs(fd).min():.3e} .. {np.abs(fd).max():.3e}")
    assert rel.max() <= 1e-3, rel.max()
