"""Consumers of the solver's particles on the GPU against the reference's
own classes (built from its sources into oracle/_ref) and the oracle's
restatements, on the same particles:
  * SPH-MPM contact coupling (SPHMPMCouplingSystem, src/sph_mpm_coupling.h:
    453-575): pair count exact; forces to 1e-5 of the largest (the GPU sums
    a particle's pair forces in another order); energy to 1e-5 relative;
  * the FSI energy monitor (FSISimulationManager::computeTotalEnergy,
    src/fsi_coupling.h:837-858): 1e-5 relative (float sums there).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _drop(gpu, steps=5, n=40000, seed=61):
    from physgrad_b200 import workloads as W

    scenes, counts, mats, st, _ = W.two_material_drop(n_particles=n, n=64, seed=seed)
    sim = gpu.Simulator(scenes, counts, mats)
    sim.upload(st["x"], st["v"], None, None, st["m"], st["V0"], st["mat"])
    sim.step(steps)
    return sim, st


@pytest.mark.parametrize("device_arrays,two_way,radius", [(False, True, 0.02), (True, True, 0.03),
                                                          (False, False, 0.02)])
def test_sph_coupling_matches_reference_class(gpu, oracle, device_arrays, two_way, radius):
    if not oracle.ref_coupling_available():
        pytest.skip("oracle/_ref not built")
    import torch

    sim, st = _drop(gpu)
    out = sim.download()
    rng = np.random.default_rng(62)
    nq = 3000
    sx = rng.uniform(0.15, 0.9, (nq, 3)).astype(np.float32)
    sv = rng.normal(0.0, 0.5, (nq, 3)).astype(np.float32)
    kw = dict(stiffness=2e4, damping=50.0, friction=0.4, radius=radius, two_way=two_way)
    if device_arrays:
        f, fm, npairs, energy = sim.sph_coupling(torch.tensor(sx, device="cuda"), torch.tensor(sv, device="cuda"),
                                                 **kw)
        f, fm = f.cpu().numpy(), fm.cpu().numpy()
    else:
        f, fm, npairs, energy = sim.sph_coupling(sx, sv, **kw)
    ref = oracle.ref_sph_coupling(sx, sv, out["x"], out["v"], **kw)
    res = oracle.sph_coupling(sx, sv, out["x"], out["v"], **kw)
    assert res["n_pairs"] == ref["n_pairs"]
    print(f"coupling r={radius}: {npairs} pairs (reference {ref['n_pairs']}), energy {energy:.6e} "
          f"(reference {ref['energy']:.6e})")
    assert npairs == ref["n_pairs"] > 0
    assert abs(energy - ref["energy"]) <= 1e-5 * abs(ref["energy"])
    fmax = np.abs(ref["mpm_force"]).max()
    assert np.abs(fm - ref["mpm_force"]).max() <= 1e-5 * fmax
    if two_way:
        assert np.abs(f - ref["sph_force"]).max() <= 1e-5 * np.abs(ref["sph_force"]).max()
    else:
        assert not np.any(f)


def test_sph_coupling_adds_to_existing_forces(gpu):
    """The fluid forces are added to the forces passed in, as the reference
    adds them to SPHParticle::force."""
    sim, _ = _drop(gpu, steps=1, n=10000, seed=63)
    rng = np.random.default_rng(64)
    sx = rng.uniform(0.2, 0.5, (500, 3)).astype(np.float32)
    sv = np.zeros_like(sx)
    base = rng.normal(0, 1, (500, 3)).astype(np.float32)
    f0, _, _, _ = sim.sph_coupling(sx, sv, radius=0.03)
    f1, _, _, _ = sim.sph_coupling(sx, sv, sph_force=base.copy(), radius=0.03)
    assert np.abs(f1 - (base + f0)).max() <= 1e-5 * (np.abs(f0).max() + 1.0)


def _float_running_sum(v, m):
    """The reference monitor's accumulation: a float total, each term
    0.5 * m * |v|^2 formed in double and added in order (src/fsi_coupling.h:
    841-856)."""
    total = np.float32(0.0)
    terms = 0.5 * m.astype(np.float64) * (v.astype(np.float32) ** 2).sum(1, dtype=np.float32).astype(np.float64)
    for t in terms:
        total = np.float32(np.float64(total) + t)
    return total


def test_kinetic_energy_matches_reference_monitor(gpu, oracle):
    """The GPU sums in FP64 and equals the oracle's FP64 sum to 1e-9.  The
    reference monitor keeps a float total: on nearly equal terms (the solid
    falls at one speed) its rounding drifts one way, here by ~3e-4 relative.
    It is pinned instead by replaying its float running sum on the same
    particles, which it must equal to one float rounding."""
    if not oracle.ref_fsi_available():
        pytest.skip("oracle/_ref not built")
    sim, st = _drop(gpu, steps=20)
    out = sim.download()
    per, tot = sim.kinetic_energy()
    mat = st["mat"]
    vf, mf, vs, ms = out["v"][mat == 1], st["m"][mat == 1], out["v"][mat == 0], st["m"][mat == 0]
    ref = oracle.ref_fsi_energy(vf, mf, vs, ms)
    ours = oracle.kinetic_energy(out["v"].astype(np.float64), st["m"].astype(np.float64), mat, 2)
    replay = _float_running_sum(np.concatenate([vf, vs]), np.concatenate([mf, ms]))
    print(f"kinetic energy: GPU {tot:.10e} (solid {per[0]:.6e}, fluid {per[1]:.6e}); FP64 oracle "
          f"{ours.sum():.10e}; reference monitor {ref:.10e} (its float running sum replayed {float(replay):.10e})")
    assert np.allclose(per, ours, rtol=1e-9)
    assert abs(float(replay) - ref) <= 2 * np.spacing(np.float32(ref))
    assert abs(tot - ref) <= 1e-3 * ref


@pytest.mark.parametrize("n_mats", [1, 5, 20, 70])
def test_kinetic_energy_per_material_counts(gpu, oracle, n_mats):
    """The monitor's per-material sums take three routes by the number of
    materials (register sums up to 8, shared-memory sums up to 64, global
    atomics above); each equals the FP64 oracle's sums to 1e-9, including
    materials that no particle uses."""
    from physgrad_b200 import workloads as W

    scenes, counts, _, st, _ = W.elastic_cube(n_particles=50000, n=32, v_sigma=0.3, seed=12)
    N = counts[0]
    rng = np.random.default_rng(13)
    mats = [gpu.createElasticMaterial(1000.0, 1e4 * (1 + 0.1 * k), 0.3) for k in range(n_mats)]
    # the last material, if there are several, is left without particles
    mat = rng.integers(0, max(1, n_mats - 1), N).astype(np.int32) if n_mats > 1 else None
    sim = gpu.Simulator(scenes, counts, mats)
    sim.upload(st["x"], st["v"], None, None, st["m"], st["V0"], mat)
    sim.step(3)
    out = sim.download()
    per, tot = sim.kinetic_energy()
    ref = oracle.kinetic_energy(out["v"].astype(np.float64), st["m"].astype(np.float64),
                                mat if mat is not None else np.zeros(N, np.int32), n_mats)
    assert per.shape == (n_mats,)
    assert np.allclose(per, ref, rtol=1e-9, atol=1e-300)
    if n_mats > 1:
        assert per[-1] == 0.0
    assert abs(tot - ref.sum()) <= 1e-9 * ref.sum()
