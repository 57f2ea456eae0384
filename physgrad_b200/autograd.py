"""torch.autograd.Functions over the MPM step.

* MPMSimulate: the checkpointed MLS-MPM forward / backward over many steps.
  It replaces the reference's PhysicsSimulationFunction pattern
  (src/pytorch_autograd.h:146-226: save inputs, run forward, backward by the
  adjoint) for the MPM path, whose reference adjoint records an empty backward
  (src/differentiable_mpm.h:871-876).
* MPMTimestep: one step of the reference's PIC step through the extern-C
  launchers launch_mpm_timestep_forward / _backward
  (src/pytorch_autograd.cu:371-402).

Device tensors cross the C-ABI by pointer (no copies); work runs on torch's
current stream.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional

import torch

from ._capi import PGMPMError, lib
from .solver import Simulator


class MPMSimulate(torch.autograd.Function):
    """(x0, v0, C0, F0, E) -> (x, v, C, F) after ``n_steps`` steps.

    ``E`` is a float32 tensor [n_materials] of Young's moduli (bulk modulus
    for FLUID materials); gradients flow to x0, v0, C0, F0 and E.  m, V0 and
    the material ids are constants of the simulation.  The Simulator holds
    one recording, so two rollouts in one autograd graph need two
    Simulators: a backward whose recording was replaced raises PGMPMError."""

    @staticmethod
    def forward(ctx, sim: Simulator, n_steps: int, checkpoint_every: int, x0, v0, C0, F0, E, m, V0,
                mat: Optional[torch.Tensor] = None):
        if not x0.is_cuda:
            raise ValueError("MPMSimulate expects CUDA tensors")
        N = x0.shape[0]
        Evals = E.detach().float().cpu().tolist()
        if len(Evals) != len(sim.materials):
            raise ValueError("E must have one entry per material")
        sim.set_materials([dataclasses.replace(mt, youngs_modulus=float(e)) for mt, e in zip(sim.materials, Evals)])
        stream = torch.cuda.current_stream()
        f32 = lambda t: t.detach().to(torch.float32).contiguous()
        sim.upload(f32(x0), f32(v0), f32(C0).reshape(N, 9), f32(F0).reshape(N, 9), f32(m), f32(V0),
                   mat.detach().to(torch.int32).contiguous() if mat is not None else None, stream=stream)
        sim.forward_checkpointed(int(n_steps), int(checkpoint_every), stream=stream)
        out = {"x": torch.empty(N, 3, device=x0.device), "v": torch.empty(N, 3, device=x0.device),
               "C": torch.empty(N, 3, 3, device=x0.device), "F": torch.empty(N, 3, 3, device=x0.device)}
        sim.download(out, stream=stream)
        ctx.sim = sim
        ctx.N = N
        ctx.generation = sim.forward_generation
        return out["x"], out["v"], out["C"], out["F"]

    @staticmethod
    def backward(ctx, gx, gv, gC, gF):
        sim, N = ctx.sim, ctx.N
        if sim.forward_generation != ctx.generation:
            # the solver keeps one recording: a later forward on the same
            # Simulator replaced the one this node needs
            raise PGMPMError(-3, "MPMSimulate.backward: the Simulator has run another forward since this rollout "
                                 "(it keeps one recording); use one Simulator per rollout in a graph")
        c = lambda t: None if t is None else t.detach().to(torch.float32).contiguous()
        stream = torch.cuda.current_stream()
        grads = sim.backward({"x": c(gx), "v": c(gv), "C": None if gC is None else c(gC).reshape(N, 9),
                              "F": None if gF is None else c(gF).reshape(N, 9)}, stream=stream)
        return (None, None, None, grads["x"], grads["v"], grads["C"].reshape(N, 3, 3), grads["F"].reshape(N, 3, 3),
                grads["E"], None, None, None)


def simulate(sim: Simulator, x0, v0, E, m, V0, n_steps: int, checkpoint_every: int = 16, C0=None, F0=None, mat=None):
    """Differentiable rollout: returns (x, v, C, F) after n_steps."""
    N = x0.shape[0]
    if C0 is None:
        C0 = torch.zeros(N, 3, 3, device=x0.device)
    if F0 is None:
        F0 = torch.eye(3, device=x0.device).expand(N, 3, 3).contiguous()
    return MPMSimulate.apply(sim, n_steps, checkpoint_every, x0, v0, C0, F0, E, m, V0, mat)


def _launch(name: str, *args):
    """Calls a void launch_* entry point; raises if it reported an error."""
    L = lib()
    L.pgmpm_clear_error()
    getattr(L, name)(*args)
    msg = L.pgmpm_last_error()
    if msg:
        raise PGMPMError(-1, msg.decode())


class MPMTimestep(torch.autograd.Function):
    """One step of the reference's PIC MPM step (REF_COMPAT physics) on the
    unit cube with a grid_resolution^3 grid, through the extern-C launchers
    launch_mpm_timestep_forward / launch_mpm_timestep_backward
    (src/pytorch_autograd.cu:371-402): (positions [N,3], velocities [N,3],
    masses [N], gravity [3]) -> (positions, velocities); gradients flow to
    all four.  Chains into rollouts like any torch op."""

    @staticmethod
    def forward(ctx, positions, velocities, masses, gravity, grid_resolution: int, dt: float):
        if not positions.is_cuda:
            raise ValueError("MPMTimestep expects CUDA tensors")
        f32 = lambda t: t.detach().to(torch.float32).contiguous()
        x0, v0, m, g = f32(positions), f32(velocities), f32(masses), f32(gravity)
        x, v = x0.clone(), v0.clone()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _launch("launch_mpm_timestep_forward", x.data_ptr(), v.data_ptr(), m.data_ptr(), x.shape[0],
                int(grid_resolution), float(dt), g.data_ptr(), stream)
        ctx.save_for_backward(x0, v0, m, g)
        ctx.res, ctx.dt = int(grid_resolution), float(dt)
        return x, v

    @staticmethod
    def backward(ctx, gx, gv):
        x0, v0, m, g = ctx.saved_tensors
        N = x0.shape[0]
        z = lambda t: torch.zeros_like(x0) if t is None else t.detach().to(torch.float32).contiguous()
        gx, gv = z(gx), z(gv)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        # the backward launcher uses the masses and gravity of the last forward
        # call with this particle count and resolution: make that this step's
        xs, vs = x0.clone(), v0.clone()
        _launch("launch_mpm_timestep_forward", xs.data_ptr(), vs.data_ptr(), m.data_ptr(), N, ctx.res, ctx.dt,
                g.data_ptr(), stream)
        gix, giv = torch.empty_like(x0), torch.empty_like(v0)
        gim, gg = torch.empty_like(m), torch.zeros_like(g)
        _launch("launch_mpm_timestep_backward", gx.data_ptr(), gv.data_ptr(), gix.data_ptr(), giv.data_ptr(),
                gim.data_ptr(), gg.data_ptr(), x0.data_ptr(), v0.data_ptr(), N, ctx.res, ctx.dt, stream)
        return gix, giv, gim, gg, None, None
