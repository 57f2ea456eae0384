"""Host-side mirror of the reference's MPM solver interfaces over the C-ABI.

``Simulator`` is the thin handle wrapper (one or many scenes, numpy host
arrays or CUDA torch tensors).  ``MPMSolver`` / ``MPMSolverConfig`` /
``MaterialParameters`` / ``MaterialType`` keep the names, argument meaning
and error behaviour of physgrad's ``physgrad::mpm::MPMSolver<T>``
(src/mpm_solver.h:29-329) and ``src/mpm_data_structures.h:54-96``;
``RefCompatSolver`` mirrors ``MPMSolver<T,64>`` of
src/material_point_method.h:430-506 (PIC physics of the reference CPU path).
"""
from __future__ import annotations

import ctypes
import os
import enum
import dataclasses
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _capi as C
from ._capi import check, lib

try:  # torch is optional for the numpy path
    import torch
except Exception:  # pragma: no cover
    torch = None


class MaterialType(enum.IntEnum):
    """src/mpm_data_structures.h:54-61."""
    ELASTIC = 0
    ELASTOPLASTIC = 1
    FLUID = 2
    SAND = 3
    SNOW = 4
    JELLY = 5


class ConstitutiveModel(enum.IntEnum):
    FIXED_COROTATED = C.MODEL_FIXED_COROTATED
    NEO_HOOKEAN = C.MODEL_NEO_HOOKEAN
    EOS_FLUID = C.MODEL_EOS_FLUID


class BoundaryType(enum.IntEnum):
    NONE = C.BC_NONE
    STICKY = C.BC_STICKY
    SLIP = C.BC_SLIP
    SEPARATE = C.BC_SEPARATE


@dataclass
class MaterialParameters:
    """Subset of src/mpm_data_structures.h:63-75 used by the step, with the
    reference's defaults.

    For FLUID the bulk modulus is carried in ``youngs_modulus`` (the
    reference's convention, src/mpm_data_structures.h:87-94) and
    ``viscosity`` adds a Newtonian viscous stress.  ELASTOPLASTIC is the
    neo-Hookean predictor with a von Mises cap at ``yield_stress``
    (``model`` is ignored for it)."""
    density: float = 1000.0
    youngs_modulus: float = 1e6
    poisson_ratio: float = 0.3
    type: MaterialType = MaterialType.ELASTIC
    model: ConstitutiveModel = ConstitutiveModel.FIXED_COROTATED
    yield_stress: float = 1e5
    viscosity: float = 0.001

    def to_c(self) -> C.Material:
        m = C.Material()
        m.type = int(self.type)
        m.model = int(self.model)
        m.youngs_modulus = float(self.youngs_modulus)
        m.poisson_ratio = float(self.poisson_ratio)
        m.density = float(self.density)
        m.yield_stress = float(self.yield_stress)
        m.viscosity = float(self.viscosity)
        return m


def createElasticMaterial(density, youngs_modulus, poisson_ratio,
                          model: ConstitutiveModel = ConstitutiveModel.FIXED_COROTATED) -> MaterialParameters:
    """src/mpm_data_structures.h:78-85."""
    return MaterialParameters(density, youngs_modulus, poisson_ratio, MaterialType.ELASTIC, model)


def createFluidMaterial(density, viscosity, gamma=7.0) -> MaterialParameters:
    """src/mpm_data_structures.h:87-94: the third argument (the bulk modulus
    K of p = -K (J - 1)) is stored in youngs_modulus, as there."""
    return MaterialParameters(density, gamma, 0.0, MaterialType.FLUID, ConstitutiveModel.EOS_FLUID,
                              viscosity=viscosity)


@dataclass
class Scene:
    """One background grid: n nodes per axis, spacing dx, origin."""
    n: Sequence[int] = (64, 64, 64)
    dx: float = 1.0 / 64
    dt: float = 1e-4
    gravity: Sequence[float] = (0.0, -9.8, 0.0)
    origin: Sequence[float] = (0.0, 0.0, 0.0)
    physics: int = C.PHYSICS_MLS
    boundary: int = C.BC_STICKY
    boundary_thickness: int = 3

    def to_c(self) -> C.SceneDesc:
        d = C.SceneDesc()
        for a in range(3):
            d.n[a] = int(self.n[a])
            d.origin[a] = float(self.origin[a])
            d.gravity[a] = float(self.gravity[a])
        d.physics = int(self.physics)
        d.boundary = int(self.boundary)
        d.boundary_thickness = int(self.boundary_thickness)
        d.dx = float(self.dx)
        d.dt = float(self.dt)
        return d


def _is_torch(a) -> bool:
    return torch is not None and isinstance(a, torch.Tensor)


def _ptr(a, n_rows: int, n_cols: int, dtype, name: str, keep: list, kind: list):
    """Validated pointer of a numpy array (host) or CUDA torch tensor (device)."""
    if a is None:
        return None
    if _is_torch(a):
        if not a.is_cuda:
            a = a.detach().cpu().numpy()
        else:
            want = torch.float32 if dtype == np.float32 else torch.int32
            if a.dtype != want:
                raise TypeError(f"{name} must be {want}")
            if not a.is_contiguous():
                raise ValueError(f"{name} must be contiguous")
            if a.numel() != n_rows * n_cols:
                raise ValueError(f"{name} must have {n_rows}x{n_cols} elements, got {tuple(a.shape)}")
            kind.append(C.PTR_DEVICE)
            keep.append(a)
            return a.data_ptr()
    a = np.ascontiguousarray(a, dtype=dtype)
    if a.size != n_rows * n_cols:
        raise ValueError(f"{name} must have {n_rows}x{n_cols} elements, got {a.shape}")
    kind.append(C.PTR_HOST)
    keep.append(a)
    return a.ctypes.data


def _stream_handle(stream):
    if stream is None:
        return None
    if torch is not None and isinstance(stream, torch.cuda.Stream):
        return ctypes.c_void_p(stream.cuda_stream)
    return ctypes.c_void_p(int(stream))


class Simulator:
    """Handle over pgmpm_* for one or more scenes (batched when > 1)."""

    def __init__(self, scenes: Sequence[Scene], counts: Sequence[int], materials: Sequence[MaterialParameters],
                 device: int = 0, tuning: Optional[dict] = None, sparse_tiles: Optional[int] = None):
        """sparse_tiles: None for dense grids; else a sparse grid whose tile
        pool holds that many 4^3 tiles (0: the library's default sizing)."""
        L = lib()
        self.scenes = list(scenes)
        self.counts = [int(c) for c in counts]
        self.materials = list(materials)
        self.N = int(sum(self.counts))
        sd = (C.SceneDesc * len(self.scenes))(*[s.to_c() for s in self.scenes])
        cn = (ctypes.c_int64 * len(self.counts))(*self.counts)
        md = (C.Material * len(self.materials))(*[m.to_c() for m in self.materials])
        h = ctypes.c_void_p()
        self.sparse = sparse_tiles is not None
        if self.sparse:
            opt = C.CreateOptions(1, 0, int(sparse_tiles))
            check(L.pgmpm_create_ex(sd, len(self.scenes), cn, md, len(self.materials), int(device), ctypes.byref(opt),
                                    ctypes.byref(h)))
        else:
            check(L.pgmpm_create(sd, len(self.scenes), cn, md, len(self.materials), int(device), ctypes.byref(h)))
        self._h = h
        self.device = device
        # incremented by every forward_checkpointed: a recording's identity,
        # so that a backward can tell whether the recording it was made for
        # is still the one the solver holds
        self.forward_generation = 0
        if tuning:
            self.set_tuning(**tuning)

    # -- lifecycle
    def close(self):
        if getattr(self, "_h", None):
            lib().pgmpm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # -- data
    def upload(self, x, v=None, C_=None, F=None, m=None, V0=None, mat=None, stream=None):
        N = self.N
        keep, kind = [], []
        px = _ptr(x, N, 3, np.float32, "x", keep, kind)
        pv = _ptr(v, N, 3, np.float32, "v", keep, kind)
        pC = _ptr(C_, N, 9, np.float32, "C", keep, kind)
        pF = _ptr(F, N, 9, np.float32, "F", keep, kind)
        pm = _ptr(m, N, 1, np.float32, "m", keep, kind)
        pV = _ptr(V0, N, 1, np.float32, "V0", keep, kind)
        pmat = _ptr(mat, N, 1, np.int32, "mat", keep, kind)
        if len(set(kind)) > 1:
            raise ValueError("mix of host and device inputs")
        k = kind[0] if kind else C.PTR_HOST
        check(lib().pgmpm_upload(self._h, px, pv, pC, pF, pm, pV, pmat, k, _stream_handle(stream)))

    def write_vtk(self, path: str, time: float = 0.0, stream=None):
        """The particles (upload order) as a legacy binary VTK file: points,
        velocity, J = det F and, with several materials, the material id."""
        check(lib().pgmpm_write_vtk(self._h, os.fsencode(path), float(time), _stream_handle(stream)))

    def download(self, out: Optional[dict] = None, stream=None):
        """State in upload order: numpy arrays, or into the CUDA tensors of ``out``."""
        N = self.N
        if out is not None:
            keep, kind = [], []
            ptrs = [_ptr(out.get(k), N, c, np.float32, k, keep, kind) for k, c in (("x", 3), ("v", 3), ("C", 9), ("F", 9))]
            if any(kd != C.PTR_DEVICE for kd in kind):
                raise ValueError("out= tensors must be CUDA tensors")
            check(lib().pgmpm_download(self._h, *ptrs, C.PTR_DEVICE, _stream_handle(stream)))
            return out
        x = np.empty((N, 3), np.float32)
        v = np.empty((N, 3), np.float32)
        Cm = np.empty((N, 3, 3), np.float32)
        F = np.empty((N, 3, 3), np.float32)
        check(lib().pgmpm_download(self._h, x.ctypes.data, v.ctypes.data, Cm.ctypes.data, F.ctypes.data, C.PTR_HOST,
                                   _stream_handle(stream)))
        return {"x": x, "v": v, "C": Cm, "F": F}

    def grid(self, scene: int = 0):
        s = self.scenes[scene]
        nodes = int(s.n[0]) * int(s.n[1]) * int(s.n[2])
        m = np.empty(nodes, np.float32)
        v = np.empty((nodes, 3), np.float32)
        check(lib().pgmpm_download_grid(self._h, scene, m.ctypes.data, v.ctypes.data, C.PTR_HOST, None))
        return m, v

    # -- simulation
    def step(self, n: int = 1, stream=None):
        check(lib().pgmpm_step(self._h, int(n), _stream_handle(stream)))

    def status(self, stream=None) -> int:
        f = ctypes.c_uint32()
        check(lib().pgmpm_check_status(self._h, ctypes.byref(f), _stream_handle(stream)))
        return f.value

    def set_materials(self, materials: Sequence[MaterialParameters]):
        md = (C.Material * len(materials))(*[m.to_c() for m in materials])
        check(lib().pgmpm_set_materials(self._h, md, len(materials)))
        self.materials = list(materials)

    def set_scene_params(self, scene: int = 0, dt: float | None = None, gravity: Sequence[float] | None = None):
        """New time step and/or gravity for one scene between steps (the
        per-call dt, gravity of DifferentiableMPMSystem::simulationStep,
        src/differentiable_mpm.h:748).  Invalidates a recording made by
        forward_checkpointed before the change."""
        s = self.scenes[scene] if 0 <= scene < len(self.scenes) else None  # the C-ABI rejects the index
        new_dt = float(dt) if dt is not None else (float(s.dt) if s is not None else 0.0)
        g = None
        if gravity is not None:
            g = (ctypes.c_float * 3)(*[float(a) for a in gravity])
        check(lib().pgmpm_set_scene_params(self._h, int(scene), new_dt, g))
        self.scenes[scene] = dataclasses.replace(s, dt=new_dt,
                                                 gravity=tuple(s.gravity) if gravity is None else tuple(gravity))

    def set_tuning(self, p2g_block=0, ppt=0, g2p_block=0, use_graph=-1):
        check(lib().pgmpm_set_tuning(self._h, int(p2g_block), int(ppt), int(g2p_block), int(use_graph)))

    def set_variants(self, p2g_variant=-1, g2p_variant=-1, p2g_tiles_per_sm=0, g2p_tiles_per_sm=0):
        check(lib().pgmpm_set_kernel_variants(self._h, int(p2g_variant), int(g2p_variant), int(p2g_tiles_per_sm),
                                              int(g2p_tiles_per_sm)))

    def set_step_sort(self, kind: int):
        """C.SORT_BINS (default) or C.SORT_RADIX (stable order within a cell)."""
        check(lib().pgmpm_set_step_sort(self._h, int(kind)))

    def set_sort_record(self, on):
        """Record every step's sort in forward_checkpointed (default on), so
        that backward's replays keep it instead of sorting again; 2: record,
        but every replayed step after a segment's first sorts again."""
        check(lib().pgmpm_set_sort_record(self._h, int(on)))

    def replay_resorts(self) -> int:
        """Replayed steps that sorted again because a key changed."""
        n = ctypes.c_int64(0)
        check(lib().pgmpm_get_replay_resorts(self._h, ctypes.byref(n)))
        return int(n.value)

    def autotune(self, reps: int = 3, stream=None) -> dict:
        check(lib().pgmpm_autotune(self._h, int(reps), _stream_handle(stream)))
        m = self.metrics()
        return {k: m[k] for k in ("p2g_variant", "p2g_block", "p2g_ppt", "p2g_tiles_per_sm", "g2p_variant",
                                  "g2p_block", "g2p_tiles_per_sm")}

    def get_array(self, which: int) -> np.ndarray:
        """u32 array of N entries (C.ARRAY_*): physical order, keys, last sort."""
        out = np.empty(self.N, np.uint32)
        check(lib().pgmpm_get_array(self._h, int(which), out.ctypes.data, C.PTR_HOST, None))
        return out

    def set_profiling(self, on: bool):
        check(lib().pgmpm_set_profiling(self._h, 1 if on else 0))

    def metrics(self) -> dict:
        m = C.Metrics()
        check(lib().pgmpm_get_metrics(self._h, ctypes.byref(m)))
        return {k: getattr(m, k) for k, _ in C.Metrics._fields_}

    # -- consumers of the particles
    def sph_coupling(self, sph_x, sph_v, sph_force=None, mpm_force=None, stiffness=1e5, damping=1e3, friction=0.3,
                     radius=0.15, two_way=True, stream=None):
        """SPH-MPM contact coupling (SPHMPMCouplingSystem of the reference,
        src/sph_mpm_coupling.h:453-575) with this solver's particles as the
        MPM side.  The fluid forces are added to ``sph_force`` (zeros when
        None); ``mpm_force`` receives each particle's summed solid force.
        Arrays are numpy (host) or CUDA tensors, [n][3] float32.  Returns
        (sph_force, mpm_force, n_pairs, energy)."""
        n = int(sph_x.shape[0])
        keep, kind = [], []
        host = not _is_torch(sph_x)
        if sph_force is None:
            sph_force = np.zeros((n, 3), np.float32) if host else torch.zeros((n, 3), dtype=torch.float32,
                                                                                device=sph_x.device)
        if mpm_force is None:
            mpm_force = np.zeros((self.N, 3), np.float32) if host else torch.zeros((self.N, 3), dtype=torch.float32,
                                                                                     device=sph_x.device)
        px = _ptr(sph_x, n, 3, np.float32, "sph_x", keep, kind)
        pv = _ptr(sph_v, n, 3, np.float32, "sph_v", keep, kind)
        pf = _ptr(sph_force, n, 3, np.float32, "sph_force", keep, kind)
        pm = _ptr(mpm_force, self.N, 3, np.float32, "mpm_force", keep, kind)
        if len(set(kind)) > 1:
            raise ValueError("mix of host and device arrays")
        cfg = C.SPHCouplingConfig(float(stiffness), float(damping), float(friction), float(radius), int(bool(two_way)),
                                  0)
        npairs = ctypes.c_int64()
        energy = ctypes.c_double()
        check(lib().pgmpm_sph_coupling(self._h, ctypes.byref(cfg), px, pv, n, pf, pm, ctypes.byref(npairs),
                                       ctypes.byref(energy), kind[0] if kind else C.PTR_HOST, _stream_handle(stream)))
        return keep[2], keep[3], npairs.value, energy.value  # the arrays written (a float32 copy if converted)

    def kinetic_energy(self, stream=None):
        """(per-material kinetic energies, total): the FSI energy monitor's
        sum of m |v|^2 / 2 (src/fsi_coupling.h:837-858)."""
        per = (ctypes.c_double * len(self.materials))()
        tot = ctypes.c_double()
        check(lib().pgmpm_kinetic_energy(self._h, per, ctypes.byref(tot), _stream_handle(stream)))
        return np.array(per[:]), tot.value

    # -- differentiation
    def forward_checkpointed(self, n_steps: int, checkpoint_every: int, stream=None):
        """Runs n_steps from the current state and records them for backward();
        each call replaces the previous recording (forward_generation + 1)."""
        self.forward_generation += 1
        check(lib().pgmpm_forward_checkpointed(self._h, int(n_steps), int(checkpoint_every), _stream_handle(stream)))

    def backward(self, grads_out: dict, grads_in: Optional[dict] = None, gE=None, stream=None):
        """Reverse pass: ``grads_out`` dL/d(final x, v, C, F) -> dL/d(initial), dL/dE."""
        N = self.N
        keep, kind = [], []
        gin = [_ptr(grads_out.get(k), N, c, np.float32, "g" + k, keep, kind)
               for k, c in (("x", 3), ("v", 3), ("C", 9), ("F", 9))]
        host = (not kind) or kind[0] == C.PTR_HOST
        if grads_in is None:
            if host:
                grads_in = {"x": np.zeros((N, 3), np.float32), "v": np.zeros((N, 3), np.float32),
                            "C": np.zeros((N, 3, 3), np.float32), "F": np.zeros((N, 3, 3), np.float32)}
            else:
                dev = next(t for t in keep if _is_torch(t)).device
                grads_in = {k: torch.zeros(sh, dtype=torch.float32, device=dev)
                            for k, sh in (("x", (N, 3)), ("v", (N, 3)), ("C", (N, 3, 3)), ("F", (N, 3, 3)))}
        gout = [_ptr(grads_in.get(k), N, c, np.float32, "gin_" + k, keep, kind)
                for k, c in (("x", 3), ("v", 3), ("C", 9), ("F", 9))]
        M = len(self.materials)
        if gE is None:
            gE = np.zeros(M, np.float32) if host else torch.zeros(M, dtype=torch.float32, device=keep[0].device)
        pE = _ptr(gE, M, 1, np.float32, "gE", keep, kind)
        if len(set(kind)) > 1:
            raise ValueError("mix of host and device gradient buffers")
        check(lib().pgmpm_backward(self._h, *gin, *gout, pE, kind[0], _stream_handle(stream)))
        grads_in["E"] = gE
        return grads_in


def radix_sort_pairs(keys, vals=None, key_bits: int = 32, stream=None):
    """Stable radix sort of CUDA uint32/int32 tensors (device pointers)."""
    n = keys.numel()
    ko = torch.empty_like(keys)
    vo = torch.empty_like(keys)
    check(lib().pgmpm_radix_sort_pairs(keys.data_ptr(), vals.data_ptr() if vals is not None else None, ko.data_ptr(),
                                       vo.data_ptr(), n, int(key_bits), _stream_handle(stream)))
    return ko, vo


# ---------------------------------------------------------------------------
# Reference-shaped solver classes
# ---------------------------------------------------------------------------

@dataclass
class MPMSolverConfig:
    """src/mpm_solver.h:29-66 (fields the step uses, plus physics/walls)."""
    grid_dimensions: Sequence[int] = (64, 64, 64)
    grid_spacing: Sequence[float] = (0.01, 0.01, 0.01)
    domain_origin: Sequence[float] = (0.0, 0.0, 0.0)
    time_step: float = 1e-4
    simulation_time: float = 1.0
    max_particles: int = 1000000
    enable_gravity: bool = True
    gravity: Sequence[float] = (0.0, -9.81, 0.0)
    cuda_block_size: int = 256
    enable_g2p2g_fusion: bool = True
    enable_profiling: bool = False
    physics: int = C.PHYSICS_MLS
    boundary: int = C.BC_STICKY
    boundary_thickness: int = 3
    device: int = 0
    materials: list = field(default_factory=lambda: [
        createElasticMaterial(1000.0, 1e4, 0.3)])


class MPMSolver:
    """``physgrad::mpm::MPMSolver<T>`` (src/mpm_solver.h:107-329) on the GPU path."""

    def __init__(self, config: MPMSolverConfig = None):
        self.config = config or MPMSolverConfig()
        self._pos, self._vel, self._mass, self._vol, self._mat = [], [], [], [], []
        self._sim: Optional[Simulator] = None
        self._time = 0.0
        self._step = 0
        self._initialized = False

    def addParticles(self, positions, velocities, masses, material_type: int = 0, volumes=None):
        """Append particles; ``material_type`` indexes ``config.materials``.
        Raises like src/mpm_solver.h:199 when max_particles is exceeded."""
        positions = np.asarray(positions, np.float32).reshape(-1, 3)
        n = positions.shape[0]
        if sum(len(p) for p in self._pos) + n > self.config.max_particles:
            raise RuntimeError("Exceeded maximum particle count")
        if self._initialized:
            raise RuntimeError("addParticles after initialize() is not supported")
        mats = self.config.materials
        if not (0 <= int(material_type) < len(mats)):
            raise ValueError("material_type out of range of config.materials")
        masses = np.asarray(masses, np.float32).reshape(n)
        self._pos.append(positions)
        self._vel.append(np.asarray(velocities, np.float32).reshape(n, 3))
        self._mass.append(masses)
        # src/mpm_solver.h:472-475: V = m / density
        self._vol.append(np.asarray(volumes, np.float32).reshape(n) if volumes is not None
                         else masses / np.float32(mats[int(material_type)].density))
        self._mat.append(np.full(n, int(material_type), np.int32))

    def initialize(self):
        if self._initialized:
            return
        cfg = self.config
        g = cfg.gravity if cfg.enable_gravity else (0.0, 0.0, 0.0)
        scene = Scene(cfg.grid_dimensions, float(cfg.grid_spacing[0]), cfg.time_step, g, cfg.domain_origin,
                      cfg.physics, cfg.boundary, cfg.boundary_thickness)
        N = sum(len(p) for p in self._pos)
        self._sim = Simulator([scene], [N], cfg.materials, cfg.device)
        if N:
            cat = lambda xs: np.concatenate(xs, 0)
            self._sim.upload(cat(self._pos), cat(self._vel), None, None, cat(self._mass), cat(self._vol),
                             cat(self._mat) if len(cfg.materials) > 1 else None)
        self._sim.set_tuning(p2g_block=cfg.cuda_block_size if cfg.cuda_block_size % 64 == 0 else 0)
        if cfg.enable_profiling:
            self._sim.set_profiling(True)
        self._initialized = True

    def step(self):
        if not self._initialized:
            raise RuntimeError("Solver not initialized")  # src/mpm_solver.h:231
        self._sim.step(1)
        self._time += self.config.time_step
        self._step += 1

    def run(self, num_steps: Optional[int] = None):
        self.initialize()
        n = num_steps if num_steps is not None else int(round(self.config.simulation_time / self.config.time_step))
        self._sim.step(n)
        self._time += n * self.config.time_step
        self._step += n

    def getParticles(self) -> dict:
        return self._sim.download()

    def getGrid(self) -> dict:
        m, v = self._sim.grid(0)
        dims = tuple(int(d) for d in self.config.grid_dimensions)
        return {"mass": m, "velocity": v, "momentum": v * m[:, None], "dimensions": dims}

    def getMetrics(self) -> dict:
        return self._sim.metrics()

    def getCurrentTime(self) -> float:
        return self._time

    def getCurrentStep(self) -> int:
        return self._step

    @property
    def simulator(self) -> Simulator:
        return self._sim


class RefCompatSolver:
    """``MPMSolver<T,64>`` (src/material_point_method.h:430-506): the reference
    CPU path's physics (PIC, floor-based stencil, gravity only) on the GPU."""

    @dataclass
    class SimulationParams:
        timestep: float = 1e-4
        gravity: Sequence[float] = (0.0, -9.81, 0.0)
        interpolation_order: int = 2

    def __init__(self, grid_dims, cell_size, origin=(0.0, 0.0, 0.0), params: "RefCompatSolver.SimulationParams" = None,
                 device: int = 0):
        self.params = params or RefCompatSolver.SimulationParams()
        if self.params.interpolation_order != 2:
            raise NotImplementedError("only the quadratic stencil (interpolation_order=2) is built")
        cs = cell_size if np.ndim(cell_size) else (cell_size,) * 3
        if not (cs[0] == cs[1] == cs[2]):
            raise ValueError("cubic cells required")
        self.scene = Scene(tuple(grid_dims), float(cs[0]), float(self.params.timestep), tuple(self.params.gravity),
                           tuple(origin), C.PHYSICS_REF_COMPAT, C.BC_NONE, 0)
        self.device = device
        self._x, self._v, self._m, self._V = [], [], [], []
        self._sim: Optional[Simulator] = None
        self._time = 0.0
        self._count = 0

    def addParticles(self, positions, velocities, masses, volumes, young_modulus=1e6, poisson_ratio=0.3,
                     density=1000.0):
        self._x.append(np.asarray(positions, np.float32).reshape(-1, 3))
        self._v.append(np.asarray(velocities, np.float32).reshape(-1, 3))
        self._m.append(np.asarray(masses, np.float32).reshape(-1))
        self._V.append(np.asarray(volumes, np.float32).reshape(-1))
        self._sim = None

    def _ensure(self):
        if self._sim is None:
            x = np.concatenate(self._x, 0)
            mats = [createElasticMaterial(1000.0, 1e6, 0.3)]
            self._sim = Simulator([self.scene], [x.shape[0]], mats, self.device)
            self._sim.upload(x, np.concatenate(self._v, 0), None, None, np.concatenate(self._m, 0),
                             np.concatenate(self._V, 0))

    def step(self, n: int = 1):
        self._ensure()
        self._sim.step(n)
        self._time += n * self.params.timestep
        self._count += n

    def getParticles(self) -> dict:
        self._ensure()
        return self._sim.download()

    def getGrid(self) -> dict:
        self._ensure()
        m, v = self._sim.grid(0)
        return {"mass": m, "velocity": v}

    def getCurrentTime(self) -> float:
        return self._time

    def getStepCount(self) -> int:
        return self._count
