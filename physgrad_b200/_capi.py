"""ctypes declarations of the C-ABI in include/pgmpm.h (libpgmpm.so).

The shared library is built in-tree by ``physgrad_b200.build``.  Loading
fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpgmpm.so")

PGMPM_OK = 0
PGMPM_ERR_ARG = -1
PGMPM_ERR_CUDA = -2
PGMPM_ERR_STATE = -3
PGMPM_ERR_UNSUPPORTED = -4
PGMPM_ERR_OOM = -5
PGMPM_ERR_SIMULATION = -6

FLAG_ESCAPE = 1
FLAG_NONFINITE = 2
FLAG_TILE_RANGE = 4
FLAG_BAD_MATERIAL = 8
FLAG_TILE_POOL = 16

PHYSICS_MLS = 0
PHYSICS_REF_COMPAT = 1

BC_NONE = 0
BC_STICKY = 1
BC_SLIP = 2
BC_SEPARATE = 3

MAT_ELASTIC = 0
MAT_ELASTOPLASTIC = 1
MAT_FLUID = 2
MAT_SAND = 3
MAT_SNOW = 4
MAT_JELLY = 5

MODEL_FIXED_COROTATED = 0
MODEL_NEO_HOOKEAN = 1
MODEL_EOS_FLUID = 2

ARRAY_USER_INDEX = 0
ARRAY_KEYS = 1
ARRAY_SORTED_KEYS = 2
ARRAY_SORTED_ORDER = 3

SORT_BINS = 0
SORT_RADIX = 1

PTR_HOST = 0
PTR_DEVICE = 1



def _header_define(name: str) -> int:
    """Integer value of a #define in include/pgmpm.h (the C-ABI's own header),
    so that Python never carries a second copy of a limit the library uses."""
    import re

    hdr = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "pgmpm.h")
    with open(hdr) as f:
        m = re.search(r"^#define\s+" + name + r"\s+\(?\s*(\d+)\s*(?:<<\s*(\d+))?\s*\)?", f.read(), re.M)
    if not m:
        raise RuntimeError(f"{name} not found in {hdr}")
    v = int(m.group(1))
    return v << int(m.group(2)) if m.group(2) else v


# maximum pairs of pgmpm_radix_sort_pairs_noalloc (PGMPM_NOALLOC_MAX_PAIRS)
NOALLOC_MAX_PAIRS = _header_define("PGMPM_NOALLOC_MAX_PAIRS")


class SceneDesc(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32 * 3),
        ("physics", ctypes.c_int32),
        ("boundary", ctypes.c_int32),
        ("boundary_thickness", ctypes.c_int32),
        ("dx", ctypes.c_float),
        ("origin", ctypes.c_float * 3),
        ("dt", ctypes.c_float),
        ("gravity", ctypes.c_float * 3),
    ]


class Material(ctypes.Structure):
    _fields_ = [
        ("type", ctypes.c_int32),
        ("model", ctypes.c_int32),
        ("youngs_modulus", ctypes.c_float),
        ("poisson_ratio", ctypes.c_float),
        ("density", ctypes.c_float),
        ("yield_stress", ctypes.c_float),
        ("viscosity", ctypes.c_float),
    ]


class CreateOptions(ctypes.Structure):
    _fields_ = [
        ("sparse_grid", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("max_tiles", ctypes.c_int64),
    ]


class SPHCouplingConfig(ctypes.Structure):
    _fields_ = [
        ("coupling_stiffness", ctypes.c_float),
        ("coupling_damping", ctypes.c_float),
        ("friction_coefficient", ctypes.c_float),
        ("coupling_radius", ctypes.c_float),
        ("enable_two_way_coupling", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class Metrics(ctypes.Structure):
    _fields_ = [
        ("total_steps", ctypes.c_int64),
        ("num_particles", ctypes.c_int64),
        ("active_nodes", ctypes.c_int64),
        ("last_step_ms", ctypes.c_double),
        ("average_step_ms", ctypes.c_double),
        ("particle_steps_per_s", ctypes.c_double),
        ("sort_ms", ctypes.c_double),
        ("p2g_ms", ctypes.c_double),
        ("grid_ms", ctypes.c_double),
        ("g2p_ms", ctypes.c_double),
        ("p2g_block", ctypes.c_int32),
        ("p2g_ppt", ctypes.c_int32),
        ("g2p_block", ctypes.c_int32),
        ("graph_enabled", ctypes.c_int32),
        ("p2g_variant", ctypes.c_int32),
        ("g2p_variant", ctypes.c_int32),
        ("p2g_tiles_per_sm", ctypes.c_int32),
        ("g2p_tiles_per_sm", ctypes.c_int32),
    ]


class HashGridInfo(ctypes.Structure):
    _fields_ = [
        ("average_particles_per_cell", ctypes.c_float),
        ("load_factor", ctypes.c_float),
        ("max_particles_per_cell", ctypes.c_uint32),
        ("occupied_cells", ctypes.c_uint32),
        ("memory_usage_mb", ctypes.c_float),
        ("total_cells", ctypes.c_uint32),
        ("resolution", ctypes.c_uint32 * 3),
    ]


# name -> (restype, argtypes)
_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
SIGNATURES = {
    "pgmpm_last_error": (ctypes.c_char_p, []),
    "pgmpm_abi_version": (ctypes.c_int, []),
    "pgmpm_clear_error": (None, []),
    "pgmpm_create": (ctypes.c_int, [ctypes.POINTER(SceneDesc), _i32, ctypes.POINTER(_i64), ctypes.POINTER(Material),
                                    _i32, _i32, ctypes.POINTER(_vp)]),
    "pgmpm_create_ex": (ctypes.c_int, [ctypes.POINTER(SceneDesc), _i32, ctypes.POINTER(_i64),
                                       ctypes.POINTER(Material), _i32, _i32, ctypes.POINTER(CreateOptions),
                                       ctypes.POINTER(_vp)]),
    "pgmpm_destroy": (ctypes.c_int, [_vp]),
    "pgmpm_sph_coupling": (ctypes.c_int, [_vp, ctypes.POINTER(SPHCouplingConfig), _vp, _vp, _i64, _vp, _vp,
                                          ctypes.POINTER(_i64), ctypes.POINTER(ctypes.c_double), _i32, _vp]),
    "pgmpm_kinetic_energy": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ctypes.c_double), _vp]),
    "pgmpm_set_materials": (ctypes.c_int, [_vp, ctypes.POINTER(Material), _i32]),
    "pgmpm_set_scene_params": (ctypes.c_int, [_vp, _i32, ctypes.c_float, _vp]),
    "pgmpm_upload": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _vp]),
    "pgmpm_download": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _i32, _vp]),
    "pgmpm_vtk_write_particles": (ctypes.c_int, [ctypes.c_char_p, _i64, _vp, _vp, _vp, _vp, ctypes.c_double]),
    "pgmpm_write_vtk": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_double, _vp]),
    "pgmpm_hashgrid_create": (ctypes.c_int, [ctypes.c_float, _vp, _vp, _i64, _i32, ctypes.POINTER(_vp)]),
    "pgmpm_hashgrid_destroy": (ctypes.c_int, [_vp]),
    "pgmpm_hashgrid_build": (ctypes.c_int, [_vp, _vp, _i64, _i32, _vp]),
    "pgmpm_hashgrid_neighbors": (ctypes.c_int, [_vp, _vp, _i64, ctypes.c_float, _vp, _vp, _i64,
                                                ctypes.POINTER(_i64), _i32, _vp]),
    "pgmpm_hashgrid_get_table": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _i32, _vp]),
    "pgmpm_hashgrid_stats": (ctypes.c_int, [_vp, ctypes.POINTER(HashGridInfo)]),
    "pgmpm_download_grid": (ctypes.c_int, [_vp, _i32, _vp, _vp, _i32, _vp]),
    "pgmpm_step": (ctypes.c_int, [_vp, _i32, _vp]),
    "pgmpm_advance_host": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _vp, _vp, _vp, _vp, _vp]),
    "pgmpm_check_status": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_uint32), _vp]),
    "pgmpm_set_tuning": (ctypes.c_int, [_vp, _i32, _i32, _i32, _i32]),
    "pgmpm_autotune": (ctypes.c_int, [_vp, _i32, _vp]),
    "pgmpm_set_kernel_variants": (ctypes.c_int, [_vp, _i32, _i32, _i32, _i32]),
    "pgmpm_set_step_sort": (ctypes.c_int, [_vp, _i32]),
    "pgmpm_set_sort_record": (ctypes.c_int, [_vp, _i32]),
    "pgmpm_get_replay_resorts": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "pgmpm_set_profiling": (ctypes.c_int, [_vp, _i32]),
    "pgmpm_get_metrics": (ctypes.c_int, [_vp, ctypes.POINTER(Metrics)]),
    "pgmpm_forward_checkpointed": (ctypes.c_int, [_vp, _i32, _i32, _vp]),
    "pgmpm_backward": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _vp]),
    "pgmpm_get_array": (ctypes.c_int, [_vp, _i32, _vp, _i32, _vp]),
    "pgmpm_radix_sort_pairs": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, _i32, _vp]),
    "pgmpm_radix_sort_pairs_noalloc": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, _i32, _vp]),
    "launch_mpm_timestep_forward": (None, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, _vp, _vp]),
    "launch_mpm_timestep_backward": (None, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_float, _vp]),
}

_lib = None


class PGMPMError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"pgmpm error {code}: {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    """Load libpgmpm.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m physgrad_b200.build` "
                               "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != PGMPM_OK:
        msg = lib().pgmpm_last_error()
        raise PGMPMError(rc, msg.decode() if msg else "")
