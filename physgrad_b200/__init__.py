"""physgrad_b200 -- B200-native (sm_100a) MLS-MPM step behind physgrad's MPM
solver interfaces.  The compute path is libpgmpm.so (hand-written CUDA
kernels + a C-ABI, include/pgmpm.h); this package is its host-side mirror.
"""
from ._capi import PGMPMError, lib  # noqa: F401
from .solver import (  # noqa: F401
    BoundaryType,
    ConstitutiveModel,
    MaterialParameters,
    MaterialType,
    MPMSolver,
    MPMSolverConfig,
    RefCompatSolver,
    Scene,
    Simulator,
    createElasticMaterial,
    createFluidMaterial,
    radix_sort_pairs,
)
from .hashgrid import SpatialHashGrid  # noqa: F401

__all__ = [
    "PGMPMError", "lib", "BoundaryType", "ConstitutiveModel", "MaterialParameters", "MaterialType", "MPMSolver",
    "MPMSolverConfig", "RefCompatSolver", "Scene", "Simulator", "createElasticMaterial", "createFluidMaterial",
    "radix_sort_pairs", "SpatialHashGrid",
]
