"""B200-native (sm_100a) engine for ArtiSynth's FEM force/stiffness assembly
and BackwardEuler step.  The compute lives in libb200fem.so (C ABI,
include/b200fem.h); this package is the host-side mirror of the reference
interface around it."""
from . import _lib
from ._lib import B200FemError, lib
from .femmodel import (FemEngine, FemFactory, FemModel3d, FemPack, LinearMaterial, MechSystemSolver,
                       MooneyRivlinMaterial, NeoHookeanMaterial, StVenantKirchoffMaterial, create_grid,
                       jitter_grid)

__all__ = [
    "B200FemError", "FemEngine", "FemFactory", "FemModel3d", "FemPack", "LinearMaterial", "MechSystemSolver",
    "MooneyRivlinMaterial", "NeoHookeanMaterial", "StVenantKirchoffMaterial", "create_grid", "jitter_grid",
    "lib", "_lib",
]
