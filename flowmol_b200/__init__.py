"""B200 (sm_100a) per-timestep MD hot path of Flowmol: pair forces, cell and
neighbour lists, velocity-Verlet integration, behind a C ABI
(include/flowmol_b200.h) that mirrors the reference's subroutines."""
from .api import (MDSystem, FlowmolError, make_params, derive_geometry, global_domain, lib,  # noqa: F401
                  FORCE_LIST_ALLPAIRS, FORCE_LIST_FULL, FORCE_LIST_HALF, PRECISION_FP64, PRECISION_FP32)
from . import lattice  # noqa: F401
