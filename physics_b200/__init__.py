"""B200-native SPH fluid step with the reference's FluidWorld / phy-ffi API.

The mechanics live in ``lib/libphysph.so`` (CUDA kernels for sm_100a plus the
C ABI declared in ``include/phy_ffi.h`` and ``include/phy_fluid.h``).  Importing
this package loads that library and fails if it is missing: there is no CPU
fallback.
"""
from . import _lib
from ._lib import (FIELD_ACC, FIELD_BODY_ACC, FIELD_MASS, FIELD_MATERIAL, FIELD_MU_EFF, FIELD_P, FIELD_POS,
                   FIELD_RHO, FIELD_VEL, FIELD_XSPH, PRECISION_F32_COMP, PRECISION_F64_PLAIN, PhyError)
from .fluid import FluidSubsystem, FluidWorld, SphParams, World

_lib.load()

__all__ = [
    "FluidSubsystem", "FluidWorld", "SphParams", "World", "PhyError",
    "PRECISION_F64_PLAIN", "PRECISION_F32_COMP",
    "FIELD_POS", "FIELD_VEL", "FIELD_ACC", "FIELD_BODY_ACC", "FIELD_RHO", "FIELD_P", "FIELD_MASS",
    "FIELD_MU_EFF", "FIELD_XSPH", "FIELD_MATERIAL",
]
