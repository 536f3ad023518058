"""ccoil_b200 -- B200-native (sm_100a) field and coil-pair hot path of C-Coil.

The Python surface mirrors the reference's `c_coil.coil` / `c_coil.coil_group`
modules for ComputeMethod.GPU; the work runs in libccoil_b200.so (include/ccoil_gpu.h).
"""
from ._lib import CCoilError, lib, LIB_PATH  # noqa: F401
from .batch import BatchPlan  # noqa: F401
from .coil import (Coil, CoilGroup, CoilPairArguments, CoilType, ComputeMethod, FieldPlan,  # noqa: F401
                   PrecisionArguments, PrecisionFactor, PrecisionMode, legendre)

__all__ = ["BatchPlan", "Coil", "CoilGroup", "CoilPairArguments", "CoilType", "ComputeMethod", "FieldPlan",
           "PrecisionArguments", "PrecisionFactor", "PrecisionMode", "legendre", "CCoilError", "lib"]
