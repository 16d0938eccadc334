"""emfem_b200: B200-native EMFEM forward-solve path.

The product is ``libemfem_b200.so`` (host C++ + sm_100a CUDA behind the C ABI
declared in ``include/emfem_b200.h``).  This package loads it with ctypes and
mirrors the reference's entry points (``src/em_fwd.h``, ``src/em_la.h``) on
an :class:`EMContext` object.  There is no CPU fallback: without the built
library or without a GPU every compute call raises.
"""

from .api import (EMContext, EMGError, SolveInfo, lib, library_path, refine_fixed_fraction,
                  refine_fixed_number, launch_count, profile_enable, profile_get, spmm_layouts, XY_POLAR, YX_POLAR,
                  SOL_CSEM, SOL_DUAL, calculate_response_mt, calculate_response_csem, PointIndex, Survey)
from . import meshgen

__all__ = ["EMContext", "EMGError", "SolveInfo", "lib", "library_path", "refine_fixed_fraction",
           "refine_fixed_number", "launch_count", "profile_enable", "profile_get", "spmm_layouts", "XY_POLAR", "YX_POLAR", "SOL_CSEM", "SOL_DUAL", "calculate_response_mt",
           "calculate_response_csem", "PointIndex", "Survey", "meshgen"]
