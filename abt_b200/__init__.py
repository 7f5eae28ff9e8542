"""abt_b200 -- B200-native far-field vector diffraction for PBT (hballington12/abt).

The package replaces the reference's diff_mod + outputs_mod hot path with
CUDA sm_100a kernels behind a C ABI (include/pbt_diff.h, libpbt_b200.so):

  Context.diff_main / diffraction     diff_mod (FP64 reference-exact or FP32)
  Context.finalise / summation /      outputs_mod epilogue
    divide_by_num_orientations
  Context.diff_batch                   batched orientation averaging

There is no CPU fallback: importing the compute entry points requires the
built library (python abt_b200/build.py).
"""
from ._lib import OUTBEAM_DTYPE, PARAMS_DTYPE, PARAM_NAMES, PbtError  # noqa: F401
from .diff import (Context, PI_REF, make_angles, make_far_field_bins, make_geometry, params,  # noqa: F401
                   params_dict)

__all__ = ["Context", "OUTBEAM_DTYPE", "PARAMS_DTYPE", "PARAM_NAMES", "PbtError", "PI_REF",
           "make_angles", "make_far_field_bins", "make_geometry", "params", "params_dict"]
