"""ctypes binding of libpbt_b200.so (include/pbt_diff.h).

The shared library is built in-tree by abt_b200/build.py.  Loading fails
loudly when it is missing: there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpbt_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "pbt_diff.h")

PBT_OK, PBT_EINVAL, PBT_ENOMEM, PBT_ECUDA, PBT_ETIMEOUT, PBT_ENODEV, PBT_ESTATE = range(7)
PBT_DEVICE_LOCAL_RANK = -1  # pbt_ctx_create: the node-local rank modulo the visible devices
PBT_PREC_FP64, PBT_PREC_FP32 = 0, 1
STATUS_NAMES = {0: "PBT_OK", 1: "PBT_EINVAL", 2: "PBT_ENOMEM", 3: "PBT_ECUDA",
                4: "PBT_ETIMEOUT", 5: "PBT_ENODEV", 6: "PBT_ESTATE"}

# pbt_outbeam: the fields of outbeamtype (src/types_mod.f90:8-17) read by diffraction
OUTBEAM_DTYPE = np.dtype([("ampl", "<f8", (8,)), ("vk7", "<f8", (3,)),
                          ("prop_out", "<f8", (3,)), ("fov", "<f8"), ("fi", "<i8")])
assert OUTBEAM_DTYPE.itemsize == 128

# pbt_output_params: output_parameters_type (src/types_mod.f90:32-53)
PARAM_NAMES = ("abs", "scatt", "ext", "albedo", "asymmetry", "abs_eff", "scatt_eff",
               "ext_eff", "geo_cross_sec", "back_scatt", "beam_energy_out",
               "ext_energy_out", "scatt_beam", "scatt_ext_diff", "asymmetry_beam",
               "asymmetry_ext_diff", "scatt_eff_beam", "scatt_eff_ext_diff")
PARAMS_DTYPE = np.dtype([(n, "<f8") for n in PARAM_NAMES])
assert PARAMS_DTYPE.itemsize == 144

# every function declared in include/pbt_diff.h
EXPORTS = ("pbt_ctx_create", "pbt_ctx_device", "pbt_ctx_destroy", "pbt_last_error_string", "pbt_version",
           "pbt_diff_main_c", "pbt_diffraction_c", "pbt_finalise_c", "pbt_summation_c",
           "pbt_divide_by_num_orientations_c", "pbt_totals_reset_c", "pbt_diff_batch_c",
           "pbt_diff_batch_dev_c", "pbt_last_launch_count", "pbt_set_kernel_timing",
           "pbt_kernel_time_ms", "pbt_diffraction_noalloc_c", "pbt_set_plan",
           "pbt_diff_adjoint_c", "pbt_diff_batch_dev_graph_c", "pbt_graph_launch_c",
           "pbt_graph_kernel_count", "pbt_graph_destroy_c", "pbt_beamlist_writer_open",
           "pbt_beamlist_writer_add", "pbt_beamlist_writer_close", "pbt_beamlist_read",
           "pbt_beamlist_info", "pbt_beamlist_arrays", "pbt_beamlist_free",
           "pbt_make_far_field_bins_c", "pbt_selftest_bounded_wait_c", "pbt_diff_batch_list_c",
           "pbt_particle_create", "pbt_particle_info", "pbt_particle_verts",
           "pbt_particle_destroy", "pbt_trace_orientation_c", "pbt_trace_batch_c", "pbt_trace_sizes",
           "pbt_trace_copy", "pbt_trace_destroy", "pbt_test_fail_next_alloc")

# pbt_trace_params / pbt_trace_energy
TRACE_PARAMS_DTYPE = np.dtype([("lambda", "<f8"), ("rbi", "<f8"), ("ibi", "<f8"), ("rec", "<i8"),
                               ("refl", "<i8"), ("thresh_area", "<f8"),
                               ("thresh_energy", "<f8")])
TRACE_ENERGY_DTYPE = np.dtype([("abs", "<f8"), ("geo_cross_sec", "<f8"),
                               ("beam_energy_out", "<f8"), ("ext_energy_out", "<f8"),
                               ("nbeams", "<i8")])


class PbtError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), message))
        self.status = status


_lib = None


def lib():
    """Load the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libpbt_b200.so is not built; run `python abt_b200/build.py`")
    L = ctypes.CDLL(LIB_PATH)
    P, I64, I32, D = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_double
    C = ctypes.c_int
    sig = {
        "pbt_ctx_create": (C, [C, ctypes.POINTER(P)]),
        "pbt_ctx_destroy": (C, [P]),
        "pbt_ctx_device": (C, [P, ctypes.POINTER(C)]),
        "pbt_last_error_string": (ctypes.c_char_p, []),
        "pbt_version": (C, []),
        "pbt_diff_main_c": (C, [P, P, I64, P, I64, P, I64, P, P, I64, P, I64, P, I64, D, I32, I32,
                                P, P]),
        "pbt_diffraction_c": (C, [P, P, P, I64, P, P, I64, P, I64, P, I64, D, I32, P]),
        "pbt_finalise_c": (C, [P, P, P, P, I64, P, I64, D, I32, P, P, P, I32]),
        "pbt_summation_c": (C, [P, P, P, P, I64, I64]),
        "pbt_divide_by_num_orientations_c": (C, [P, I64, P, P, P]),
        "pbt_totals_reset_c": (C, [P]),
        "pbt_diff_batch_c": (C, [P, I64, P, P, P, P, P, I64, P, P, I64, P, I64, P, I64, D, I32,
                                 I32, I32, P, P, P, P, P]),
        "pbt_diff_batch_dev_c": (C, [P, P, I64, P, P, P, P, P, I64, P, P, I64, P, I64, P, I64, D,
                                     I32, I32, I32, P, P, P, P, P]),
        "pbt_diff_batch_dev_graph_c": (C, [P, P, I64, P, P, P, P, P, I64, P, P, I64, P, I64, P,
                                           I64, D, I32, I32, P, P, P, P, P, P]),
        "pbt_graph_launch_c": (C, [P, P]),
        "pbt_beamlist_writer_open": (C, [ctypes.c_char_p, P, I64, P, I64, I64, P, P, I64, D, P]),
        "pbt_beamlist_writer_add": (C, [P, P, I64, P, I64, P, P]),
        "pbt_beamlist_writer_close": (C, [P]),
        "pbt_beamlist_read": (C, [ctypes.c_char_p, P]),
        "pbt_beamlist_info": (C, [P, P, P]),
        "pbt_beamlist_arrays": (C, [P] + [P] * 10),
        "pbt_beamlist_free": (C, [P]),
        "pbt_make_far_field_bins_c": (C, [P, I64, P, I64, P, P, P]),
        "pbt_selftest_bounded_wait_c": (C, [P, I32]),
        "pbt_test_fail_next_alloc": (C, [I32]),
        "pbt_diff_batch_list_c": (C, [P, I64, P, P, P, P, P, I64, P, P, I64, P, I64, P, I64, D,
                                      I32, I32, I32, P, P, P, P, P]),
        "pbt_graph_kernel_count": (I64, [P]),
        "pbt_graph_destroy_c": (C, [P]),
        "pbt_last_launch_count": (I64, [P]),
        "pbt_set_kernel_timing": (C, [P, I32]),
        "pbt_kernel_time_ms": (C, [P, ctypes.POINTER(D), ctypes.POINTER(I64)]),
        "pbt_diffraction_noalloc_c": (C, [P, P, I64, P, P, I64, P, I64, P, I64, D, I32, P]),
        "pbt_set_plan": (C, [P, I32, I32, I64]),
        "pbt_diff_adjoint_c": (C, [P, P, I64, P, I64, P, I64, P, P, I64, P, I64, P, I64, D, I32,
                                   P, P, P, P, P]),
        "pbt_particle_create": (C, [P, I64, P, P, I64, P, ctypes.POINTER(P)]),
        "pbt_particle_info": (C, [P, P, P, P, P]),
        "pbt_particle_verts": (C, [P, P]),
        "pbt_particle_destroy": (C, [P]),
        "pbt_trace_orientation_c": (C, [P, P, P, ctypes.POINTER(P)]),
        "pbt_trace_batch_c": (C, [P, I64, P, P, P]),
        "pbt_trace_sizes": (C, [P, P, P]),
        "pbt_trace_copy": (C, [P, P, P, P, P]),
        "pbt_trace_destroy": (C, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status):
    if status != PBT_OK:
        msg = lib().pbt_last_error_string()
        raise PbtError(status, msg.decode() if msg else "")


def ptr(a):
    """Data pointer of a numpy array (None for None / empty)."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):  # torch tensor
        return a.data_ptr() or None
    return a.ctypes.data if a.size else None
