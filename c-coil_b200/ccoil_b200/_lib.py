"""ctypes binding of libccoil_b200.so (the C-ABI declared in include/ccoil_gpu.h).

The shared library is built in-tree by c-coil_b200/build.py.  Loading fails
loudly when it is missing: there is no CPU fallback anywhere in this package.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# CCOIL_B200_LIB selects another build of the same library (a variant build)
LIB_PATH = os.environ.get("CCOIL_B200_LIB") or os.path.join(HERE, "libccoil_b200.so")

CCOIL_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "INVALID_ARGUMENT", 2: "CUDA", 3: "OUT_OF_MEMORY", 4: "NOT_SUPPORTED", 5: "TIMEOUT",
    6: "NO_DEVICE",
}

FIELD_A, FIELD_B, FIELD_E, FIELD_G = 0, 1, 2, 3
PRECISION_FP64, PRECISION_FP32_COMPENSATED, PRECISION_FP32_REFINED = 0, 1, 2
MEMORY_HOST, MEMORY_DEVICE = 0, 1


class PrecisionArgsStruct(ctypes.Structure):
    _fields_ = [("angular_blocks", ctypes.c_int), ("thickness_blocks", ctypes.c_int),
                ("length_blocks", ctypes.c_int), ("angular_increments", ctypes.c_int),
                ("thickness_increments", ctypes.c_int), ("length_increments", ctypes.c_int)]

    def as_tuple(self):
        return (self.angular_blocks, self.thickness_blocks, self.length_blocks, self.angular_increments,
                self.thickness_increments, self.length_increments)


class CoilStruct(ctypes.Structure):
    _fields_ = [("inner_radius", ctypes.c_double), ("thickness", ctypes.c_double), ("length", ctypes.c_double),
                ("current_density", ctypes.c_double), ("current", ctypes.c_double),
                ("sine_frequency", ctypes.c_double), ("position", ctypes.c_double * 3),
                ("y_axis_angle", ctypes.c_double), ("z_axis_angle", ctypes.c_double),
                ("transform", ctypes.c_double * 9), ("inverse_transform", ctypes.c_double * 9),
                ("num_turns", ctypes.c_int), ("use_fast_method", ctypes.c_int), ("coil_type", ctypes.c_int),
                ("precision", PrecisionArgsStruct)]


class PoseStruct(ctypes.Structure):
    _fields_ = [("position", ctypes.c_double * 3), ("y_axis_angle", ctypes.c_double),
                ("z_axis_angle", ctypes.c_double)]


PAIR_MUTUAL_INDUCTANCE, PAIR_FORCE_TORQUE, PAIR_MUTUAL_INDUCTANCE_GRADIENT = 0, 1, 2
PAIR_MUTUAL_INDUCTANCE_PARAMETER_GRADIENT = 3


class CCoilError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("ccoil status %s (%d): %s" % (STATUS_NAMES.get(status, "?"), status, message))
        self.status = status


_lib = None


def lib():
    """Load the library once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libccoil_b200.so is not built (run python c-coil_b200/build.py): " + LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    dp = ctypes.POINTER(ctypes.c_double)
    vp = ctypes.c_void_p
    cp = ctypes.POINTER(CoilStruct)
    pp = ctypes.POINTER(PrecisionArgsStruct)
    L.ccoil_abi_version.restype = ctypes.c_int
    L.ccoil_last_error_message.restype = ctypes.c_char_p
    L.ccoil_coil_init.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_double, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_int, cp]
    L.ccoil_precision_arguments.argtypes = [cp, ctypes.c_double, ctypes.c_int, pp]
    L.ccoil_pair_arguments.argtypes = [cp, cp, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, pp, pp]
    L.ccoil_legendre.argtypes = [ctypes.c_int, dp, dp]
    L.ccoil_compute_fields.argtypes = [cp, ctypes.c_int, vp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, vp,
                                       ctypes.c_int, vp]
    L.ccoil_field_plan_create.argtypes = [cp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    L.ccoil_field_plan_execute.argtypes = [vp, vp, ctypes.c_longlong, vp, ctypes.c_int, ctypes.c_int, vp]
    L.ccoil_field_plan_destroy.argtypes = [vp]
    L.ccoil_field_plan_segment_count.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.ccoil_timeout_count.restype = ctypes.c_longlong
    L.ccoil_check_bounded_wait.argtypes = [ctypes.c_longlong, vp]
    L.ccoil_set_point_ordering.argtypes = [ctypes.c_int]
    L.ccoil_set_refine_fraction.argtypes = [ctypes.c_double]
    L.ccoil_refine_fraction.restype = ctypes.c_double
    L.ccoil_field_plan_refined_pairs.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.ccoil_inject_allocation_failures.argtypes = [ctypes.c_int]
    L.ccoil_batch_plan_create.argtypes = [cp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong),
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    L.ccoil_batch_plan_execute.argtypes = [vp, vp, vp, vp, vp, vp]
    L.ccoil_batch_plan_tune.argtypes = [vp, vp, vp, vp, vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)]
    L.ccoil_batch_plan_set_split.argtypes = [vp, ctypes.c_int]
    L.ccoil_batch_plan_destroy.argtypes = [vp]
    L.ccoil_b_field_adjoint.argtypes = [dp, pp, ctypes.c_int, vp, ctypes.c_longlong, vp, vp, vp]
    L.ccoil_pair_arrangements.argtypes = [cp, ctypes.c_int, cp, pp, vp, vp, ctypes.c_longlong, ctypes.c_int,
                                          ctypes.c_int, vp, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int, vp]
    L.ccoil_self_inductances.argtypes = [cp, pp, ctypes.c_int, vp, vp]
    L.ccoil_eval_log64.argtypes = [vp, vp, ctypes.c_longlong, vp]
    L.ccoil_eval_fp64_op.argtypes = [ctypes.c_int, vp, vp, vp, ctypes.c_longlong, vp]
    L.ccoil_pair_arrangements_zaxis.argtypes = [cp, ctypes.c_int, cp, pp, pp, vp, vp, ctypes.c_longlong,
                                                ctypes.c_int, ctypes.c_int, vp, ctypes.POINTER(ctypes.c_longlong),
                                                ctypes.c_int, vp]
    _lib = L
    return L


def check(status):
    if status != CCOIL_OK:
        msg = lib().ccoil_last_error_message()
        raise CCoilError(status, msg.decode() if msg else "")
    return status
