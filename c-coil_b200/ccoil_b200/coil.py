"""Host-side mirror of the reference's Coil / CoilGroup field API for the GPU path.

Names and argument meaning follow the reference's Python module `c_coil.coil`
and `c_coil.coil_group` (src/Coil/PyBindings.cxx, src/CoilGroup/PyBindings.cxx)
and its C++ API (src/Coil/Coil.h, src/CoilGroup/CoilGroup.h).  Every
computation goes through the C-ABI of libccoil_b200.so; only ComputeMethod.GPU
is provided here (the CPU methods are the reference's own code).

Points are (n, 3) float64 arrays (numpy on the host, or torch CUDA tensors for
device-resident data); vector results are (n, 3) and gradients (n, 3, 3).

Precision.  The reference's GPU kernels cap every layer at GPU_INCREMENTS nodes
in one block (PrecisionArguments.cxx:124-141); the kernels here have no such
cap, so GPU calls use the reference's CPU PrecisionArguments for the same
PrecisionFactor and reproduce the CPU double path.  `used_precision` overrides
this per call exactly as in the reference.
"""
import ctypes
import enum

import numpy as np

from . import _lib
from ._lib import check, lib


class ComputeMethod(enum.IntEnum):
    CPU_ST = 0
    CPU_MT = 1
    GPU = 2


class CoilType(enum.IntEnum):
    RECTANGULAR = 0
    THIN = 1
    FLAT = 2
    FILAMENT = 3


class PrecisionMode(enum.IntEnum):
    """Arithmetic of the quadrature (runtime choice; the reference fixes it with the TYPE macro)."""
    FP64 = _lib.PRECISION_FP64
    FP32_COMPENSATED = _lib.PRECISION_FP32_COMPENSATED
    FP32_REFINED = _lib.PRECISION_FP32_REFINED


class PrecisionFactor:
    """PrecisionFactor (src/Coil/Coil.h:30-40): values outside [1, 15] become 5."""

    def __init__(self, relative_precision=5.0):
        rp = float(relative_precision)
        self.relative_precision = rp if 1.0 <= rp <= 15.0 else 5.0

    def __repr__(self):
        return "PrecisionFactor(relative_precision=%g)" % self.relative_precision


def _factor(pf):
    return pf.relative_precision if isinstance(pf, PrecisionFactor) else PrecisionFactor(pf).relative_precision


class PrecisionArguments:
    """PrecisionArguments (src/Coil/Coil.h:47-94) with the reference's constructor clamps."""

    def __init__(self, angular_blocks=1, thickness_blocks=1, length_blocks=1, angular_increments=20,
                 thickness_increments=20, length_increments=20):
        self.angular_blocks = angular_blocks if angular_blocks >= 1 else 1
        self.thickness_blocks = thickness_blocks if thickness_blocks >= 1 else 1
        self.length_blocks = length_blocks if length_increments >= 1 else 1
        self.angular_increments = angular_increments if 1 <= angular_increments <= 100 else 20
        self.thickness_increments = thickness_increments if 1 <= thickness_increments <= 100 else 20
        self.length_increments = length_increments if 1 <= length_increments <= 100 else 20

    # the reference's Python names for the same fields
    angular_block_count = property(lambda s: s.angular_blocks)
    thickness_block_count = property(lambda s: s.thickness_blocks)
    length_block_count = property(lambda s: s.length_blocks)
    angular_increment_count = property(lambda s: s.angular_increments)
    thickness_increment_count = property(lambda s: s.thickness_increments)
    length_increment_count = property(lambda s: s.length_increments)

    def as_tuple(self):
        return (self.angular_blocks, self.thickness_blocks, self.length_blocks, self.angular_increments,
                self.thickness_increments, self.length_increments)

    @classmethod
    def from_struct(cls, s):
        return cls(*s.as_tuple())

    def to_struct(self):
        return _lib.PrecisionArgsStruct(*self.as_tuple())

    def __eq__(self, other):
        return isinstance(other, PrecisionArguments) and self.as_tuple() == other.as_tuple()

    def __repr__(self):
        return ("PrecisionArguments(angular_block_count=%d, thickness_block_count=%d, length_block_count=%d, "
                "angular_increment_count=%d, thickness_increment_count=%d, length_increment_count=%d)"
                % self.as_tuple())

    @staticmethod
    def get_coil_precision_arguments_CPU(coil, precision_factor):
        return coil._precision(_factor(precision_factor), 0)

    @staticmethod
    def get_coil_precision_arguments_GPU(coil, precision_factor, gpu_increments=80):
        """The reference's capped GPU variant (GPU_INCREMENTS, 80 in its CMake build)."""
        return coil._precision(_factor(precision_factor), gpu_increments)


class CoilPairArguments:
    def __init__(self, primary_precision=None, secondary_precision=None):
        self.primary_precision = primary_precision or PrecisionArguments()
        self.secondary_precision = secondary_precision or PrecisionArguments()

    @staticmethod
    def get_appropriate_coil_pair_arguments(primary, secondary, precision_factor, compute_method=ComputeMethod.CPU_ST,
                                            z_axis_case=False, pure_gpu=False, gpu_increments=80):
        p, s = _lib.PrecisionArgsStruct(), _lib.PrecisionArgsStruct()
        cap = gpu_increments if compute_method == ComputeMethod.GPU else 0
        check(lib().ccoil_pair_arguments(ctypes.byref(primary._s), ctypes.byref(secondary._s),
                                         _factor(precision_factor), cap, int(z_axis_case), int(pure_gpu),
                                         ctypes.byref(p), ctypes.byref(s)))
        return CoilPairArguments(PrecisionArguments.from_struct(p), PrecisionArguments.from_struct(s))


# ---------------------------------------------------------------------------
# point / result marshalling
# ---------------------------------------------------------------------------
def _is_torch_cuda(x):
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _points_host(points):
    a = np.ascontiguousarray(points, dtype=np.float64)
    if a.ndim != 2 or a.shape[1] != 3:
        raise ValueError("points must have shape (n, 3)")
    return a


def _evaluate(coil_structs, points, field, precision, lanes=0, stream=None):
    """Runs one field evaluation through a temporary plan."""
    plan = FieldPlan(coil_structs, field, precision)
    try:
        return plan(points, lanes=lanes, stream=stream)
    finally:
        plan.close()


class FieldPlan:
    """A prepared coil set (ccoil_field_plan_t): node tables resident in device memory."""

    def __init__(self, coil_structs, field, precision=PrecisionMode.FP64):
        n = len(coil_structs)
        arr = (_lib.CoilStruct * max(n, 1))(*coil_structs)
        self.field = int(field)
        self.width = 9 if self.field == _lib.FIELD_G else 3
        self._h = ctypes.c_void_p()
        check(lib().ccoil_field_plan_create(arr, n, self.field, int(precision), ctypes.byref(self._h)))

    def __call__(self, points, lanes=0, stream=None, out=None):
        if _is_torch_cuda(points):
            import torch
            pts = points.contiguous().to(torch.float64)
            if pts.ndim != 2 or pts.shape[1] != 3:
                raise ValueError("points must have shape (n, 3)")
            if out is None:
                out = torch.empty((pts.shape[0], self.width), dtype=torch.float64, device=pts.device)
            st = stream if stream is not None else torch.cuda.current_stream(pts.device).cuda_stream
            check(lib().ccoil_field_plan_execute(self._h, ctypes.c_void_p(pts.data_ptr()), pts.shape[0],
                                                 ctypes.c_void_p(out.data_ptr()), _lib.MEMORY_DEVICE, int(lanes),
                                                 ctypes.c_void_p(st)))
            return out
        pts = _points_host(points)
        res = np.empty((pts.shape[0], self.width), dtype=np.float64) if out is None else out
        check(lib().ccoil_field_plan_execute(self._h, pts.ctypes.data_as(ctypes.c_void_p), pts.shape[0],
                                             res.ctypes.data_as(ctypes.c_void_p), _lib.MEMORY_HOST, int(lanes),
                                             ctypes.c_void_p(stream or 0)))
        return res

    def segment_count(self):
        """Segments the plan evaluates per point (one per coil, more for coils whose
        node tables exceed one segment)."""
        n = ctypes.c_int()
        check(lib().ccoil_field_plan_segment_count(self._h, ctypes.byref(n)))
        return n.value

    def refined_pairs(self):
        """(point, coil segment) pairs the last execution re-evaluated in FP64
        (FP32_REFINED plans)."""
        n = ctypes.c_longlong()
        check(lib().ccoil_field_plan_refined_pairs(self._h, ctypes.byref(n)))
        return n.value

    def close(self):
        if self._h:
            lib().ccoil_field_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _shape(res, field):
    if field == _lib.FIELD_G:
        return res.reshape(-1, 3, 3)
    return res


def _poses(positions, y_angles, z_angles):
    pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
    y = np.ascontiguousarray(y_angles, dtype=np.float64).reshape(-1)
    z = np.ascontiguousarray(z_angles, dtype=np.float64).reshape(-1)
    if not (len(pos) == len(y) == len(z)):
        raise ValueError("Array sizes do not match!")
    return np.ascontiguousarray(np.concatenate([pos, y[:, None], z[:, None]], axis=1))


def _pair_arrangements(primaries, secondary, sec_precisions, primary_poses, secondary_poses, quantity,
                       precision_mode=PrecisionMode.FP64, zaxis_precisions=None):
    """Runs ccoil_pair_arrangements (ccoil_pair_arrangements_zaxis when z-axis pair arguments
    [primary, secondary] per primary are given); returns (values, number of exact z-axis pairs)."""
    n = len(secondary_poses)
    width = {_lib.PAIR_MUTUAL_INDUCTANCE: 1, _lib.PAIR_FORCE_TORQUE: 6,
             _lib.PAIR_MUTUAL_INDUCTANCE_GRADIENT: 3, _lib.PAIR_MUTUAL_INDUCTANCE_PARAMETER_GRADIENT: 14}[quantity]
    out = np.zeros((n, width))
    prim = (_lib.CoilStruct * max(len(primaries), 1))(*primaries)
    secp = (_lib.PrecisionArgsStruct * max(len(sec_precisions), 1))(*sec_precisions)
    zc = ctypes.c_longlong(0)
    pposes = None if primary_poses is None else primary_poses.ctypes.data_as(ctypes.c_void_p)
    if zaxis_precisions is None:
        check(lib().ccoil_pair_arrangements(
            prim, len(primaries), ctypes.byref(secondary), secp, pposes,
            secondary_poses.ctypes.data_as(ctypes.c_void_p), n, quantity, int(precision_mode),
            out.ctypes.data_as(ctypes.c_void_p), ctypes.byref(zc), _lib.MEMORY_HOST, None))
    else:
        zp = (_lib.PrecisionArgsStruct * max(len(zaxis_precisions), 1))(*zaxis_precisions)
        check(lib().ccoil_pair_arrangements_zaxis(
            prim, len(primaries), ctypes.byref(secondary), secp, zp, pposes,
            secondary_poses.ctypes.data_as(ctypes.c_void_p), n, quantity, int(precision_mode),
            out.ctypes.data_as(ctypes.c_void_p), ctypes.byref(zc), _lib.MEMORY_HOST, None))
    return (out[:, 0] if width == 1 else out), zc.value


def pair_arrangements_device(primaries, secondary, sec_precisions, primary_poses, secondary_poses, quantity,
                             out, stream=None, precision_mode=PrecisionMode.FP64):
    """Device-memory variant: poses (n, 5) and out are torch CUDA float64 tensors
    (primary_poses may be None for fixed primaries); asynchronous on `stream`
    up to the library's own completion wait."""
    import torch
    n = secondary_poses.shape[0]
    prim = (_lib.CoilStruct * max(len(primaries), 1))(*primaries)
    secp = (_lib.PrecisionArgsStruct * max(len(sec_precisions), 1))(*sec_precisions)
    zc = ctypes.c_longlong(0)
    st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    check(lib().ccoil_pair_arrangements(
        prim, len(primaries), ctypes.byref(secondary), secp,
        None if primary_poses is None else ctypes.c_void_p(primary_poses.data_ptr()),
        ctypes.c_void_p(secondary_poses.data_ptr()), n, quantity, int(precision_mode),
        ctypes.c_void_p(out.data_ptr()), ctypes.byref(zc), _lib.MEMORY_DEVICE, ctypes.c_void_p(st)))
    return zc.value


_next_id = [0]


class Coil:
    """Circular coil with rectangular cross-section (src/Coil/Coil.h:152-814).

    Coil(inner_radius, thickness, length, num_of_turns, current=1.0, sine_frequency=50.0,
         precision_factor=PrecisionFactor(), thread_count=8, coordinate_position=(0, 0, 0),
         y_axis_angle=0.0, z_axis_angle=0.0)
    """

    def __init__(self, inner_radius, thickness, length, num_of_turns, current=1.0, sine_frequency=50.0,
                 precision_factor=None, thread_count=8, coordinate_position=(0.0, 0.0, 0.0), y_axis_angle=0.0,
                 z_axis_angle=0.0):
        self._args = (float(inner_radius), float(thickness), float(length), int(num_of_turns), float(current),
                      float(sine_frequency))
        _next_id[0] += 1
        self._id = _next_id[0]
        self.thread_count = thread_count
        self._pf = _factor(precision_factor if precision_factor is not None else PrecisionFactor())
        self._s = _lib.CoilStruct()
        self._init(coordinate_position, y_axis_angle, z_axis_angle)
        self.default_precision_CPU = self._precision(self._pf, 0)
        self.default_precision_GPU = self.default_precision_CPU

    def _init(self, position, y_angle, z_angle):
        pos = (ctypes.c_double * 3)(*[float(v) for v in position])
        R, a, b, N, I, f = self._args
        check(lib().ccoil_coil_init(R, a, b, N, I, f, pos, float(y_angle), float(z_angle), self._pf, 0,
                                    ctypes.byref(self._s)))

    def _precision(self, pf, cap):
        out = _lib.PrecisionArgsStruct()
        check(lib().ccoil_precision_arguments(ctypes.byref(self._s), pf, cap, ctypes.byref(out)))
        return PrecisionArguments.from_struct(out)

    # --- getters mirroring the reference -------------------------------------------------
    def get_id(self): return self._id
    def get_inner_radius(self): return self._s.inner_radius
    def get_thickness(self): return self._s.thickness
    def get_length(self): return self._s.length
    def get_num_of_turns(self): return self._s.num_turns
    def get_current(self): return self._s.current
    def get_current_density(self): return self._s.current_density
    def get_sine_frequency(self): return self._s.sine_frequency
    def is_using_fast_method(self): return bool(self._s.use_fast_method)
    def get_coil_type(self): return CoilType(self._s.coil_type)
    def get_position_vector(self): return np.array(self._s.position[:])
    def get_rotation_angles(self): return (self._s.y_axis_angle, self._s.z_axis_angle)
    def get_transformation_matrix(self): return np.array(self._s.transform[:]).reshape(3, 3)
    def get_inverse_transformation_matrix(self): return np.array(self._s.inverse_transform[:]).reshape(3, 3)

    def set_current(self, current):
        R, a, b, N, _, f = self._args
        self._args = (R, a, b, N, float(current), f)
        self._s.current = float(current)
        self._s.current_density = float(current) * N / (self._s.length * self._s.thickness)

    def set_position_and_orientation(self, position_vector=(0.0, 0.0, 0.0), y_axis_angle=0.0, z_axis_angle=0.0):
        prec = self._s.precision
        self._init(position_vector, y_axis_angle, z_axis_angle)
        self._s.precision = prec

    def set_default_precision(self, precision_factor=None):
        self._pf = _factor(precision_factor if precision_factor is not None else PrecisionFactor())
        self.default_precision_CPU = self._precision(self._pf, 0)
        self.default_precision_GPU = self.default_precision_CPU

    def struct(self, precision=None):
        """The ccoil_coil_t of this coil with the given (default) PrecisionArguments."""
        s = _lib.CoilStruct()
        ctypes.pointer(s)[0] = self._s
        s.precision = (precision or self.default_precision_GPU).to_struct()
        return s

    # --- field evaluation ---------------------------------------------------------------
    def _compute(self, points, field, compute_method, used_precision, precision_mode):
        if ComputeMethod(compute_method) != ComputeMethod.GPU:
            raise NotImplementedError("this package provides the ComputeMethod.GPU path only")
        return _shape(_evaluate([self.struct(used_precision)], points, field, precision_mode), field)

    def compute_all_A_potential_vectors(self, point_vectors, compute_method=ComputeMethod.GPU, used_precision=None,
                                        precision_mode=PrecisionMode.FP64):
        return self._compute(point_vectors, _lib.FIELD_A, compute_method, used_precision, precision_mode)

    def compute_all_B_field_vectors(self, point_vectors, compute_method=ComputeMethod.GPU, used_precision=None,
                                    precision_mode=PrecisionMode.FP64):
        return self._compute(point_vectors, _lib.FIELD_B, compute_method, used_precision, precision_mode)

    def compute_all_E_field_vectors(self, point_vectors, compute_method=ComputeMethod.GPU, used_precision=None,
                                    precision_mode=PrecisionMode.FP64):
        return self._compute(point_vectors, _lib.FIELD_E, compute_method, used_precision, precision_mode)

    def compute_all_B_gradient_matrices(self, point_vectors, compute_method=ComputeMethod.GPU, used_precision=None,
                                        precision_mode=PrecisionMode.FP64):
        return self._compute(point_vectors, _lib.FIELD_G, compute_method, used_precision, precision_mode)

    # --- coil pairs ------------------------------------------------------------------------
    @staticmethod
    def _pair_args(primary, secondary, pf):
        """CPU pair arguments (computeMethod != GPU, general case), as the CPU path uses."""
        a = CoilPairArguments.get_appropriate_coil_pair_arguments(primary, secondary, pf, ComputeMethod.CPU_ST)
        return a.primary_precision, a.secondary_precision

    @staticmethod
    def _arrangements(primary, secondary, primary_positions, secondary_positions, primary_y_angles,
                      primary_z_angles, secondary_y_angles, secondary_z_angles, precision_factor, compute_method,
                      quantity, precision_mode=PrecisionMode.FP64):
        if ComputeMethod(compute_method) != ComputeMethod.GPU:
            raise NotImplementedError("this package provides the ComputeMethod.GPU path only")
        pp, sp = Coil._pair_args(primary, secondary, _factor(precision_factor))
        ppose = _poses(primary_positions, primary_y_angles, primary_z_angles)
        spose = _poses(secondary_positions, secondary_y_angles, secondary_z_angles)
        if len(ppose) != len(spose):
            raise ValueError("Array sizes do not match!")
        zargs = None
        if quantity in (_lib.PAIR_MUTUAL_INDUCTANCE, _lib.PAIR_FORCE_TORQUE):
            # coaxial arrangements take the reference CPU path's z-axis formulas and arguments
            za = CoilPairArguments.get_appropriate_coil_pair_arguments(primary, secondary, _factor(precision_factor),
                                                                       ComputeMethod.CPU_ST, z_axis_case=True)
            zargs = [za.primary_precision.to_struct(), za.secondary_precision.to_struct()]
        vals, _ = _pair_arrangements([primary.struct(pp)], secondary.struct(sp), [sp.to_struct()], ppose, spose,
                                     quantity, precision_mode, zargs)
        return vals

    @staticmethod
    def compute_all_mutual_inductance_arrangements(primary, secondary, primary_positions, secondary_positions,
                                                   primary_y_angles, primary_z_angles, secondary_y_angles,
                                                   secondary_z_angles, precision_factor=None,
                                                   compute_method=ComputeMethod.GPU,
                                                   precision_mode=PrecisionMode.FP64):
        """Coil::computeAllMutualInductanceArrangements (ComputeMInductanceMethods.cxx:200-260): (n,) array.
        precision_mode FP32_COMPENSATED runs the primary quadrature in FP32 away from its winding;
        FP32_REFINED also re-evaluates in FP64 the secondary nodes whose contributions dominate."""
        return Coil._arrangements(primary, secondary, primary_positions, secondary_positions, primary_y_angles,
                                  primary_z_angles, secondary_y_angles, secondary_z_angles,
                                  precision_factor or PrecisionFactor(), compute_method,
                                  _lib.PAIR_MUTUAL_INDUCTANCE, precision_mode)

    @staticmethod
    def compute_all_mutual_inductance_gradient_arrangements(primary, secondary, primary_positions,
                                                            secondary_positions, primary_y_angles, primary_z_angles,
                                                            secondary_y_angles, secondary_z_angles,
                                                            precision_factor=None, compute_method=ComputeMethod.GPU):
        """dM/d(secondary position) per arrangement, (n, 3): the exact derivative of the mutual
        inductance quadrature (no counterpart in the reference)."""
        return Coil._arrangements(primary, secondary, primary_positions, secondary_positions, primary_y_angles,
                                  primary_z_angles, secondary_y_angles, secondary_z_angles,
                                  precision_factor or PrecisionFactor(), compute_method,
                                  _lib.PAIR_MUTUAL_INDUCTANCE_GRADIENT)

    @staticmethod
    def compute_all_mutual_inductance_parameter_gradient_arrangements(
            primary, secondary, primary_positions, secondary_positions, primary_y_angles, primary_z_angles,
            secondary_y_angles, secondary_z_angles, precision_factor=None, compute_method=ComputeMethod.GPU):
        """M and its exact derivatives with respect to both coils' parameters per arrangement, (n, 14):
        M, dM/d(R1, a1, b1, y_angle1, z_angle1, R2, a2, b2, x2, y2, z2, y_angle2, z_angle2) (no
        counterpart in the reference).  The primary's position gradient is -dM/d(x2, y2, z2) and
        dM/dN = M / N for either coil."""
        return Coil._arrangements(primary, secondary, primary_positions, secondary_positions, primary_y_angles,
                                  primary_z_angles, secondary_y_angles, secondary_z_angles,
                                  precision_factor or PrecisionFactor(), compute_method,
                                  _lib.PAIR_MUTUAL_INDUCTANCE_PARAMETER_GRADIENT)

    @staticmethod
    def compute_all_force_torque_arrangements(primary, secondary, primary_positions, secondary_positions,
                                              primary_y_angles, primary_z_angles, secondary_y_angles,
                                              secondary_z_angles, precision_factor=None,
                                              compute_method=ComputeMethod.GPU,
                                              precision_mode=PrecisionMode.FP64):
        """Coil::computeAllForceTorqueArrangements (ComputeForceMethods.cxx:189-248): (n, 6) array of
        force xyz and torque xyz on the secondary."""
        return Coil._arrangements(primary, secondary, primary_positions, secondary_positions, primary_y_angles,
                                  primary_z_angles, secondary_y_angles, secondary_z_angles,
                                  precision_factor or PrecisionFactor(), compute_method, _lib.PAIR_FORCE_TORQUE,
                                  precision_mode)

    # --- self inductance ----------------------------------------------------------------------
    def compute_and_set_self_inductance(self, precision_factor=None):
        """Coil::computeAndSetSelfInductance (ComputeMInductanceMethods.cxx:55-81): the coil's self
        inductance at its z-axis pair arguments with itself; stored and returned."""
        self._self_inductance = float(Coil.compute_all_self_inductances([self], precision_factor)[0])
        return self._self_inductance

    def get_self_inductance(self):
        return getattr(self, "_self_inductance", 0.0)

    @staticmethod
    def compute_all_self_inductances(coils, precision_factor=None):
        """Self inductances of many coils in one launch (no counterpart in the reference)."""
        pf = _factor(precision_factor or PrecisionFactor())
        structs, args = [], []
        for c in coils:
            a = CoilPairArguments.get_appropriate_coil_pair_arguments(c, c, pf, ComputeMethod.CPU_ST,
                                                                      z_axis_case=True)
            structs.append(c.struct(a.primary_precision))
            args += [a.primary_precision.to_struct(), a.secondary_precision.to_struct()]
        out = np.zeros(len(structs))
        if not structs:
            return out
        arr = (_lib.CoilStruct * len(structs))(*structs)
        pa = (_lib.PrecisionArgsStruct * len(args))(*args)
        check(lib().ccoil_self_inductances(arr, pa, len(structs), out.ctypes.data_as(ctypes.c_void_p), None))
        return out

    def _pose_row(self):
        return self.get_position_vector(), self._s.y_axis_angle, self._s.z_axis_angle

    @staticmethod
    def compute_mutual_inductance(primary, secondary, precision_factor=None, compute_method=ComputeMethod.GPU):
        """Coil::computeMutualInductance for the pair as placed (general case)."""
        pp, py, pz = primary._pose_row()
        sp, sy, sz = secondary._pose_row()
        return float(Coil.compute_all_mutual_inductance_arrangements(
            primary, secondary, [pp], [sp], [py], [pz], [sy], [sz], precision_factor, compute_method)[0])

    @staticmethod
    def compute_force_torque(primary, secondary, precision_factor=None, compute_method=ComputeMethod.GPU):
        """Coil::computeForceTorque for the pair as placed: (force xyz, torque xyz)."""
        pp, py, pz = primary._pose_row()
        sp, sy, sz = secondary._pose_row()
        v = Coil.compute_all_force_torque_arrangements(primary, secondary, [pp], [sp], [py], [pz], [sy], [sz],
                                                       precision_factor, compute_method)[0]
        return v[:3].copy(), v[3:].copy()

    def __repr__(self):
        R, a, b, N, I, f = self._args
        return "Coil(inner_radius=%g, thickness=%g, length=%g, num_of_turns=%d, current=%g)" % (R, a, b, N, I)


class CoilGroup:
    """A set of coils whose fields add (src/CoilGroup/CoilGroup.h:19-283).

    Each member is evaluated at its own PrecisionArguments for the group's
    PrecisionFactor (CoilGroup::setDefaultPrecisionFactor, CoilGroup.cxx:31-37)
    and the whole group is one kernel launch (coils inner, points outer).
    """

    def __init__(self, member_coils=None, precision_factor=None, thread_count=8):
        self.member_coils = list(member_coils or [])
        self.thread_count = thread_count
        self.default_precision_factor = precision_factor if precision_factor is not None else PrecisionFactor()
        for c in self.member_coils:
            c.set_default_precision(self.default_precision_factor)

    def add_coil(self, inner_radius, thickness, length, num_of_turns, current=1.0, precision_factor=None,
                 coil_threads=8, coordinate_position=(0.0, 0.0, 0.0), y_axis_angle=0.0, z_axis_angle=0.0,
                 sine_frequency=50.0):
        self.member_coils.append(Coil(inner_radius, thickness, length, num_of_turns, current, sine_frequency,
                                      precision_factor, coil_threads, coordinate_position, y_axis_angle,
                                      z_axis_angle))

    def remove_coil(self, index):
        if index >= len(self.member_coils):
            raise IndexError("Coil index out of range!")
        del self.member_coils[index]

    def __getitem__(self, index):
        return self.member_coils[index]

    def set_default_precision_factor(self, precision_factor=None):
        self.default_precision_factor = precision_factor if precision_factor is not None else PrecisionFactor()
        for c in self.member_coils:
            c.set_default_precision(self.default_precision_factor)

    def get_default_precision_factor(self):
        return self.default_precision_factor

    def structs(self):
        return [c.struct() for c in self.member_coils]

    def plan(self, field, precision_mode=PrecisionMode.FP64):
        return FieldPlan(self.structs(), field, precision_mode)

    def _compute(self, points, field, compute_method, precision_mode):
        if ComputeMethod(compute_method) != ComputeMethod.GPU:
            raise NotImplementedError("this package provides the ComputeMethod.GPU path only")
        return _shape(_evaluate(self.structs(), points, field, precision_mode), field)

    def compute_all_A_potential_vectors(self, point_vectors, compute_method=ComputeMethod.GPU,
                                        precision_mode=PrecisionMode.FP64):
        return self._compute(point_vectors, _lib.FIELD_A, compute_method, precision_mode)

    def compute_all_B_field_vectors(self, point_vectors, compute_method=ComputeMethod.GPU,
                                    precision_mode=PrecisionMode.FP64):
        return self._compute(point_vectors, _lib.FIELD_B, compute_method, precision_mode)

    def compute_all_E_field_vectors(self, point_vectors, compute_method=ComputeMethod.GPU,
                                    precision_mode=PrecisionMode.FP64):
        return self._compute(point_vectors, _lib.FIELD_E, compute_method, precision_mode)

    def compute_all_B_gradient_matrices(self, point_vectors, compute_method=ComputeMethod.GPU,
                                        precision_mode=PrecisionMode.FP64):
        return self._compute(point_vectors, _lib.FIELD_G, compute_method, precision_mode)

    # --- coil pairs: the secondary against every member except itself ---------------------
    def _group_arrangements(self, secondary, positions, y_angles, z_angles, precision_factor, compute_method,
                            quantity, precision_mode=PrecisionMode.FP64):
        if ComputeMethod(compute_method) != ComputeMethod.GPU:
            raise NotImplementedError("this package provides the ComputeMethod.GPU path only")
        pf = _factor(precision_factor or PrecisionFactor())
        prims, secs, zargs = [], [], []
        for m in self.member_coils:
            if m.get_id() == secondary.get_id():
                continue  # CoilGroup::computeMutualInductance skips the secondary (ComputeMInductance.cxx:15)
            pp, sp = Coil._pair_args(m, secondary, pf)
            prims.append(m.struct(pp))
            secs.append(sp.to_struct())
            za = CoilPairArguments.get_appropriate_coil_pair_arguments(m, secondary, pf, ComputeMethod.CPU_ST,
                                                                       z_axis_case=True)
            zargs += [za.primary_precision.to_struct(), za.secondary_precision.to_struct()]
        spose = _poses(positions, y_angles, z_angles)
        vals, _ = _pair_arrangements(prims, secondary.struct(), secs, None, spose, quantity, precision_mode,
                                     zargs if quantity in (_lib.PAIR_MUTUAL_INDUCTANCE, _lib.PAIR_FORCE_TORQUE)
                                     else None)
        return vals

    def compute_all_mutual_inductance_arrangements(self, secondary, secondary_positions, secondary_y_angles,
                                                   secondary_z_angles, precision_factor=None,
                                                   compute_method=ComputeMethod.GPU,
                                                   precision_mode=PrecisionMode.FP64):
        """CoilGroup::computeAllMutualInductanceArrangements (ComputeMInductance.cxx:23-64)."""
        return self._group_arrangements(secondary, secondary_positions, secondary_y_angles, secondary_z_angles,
                                        precision_factor, compute_method, _lib.PAIR_MUTUAL_INDUCTANCE,
                                        precision_mode)

    def compute_all_force_torque_arrangements(self, secondary, secondary_positions, secondary_y_angles,
                                              secondary_z_angles, precision_factor=None,
                                              compute_method=ComputeMethod.GPU,
                                              precision_mode=PrecisionMode.FP64):
        """CoilGroup::computeAllForceTorqueArrangements (ComputeForce.cxx:47-89): (n, 6)."""
        return self._group_arrangements(secondary, secondary_positions, secondary_y_angles, secondary_z_angles,
                                        precision_factor, compute_method, _lib.PAIR_FORCE_TORQUE, precision_mode)

    def compute_mutual_inductance(self, secondary, precision_factor=None, compute_method=ComputeMethod.GPU):
        p, y, z = secondary._pose_row()
        return float(self.compute_all_mutual_inductance_arrangements(secondary, [p], [y], [z], precision_factor,
                                                                     compute_method)[0])

    def compute_force_torque(self, secondary, precision_factor=None, compute_method=ComputeMethod.GPU):
        p, y, z = secondary._pose_row()
        v = self.compute_all_force_torque_arrangements(secondary, [p], [y], [z], precision_factor,
                                                       compute_method)[0]
        return v[:3].copy(), v[3:].copy()


def legendre(order):
    """Gauss-Legendre nodes and weights of the given order (1..100), ascending nodes."""
    x, w = np.zeros(order), np.zeros(order)
    check(lib().ccoil_legendre(order, x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                               w.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return x, w
