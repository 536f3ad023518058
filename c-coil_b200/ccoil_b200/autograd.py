"""Differentiable coil fields: torch.autograd.Function over the B-field kernels
and the hand-written adjoint kernel (ccoil_b_field_adjoint).

    params = torch.tensor([[R, a, b, N*I, x, y, z, y_angle, z_angle], ...], requires_grad=True)
    B = b_field(params, points)          # (n, 3), float64 or float32 like `points`
    loss = ...; loss.backward()          # params.grad: (C, 9)

The node counts (PrecisionArguments) are fixed at the values of the given
parameters (or passed explicitly), so the quadrature is a smooth function of
the parameters.  Forward: FP64 kernel for float64 points, FP32-compensated for
float32 points; backward: the FP64 adjoint in both cases.

`mutual_inductance_position_gradient` is the exact derivative of the mutual
inductance quadrature with respect to the secondary's position (the pair
kernel differentiates the primary's A at every secondary node).  Physically
it equals F / (I1 I2), the Ampere force of
src/Coil/ForceAndTorque/CalculateForceGeneral.cxx:9-131 divided by the
currents; the two quadratures agree up to the quadrature error of the
reference's precision settings (`mutual_inductance_position_gradient_from_force`).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, lib
from .coil import Coil, PrecisionArguments, PrecisionFactor, PrecisionMode, _factor

PARAMS = ("R", "a", "b", "NI", "x", "y", "z", "y_angle", "z_angle")


def _structs(params, precisions):
    out = []
    for q, pa in zip(params, precisions):
        s = _lib.CoilStruct()
        pos = (ctypes.c_double * 3)(q[4], q[5], q[6])
        check(lib().ccoil_coil_init(q[0], q[1], q[2], 1, q[3], 0.0, pos, q[7], q[8], 5.0, 0, ctypes.byref(s)))
        s.precision = pa.to_struct()
        out.append(s)
    return out


def precisions_for(params, precision_factor=5.0):
    """CPU PrecisionArguments of each parameter row at precision_factor."""
    pf = _factor(precision_factor)
    res = []
    for q in np.asarray(params, dtype=np.float64):
        c = Coil(q[0], q[1], q[2], 1, q[3], 0.0, PrecisionFactor(pf), 8, (q[4], q[5], q[6]), q[7], q[8])
        res.append(c.default_precision_CPU)
    return res


class _BField(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, points, precisions):
        q = params.detach().to("cpu", torch.float64).numpy()
        structs = _structs(q, precisions)
        pts = points.detach().to(torch.float64).contiguous()
        mode = PrecisionMode.FP32_COMPENSATED if points.dtype == torch.float32 else PrecisionMode.FP64
        out = torch.empty((pts.shape[0], 3), dtype=torch.float64, device=pts.device)
        arr = (_lib.CoilStruct * max(len(structs), 1))(*structs)
        st = torch.cuda.current_stream(pts.device).cuda_stream
        check(lib().ccoil_compute_fields(arr, len(structs), ctypes.c_void_p(pts.data_ptr()), pts.shape[0],
                                         _lib.FIELD_B, int(mode), ctypes.c_void_p(out.data_ptr()),
                                         _lib.MEMORY_DEVICE, ctypes.c_void_p(st)))
        ctx.save_for_backward(params, pts)
        ctx.precisions = precisions
        ctx.points_dtype = points.dtype
        return out.to(points.dtype)

    @staticmethod
    def backward(ctx, grad_b):
        params, pts = ctx.saved_tensors
        q = np.ascontiguousarray(params.detach().to("cpu", torch.float64).numpy())
        g = grad_b.detach().to(torch.float64).contiguous()
        gp = torch.zeros((q.shape[0], 9), dtype=torch.float64, device=pts.device)
        precs = (_lib.PrecisionArgsStruct * max(len(ctx.precisions), 1))(*[p.to_struct() for p in ctx.precisions])
        st = torch.cuda.current_stream(pts.device).cuda_stream
        check(lib().ccoil_b_field_adjoint(q.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), precs, q.shape[0],
                                          ctypes.c_void_p(pts.data_ptr()), pts.shape[0],
                                          ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(gp.data_ptr()),
                                          ctypes.c_void_p(st)))
        return gp.to(params.dtype).to(params.device), None, None


def b_field(params, points, precisions=None, precision_factor=5.0):
    """Differentiable group B field at `points` (CUDA tensor) for coil parameter rows `params`."""
    if precisions is None:
        precisions = precisions_for(params.detach().cpu().numpy(), precision_factor)
    return _BField.apply(params, points, list(precisions))


def mutual_inductance_position_gradient(primary, secondary, precision_factor=None):
    """dM/d(secondary position) of the pair as placed: exact derivative of the M quadrature."""
    pp, py, pz = primary._pose_row()
    sp, sy, sz = secondary._pose_row()
    return Coil.compute_all_mutual_inductance_gradient_arrangements(
        primary, secondary, [pp], [sp], [py], [pz], [sy], [sz], precision_factor or PrecisionFactor())[0]


def mutual_inductance_position_gradient_from_force(primary, secondary, precision_factor=None):
    """F / (I1 I2) with F the force on the secondary (src/Coil/ForceAndTorque/CalculateForceGeneral.cxx)."""
    F, _ = Coil.compute_force_torque(primary, secondary, precision_factor or PrecisionFactor())
    return F / (primary.get_current() * secondary.get_current())
