"""Differentiable coil fields: torch.autograd.Function over the B-field kernels
and the hand-written adjoint kernel (ccoil_b_field_adjoint).

    params = torch.tensor([[R, a, b, N*I, x, y, z, y_angle, z_angle], ...], requires_grad=True)
    B = b_field(params, points)          # (n, 3), float64 or float32 like `points`
    loss = ...; loss.backward()          # params.grad: (C, 9)

The node counts (PrecisionArguments) are fixed at the values of the given
parameters (or passed explicitly), so the quadrature is a smooth function of
the parameters.  Forward: FP64 kernel for float64 points, FP32-compensated for
float32 points; backward: the FP64 adjoint in both cases.

    M = mutual_inductance(geom1, geom2, poses1, poses2)   # (n,)
    geom = [R, a, b, N] per coil (tensors), poses = (n, 5) [x, y, z, y_angle, z_angle]

differentiates the mutual inductance of n arrangements of one primary and one
secondary with respect to both coils' R, a, b, N and every arrangement's
poses, through the pair kernel's exact parameter gradient (node counts fixed
at the given geometry; FP64 for float64 poses, the primary's quadrature in
FP32 for float32 poses).

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


def pair_precisions_for(geom1, geom2, precision_factor=5.0):
    """CPU pair PrecisionArguments (primary, secondary) of two coil geometries [R, a, b, N]."""
    g1 = [float(v) for v in geom1]
    g2 = [float(v) for v in geom2]
    c1 = Coil(g1[0], g1[1], g1[2], int(round(g1[3])), 1.0)
    c2 = Coil(g2[0], g2[1], g2[2], int(round(g2[3])), 1.0)
    return Coil._pair_args(c1, c2, _factor(precision_factor))


def _pair_structs(g1, g2, pp, sp):
    zero = (ctypes.c_double * 3)(0.0, 0.0, 0.0)
    s1, s2 = _lib.CoilStruct(), _lib.CoilStruct()
    check(lib().ccoil_coil_init(g1[0], g1[1], g1[2], 1, 1.0, 0.0, zero, 0.0, 0.0, 5.0, 0, ctypes.byref(s1)))
    check(lib().ccoil_coil_init(g2[0], g2[1], g2[2], 1, 1.0, 0.0, zero, 0.0, 0.0, 5.0, 0, ctypes.byref(s2)))
    # turns enter M as N1 N2: run with N = 1 and scale, so non-integer N stay differentiable
    s1.precision = pp.to_struct()
    s2.precision = sp.to_struct()
    return s1, s2


class _MutualInductance(torch.autograd.Function):
    @staticmethod
    def forward(ctx, geom1, geom2, poses1, poses2, precisions):
        from .coil import _pair_arrangements
        g1 = geom1.detach().to("cpu", torch.float64).numpy()
        g2 = geom2.detach().to("cpu", torch.float64).numpy()
        p1 = np.ascontiguousarray(poses1.detach().to("cpu", torch.float64).numpy())
        p2 = np.ascontiguousarray(poses2.detach().to("cpu", torch.float64).numpy())
        if p1.shape != p2.shape or p1.ndim != 2 or p1.shape[1] != 5:
            raise ValueError("poses must be (n, 5) arrays of equal shape")
        pp, sp = precisions
        s1, s2 = _pair_structs(g1, g2, pp, sp)
        # float32 poses: the primary's quadrature in FP32 (FP64 near its winding and in the sums)
        mode = PrecisionMode.FP32_COMPENSATED if poses2.dtype == torch.float32 else PrecisionMode.FP64
        out, _ = _pair_arrangements([s1], s2, [sp.to_struct()], p1, p2,
                                    _lib.PAIR_MUTUAL_INDUCTANCE_PARAMETER_GRADIENT, precision_mode=mode)
        out = out * (g1[3] * g2[3])
        ctx.out = out
        ctx.turns = (g1[3], g2[3])
        ctx.devices = (geom1.device, geom2.device, poses1.device, poses2.device)
        ctx.dtypes = (geom1.dtype, geom2.dtype, poses1.dtype, poses2.dtype)
        return torch.from_numpy(out[:, 0].copy()).to(poses2.device, poses2.dtype)

    @staticmethod
    def backward(ctx, grad_m):
        out = ctx.out
        n1, n2 = ctx.turns
        g = grad_m.detach().to("cpu", torch.float64).numpy()
        M = out[:, 0]
        d1 = np.array([g @ out[:, 1], g @ out[:, 2], g @ out[:, 3], g @ M / n1])
        d2 = np.array([g @ out[:, 6], g @ out[:, 7], g @ out[:, 8], g @ M / n2])
        dp2 = np.concatenate([out[:, 9:12], out[:, 12:14]], axis=1) * g[:, None]
        dp1 = np.concatenate([-out[:, 9:12], out[:, 4:6]], axis=1) * g[:, None]
        res = [torch.from_numpy(v).to(dev, dt) for v, dev, dt in zip((d1, d2, dp1, dp2), ctx.devices, ctx.dtypes)]
        return res[0], res[1], res[2], res[3], None


def mutual_inductance(geom1, geom2, poses1, poses2, precisions=None, precision_factor=5.0):
    """Differentiable mutual inductance of n arrangements: geom = [R, a, b, N] per coil, poses (n, 5)
    = [x, y, z, y_angle, z_angle] per arrangement (primary 1, secondary 2).  Gradients flow to
    both geometries and both pose arrays."""
    if precisions is None:
        precisions = pair_precisions_for(geom1.detach().cpu().numpy(), geom2.detach().cpu().numpy(),
                                         precision_factor)
    return _MutualInductance.apply(geom1, geom2, poses1, poses2, tuple(precisions))
