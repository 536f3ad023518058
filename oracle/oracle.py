"""TEST INFRASTRUCTURE ONLY -- ctypes bindings for the two CPU checkers.

* ``Oracle``   : the project's C restatement of the reference's CPU algorithm
                 (oracle/ccoil_oracle.c -> oracle/liboracle.so).
* ``Reference``: the reference's own CPU sources compiled unmodified
                 (oracle/ref_capi.cpp + C-Coil src/ -> oracle/_ref/libccoil_ref.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module.  Coils are 11-float rows {R, a, b, N, I, f, x, y, z, yAngle, zAngle};
points are (n, 3) float64 arrays; quantities are 0=A, 1=B, 2=E, 3=G.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libccoil_ref.so")
# the same reference sources built with USE_GPU: its own GPU glue, linked against
# libccoil_b200.so (oracle/Makefile, target ref-gpu)
REF_GPU_SO = os.path.join(HERE, "_ref", "libccoil_ref_gpu.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_d = ctypes.c_double
_i = ctypes.c_int
_ll = ctypes.c_longlong


def _ptr(a, t=_dp):
    return None if a is None else a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


def coil_row(R, a, b, N, I=1.0, f=0.0, pos=(0.0, 0.0, 0.0), y_angle=0.0, z_angle=0.0):
    return np.array([R, a, b, N, I, f, pos[0], pos[1], pos[2], y_angle, z_angle], dtype=np.float64)


class Oracle:
    """C restatement (always available once `make -C oracle` has run)."""

    def __init__(self, path=ORACLE_SO):
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.oracle_legendre.argtypes = [_i, _dp, _dp]
        L.oracle_coil_info.argtypes = [_dp, _dp]
        L.oracle_precision_args.argtypes = [_dp, _d, _i, _ip]
        L.oracle_pair_args.argtypes = [_dp, _dp, _d, _i, _i, _i, _ip]
        L.oracle_coil_fields.argtypes = [_dp, _d, _ip, _i, _ll, _dp, _dp]
        L.oracle_group_fields.argtypes = [_i, _dp, _d, _i, _ll, _dp, _dp]
        L.oracle_mutual_inductance.argtypes = [_dp, _dp, _d, _ip, _dp]
        L.oracle_force_torque.argtypes = [_dp, _dp, _d, _ip, _dp]
        L.oracle_z_axis_case.argtypes = [_dp, _dp]
        L.oracle_self_inductance.argtypes = [_dp, _d, _ip, _dp]

    def legendre(self, order):
        p, w = np.zeros(order), np.zeros(order)
        assert self.lib.oracle_legendre(order, _ptr(p), _ptr(w)) == 0
        return p, w

    def coil_info(self, coil):
        out = np.zeros(24)
        self.lib.oracle_coil_info(_ptr(_f64(coil)), _ptr(out))
        return out

    def precision_args(self, coil, pf, gpu_cap=0):
        out = np.zeros(6, dtype=np.int32)
        self.lib.oracle_precision_args(_ptr(_f64(coil)), pf, gpu_cap, _ptr(out, _ip))
        return out

    def pair_args(self, prim, sec, pf, gpu_cap=0, z_axis=False, pure_gpu=False):
        out = np.zeros(12, dtype=np.int32)
        self.lib.oracle_pair_args(_ptr(_f64(prim)), _ptr(_f64(sec)), pf, gpu_cap, int(z_axis), int(pure_gpu),
                                  _ptr(out, _ip))
        return out

    def coil_fields(self, coil, points, qty, pf=5.0, prec=None):
        pts = _f64(points)
        n = pts.shape[0]
        out = np.zeros((n, 9 if qty == 3 else 3))
        prec = _i32(prec)
        self.lib.oracle_coil_fields(_ptr(_f64(coil)), pf, _ptr(prec, _ip), qty, n, _ptr(pts), _ptr(out))
        return out

    def group_fields(self, coils, points, qty, pf=5.0):
        pts = _f64(points)
        coils = _f64(coils)
        n = pts.shape[0]
        out = np.zeros((n, 9 if qty == 3 else 3))
        self.lib.oracle_group_fields(coils.shape[0], _ptr(coils), pf, qty, n, _ptr(pts), _ptr(out))
        return out

    def z_axis_case(self, prim, sec):
        return bool(self.lib.oracle_z_axis_case(_ptr(_f64(prim)), _ptr(_f64(sec))))

    def mutual_inductance(self, prim, sec, pf=5.0, args=None):
        out = np.zeros(1)
        rc = self.lib.oracle_mutual_inductance(_ptr(_f64(prim)), _ptr(_f64(sec)), pf, _ptr(_i32(args), _ip),
                                               _ptr(out))
        if rc != 0:
            raise ValueError("oracle pair evaluation failed (invalid coils or arguments)")
        return float(out[0])

    def self_inductance(self, coil, pf=5.0, args=None):
        out = np.zeros(1)
        rc = self.lib.oracle_self_inductance(_ptr(_f64(coil)), pf, _ptr(_i32(args), _ip), _ptr(out))
        if rc != 0:
            raise ValueError("a filament has no self inductance (divergent integral)")
        return float(out[0])

    def force_torque(self, prim, sec, pf=5.0, args=None):
        out = np.zeros(6)
        rc = self.lib.oracle_force_torque(_ptr(_f64(prim)), _ptr(_f64(sec)), pf, _ptr(_i32(args), _ip), _ptr(out))
        if rc != 0:
            raise ValueError("oracle pair evaluation failed (invalid coils or arguments)")
        return out


class Reference:
    """The reference's own CPU code (needs oracle/_ref/libccoil_ref.so)."""

    def __init__(self, path=REF_SO, threads=None):
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.ref_set_threads.argtypes = [_i]
        L.ref_legendre.argtypes = [_i, _dp, _dp]
        L.ref_coil_info.argtypes = [_dp, _dp]
        L.ref_precision_args.argtypes = [_dp, _d, _i, _ip]
        L.ref_secondary_precision_gpu.argtypes = [_dp, _d, _ip]
        L.ref_pair_args.argtypes = [_dp, _dp, _d, _i, _i, _i, _ip]
        L.ref_coil_fields.argtypes = [_dp, _d, _ip, _i, _i, _ll, _dp, _dp]
        L.ref_group_fields.argtypes = [_i, _dp, _d, _i, _i, _ll, _dp, _dp]
        if hasattr(L, "ref_group_fields_dispatch"):
            L.ref_group_fields_dispatch.argtypes = [_i, _dp, _d, _i, _i, _ll, _dp, _dp]
        L.ref_mutual_inductance.argtypes = [_dp, _dp, _d, _i, _dp]
        L.ref_mutual_inductance_args.argtypes = [_dp, _dp, _ip, _i, _dp]
        L.ref_force_torque.argtypes = [_dp, _dp, _d, _i, _dp]
        L.ref_force_torque_args.argtypes = [_dp, _dp, _ip, _i, _dp]
        arr = [_dp, _dp, _ll, _dp, _dp, _dp, _dp, _dp, _dp, _d, _i, _dp]
        L.ref_m_arrangements.argtypes = arr
        L.ref_ft_arrangements.argtypes = arr
        garr = [_i, _dp, _dp, _i, _ll, _dp, _dp, _dp, _d, _i, _dp]
        L.ref_group_m_arrangements.argtypes = garr
        L.ref_group_ft_arrangements.argtypes = garr
        L.ref_self_inductance.argtypes = [_dp, _d, _dp]
        if threads:
            self.set_threads(threads)

    @staticmethod
    def available(path=REF_SO):
        return os.path.exists(path)

    def set_threads(self, n):
        self.lib.ref_set_threads(int(n))

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError("the reference raised an exception")

    def legendre(self, order):
        p, w = np.zeros(order), np.zeros(order)
        self._check(self.lib.ref_legendre(order, _ptr(p), _ptr(w)))
        return p, w

    def coil_info(self, coil):
        out = np.zeros(24)
        self._check(self.lib.ref_coil_info(_ptr(_f64(coil)), _ptr(out)))
        return out

    def precision_args(self, coil, pf, gpu=False):
        out = np.zeros(6, dtype=np.int32)
        self._check(self.lib.ref_precision_args(_ptr(_f64(coil)), pf, int(gpu), _ptr(out, _ip)))
        return out

    def secondary_precision_gpu(self, coil, pf):
        """PrecisionArguments::getSecondaryCoilPrecisionArgumentsGPU"""
        out = np.zeros(6, dtype=np.int32)
        self._check(self.lib.ref_secondary_precision_gpu(_ptr(_f64(coil)), pf, _ptr(out, _ip)))
        return out

    def pair_args(self, prim, sec, pf, gpu=False, z_axis=False, pure_gpu=False):
        out = np.zeros(12, dtype=np.int32)
        self._check(self.lib.ref_pair_args(_ptr(_f64(prim)), _ptr(_f64(sec)), pf, int(gpu), int(z_axis),
                                           int(pure_gpu), _ptr(out, _ip)))
        return out

    def coil_fields(self, coil, points, qty, pf=5.0, prec=None, method=0):
        pts = _f64(points)
        n = pts.shape[0]
        out = np.zeros((n, 9 if qty == 3 else 3))
        prec = _i32(prec)
        self._check(self.lib.ref_coil_fields(_ptr(_f64(coil)), pf, _ptr(prec, _ip), qty, method, n, _ptr(pts),
                                             _ptr(out)))
        return out

    def group_fields(self, coils, points, qty, pf=5.0, method=0):
        pts = _f64(points)
        coils = _f64(coils)
        n = pts.shape[0]
        out = np.zeros((n, 9 if qty == 3 else 3))
        self._check(self.lib.ref_group_fields(coils.shape[0], _ptr(coils), pf, qty, method, n, _ptr(pts),
                                              _ptr(out)))
        return out

    def group_fields_dispatch(self, coils, points, qty, pf=5.0, method=0):
        """CoilGroup::computeAll*(points, method) through the group's own dispatch
        (method 2: its GPU glue)."""
        pts = _f64(points)
        coils = _f64(coils)
        n = pts.shape[0]
        out = np.zeros((n, 9 if qty == 3 else 3))
        self._check(self.lib.ref_group_fields_dispatch(coils.shape[0], _ptr(coils), pf, qty, method, n, _ptr(pts),
                                                       _ptr(out)))
        return out

    def mutual_inductance(self, prim, sec, pf=5.0, args=None, method=0):
        out = np.zeros(1)
        if args is None:
            self._check(self.lib.ref_mutual_inductance(_ptr(_f64(prim)), _ptr(_f64(sec)), pf, method, _ptr(out)))
        else:
            self._check(self.lib.ref_mutual_inductance_args(_ptr(_f64(prim)), _ptr(_f64(sec)),
                                                            _ptr(_i32(args), _ip), method, _ptr(out)))
        return float(out[0])

    def force_torque(self, prim, sec, pf=5.0, args=None, method=0):
        out = np.zeros(6)
        if args is None:
            self._check(self.lib.ref_force_torque(_ptr(_f64(prim)), _ptr(_f64(sec)), pf, method, _ptr(out)))
        else:
            self._check(self.lib.ref_force_torque_args(_ptr(_f64(prim)), _ptr(_f64(sec)), _ptr(_i32(args), _ip),
                                                       method, _ptr(out)))
        return out

    def _arr(self, fn, width, prim, sec, prim_pos, sec_pos, py, pz, sy, sz, pf, method):
        n = len(py)
        out = np.zeros((n, width)) if width > 1 else np.zeros(n)
        self._check(fn(_ptr(_f64(prim)), _ptr(_f64(sec)), n, _ptr(_f64(prim_pos)), _ptr(_f64(sec_pos)),
                       _ptr(_f64(py)), _ptr(_f64(pz)), _ptr(_f64(sy)), _ptr(_f64(sz)), pf, method, _ptr(out)))
        return out

    def m_arrangements(self, prim, sec, prim_pos, sec_pos, py, pz, sy, sz, pf=5.0, method=0):
        return self._arr(self.lib.ref_m_arrangements, 1, prim, sec, prim_pos, sec_pos, py, pz, sy, sz, pf, method)

    def ft_arrangements(self, prim, sec, prim_pos, sec_pos, py, pz, sy, sz, pf=5.0, method=0):
        return self._arr(self.lib.ref_ft_arrangements, 6, prim, sec, prim_pos, sec_pos, py, pz, sy, sz, pf,
                         method)

    def group_m_arrangements(self, coils, sec, sec_pos, sy, sz, pf=5.0, method=0, sec_member=-1):
        coils = _f64(coils)
        n = len(sy)
        out = np.zeros(n)
        self._check(self.lib.ref_group_m_arrangements(coils.shape[0], _ptr(coils), _ptr(_f64(sec)), sec_member, n,
                                                      _ptr(_f64(sec_pos)), _ptr(_f64(sy)), _ptr(_f64(sz)), pf,
                                                      method, _ptr(out)))
        return out

    def group_ft_arrangements(self, coils, sec, sec_pos, sy, sz, pf=5.0, method=0, sec_member=-1):
        coils = _f64(coils)
        n = len(sy)
        out = np.zeros((n, 6))
        self._check(self.lib.ref_group_ft_arrangements(coils.shape[0], _ptr(coils), _ptr(_f64(sec)), sec_member, n,
                                                       _ptr(_f64(sec_pos)), _ptr(_f64(sy)), _ptr(_f64(sz)), pf,
                                                       method, _ptr(out)))
        return out

    def self_inductance(self, coil, pf=5.0):
        out = np.zeros(1)
        self._check(self.lib.ref_self_inductance(_ptr(_f64(coil)), pf, _ptr(out)))
        return float(out[0])
