"""Batched evaluation of many independent coil systems in one persistent launch,
replayed from a captured CUDA graph (ccoil_batch_plan_*, include/ccoil_gpu.h).

    plan = BatchPlan([(coils_0, points_0), (coils_1, points_1), ...], fields=("B", "G"))
    plan.tune()                  # optional: the autotuner picks the work split
    out = plan.run()             # {"B": (n_total, 3), "G": (n_total, 9)} torch CUDA tensors
    plan.split(out["B"])         # per-system views

Each system is a list of Coil objects (evaluated at their default precision)
and an (n, 3) array of points.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib
from .coil import PrecisionMode

_FIELDS = {"A": _lib.FIELD_A, "B": _lib.FIELD_B, "G": _lib.FIELD_G}


class BatchPlan:
    def __init__(self, systems, fields=("B", "G"), precision=PrecisionMode.FP64, device=None):
        import torch
        self.device = torch.device(device or "cuda")
        structs, coil_off, point_off, pts = [], [0], [0], []
        for coils, points in systems:
            structs.extend(c.struct() for c in coils)
            coil_off.append(len(structs))
            p = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
            pts.append(p)
            point_off.append(point_off[-1] + len(p))
        self.point_offsets = point_off
        self.fields = tuple(fields)
        mask = 0
        for f in self.fields:
            mask |= 1 << _FIELDS[f]
        arr = (_lib.CoilStruct * max(len(structs), 1))(*structs)
        co = (ctypes.c_int * len(coil_off))(*coil_off)
        po = (ctypes.c_longlong * len(point_off))(*point_off)
        self._h = ctypes.c_void_p()
        check(lib().ccoil_batch_plan_create(arr, co, po, len(systems), mask, int(precision), ctypes.byref(self._h)))
        allpts = np.concatenate(pts) if pts else np.zeros((0, 3))
        self.points = torch.from_numpy(allpts).to(self.device)
        n = len(allpts)
        self.out = {f: torch.zeros((n, 9 if f == "G" else 3), dtype=torch.float64, device=self.device)
                    for f in self.fields}

    def _ptrs(self):
        def p(t):
            return ctypes.c_void_p(t.data_ptr()) if t is not None else None
        return (p(self.points), p(self.out.get("A")), p(self.out.get("B")), p(self.out.get("G")))

    def run(self, stream=None):
        import torch
        st = stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        check(lib().ccoil_batch_plan_execute(self._h, *self._ptrs(), ctypes.c_void_p(st)))
        return self.out

    def tune(self):
        """Runs the autotuner; returns (chosen split, best time in ms)."""
        import torch
        torch.cuda.synchronize(self.device)
        split = ctypes.c_int(0)
        ms = ctypes.c_float(0)
        check(lib().ccoil_batch_plan_tune(self._h, *self._ptrs(), ctypes.byref(split), ctypes.byref(ms)))
        return split.value, ms.value

    def set_split(self, split):
        check(lib().ccoil_batch_plan_set_split(self._h, int(split)))

    def split(self, tensor):
        o = self.point_offsets
        return [tensor[o[i]:o[i + 1]] for i in range(len(o) - 1)]

    def close(self):
        if self._h:
            lib().ccoil_batch_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
