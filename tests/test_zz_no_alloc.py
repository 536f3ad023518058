"""The allocation-free entry point (ccoil_fields_fp32c_static) against the
plan-based FP32_COMPENSATED path, through the C-ABI, on two calls in a row.

It serves callers that cannot allocate device memory (host programs that own
every device allocation, real-time loops that must not stall on one); its scratch is a fixed array in device
memory shared by all calls, so the second call also checks that the state the
first one left behind does not leak into the result."""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def test_static_entry_point_matches_plan_path(ccoil):
    import torch
    from ccoil_b200 import workloads

    L = ccoil.lib()
    fn = L.ccoil_fields_fp32c_static
    fn.argtypes = [ctypes.POINTER(ccoil._lib.CoilStruct), ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong,
                   ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    rows = workloads.coil_rows_mixed(24, seed=314)
    coils = workloads.coils_from_rows(rows, 5.0)
    structs = (ccoil._lib.CoilStruct * len(coils))(*[c.struct() for c in coils])
    # points near and far from the windings, so the near-field work list is used
    pts = np.concatenate([workloads.points_cube(6000, seed=315),
                          workloads.points_cube(2000, seed=316, half=0.5) + 0.5])
    dpts = torch.from_numpy(pts).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    # B, G, A and E (E = 2 pi f A: the rows carry f = 50 Hz); the rows mix all four
    # coil types, so both the fast (RECTANGULAR, THIN) and slow integrands run
    for field in (1, 3, 0, 2):
        width = 9 if field == 3 else 3
        plan = ccoil.FieldPlan([c.struct() for c in coils], field, ccoil.PrecisionMode.FP32_COMPENSATED)
        expected = plan(pts)
        plan.close()
        for call in range(2):
            out = torch.full((len(pts), width), float("nan"), dtype=torch.float64, device="cuda")
            rc = fn(structs, len(coils), ctypes.c_void_p(dpts.data_ptr()), len(pts), field,
                    ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
            assert rc == 0, L.ccoil_last_error_message()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got)), (field, call)
            assert rel_err(got, expected).max() < 1e-14, (field, call)


def test_static_entry_point_rejects_oversized_requests(ccoil):
    import torch
    L = ccoil.lib()
    fn = L.ccoil_fields_fp32c_static
    fn.argtypes = [ctypes.POINTER(ccoil._lib.CoilStruct), ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong,
                   ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    # 1200 coils at PrecisionFactor 9 need far more than 1 MiB of node tables
    coil = ccoil.Coil(0.1, 0.05, 0.05, 10, precision_factor=9.0)
    structs = (ccoil._lib.CoilStruct * 1200)(*([coil.struct()] * 1200))
    pts = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    out = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    rc = fn(structs, 1200, ctypes.c_void_p(pts.data_ptr()), 4, 1, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1
    assert b"1 MiB" in L.ccoil_last_error_message()


def test_static_entry_point_refuses_stream_capture(ccoil):
    """Inside a stream capture the entry point returns CCOIL_ERR_NOT_SUPPORTED
    before it touches the stream (a captured call would record copies from the
    shared host staging buffers), and the capture itself stays usable."""
    import torch
    from ccoil_b200 import workloads

    L = ccoil.lib()
    fn = L.ccoil_fields_fp32c_static
    fn.argtypes = [ctypes.POINTER(ccoil._lib.CoilStruct), ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong,
                   ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    coils = workloads.coils_from_rows(workloads.coil_rows_mixed(4, seed=317), 5.0)
    structs = (ccoil._lib.CoilStruct * len(coils))(*[c.struct() for c in coils])
    dpts = torch.from_numpy(workloads.points_cube(256, seed=318)).cuda()
    dout = torch.empty((256, 3), dtype=torch.float64, device="cuda")
    x = torch.zeros(1, device="cuda")
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        x.add_(1.0)
        rc = fn(structs, len(coils), ctypes.c_void_p(dpts.data_ptr()), 256, 1, ctypes.c_void_p(dout.data_ptr()),
                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 4, rc  # CCOIL_ERR_NOT_SUPPORTED
    assert b"capture" in L.ccoil_last_error_message()
    g.replay()
    torch.cuda.synchronize()
    assert x.item() == 1.0
    # outside a capture the same call runs
    assert fn(structs, len(coils), ctypes.c_void_p(dpts.data_ptr()), 256, 1, ctypes.c_void_p(dout.data_ptr()),
              None) == 0
    torch.cuda.synchronize()
    assert torch.isfinite(dout).all()
