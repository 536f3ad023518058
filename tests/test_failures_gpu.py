"""Failure paths, exercised without faulting the GPU: the reference ends the
process on any CUDA error (src/CUDAUtils/ErrorCheck/ErrorCheck.cu:15); this
library returns a status code and stays usable.

  - a bounded device-side wait on a barrier that nothing completes gives up,
    returns CCOIL_ERR_TIMEOUT and is counted by ccoil_timeout_count();
  - injected allocation failures of the library's memory pool surface as
    CCOIL_ERR_OUT_OF_MEMORY, and the next call succeeds;
  - NaN and infinite point coordinates give NaN results in their rows only
    (the kernels' loops run over node counts, never over values)."""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

OK, TIMEOUT, OOM = 0, 5, 3


def group(ccoil, n=6, seed=3):
    from ccoil_b200 import workloads
    return [c.struct() for c in workloads.coils_from_rows(workloads.coil_rows_mixed(n, seed), 5.0)]


def fields_host(ccoil, structs, pts, field, precision):
    from ccoil_b200 import _lib
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    out = np.zeros((len(pts), 9 if field == 3 else 3))
    arr = (_lib.CoilStruct * len(structs))(*structs)
    rc = ccoil.lib().ccoil_compute_fields(arr, len(structs), pts.ctypes.data_as(ctypes.c_void_p), len(pts), field,
                                          precision, out.ctypes.data_as(ctypes.c_void_p), 0, None)
    return rc, out


def test_bounded_wait_gives_up_and_the_context_survives(ccoil):
    L = ccoil.lib()
    before = L.ccoil_timeout_count()
    rc = L.ccoil_check_bounded_wait(2_000_000, None)  # ~1 ms of polling
    assert rc == TIMEOUT, (rc, L.ccoil_last_error_message())
    assert L.ccoil_timeout_count() == before + 1
    structs = group(ccoil)
    pts = np.random.default_rng(1).uniform(-1, 1, (1000, 3))
    rc, out = fields_host(ccoil, structs, pts, 1, 0)
    assert rc == OK and np.all(np.isfinite(out))
    assert L.ccoil_check_bounded_wait(-1, None) == 1


@pytest.mark.parametrize("precision", [0, 1])
def test_injected_allocation_failure(ccoil, precision):
    L = ccoil.lib()
    structs = group(ccoil)
    pts = np.random.default_rng(2).uniform(-1, 1, (2000, 3))
    rc, want = fields_host(ccoil, structs, pts, 1, precision)
    assert rc == OK
    assert L.ccoil_inject_allocation_failures(1) == OK
    rc, _ = fields_host(ccoil, structs, pts, 1, precision)
    assert rc == OOM, (rc, L.ccoil_last_error_message())
    assert b"memory" in L.ccoil_last_error_message().lower()
    rc, got = fields_host(ccoil, structs, pts, 1, precision)
    assert rc == OK and rel_err(got, want).max() < 1e-14
    # the pair path takes the same pool
    from ccoil_b200 import workloads
    prim_row, sec_row, ppos, spos, py, pz, sy, sz = workloads.pair_config(arrangements=64, seed=4)
    prim, sec = workloads.coils_from_rows(prim_row, 5.0)[0], workloads.coils_from_rows(sec_row, 5.0)[0]
    m0 = ccoil.Coil.compute_all_mutual_inductance_arrangements(prim, sec, ppos, spos, py, pz, sy, sz)
    assert L.ccoil_inject_allocation_failures(1) == OK
    with pytest.raises(Exception):
        ccoil.Coil.compute_all_mutual_inductance_arrangements(prim, sec, ppos, spos, py, pz, sy, sz)
    m1 = ccoil.Coil.compute_all_mutual_inductance_arrangements(prim, sec, ppos, spos, py, pz, sy, sz)
    assert np.array_equal(m0, m1)
    assert L.ccoil_inject_allocation_failures(0) == OK


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("field", [0, 1, 3])
def test_nan_and_infinite_points(ccoil, precision, field):
    """The other rows keep their values: exactly in FP64; in FP32_COMPENSATED to its
    rounding level, because a warp picks some integrand forms by a vote of its
    lanes (a NaN lane votes for the general form)."""
    structs = group(ccoil)
    pts = np.random.default_rng(5).uniform(-1, 1, (512, 3))
    rc, clean = fields_host(ccoil, structs, pts, field, precision)
    assert rc == OK
    bad = pts.copy()
    rows = [3, 100, 257, 511]
    bad[3, 0] = np.nan
    bad[100, 2] = np.inf
    bad[257, 1] = -np.inf
    bad[511] = np.nan
    rc, got = fields_host(ccoil, structs, bad, field, precision)
    assert rc == OK
    keep = np.setdiff1d(np.arange(len(pts)), rows)
    assert np.all(~np.isfinite(got[rows]).all(axis=1))
    assert rel_err(got[keep], clean[keep]).max() < (1e-14 if precision == 0 else 1e-7)
