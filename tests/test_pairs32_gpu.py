"""FP32-compensated mutual inductance and force/torque arrangements against the
FP64 kernel (itself held to 1e-12 of the reference by test_pairs_gpu.py).

Bars, relative error against max(|FP64|, 1e-3 x batch max) per arrangement
(norm-wise for force and torque): median below 1e-7, maximum below 2e-5.
Where a secondary node lies in the primary's near-field box the primary's
quadrature is FP64, which the near-field case checks at 1e-9."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

MEDIAN, MAX = 1e-7, 2e-5


def coils(ccoil, prim_row, sec_row, pf=5.0):
    from ccoil_b200 import workloads
    return workloads.coils_from_rows(prim_row, pf)[0], workloads.coils_from_rows(sec_row, pf)[0]


def both(ccoil, fn, *args):
    a = fn(*args, precision_mode=ccoil.PrecisionMode.FP32_COMPENSATED)
    b = fn(*args, precision_mode=ccoil.PrecisionMode.FP64)
    return a, b


def check_m(a, b, median=MEDIAN, worst=MAX):
    e = rel_err(a, b)
    assert np.median(e) < median and e.max() < worst, (np.median(e), e.max())


def check_ft(a, b, median=MEDIAN, worst=MAX):
    for lo in (0, 3):
        e = rel_err(a[:, lo:lo + 3], b[:, lo:lo + 3])
        assert np.median(e) < median and e.max() < worst, (lo, np.median(e), e.max())


def test_seeded_arrangements(ccoil):
    from ccoil_b200 import workloads
    prim_row, sec_row, ppos, spos, py, pz, sy, sz = workloads.pair_config(arrangements=2048, seed=17,
                                                                          coaxial_fraction=0.05)
    prim, sec = coils(ccoil, prim_row, sec_row)
    args = (prim, sec, ppos, spos, py, pz, sy, sz, ccoil.PrecisionFactor(5.0))
    a, b = both(ccoil, ccoil.Coil.compute_all_mutual_inductance_arrangements, *args)
    check_m(a, b)
    a, b = both(ccoil, ccoil.Coil.compute_all_force_torque_arrangements, *args)
    check_ft(a, b)


@pytest.mark.parametrize("pf", [1.0, 4.0, 7.0])
def test_odd_primary_angular_counts(ccoil, pf):
    """At these PrecisionFactors the primary's angular node count is odd (17, 29,
    49), so its FP32 mirror-pair table ends in a middle node of its own."""
    from ccoil_b200 import workloads
    prim_row, sec_row, ppos, spos, py, pz, sy, sz = workloads.pair_config(arrangements=1024, seed=19,
                                                                          coaxial_fraction=0.05)
    prim, sec = coils(ccoil, prim_row, sec_row, pf=pf)
    pp, _ = ccoil.Coil._pair_args(prim, sec, pf)
    assert (pp.angular_blocks * pp.angular_increments) % 2 == 1
    args = (prim, sec, ppos, spos, py, pz, sy, sz, ccoil.PrecisionFactor(pf))
    a, b = both(ccoil, ccoil.Coil.compute_all_mutual_inductance_arrangements, *args)
    check_m(a, b)
    a, b = both(ccoil, ccoil.Coil.compute_all_force_torque_arrangements, *args)
    check_ft(a, b)


def test_slow_method_primary(ccoil):
    """FLAT primary (slow method, length x thickness x angle) and FILAMENT secondary."""
    from ccoil_b200 import workloads
    prim_row, sec_row, ppos, spos, py, pz, sy, sz = workloads.pair_config(arrangements=512, seed=23)
    prim_row = prim_row.copy(); prim_row[2] = 0.0      # FLAT: no length
    sec_row = sec_row.copy(); sec_row[2] = 0.0         # FILAMENT
    prim, sec = coils(ccoil, prim_row, sec_row, pf=3.0)
    args = (prim, sec, ppos, spos, py, pz, sy, sz, ccoil.PrecisionFactor(3.0))
    a, b = both(ccoil, ccoil.Coil.compute_all_mutual_inductance_arrangements, *args)
    check_m(a, b)
    a, b = both(ccoil, ccoil.Coil.compute_all_force_torque_arrangements, *args)
    check_ft(a, b)


def test_near_field_pairs_take_fp64(ccoil):
    """Secondary rings running through the primary's winding: every warp iteration
    has a node in the near-field box, so FP32 mode reproduces FP64."""
    prim_row = np.array([0.1, 0.05, 0.1, 200, 1.0, 0, 0, 0, 0, 0, 0], dtype=float)
    sec_row = np.array([0.12, 0.01, 0.05, 50, 2.0, 0, 0, 0, 0, 0, 0], dtype=float)
    prim, sec = coils(ccoil, prim_row, sec_row)
    g = np.random.default_rng(3)
    n = 64
    spos = np.stack([g.uniform(-2e-3, 2e-3, n), g.uniform(-2e-3, 2e-3, n), g.uniform(-0.02, 0.02, n)], 1)
    zeros = np.zeros(n)
    args = (prim, sec, np.zeros((n, 3)), spos, zeros, zeros, g.uniform(0, 0.05, n), g.uniform(0, 6.28, n),
            ccoil.PrecisionFactor(5.0))
    a, b = both(ccoil, ccoil.Coil.compute_all_mutual_inductance_arrangements, *args)
    check_m(a, b, 1e-9, 1e-9)
    a, b = both(ccoil, ccoil.Coil.compute_all_force_torque_arrangements, *args)
    check_ft(a, b, 1e-9, 1e-9)


def test_group_arrangements(ccoil, golden):
    from ccoil_b200 import workloads
    group = ccoil.CoilGroup(workloads.coils_from_rows(golden["garr_coils"], 5.0), ccoil.PrecisionFactor(5.0))
    sy, sz = golden["garr_angles"]
    args = (group[0], golden["garr_sec_pos"], sy, sz, ccoil.PrecisionFactor(4.0))
    a, b = both(ccoil, group.compute_all_mutual_inductance_arrangements, *args)
    check_m(a, b)
    assert rel_err(b, golden["garr_M"]).max() < 1e-12
    a, b = both(ccoil, group.compute_all_force_torque_arrangements, *args)
    check_ft(a, b)


def test_gradient_is_fp64_only(ccoil):
    from ccoil_b200 import _lib
    from ccoil_b200.coil import _pair_arrangements
    prim = ccoil.Coil(0.1, 0.05, 0.1, 100)
    sec = ccoil.Coil(0.05, 0.0, 0.1, 50)
    pp, sp = ccoil.Coil._pair_args(prim, sec, 5.0)
    with pytest.raises(ccoil.CCoilError):
        _pair_arrangements([prim.struct(pp)], sec.struct(sp), [sp.to_struct()],
                           np.zeros((1, 5)), np.array([[0, 0, 0.3, 0, 0]], dtype=float),
                           _lib.PAIR_MUTUAL_INDUCTANCE_GRADIENT, ccoil.PrecisionMode.FP32_COMPENSATED)


def test_refined_arrangements(ccoil):
    """FP32_REFINED arrangements re-evaluate in FP64 every secondary node whose FP32
    contribution exceeds the set fraction of the arrangement's M (for F/T: of its
    force or torque).  At the default 0.1 the worst arrangement of the seeded
    workload improves at least 5x on FP32_COMPENSATED's (4-10e-6) to below 1e-6,
    99th percentile below 3e-7 (the 374 secondary nodes each keep their FP32 error,
    and the ring sum's own cancellation magnifies what is left: 1e-7 takes a fraction
    near 0.005, at about FP64's cost); at fraction 0 every node is FP64 and the
    result is FP64's up to summation order; the gradients are not refined."""
    import ctypes
    from ccoil_b200 import workloads
    from ccoil_b200 import _lib
    L = ccoil.lib()
    prim_row, sec_row, ppos, spos, py, pz, sy, sz = workloads.pair_config(arrangements=4096, seed=23,
                                                                          coaxial_fraction=0.05)
    prim, sec = coils(ccoil, prim_row, sec_row)
    args = (prim, sec, ppos, spos, py, pz, sy, sz, ccoil.PrecisionFactor(5.0))
    PM = ccoil.PrecisionMode
    for fn, check in ((ccoil.Coil.compute_all_mutual_inductance_arrangements, check_m),
                      (ccoil.Coil.compute_all_force_torque_arrangements, check_ft)):
        b = fn(*args, precision_mode=PM.FP64)
        c = fn(*args, precision_mode=PM.FP32_COMPENSATED)
        r = fn(*args, precision_mode=PM.FP32_REFINED)
        cols = [(0, 1)] if b.ndim == 1 or b.shape[-1] == 1 else [(0, 3), (3, 6)]
        b2, c2, r2 = (np.asarray(x).reshape(len(x), -1) for x in (b, c, r))
        for lo, hi in cols:
            er, ec = rel_err(r2[:, lo:hi], b2[:, lo:hi]), rel_err(c2[:, lo:hi], b2[:, lo:hi])
            print(fn.__name__, lo, "refined max %.1e p99 %.1e (FP32c max %.1e)" % (er.max(), np.quantile(er, 0.99),
                                                                                 ec.max()))
            assert er.max() < 1e-6 and er.max() < ec.max() / 5 and np.quantile(er, 0.99) < 3e-7, \
                (lo, er.max(), ec.max(), np.quantile(er, 0.99))
        default = L.ccoil_refine_fraction()
        try:
            L.ccoil_set_refine_fraction(ctypes.c_double(0.0))
            z = np.asarray(fn(*args, precision_mode=PM.FP32_REFINED)).reshape(len(b), -1)
        finally:
            L.ccoil_set_refine_fraction(ctypes.c_double(default))
        check(z, b2, median=1e-13, worst=1e-11)
    with pytest.raises(ccoil.CCoilError) as ei:
        ccoil.Coil._arrangements(prim, sec, ppos, spos, py, pz, sy, sz, ccoil.PrecisionFactor(5.0),
                                 ccoil.ComputeMethod.GPU, _lib.PAIR_MUTUAL_INDUCTANCE_GRADIENT, PM.FP32_REFINED)
    assert ei.value.status == 4
