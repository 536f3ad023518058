"""FP32-compensated field path against the FP64 path (which reproduces the
reference's double CPU results to 1e-12, see test_fields_gpu.py).

Error is the norm-wise relative error per point.  One coil at a time, the
closed-form mirror differences keep the error flat with distance
(test_single_coil_far_field: max below 1e-6 out to 40 coil radii, where
subtracting the mirror nodes lost up to 2e-5).  A group adds the cancellation
between coils of opposite current, which multiplies the per-coil error by
sum |F_c| / |sum F_c| (up to ~100 on the benchmark workload).  The 16-coil
group workload measures median 2.4-5.0e-8, 99th percentile 1.1-1.8e-7 and
max 4.1-6.0e-7 for A, B and E; its bars sit 2-3x above that.  Near-field (point, coil) pairs
are evaluated with the FP64 integrands and must match the FP64 path exactly up
to summation order; the gradient is compared outside its ill-conditioned band,
where the FP64 reference form itself carries ~1e-7 rounding noise."""
import numpy as np
import pytest

from conftest import gradient_band, rel_err

pytestmark = pytest.mark.gpu


def modes(cc):
    return cc.PrecisionMode.FP64, cc.PrecisionMode.FP32_COMPENSATED


def evaluate(cc, coils, pts, field, mode, lanes=0):
    plan = cc.FieldPlan([c.struct() for c in coils], field, mode)
    try:
        return plan(pts, lanes=lanes)
    finally:
        plan.close()


@pytest.mark.parametrize("field", [0, 1, 2, 3])
def test_group_workload_error(ccoil, field):
    from ccoil_b200 import workloads
    rows = workloads.coil_rows_mixed(16, seed=77)
    pts = workloads.points_cube(8192, seed=78)
    coils = workloads.coils_from_rows(rows, 5.0)
    f64, f32 = (evaluate(ccoil, coils, pts, field, m) for m in modes(ccoil))
    e = rel_err(f32, f64)
    if field == 3:
        e = e[~gradient_band(rows, pts)]
    print(field, "median %.1e p99 %.1e max %.1e" % (np.median(e), np.quantile(e, 0.99), e.max()))
    assert np.median(e) < 1e-7, np.median(e)
    assert np.quantile(e, 0.99) < 4e-7, np.quantile(e, 0.99)
    assert e.max() < 2e-6, e.max()


def test_single_rect_workload_error(ccoil):
    from ccoil_b200 import workloads
    rows, pts = workloads.single_rect_config(points=16384, seed=3)
    coils = workloads.coils_from_rows(rows, 5.0)
    for field in (0, 1, 3):
        f64, f32 = (evaluate(ccoil, coils, pts, field, m) for m in modes(ccoil))
        e = rel_err(f32, f64)
        if field == 3:
            e = e[~gradient_band(rows, pts)]
        assert np.median(e) < 3e-7 and e.max() < 1e-5, (field, np.median(e), e.max())


@pytest.mark.parametrize("row", [[0.1, 0.05, 0.08, 100, 1.0, 50.0, 0, 0, 0, 0.4, 1.0],   # RECTANGULAR
                                 [0.1, 0.0, 0.08, 100, 1.0, 50.0, 0, 0, 0, 0.4, 1.0],    # THIN
                                 [0.1, 0.05, 0.0, 100, 1.0, 50.0, 0, 0, 0, 0.4, 1.0],    # FLAT
                                 [0.1, 0.0, 0.0, 100, 1.0, 50.0, 0, 0, 0, 0.4, 1.0]])    # FILAMENT
def test_single_coil_far_field(ccoil, row):
    """One coil, points at 1.5 to 40 coil radii in random directions: A and B within
    1e-6 of FP64 at every point (the far-field azimuthal cancellation is removed by
    the closed-form mirror differences), median below 1e-7."""
    from ccoil_b200 import workloads
    g = np.random.default_rng(13)
    n = 8192
    d = 0.1 * np.exp(g.uniform(np.log(1.5), np.log(40.0), n))
    v = g.normal(size=(n, 3))
    pts = v / np.linalg.norm(v, axis=1, keepdims=True) * d[:, None]
    rows = np.array([row], dtype=float)
    coils = workloads.coils_from_rows(rows, 5.0)
    for field in (0, 1):
        f64, f32 = (evaluate(ccoil, coils, pts, field, m) for m in modes(ccoil))
        e = rel_err(f32, f64)
        print(row[:3], field, "median %.1e p99 %.1e max %.1e" % (np.median(e), np.quantile(e, 0.99), e.max()))
        assert np.median(e) < 1e-7 and e.max() < 1e-6, (row[:3], field, np.median(e), e.max())


def test_near_field_pairs_use_fp64(ccoil):
    # points inside the winding of a RECTANGULAR coil: every pair is near-field
    coil = ccoil.Coil(0.1, 0.05, 0.08, 200)
    rng = np.random.default_rng(5)
    r = rng.uniform(0.1, 0.15, 2000)
    ph = rng.uniform(0, 2 * np.pi, 2000)
    z = rng.uniform(-0.04, 0.04, 2000)
    pts = np.stack([r * np.cos(ph), r * np.sin(ph), z], axis=1)
    for field in (0, 1, 3):
        f64, f32 = (evaluate(ccoil, [coil], pts, field, m) for m in modes(ccoil))
        assert rel_err(f32, f64).max() < 1e-13


def test_work_list_overflow_falls_back_in_place(ccoil):
    # 5 coincident coils x 2^20 points inside the winding = 5.2 Mi near-field pairs,
    # more than the 4 Mi-entry work list: the rest is integrated in FP64 in place
    coils = [ccoil.Coil(0.1, 0.02, 0.02, 10, precision_factor=1.0) for _ in range(5)]
    n = 1 << 20
    rng = np.random.default_rng(9)
    r = rng.uniform(0.1, 0.12, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    z = rng.uniform(-0.01, 0.01, n)
    pts = np.stack([r * np.cos(ph), r * np.sin(ph), z], axis=1)
    f64, f32 = (evaluate(ccoil, coils, pts, 1, m) for m in modes(ccoil))
    # inside the winding the 5 contributions nearly cancel; their FP64 atomic
    # additions in either order agree to rounding level
    assert rel_err(f32, f64).max() < 1e-12


@pytest.mark.parametrize("lanes", [1, 2, 4, 8, 16, 32])
def test_lane_splits(ccoil, lanes):
    from ccoil_b200 import workloads
    rows = workloads.coil_rows_mixed(8, seed=11)
    pts = workloads.points_cube(777, seed=12)
    coils = workloads.coils_from_rows(rows, 5.0)
    for field in (0, 1, 3):
        f64 = evaluate(ccoil, coils, pts, field, ccoil.PrecisionMode.FP64)
        f32 = evaluate(ccoil, coils, pts, field, ccoil.PrecisionMode.FP32_COMPENSATED, lanes)
        e = rel_err(f32, f64)
        if field == 3:
            e = e[~gradient_band(rows, pts)]
        assert np.median(e) < 3e-7 and e.max() < 1e-5, (field, lanes, e.max())


def test_repeatable(ccoil):
    from ccoil_b200 import workloads
    rows = workloads.coil_rows_mixed(8, seed=21)
    pts = workloads.points_cube(4096, seed=22, half=0.6)
    coils = workloads.coils_from_rows(rows, 5.0)
    a = evaluate(ccoil, coils, pts, 1, ccoil.PrecisionMode.FP32_COMPENSATED)
    b = evaluate(ccoil, coils, pts, 1, ccoil.PrecisionMode.FP32_COMPENSATED)
    # the near-field pass adds with FP64 atomics: run-to-run differences stay at rounding level
    assert rel_err(a, b).max() < 1e-14


@pytest.mark.parametrize("pf", [1.0, 3.0, 7.0])
def test_gradient_across_precision_factors(ccoil, pf):
    """The FP32 gradient integrands equal the reference's node by node, so the two
    paths agree at every PrecisionFactor, including the coarse ones where a
    different but equivalent integrand would differ by its quadrature error."""
    from ccoil_b200 import workloads
    rows = workloads.coil_rows_mixed(16, seed=91)
    pts = workloads.points_cube(8192, seed=92)
    coils = workloads.coils_from_rows(rows, pf)
    f64, f32 = (evaluate(ccoil, coils, pts, 3, m) for m in modes(ccoil))
    e = rel_err(f32, f64)[~gradient_band(rows, pts)]
    assert np.median(e) < 1e-7 and e.max() < 1e-5, (pf, np.median(e), e.max())


@pytest.mark.parametrize("angular", [(1, 3), (1, 7), (3, 11), (26, 99), (27, 99)])
def test_mirror_pair_tables(ccoil, angular):
    """The FP32 path evaluates angular nodes in mirror pairs (phi, pi - phi).  Odd
    node counts leave a middle node of its own (3, 7, 33, 2673 nodes), and long
    tables span several segments that must be cut between pairs (2574 and 2673
    nodes): every coil type and field still agrees with the FP64 path.  A node
    left out, counted twice or weighted wrongly shows up at 1e-3 or more; the
    bars sit below that but above the rounding of tables this short, where the
    far-field cancellation rests on one or two pairs instead of averaging over
    many (single-pair rounding reaches ~2e-5 at 3 nodes)."""
    from ccoil_b200 import workloads
    blocks, increments = angular
    prec = ccoil.PrecisionArguments(blocks, 1, 1, increments, 6, 5)
    # {R, a, b, N, I, f, x, y, z, yAngle, zAngle}: RECTANGULAR, THIN, FLAT, FILAMENT
    rows = np.array([[0.1, 0.05, 0.08, 100, 1.0, 50.0, 0.05, -0.02, 0.1, 0.7, 0.0],
                     [0.12, 0.0, 0.1, 100, 1.0, 50.0, 0.0, 0.0, 0.0, 0.0, 1.1],
                     [0.08, 0.04, 0.0, 100, 1.0, 50.0, 0.0, 0.0, 0.0, 2.0, 0.0],
                     [0.1, 0.0, 0.0, 100, 1.0, 50.0, -0.1, 0.0, 0.05, 0.0, 0.0]])
    pts = workloads.points_cube(2048, seed=31, half=0.5)
    for row, coil in zip(rows, workloads.coils_from_rows(rows, 5.0)):
        for field in (0, 1, 3):
            res = []
            for mode in modes(ccoil):
                plan = ccoil.FieldPlan([coil.struct(prec)], field, mode)
                try:
                    res.append(plan(pts))
                finally:
                    plan.close()
            e = rel_err(res[1], res[0])
            if field == 3:
                e = e[~gradient_band(row[None, :], pts)]
            assert np.median(e) < 1e-6 and e.max() < 1e-4, (angular, row[:3], field, np.median(e), e.max())


def test_refined_mode(ccoil):
    """FP32_REFINED replaces by its FP64 value every (point, coil) contribution whose
    norm exceeds the set fraction of the point's total.  With fraction 0 every pair
    is FP64: the field and the gradient are the FP64 path's up to summation order
    (the field's reciprocal square roots come from Newton steps: 1e-14); the vector
    potential (and E) takes a cancellation-free FP64 form in the refinement pass,
    which differs from the FP64 path's operation sequence (the reference's, whose
    own cancellation errors reach ~2e-10 on single pairs) by at most 1e-9, median
    below 1e-13; at the default
    0.1 the maximum error of A, B and E falls below 1e-7 on the 16-coil group
    (from the FP32 path's 4-6e-7), with part of the pairs refined; the gradient
    stays within its FP32 bars.  Fractions must be finite and
    >= 0."""
    import ctypes
    from ccoil_b200 import workloads
    L = ccoil.lib()
    default = L.ccoil_refine_fraction()
    assert default == 0.1
    rows = workloads.coil_rows_mixed(16, seed=77)
    pts = workloads.points_cube(8192, seed=78)
    coils = workloads.coils_from_rows(rows, 5.0)
    near = np.zeros(len(pts), dtype=bool)
    try:
        for field in (0, 1, 2, 3):
            f64 = evaluate(ccoil, coils, pts, field, ccoil.PrecisionMode.FP64)
            f32 = evaluate(ccoil, coils, pts, field, ccoil.PrecisionMode.FP32_COMPENSATED)
            L.ccoil_set_refine_fraction(ctypes.c_double(0.0))
            plan = ccoil.FieldPlan([c.struct() for c in coils], field, ccoil.PrecisionMode.FP32_REFINED)
            got = plan(pts)
            n_all = plan.refined_pairs()
            plan.close()
            assert 0.9 * len(pts) * len(coils) <= n_all <= len(pts) * len(coils), (field, n_all)
            e0 = rel_err(got, f64)
            print(field, "fraction 0: median %.1e max %.1e" % (np.median(e0), e0.max()))
            bar0 = {0: 1e-9, 1: 1e-13, 2: 1e-9, 3: 1e-13}[field]
            assert np.median(e0) < 1e-13 and e0.max() < bar0, (field, np.median(e0), e0.max())
            L.ccoil_set_refine_fraction(ctypes.c_double(default))
            plan = ccoil.FieldPlan([c.struct() for c in coils], field, ccoil.PrecisionMode.FP32_REFINED)
            got = plan(pts)
            n = plan.refined_pairs()
            plan.close()
            # with 16 coils each coil's share of a point's field is large: about
            # half of the pairs exceed 0.1 of the total (12 % on the 128-coil group)
            assert 0 < n < 0.7 * len(pts) * len(coils), (field, n)
            keep = ~gradient_band(rows, pts) if field == 3 else ~near
            e, e32 = rel_err(got, f64)[keep], rel_err(f32, f64)[keep]
            print(field, "refined pairs %.3f, max %.1e (FP32c %.1e), p99 %.1e" %
                  (n / (len(pts) * len(coils)), e.max(), e32.max(), np.quantile(e, 0.99)))
            if field == 3:
                assert np.median(e) < 1e-7 and e.max() < 1e-6, (field, e.max())
            else:
                assert e.max() < 1e-7 and e.max() < e32.max() / 3, (field, e.max(), e32.max())
    finally:
        L.ccoil_set_refine_fraction(ctypes.c_double(default))
    assert L.ccoil_set_refine_fraction(ctypes.c_double(-0.5)) == 1
    assert L.ccoil_set_refine_fraction(ctypes.c_double(float("nan"))) == 1
    assert L.ccoil_refine_fraction() == default


def test_refined_mode_in_chunks(ccoil):
    """FP32_REFINED stores every contribution of the points it evaluates at once: a
    gradient call whose contributions exceed 4 GiB (128 coils x 500,000 points x 9
    doubles) runs in several chunks and matches FP64 like a single chunk does."""
    from ccoil_b200 import workloads
    rows = workloads.coil_rows_mixed(128, seed=91)
    pts = workloads.points_cube(500000, seed=92)
    coils = workloads.coils_from_rows(rows, 3.0)
    f64 = evaluate(ccoil, coils, pts, 3, ccoil.PrecisionMode.FP64)
    plan = ccoil.FieldPlan([c.struct() for c in coils], 3, ccoil.PrecisionMode.FP32_REFINED)
    got = plan(pts)
    n = plan.refined_pairs()
    plan.close()
    e = rel_err(got, f64)[~gradient_band(rows, pts)]
    assert 0 < n < 0.5 * len(pts) * len(coils), n
    assert np.median(e) < 1e-9 and e.max() < 1e-6, (np.median(e), e.max())


def test_point_ordering(ccoil):
    """FP32 plans of at least 16,384 points evaluate them in Morton order and scatter
    the results back: every result lands at its caller's index (against FP64, which
    keeps the caller's order, at the group bars), ordered and unordered evaluation
    agree to FP32 rounding, the ordered results repeat exactly, and points with a
    non-finite coordinate give non-finite results at their own index only.  Ordering
    applies to FP32_REFINED too."""
    import ctypes
    from ccoil_b200 import workloads
    L = ccoil.lib()
    assert L.ccoil_point_ordering() == 1
    rows = workloads.coil_rows_mixed(16, seed=77)
    coils = workloads.coils_from_rows(rows, 5.0)
    pts = workloads.points_cube(40000, seed=31)
    bad = [5, 17000, 39999]
    pts[bad[0], 0] = np.nan
    pts[bad[1], 2] = np.inf
    pts[bad[2], 1] = -np.inf
    good = np.ones(len(pts), dtype=bool)
    good[bad] = False
    try:
        for field in (0, 1, 3):
            f64 = evaluate(ccoil, coils, pts, field, ccoil.PrecisionMode.FP64)
            on = evaluate(ccoil, coils, pts, field, ccoil.PrecisionMode.FP32_COMPENSATED)
            again = evaluate(ccoil, coils, pts, field, ccoil.PrecisionMode.FP32_COMPENSATED)
            refined = evaluate(ccoil, coils, pts, field, ccoil.PrecisionMode.FP32_REFINED)
            L.ccoil_set_point_ordering(0)
            off = evaluate(ccoil, coils, pts, field, ccoil.PrecisionMode.FP32_COMPENSATED)
            L.ccoil_set_point_ordering(1)
            assert not np.isfinite(on[bad]).any() and not np.isfinite(off[bad]).any(), field
            assert np.array_equal(on, again, equal_nan=True), field
            keep = good if field != 3 else good & ~gradient_band(rows, pts)
            for got in (on, refined):
                e = rel_err(got[keep], f64[keep])
                assert np.median(e) < 1e-7 and e.max() < 2e-6, (field, np.median(e), e.max())
            assert rel_err(on[good], off[good]).max() < 2e-6, field
    finally:
        L.ccoil_set_point_ordering(1)


def test_refined_group128_below_1e7(ccoil):
    """The bench's 128-coil group (PF 5) on 2^18 points of another seed: FP32_REFINED at
    its default fraction keeps A, B and E within 1e-7 of FP64 away from windings,
    where FP32_COMPENSATED reaches 1e-6 and more."""
    import torch
    from ccoil_b200 import workloads
    from conftest import winding_near
    rows, _ = workloads.group_config(coils=128, points=1)
    coils = workloads.coils_from_rows(rows, 5.0)
    pts = workloads.points_cube(1 << 18, seed=4242)
    away = ~winding_near(rows, pts)
    for field in (0, 1, 2):
        f64 = evaluate(ccoil, coils, pts, field, ccoil.PrecisionMode.FP64)
        f32 = evaluate(ccoil, coils, pts, field, ccoil.PrecisionMode.FP32_COMPENSATED)
        ref = evaluate(ccoil, coils, pts, field, ccoil.PrecisionMode.FP32_REFINED)
        e, e32 = rel_err(ref, f64)[away], rel_err(f32, f64)[away]
        print(field, "refined max %.1e p99 %.1e (FP32c max %.1e)" % (e.max(), np.quantile(e, 0.99), e32.max()))
        assert e.max() < 1e-7, (field, e.max())
