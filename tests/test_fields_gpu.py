"""FP64 field kernels (A, B, E, G; single coil and group) against the reference's
double CPU path, through the C-ABI of libccoil_b200.so.

Bar: norm-wise relative error <= 1e-12 per point, except the gradient at points
inside its ill-conditioned band (see conftest.gradient_band), where the bar is
the reference's own reproducibility (1e-5)."""
import numpy as np
import pytest

from conftest import gradient_band, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12
BAND_TOL = 1e-5


def group_from_rows(ccoil, rows, pf):
    coils = ccoil.workloads.coils_from_rows(rows, pf)
    return ccoil.CoilGroup(coils, ccoil.PrecisionFactor(pf))


def check(got, ref, rows, pts, field):
    e = rel_err(got.reshape(len(got), -1), ref)
    if field == 3:
        band = gradient_band(rows, pts)
        assert e[~band].max(initial=0) < TOL, e[~band].max()
        assert e[band].max(initial=0) < BAND_TOL, e[band].max()
    else:
        assert e.max() < TOL, e.max()


@pytest.fixture(scope="module")
def cc(ccoil):
    import ccoil_b200.workloads  # noqa: F401
    return ccoil


def test_single_rect_golden(cc, golden):
    rows, pts = golden["single_coil"], golden["single_points"]
    coil = cc.workloads.coils_from_rows(rows, 5.0)[0]
    fns = [coil.compute_all_A_potential_vectors, coil.compute_all_B_field_vectors,
           coil.compute_all_E_field_vectors, coil.compute_all_B_gradient_matrices]
    for q, name in enumerate("ABEG"):
        check(fns[q](pts), golden["single_" + name], rows, pts, q)


def test_group_test_fields_golden(cc, golden):
    rows, pts = golden["test_fields_coils"], golden["test_fields_points"]
    g = group_from_rows(cc, rows, 4.0)
    fns = [g.compute_all_A_potential_vectors, g.compute_all_B_field_vectors, g.compute_all_E_field_vectors,
           g.compute_all_B_gradient_matrices]
    for q, name in enumerate("ABEG"):
        check(fns[q](pts), golden["test_fields_" + name], rows, pts, q)


@pytest.mark.parametrize("pf", [1, 3, 5, 7, 9])
def test_group_mixed_golden(cc, golden, pf):
    rows, pts = golden["mixed_coils"], golden["mixed_points"]
    g = group_from_rows(cc, rows, float(pf))
    fns = [g.compute_all_A_potential_vectors, g.compute_all_B_field_vectors, g.compute_all_E_field_vectors,
           g.compute_all_B_gradient_matrices]
    for q, name in enumerate("ABEG"):
        check(fns[q](pts), golden["mixed_%s_pf%d" % (name, pf)], rows, pts, q)


def test_comparison_and_rotation_golden(cc, golden):
    c = cc.workloads.coils_from_rows(golden["comp_coil"], 6.0)[0]
    check(c.compute_all_A_potential_vectors(golden["comp_points"]), golden["comp_A"], golden["comp_coil"],
          golden["comp_points"], 0)
    check(c.compute_all_B_field_vectors(golden["comp_points"]), golden["comp_B"], golden["comp_coil"],
          golden["comp_points"], 1)
    c1 = cc.workloads.coils_from_rows(golden["rot_coil1"], 5.0)[0]
    c3 = cc.workloads.coils_from_rows(golden["rot_coil3"], 5.0)[0]
    check(c1.compute_all_B_field_vectors(golden["rot_p1"]), golden["rot_B1"], golden["rot_coil1"],
          golden["rot_p1"], 1)
    check(c3.compute_all_B_field_vectors(golden["rot_p2"]), golden["rot_B3"], golden["rot_coil3"],
          golden["rot_p2"], 1)
    # on-axis gradient (r = 0 branch of CalculateFieldsMethods.cxx:60-65)
    check(c1.compute_all_B_gradient_matrices(golden["rot_p1"]), golden["rot_G1"], golden["rot_coil1"],
          golden["rot_p1"], 3)


@pytest.mark.parametrize("lanes", [1, 2, 4, 8, 16, 32])
def test_lane_splits_agree_with_oracle(cc, oracle, lanes):
    rows = cc.workloads.coil_rows_mixed(8, seed=101)
    pts = cc.workloads.points_cube(333, seed=102)  # ragged: not a multiple of any tile
    group = group_from_rows(cc, rows, 5.0)
    for field in range(4):
        plan = group.plan(field)
        got = plan(pts, lanes=lanes)
        plan.close()
        ref = oracle.group_fields(rows, pts, field, pf=5.0)
        check(got, ref, rows, pts, field)


def test_multi_segment_coils(cc, oracle):
    # high PrecisionFactor: angular tables span many blocks and several staging segments
    rows = np.array([[0.1, 0.0, 0.0, 10, 1.5, 50.0, 0.02, -0.01, 0.03, 0.4, 1.1],
                     [0.08, 0.0, 0.05, 30, -2.0, 50.0, -0.1, 0.05, 0.0, 1.2, 0.3]])
    pts = cc.workloads.points_cube(40, seed=7, half=0.4)
    for pf in (10.0, 12.0):
        group = group_from_rows(cc, rows, pf)
        for field in (0, 1, 3):
            plan = group.plan(field)
            got = plan(pts)
            plan.close()
            check(got, oracle.group_fields(rows, pts, field, pf=pf), rows, pts, field)


def test_custom_precision_arguments(cc, oracle):
    # user-given PrecisionArguments, including several length nodes on a slow-method coil
    row = np.array([0.12, 0.03, 0.0, 50, 1.0, 50.0, 0.0, 0.0, 0.0, 0.3, 0.2])
    coil = cc.workloads.coils_from_rows(row, 5.0)[0]
    pts = cc.workloads.points_cube(64, seed=9, half=0.5)
    for prec in [(1, 1, 1, 12, 5, 3), (3, 2, 2, 17, 9, 4), (2, 1, 1, 100, 1, 1)]:
        pa = cc.PrecisionArguments(*prec)
        for field, fn in [(0, coil.compute_all_A_potential_vectors), (1, coil.compute_all_B_field_vectors),
                          (3, coil.compute_all_B_gradient_matrices)]:
            got = fn(pts, used_precision=pa)
            check(got, oracle.coil_fields(row, pts, field, prec=np.array(prec)), row, pts, field)


def test_edge_cases(cc):
    coil = cc.Coil(0.1, 0.1, 0.1, 100)
    assert coil.compute_all_B_field_vectors(np.zeros((0, 3))).shape == (0, 3)
    one = coil.compute_all_B_field_vectors(np.array([[0.3, 0.0, 0.0]]))
    assert one.shape == (1, 3) and np.all(np.isfinite(one))
    g = cc.CoilGroup([])
    assert np.array_equal(g.compute_all_B_field_vectors(np.ones((5, 3))), np.zeros((5, 3)))


def test_device_memory_path_and_determinism(cc):
    import torch
    rows = cc.workloads.coil_rows_mixed(6, seed=55)
    pts = cc.workloads.points_cube(1000, seed=56)
    group = group_from_rows(cc, rows, 5.0)
    timeouts = cc.lib().ccoil_timeout_count()
    plan = group.plan(1)
    host = plan(pts)
    host2 = plan(pts)
    dev = plan(torch.from_numpy(pts).cuda())
    torch.cuda.synchronize()
    plan.close()
    assert np.array_equal(host, host2)
    assert np.array_equal(host, dev.cpu().numpy())
    assert cc.lib().ccoil_timeout_count() == timeouts  # no bounded wait ran out in these calls
