"""Mutual inductance and force/torque arrangements (FP64) against the reference's
CPU general-case results: golden vectors from the reference and the oracle on
seeded arrangements.  Bar: 1e-12 relative (M), norm-wise per force and torque."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rows_to_coil(cc, row, pf=5.0):
    from ccoil_b200 import workloads
    return workloads.coils_from_rows(row, pf)[0]


def check_ft(got, ref):
    got = np.atleast_2d(got)
    ref = np.atleast_2d(ref)
    assert rel_err(got[:, :3], ref[:, :3], floor_frac=0).max() < TOL
    assert rel_err(got[:, 3:], ref[:, 3:], floor_frac=1e-6).max() < TOL


def test_coil_arrangements_golden(ccoil, golden):
    prim = rows_to_coil(ccoil, golden["arr_prim"])
    sec = rows_to_coil(ccoil, golden["arr_sec"])
    py, pz, sy, sz = golden["arr_angles"]
    args = (golden["arr_prim_pos"], golden["arr_sec_pos"], py, pz, sy, sz, ccoil.PrecisionFactor(5.0))
    m = ccoil.Coil.compute_all_mutual_inductance_arrangements(prim, sec, *args)
    assert np.max(np.abs(m - golden["arr_M"]) / np.abs(golden["arr_M"])) < TOL
    ft = ccoil.Coil.compute_all_force_torque_arrangements(prim, sec, *args)
    check_ft(ft, golden["arr_FT"])


def test_pair_configuration_golden(ccoil, golden):
    prim = rows_to_coil(ccoil, golden["pairs_prim"])
    sec = rows_to_coil(ccoil, golden["pairs_sec"])
    py, pz, sy, sz = golden["pairs_angles"]
    args = (golden["pairs_prim_pos"], golden["pairs_sec_pos"], py, pz, sy, sz, ccoil.PrecisionFactor(5.0))
    m = ccoil.Coil.compute_all_mutual_inductance_arrangements(prim, sec, *args)
    assert np.max(np.abs(m - golden["pairs_M"]) / np.max(np.abs(golden["pairs_M"]))) < TOL
    ft = ccoil.Coil.compute_all_force_torque_arrangements(prim, sec, *args)
    check_ft(ft, golden["pairs_FT"])


def test_group_arrangements_golden(ccoil, golden):
    from ccoil_b200 import workloads
    coils = workloads.coils_from_rows(golden["garr_coils"], 5.0)
    group = ccoil.CoilGroup(coils, ccoil.PrecisionFactor(5.0))
    sy, sz = golden["garr_angles"]
    # the secondary is member 0: the group leaves it out of its own sum
    m = group.compute_all_mutual_inductance_arrangements(group[0], golden["garr_sec_pos"], sy, sz,
                                                         ccoil.PrecisionFactor(4.0))
    assert np.max(np.abs(m - golden["garr_M"]) / np.abs(golden["garr_M"])) < TOL
    ft = group.compute_all_force_torque_arrangements(group[0], golden["garr_sec_pos"], sy, sz,
                                                     ccoil.PrecisionFactor(4.0))
    check_ft(ft, golden["garr_FT"])


def test_parallel_axes_golden(ccoil, golden, oracle):
    if "pa_M" not in golden:
        pytest.skip("no parallel-axes fixture")
    done = 0
    for p, s, m in zip(golden["pa_prim"], golden["pa_sec"], golden["pa_M"]):
        # coaxial rows take the z-axis formulas, as in the reference
        prim, sec = rows_to_coil(ccoil, p), rows_to_coil(ccoil, s)
        # coaxial rows: the reference's -ffast-math build of its closed-form z-axis
        # formula differs from strict evaluation up to ~5e-11 (tests/test_zaxis_gpu.py)
        tol = 1e-10 if oracle.z_axis_case(p, s) else TOL
        for j, pf in enumerate((3.0, 5.0)):
            got = ccoil.Coil.compute_mutual_inductance(prim, sec, ccoil.PrecisionFactor(pf))
            assert abs(got - m[j]) <= tol * abs(m[j]), (p, s, pf, got, m[j])
        done += 1
    assert done > 10


def test_seeded_arrangements_against_oracle(ccoil, oracle):
    from ccoil_b200 import workloads
    prim_row, sec_row, ppos, spos, py, pz, sy, sz = workloads.pair_config(arrangements=12, seed=99,
                                                                          coaxial_fraction=0.25)
    prim, sec = rows_to_coil(ccoil, prim_row), rows_to_coil(ccoil, sec_row)
    args = (ppos, spos, py, pz, sy, sz, ccoil.PrecisionFactor(4.0))
    m = ccoil.Coil.compute_all_mutual_inductance_arrangements(prim, sec, *args)
    ft = ccoil.Coil.compute_all_force_torque_arrangements(prim, sec, *args)
    for i in range(len(py)):
        p = prim_row.copy(); p[6:9] = ppos[i]; p[9] = py[i]; p[10] = pz[i]
        s = sec_row.copy(); s[6:9] = spos[i]; s[9] = sy[i]; s[10] = sz[i]
        mo = oracle.mutual_inductance(p, s, pf=4.0)
        assert abs(m[i] - mo) <= TOL * abs(mo), (i, m[i], mo)
        check_ft(ft[i], oracle.force_torque(p, s, pf=4.0))


def test_empty_and_errors(ccoil):
    prim = ccoil.Coil(0.1, 0.05, 0.1, 100)
    sec = ccoil.Coil(0.05, 0.0, 0.1, 50)
    e = np.zeros((0, 3))
    z = np.zeros(0)
    assert ccoil.Coil.compute_all_mutual_inductance_arrangements(prim, sec, e, e, z, z, z, z).shape == (0,)
    with pytest.raises(ValueError):
        ccoil.Coil.compute_all_mutual_inductance_arrangements(prim, sec, np.zeros((2, 3)), np.zeros((3, 3)),
                                                              np.zeros(2), np.zeros(2), np.zeros(3), np.zeros(3))
