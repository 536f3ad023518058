"""Coaxial pairs: the arrangement kernels' z-axis pass against the reference's
z-axis formulas, for every coil-type combination, coil-level and group-level
arrangements.

Bars: 1e-12 relative against the oracle (the strict restatement, evaluated in
the reference's operation order) and 1e-10 against the golden vectors of the
compiled reference.  The closed-form fast formulas cancel between their eight
length-limit terms, and the reference is built with -Ofast -ffast-math: the
restatement and the reference's own build differ by up to 4.7e-11 there
(tests/test_oracle.py pins that difference).  Torque is exactly zero and the
force exactly axial for coaxial pairs."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12
TOL_REF = 1e-10


def rows_at(golden, c, i):
    p = golden["zax_prim"][c].copy()
    s = golden["zax_sec"][c].copy()
    py, pz, sy, sz = golden["zax_angles"][c][:, i]
    p[6:9], p[9], p[10] = golden["zax_prim_pos"][c][i], py, pz
    s[6:9], s[9], s[10] = golden["zax_sec_pos"][c][i], sy, sz
    return p, s


def coil(ccoil, row, pf):
    from ccoil_b200 import workloads
    return workloads.coils_from_rows(row, pf)[0]


@pytest.mark.parametrize("pf,key", [(3.0, "zax_M_pf3"), (5.0, "zax_M_pf5")])
def test_coaxial_mutual_inductance(ccoil, golden, oracle, pf, key):
    worst = 0.0
    for c in range(len(golden["zax_prim"])):
        prim = coil(ccoil, golden["zax_prim"][c], pf)
        sec = coil(ccoil, golden["zax_sec"][c], pf)
        py, pz, sy, sz = golden["zax_angles"][c]
        m = ccoil.Coil.compute_all_mutual_inductance_arrangements(
            prim, sec, golden["zax_prim_pos"][c], golden["zax_sec_pos"][c], py, pz, sy, sz, ccoil.PrecisionFactor(pf))
        ref = golden[key][c]
        err = np.abs(m - ref) / np.abs(ref)
        assert err.max() < TOL_REF, (c, err, m, ref)
        for i in range(len(m)):
            o = oracle.mutual_inductance(*rows_at(golden, c, i), pf=pf)
            worst = max(worst, abs(m[i] - o) / abs(o))
    print("max relative difference from the oracle: %.2e" % worst)
    assert worst < TOL, worst


def test_coaxial_force_torque(ccoil, golden, oracle):
    worst = 0.0
    for c in range(len(golden["zax_prim"])):
        prim = coil(ccoil, golden["zax_prim"][c], 5.0)
        sec = coil(ccoil, golden["zax_sec"][c], 5.0)
        py, pz, sy, sz = golden["zax_angles"][c]
        ft = ccoil.Coil.compute_all_force_torque_arrangements(
            prim, sec, golden["zax_prim_pos"][c], golden["zax_sec_pos"][c], py, pz, sy, sz, ccoil.PrecisionFactor(5.0))
        ref = golden["zax_FT_pf5"][c]
        # coaxial arrangements (the first four): axial force, no torque
        assert np.all(ft[:4, [0, 1, 3, 4, 5]] == 0.0), (c, ft[:4])
        assert rel_err(ft[:, :3], ref[:, :3], floor_frac=0).max() < TOL_REF, (c, ft[:, :3], ref[:, :3])
        assert rel_err(ft[4:, 3:], ref[4:, 3:], floor_frac=1e-6).max() < TOL, (c, ft[4:, 3:], ref[4:, 3:])
        o = np.array([oracle.force_torque(*rows_at(golden, c, i), pf=5.0) for i in range(len(ft))])
        worst = max(worst, rel_err(ft[:, :3], o[:, :3], floor_frac=0).max())
    print("max relative difference from the oracle: %.2e" % worst)
    assert worst < TOL, worst


def test_coaxial_group(ccoil, golden):
    from ccoil_b200 import workloads
    group = ccoil.CoilGroup(workloads.coils_from_rows(golden["zgrp_coils"], 4.0), ccoil.PrecisionFactor(4.0))
    sec = coil(ccoil, golden["zgrp_sec"], 4.0)
    sy, sz = golden["zgrp_angles"]
    m = group.compute_all_mutual_inductance_arrangements(sec, golden["zgrp_sec_pos"], sy, sz,
                                                         ccoil.PrecisionFactor(4.0))
    assert np.max(np.abs(m - golden["zgrp_M"]) / np.abs(golden["zgrp_M"])) < TOL_REF
    ft = group.compute_all_force_torque_arrangements(sec, golden["zgrp_sec_pos"], sy, sz, ccoil.PrecisionFactor(4.0))
    assert rel_err(ft[:, :3], golden["zgrp_FT"][:, :3], floor_frac=0).max() < TOL_REF
    assert rel_err(ft[5:, 3:], golden["zgrp_FT"][5:, 3:], floor_frac=1e-6).max() < TOL_REF


def test_coaxial_fp32c_takes_z_axis_pass(ccoil, golden):
    """In FP32-compensated mode the coaxial pairs still take the FP64 z-axis pass."""
    c = 0
    prim = coil(ccoil, golden["zax_prim"][c], 5.0)
    sec = coil(ccoil, golden["zax_sec"][c], 5.0)
    py, pz, sy, sz = golden["zax_angles"][c]
    m = ccoil.Coil.compute_all_mutual_inductance_arrangements(
        prim, sec, golden["zax_prim_pos"][c][:4], golden["zax_sec_pos"][c][:4], py[:4], pz[:4], sy[:4], sz[:4],
        ccoil.PrecisionFactor(5.0), precision_mode=ccoil.PrecisionMode.FP32_COMPENSATED)
    assert np.max(np.abs(m - golden["zax_M_pf5"][c][:4]) / np.abs(golden["zax_M_pf5"][c][:4])) < TOL_REF
