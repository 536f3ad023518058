"""The oracle (C restatement) pinned against the reference's own outputs:
the committed golden vectors, and the compiled reference where it is present."""
import numpy as np
import pytest

from conftest import gradient_band, rel_err

FIELD_TOL = 1e-12  # relative, oracle vs reference, away from the gradient's ill-conditioned band


def test_precision_arguments_golden(oracle, golden):
    coils, pfs = golden["prec_coils"], golden["prec_pf"]
    for c, pf, cpu, gpu in zip(coils, pfs, golden["prec_cpu"], golden["prec_gpu"]):
        assert list(oracle.precision_args(c, pf, 0)) == list(cpu)
        assert list(oracle.precision_args(c, pf, 80)) == list(gpu)


def test_pair_arguments_golden(oracle, golden):
    for p, s, pf, cpu, gpu in zip(golden["pprec_prim"], golden["pprec_sec"], golden["pprec_pf"],
                                  golden["pprec_cpu"], golden["pprec_gpu"]):
        assert list(oracle.pair_args(p, s, pf)) == list(cpu)
        assert list(oracle.pair_args(p, s, pf, gpu_cap=80, pure_gpu=True)) == list(gpu)


def test_fields_golden_test_fields(oracle, golden):
    coils, pts = golden["test_fields_coils"], golden["test_fields_points"]
    for q, name in enumerate("ABEG"):
        e = rel_err(oracle.group_fields(coils, pts, q, pf=4.0), golden["test_fields_" + name])
        assert e.max() < FIELD_TOL, (name, e.max())


def test_fields_golden_single_rect(oracle, golden):
    c, pts = golden["single_coil"][0], golden["single_points"]
    for q, name in enumerate("ABE"):
        e = rel_err(oracle.coil_fields(c, pts, q, pf=5.0), golden["single_" + name])
        assert e.max() < FIELD_TOL, (name, e.max())
    # the gradient's RZ term has a removable singularity where the point's radius
    # lies inside the winding's radial range; there the reference's own rounding
    # (it is built with -ffast-math) sets the floor
    e = rel_err(oracle.coil_fields(c, pts, 3, pf=5.0), golden["single_G"])
    band = gradient_band(c, pts)
    assert e[~band].max() < FIELD_TOL
    assert e[band].max() < 1e-5


def test_fields_golden_mixed(oracle, golden):
    coils, pts = golden["mixed_coils"], golden["mixed_points"]
    band = gradient_band(coils, pts)
    for pf in (1, 3, 5, 7, 9):
        for q, name in enumerate("ABE"):
            e = rel_err(oracle.group_fields(coils, pts, q, pf=float(pf)), golden["mixed_%s_pf%d" % (name, pf)])
            assert e.max() < FIELD_TOL, (name, pf, e.max())
        e = rel_err(oracle.group_fields(coils, pts, 3, pf=float(pf)), golden["mixed_G_pf%d" % pf])
        assert e[~band].max() < FIELD_TOL and e[band].max() < 1e-5, (pf, e[~band].max(), e[band].max())


def test_fields_golden_comp_and_rotation(oracle, golden):
    e = rel_err(oracle.coil_fields(golden["comp_coil"], golden["comp_points"], 0, pf=6.0), golden["comp_A"])
    assert e.max() < FIELD_TOL
    e = rel_err(oracle.coil_fields(golden["comp_coil"], golden["comp_points"], 1, pf=6.0), golden["comp_B"])
    assert e.max() < FIELD_TOL
    e = rel_err(oracle.coil_fields(golden["rot_coil1"], golden["rot_p1"], 1), golden["rot_B1"])
    assert e.max() < FIELD_TOL
    e = rel_err(oracle.coil_fields(golden["rot_coil3"], golden["rot_p2"], 1), golden["rot_B3"])
    assert e.max() < FIELD_TOL
    e = rel_err(oracle.coil_fields(golden["rot_coil1"], golden["rot_p1"], 3), golden["rot_G1"], floor=1e-30)
    assert e.max() < FIELD_TOL


def test_arrangements_golden(oracle, golden):
    prim, sec = golden["arr_prim"], golden["arr_sec"]
    ppos, spos = golden["arr_prim_pos"], golden["arr_sec_pos"]
    py, pz, sy, sz = golden["arr_angles"]
    for i in range(len(py)):
        p = prim.copy(); p[6:9] = ppos[i]; p[9] = py[i]; p[10] = pz[i]
        s = sec.copy(); s[6:9] = spos[i]; s[9] = sy[i]; s[10] = sz[i]
        m = oracle.mutual_inductance(p, s, pf=5.0)
        assert abs(m - golden["arr_M"][i]) <= 1e-12 * abs(golden["arr_M"][i])
        ft = oracle.force_torque(p, s, pf=5.0)
        assert rel_err(ft[None, :3], golden["arr_FT"][i:i + 1, :3]).max() < 1e-12
        assert rel_err(ft[None, 3:], golden["arr_FT"][i:i + 1, 3:]).max() < 1e-12


def test_parallel_axes_golden(oracle, golden):
    if "pa_M" not in golden:
        pytest.skip("no parallel-axes fixture")
    for p, s, m in zip(golden["pa_prim"], golden["pa_sec"], golden["pa_M"]):
        if oracle.z_axis_case(p, s):
            continue
        for j, pf in enumerate((3.0, 5.0)):
            assert abs(oracle.mutual_inductance(p, s, pf=pf) - m[j]) <= 1e-12 * abs(m[j])


def test_legendre_against_reference(oracle, reference):
    for n in range(1, 101):
        p1, w1 = oracle.legendre(n)
        p2, w2 = reference.legendre(n)
        assert np.max(np.abs(p1 - p2)) <= 4.5e-16
        assert np.max(np.abs(w1 - w2) / w2) <= 1e-15


def test_random_precision_against_reference(oracle, reference):
    rng = np.random.default_rng(7)
    from oracle import coil_row
    for _ in range(300):
        c = coil_row(rng.uniform(0.001, 1.0), rng.choice([0.0, rng.uniform(0, 0.5)]),
                     rng.choice([0.0, rng.uniform(0, 0.5)]), int(rng.integers(1, 5000)))
        pf = float(rng.choice([1, 2, 3, 4, 5, 6, 7, 8, 9, 11, 13, 15, rng.uniform(1, 15)]))
        assert list(oracle.precision_args(c, pf, 0)) == list(reference.precision_args(c, pf, False))
        assert list(oracle.precision_args(c, pf, 80)) == list(reference.precision_args(c, pf, True))


def test_group_arrangements_reference_semantics(oracle, golden):
    # CoilGroup arrangements with the secondary a member: the member is left out
    # (src/CoilGroup/MInductance/ComputeMInductance.cxx:14-16)
    coils, spos = golden["garr_coils"], golden["garr_sec_pos"]
    sy, sz = golden["garr_angles"]
    for i in range(len(sy)):
        s = coils[0].copy(); s[6:9] = spos[i]; s[9] = sy[i]; s[10] = sz[i]
        m = sum(oracle.mutual_inductance(c, s, pf=4.0) for c in coils[1:])
        assert abs(m - golden["garr_M"][i]) <= 1e-11 * abs(golden["garr_M"][i])


def test_oracle_z_axis_formulas_against_reference(golden, oracle):
    """The restatement's z-axis formulas (strict IEEE, the reference's operation order)
    against the compiled reference (-Ofast -ffast-math).  The closed-form fast formula
    cancels between its eight length-limit terms: the two differ by up to ~5e-11 there,
    and by <= 1e-12 for the slow (field-sum) formula."""
    worst_fast = worst_slow = 0.0
    for c in range(len(golden["zax_prim"])):
        for i in range(golden["zax_prim_pos"].shape[1]):
            p = golden["zax_prim"][c].copy()
            s = golden["zax_sec"][c].copy()
            py, pz, sy, sz = golden["zax_angles"][c][:, i]
            p[6:9], p[9], p[10] = golden["zax_prim_pos"][c][i], py, pz
            s[6:9], s[9], s[10] = golden["zax_sec_pos"][c][i], sy, sz
            fast = p[2] > 0 and s[2] > 0  # both THIN/RECTANGULAR (length > 0)
            for pf, key in ((3.0, "zax_M_pf3"), (5.0, "zax_M_pf5")):
                ref = golden[key][c][i]
                e = abs(oracle.mutual_inductance(p, s, pf=pf) - ref) / abs(ref)
                if oracle.z_axis_case(p, s) and fast:
                    worst_fast = max(worst_fast, e)
                else:
                    worst_slow = max(worst_slow, e)
            ft = oracle.force_torque(p, s, pf=5.0)
            ref = golden["zax_FT_pf5"][c][i]
            e = np.linalg.norm(ft[:3] - ref[:3]) / np.linalg.norm(ref[:3])
            if oracle.z_axis_case(p, s) and fast:
                worst_fast = max(worst_fast, e)
            else:
                worst_slow = max(worst_slow, e)
    assert worst_fast < 1e-10, worst_fast
    assert worst_slow < 1e-12, worst_slow


def test_oracle_self_inductance_against_reference(golden, oracle):
    """Coil::computeAndSetSelfInductance restated (RECTANGULAR, THIN closed form; FLAT
    through the coaxial mutual inductance with itself) against the compiled reference."""
    for c, L in zip(golden["self_coils"], golden["self_L"]):
        for j, pf in enumerate((3.0, 5.0)):
            assert abs(oracle.self_inductance(c, pf=pf) - L[j]) <= 1e-12 * abs(L[j]), (c, pf)
    with pytest.raises(ValueError):
        oracle.self_inductance(np.array([0.1, 0.0, 0.0, 10, 1.0, 0, 0, 0, 0, 0, 0]))
