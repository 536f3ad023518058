"""Self inductance (Coil::computeAndSetSelfInductance) on the GPU against the
reference's golden values and the oracle: RECTANGULAR and THIN coils through the
closed form, FLAT coils through the coaxial mutual inductance with itself, several
coils in one launch.  Bar: 1e-12 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def test_self_inductance_golden(ccoil, golden, oracle):
    from ccoil_b200 import workloads
    for j, pf in enumerate((3.0, 5.0)):
        coils = workloads.coils_from_rows(golden["self_coils"], pf)
        got = ccoil.Coil.compute_all_self_inductances(coils, ccoil.PrecisionFactor(pf))
        ref = golden["self_L"][:, j]
        assert np.max(np.abs(got - ref) / np.abs(ref)) < TOL, (pf, got, ref)
        orc = np.array([oracle.self_inductance(c, pf=pf) for c in golden["self_coils"]])
        assert np.max(np.abs(got - orc) / np.abs(orc)) < TOL, (pf, got, orc)


def test_self_inductance_single_coil_api(ccoil, golden):
    from ccoil_b200 import workloads
    c = workloads.coils_from_rows(golden["self_coils"][1], 5.0)[0]
    c.set_position_and_orientation((0.3, -0.2, 0.1), 0.7, 1.1)  # the reference centres the coil
    L = c.compute_and_set_self_inductance(ccoil.PrecisionFactor(5.0))
    assert c.get_self_inductance() == L
    assert abs(L - golden["self_L"][1, 1]) < TOL * abs(golden["self_L"][1, 1])


def test_filament_is_rejected(ccoil):
    with pytest.raises(ccoil.CCoilError):
        ccoil.Coil(0.1, 0.0, 0.0, 10).compute_and_set_self_inductance()
