"""Adjoint of the B field with respect to coil parameters (torch.autograd.Function
over ccoil_b_field_adjoint) against central finite differences, and the
mutual-inductance position gradient against finite differences of M and the
reference algorithm's force (F = I1 I2 grad M)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def loss_of(B):
    return ((B[:, 2] - 1e-3) ** 2 + B[:, 0] ** 2 + B[:, 1] ** 2).mean()


def setup_case(ccoil, ncoils=8, npts=256, seed=5):
    from ccoil_b200 import workloads
    rows, pts = workloads.adjoint_config(coils=ncoils, points=npts, seed=seed)
    params = np.stack([rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3] * rows[:, 4], rows[:, 6], rows[:, 7],
                       rows[:, 8], rows[:, 9], rows[:, 10]], axis=1)
    return params, pts


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_b_adjoint_matches_finite_differences(ccoil, dtype):
    import torch
    from ccoil_b200.autograd import b_field, precisions_for
    params, pts = setup_case(ccoil)
    precs = precisions_for(params)
    dt = getattr(torch, dtype)
    P = torch.tensor(params, dtype=dt, requires_grad=True)
    X = torch.tensor(pts, dtype=dt, device="cuda")
    loss = loss_of(b_field(P, X, precs))
    loss.backward()
    g = P.grad.double().numpy()

    # central differences in FP64 with the node counts held fixed
    X64 = torch.tensor(pts, dtype=torch.float64, device="cuda")
    base = np.array(params, dtype=np.float64)
    scale = np.array([1, 1, 1, 1, 0, 0, 0, 0, 0], dtype=float) * np.abs(base) + \
        np.array([0, 0, 0, 0, 1, 1, 1, 1, 1], dtype=float) * np.maximum(base[:, :1], 0.1)
    fd = np.zeros_like(base)
    for c in range(base.shape[0]):
        for j in range(9):
            h = 1e-6 * scale[c, j]
            up, dn = base.copy(), base.copy()
            up[c, j] += h
            dn[c, j] -= h
            lu = loss_of(b_field(torch.tensor(up), X64, precs)).item()
            ld = loss_of(b_field(torch.tensor(dn), X64, precs)).item()
            fd[c, j] = (lu - ld) / (2 * h)
    # per parameter kind, relative to the largest gradient of that kind
    for j, name in enumerate(("R", "a", "b", "NI", "x", "y", "z", "y_angle", "z_angle")):
        ref = np.max(np.abs(fd[:, j]))
        err = np.max(np.abs(g[:, j] - fd[:, j])) / ref
        bound = 1e-6 if dtype == "float64" else 1e-4
        assert err < bound, (name, err, g[:, j], fd[:, j])


def test_adjoint_is_deterministic(ccoil):
    import torch
    from ccoil_b200.autograd import b_field
    params, pts = setup_case(ccoil, ncoils=4, npts=512, seed=9)
    grads = []
    for _ in range(2):
        P = torch.tensor(params, requires_grad=True)
        loss_of(b_field(P, torch.tensor(pts, device="cuda"))).backward()
        grads.append(P.grad.numpy().copy())
    assert np.array_equal(grads[0], grads[1])


def test_mutual_inductance_position_gradient(ccoil, oracle):
    from ccoil_b200 import workloads
    from ccoil_b200.autograd import mutual_inductance_position_gradient, mutual_inductance_position_gradient_from_force
    worst_force = 0.0
    prim_row, sec_row, ppos, spos, py, pz, sy, sz = workloads.pair_config(arrangements=16, seed=21,
                                                                          coaxial_fraction=0.0)
    for i in range(len(py)):
        p_row = prim_row.copy(); p_row[4] = 2.0; p_row[6:9] = ppos[i]; p_row[9] = py[i]; p_row[10] = pz[i]
        s_row = sec_row.copy(); s_row[4] = 3.0; s_row[6:9] = spos[i]; s_row[9] = sy[i]; s_row[10] = sz[i]
        prim = workloads.coils_from_rows(p_row, 5.0)[0]
        sec = workloads.coils_from_rows(s_row, 5.0)[0]
        g = mutual_inductance_position_gradient(prim, sec, ccoil.PrecisionFactor(5.0))
        gf = mutual_inductance_position_gradient_from_force(prim, sec, ccoil.PrecisionFactor(5.0))
        # the force route reproduces the reference algorithm's force exactly ...
        fo = oracle.force_torque(p_row, s_row, pf=5.0)[:3] / (2.0 * 3.0)
        assert np.max(np.abs(gf - fo)) <= 1e-12 * np.max(np.abs(fo))
        # ... and agrees with the exact gradient up to the quadrature error at PF 5
        worst_force = max(worst_force, np.max(np.abs(g - fo)) / np.max(np.abs(fo)))
        # central differences of M in the secondary's position
        h = 1e-6 * 0.05
        fd = np.zeros(3)
        for k in range(3):
            plus, minus = spos[i].copy(), spos[i].copy()
            plus[k] += h
            minus[k] -= h
            m = ccoil.Coil.compute_all_mutual_inductance_arrangements(
                prim, sec, [ppos[i], ppos[i]], [plus, minus], [py[i]] * 2, [pz[i]] * 2, [sy[i]] * 2, [sz[i]] * 2,
                ccoil.PrecisionFactor(5.0))
            fd[k] = (m[0] - m[1]) / (2 * h)
        assert np.max(np.abs(g - fd)) <= 1e-6 * np.max(np.abs(fd)), (i, g, fd)
    assert worst_force < 1e-3, worst_force
