"""Adjoint of the B field with respect to coil parameters (torch.autograd.Function
over ccoil_b_field_adjoint) against central finite differences, and the
mutual-inductance position gradient against finite differences of M and the
reference algorithm's force (F = I1 I2 grad M)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def loss_of(B):
    return ((B[:, 2] - 1e-3) ** 2 + B[:, 0] ** 2 + B[:, 1] ** 2).mean()


def setup_case(ccoil, ncoils=8, npts=256, seed=5, types=(0,)):
    from ccoil_b200 import workloads
    rows, pts = workloads.adjoint_config(coils=ncoils, points=npts, seed=seed, types=types)
    params = np.stack([rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3] * rows[:, 4], rows[:, 6], rows[:, 7],
                       rows[:, 8], rows[:, 9], rows[:, 10]], axis=1)
    return params, pts


def adjoint_vs_fd(ccoil, params, pts, dtype):
    """Max over parameter kinds of |adjoint - central difference| / max |central difference|,
    differences in FP64 at h = 1e-6 relative with the node counts held fixed."""
    import torch
    from ccoil_b200.autograd import b_field, precisions_for
    precs = precisions_for(params)
    dt = getattr(torch, dtype)
    P = torch.tensor(params, dtype=dt, requires_grad=True)
    X = torch.tensor(pts, dtype=dt, device="cuda")
    loss = loss_of(b_field(P, X, precs))
    loss.backward()
    g = P.grad.double().numpy()
    X64 = torch.tensor(pts, dtype=torch.float64, device="cuda")
    base = np.array(params, dtype=np.float64)
    # relative steps for R, a, b, N I (thin dimensions: relative to R), 1e-6 of max(R, 0.1) for
    # positions and 1e-6 for the angles
    scale = np.abs(base).copy()
    scale[:, 1] = np.maximum(scale[:, 1], base[:, 0])
    scale[:, 2] = np.maximum(scale[:, 2], base[:, 0])
    scale[:, 4:7] = np.maximum(base[:, :1], 0.1)
    scale[:, 7:9] = 1.0
    fd = np.zeros_like(base)
    for c in range(base.shape[0]):
        for j in range(9):
            if j in (1, 2) and base[c, j] == 0.0:
                continue  # a thin dimension: its derivative is taken at 1e-25 R, not by differences at 0
            h = 1e-6 * scale[c, j]
            up, dn = base.copy(), base.copy()
            up[c, j] += h
            dn[c, j] -= h
            lu = loss_of(b_field(torch.tensor(up), X64, precs)).item()
            ld = loss_of(b_field(torch.tensor(dn), X64, precs)).item()
            fd[c, j] = (lu - ld) / (2 * h)
    errs = {}
    for j, name in enumerate(("R", "a", "b", "NI", "x", "y", "z", "y_angle", "z_angle")):
        sel = ~((j in (1, 2)) & (base[:, j] == 0.0)) if j in (1, 2) else np.ones(len(base), bool)
        ref = np.max(np.abs(fd[sel, j]))
        errs[name] = np.max(np.abs(g[sel, j] - fd[sel, j])) / ref
    return errs


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_b_adjoint_matches_finite_differences(ccoil, dtype):
    """64 RECTANGULAR coils at 4,096 points in a 5 cm ball (the adjoint workload at
    its full size).  float32 points take the FP32-compensated forward; the backward
    is the FP64 adjoint in both cases."""
    params, pts = setup_case(ccoil, ncoils=64, npts=4096)
    errs = adjoint_vs_fd(ccoil, params, pts, dtype)
    print(dtype, {k: "%.1e" % v for k, v in errs.items()})
    for name, err in errs.items():
        assert err < 1e-6, (name, err)


def test_b_adjoint_every_coil_type(ccoil):
    """RECTANGULAR, THIN, FLAT and FILAMENT coils: the slow method's length nodes and the
    thin dimensions (1e-25 R) included."""
    params, pts = setup_case(ccoil, ncoils=8, npts=512, seed=17, types=(0, 1, 2, 3))
    assert set(np.flatnonzero(params[:, 1] == 0.0)) and set(np.flatnonzero(params[:, 2] == 0.0))
    errs = adjoint_vs_fd(ccoil, params, pts, "float64")
    print({k: "%.1e" % v for k, v in errs.items()})
    for name, err in errs.items():
        assert err < 1e-6, (name, err)


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


def _pose_rows(seed, n):
    g = np.random.default_rng(seed)
    p1 = np.concatenate([g.uniform(-0.05, 0.05, (n, 3)), g.uniform(0.2, 1.2, (n, 1)),
                         g.uniform(0, 2 * np.pi, (n, 1))], axis=1)
    off = g.normal(size=(n, 3))
    off *= (0.25 / np.linalg.norm(off, axis=1))[:, None]
    p2 = np.concatenate([p1[:, :3] + off, g.uniform(0.2, 1.2, (n, 1)), g.uniform(0, 2 * np.pi, (n, 1))], axis=1)
    return p1, p2


def _frame(y, z):
    """[e1 e2 axis] of a coil's ring basis at axis angles (y, z), as the pair kernel builds the node cloud."""
    sA, cA, sB, cB = np.sin(y), np.cos(y), np.sin(z), np.cos(z)
    return np.array([[cB * cA, -sB, sA * cB], [sB * cA, cB, sA * sB], [-sA, 0.0, cA]])


@pytest.mark.parametrize("prim_geom,skip", [((0.1, 0.05, 0.1, 200.0), ()),
                                            ((0.1, 0.05, 0.0, 150.0), ("b1",))])
def test_mutual_inductance_parameter_gradient(ccoil, oracle, prim_geom, skip):
    """Adjoint of M with respect to both coils' R, a, b, N and both poses against central
    differences (node counts fixed); RECTANGULAR (fast) and FLAT (slow method) primaries."""
    import torch
    from ccoil_b200.autograd import mutual_inductance, pair_precisions_for
    n = 6
    p1, p2 = _pose_rows(31, n)
    g1 = np.array(prim_geom)
    g2 = np.array([0.05, 0.02, 0.08, 100.0])
    precs = pair_precisions_for(g1, g2, 5.0)
    coef = np.random.default_rng(7).uniform(0.5, 1.5, n)

    def loss(a, b, c, d):
        m = mutual_inductance(torch.tensor(a), torch.tensor(b), torch.tensor(c), torch.tensor(d), precs)
        return float((m.numpy() * coef).sum()), m

    G1, G2 = torch.tensor(g1, requires_grad=True), torch.tensor(g2, requires_grad=True)
    P1, P2 = torch.tensor(p1, requires_grad=True), torch.tensor(p2, requires_grad=True)
    m = mutual_inductance(G1, G2, P1, P2, precs)
    (m * torch.tensor(coef)).sum().backward()

    # M itself is the arrangement kernel's M
    prim = ccoil.Coil(g1[0], g1[1], g1[2], int(g1[3]), 1.0)
    sec = ccoil.Coil(g2[0], g2[1], g2[2], int(g2[3]), 1.0)
    ref_m = ccoil.Coil.compute_all_mutual_inductance_arrangements(
        prim, sec, p1[:, :3], p2[:, :3], p1[:, 3], p1[:, 4], p2[:, 3], p2[:, 4], ccoil.PrecisionFactor(5.0))
    assert np.max(np.abs(m.detach().numpy() - ref_m) / np.abs(ref_m)) < 1e-12

    def fd(arrs, which, idx, h):
        up = [a.copy() for a in arrs]
        dn = [a.copy() for a in arrs]
        up[which][idx] += h
        dn[which][idx] -= h
        return (loss(*up)[0] - loss(*dn)[0]) / (2 * h)

    arrs = [g1, g2, p1, p2]
    names = ("R", "a", "b", "N")
    for which, G in ((0, G1), (1, G2)):
        for k in range(4):
            if "%s%d" % (names[k], which + 1) in skip:
                continue
            h = 1e-6 * arrs[which][k]
            want = fd(arrs, which, k, h)
            got = G.grad.numpy()[k]
            print("geometry", names[k], which + 1, "rel err vs FD %.2e" % (abs(got - want) / abs(want)))
            assert abs(got - want) <= 1e-6 * abs(want) + 1e-12 * abs(loss(*arrs)[0]) / arrs[which][k], \
                (names[k], which + 1, got, want)
    for which, P in ((2, P1), (3, P2)):
        got = P.grad.numpy()
        want = np.zeros_like(got)
        for i in range(n):
            for k in range(5):
                want[i, k] = fd(arrs, which, (i, k), 1e-6 if k >= 3 else 1e-7)
        for k, scale in ((slice(0, 3), None), (slice(3, 5), None)):
            err = np.max(np.abs(got[:, k] - want[:, k])) / np.max(np.abs(want[:, k]))
            print("pose", which - 1, k, "max rel err vs FD %.2e" % err)
            assert err < 1e-6, (which, k, err, got[:, k], want[:, k])

    # against the reference algorithm's force and torque on the secondary (I1 = 2, I2 = 3):
    # F = I1 I2 dM/dc2 and T . w = I1 I2 dM/d(angle) for the rotation w that the angle turns
    # the secondary by -- equal up to the quadrature error of PF 5
    worst = 0.0
    for i in range(n):
        prow = np.array([*g1[:3], g1[3], 2.0, 0.0, *p1[i]])
        srow = np.array([*g2[:3], g2[3], 3.0, 0.0, *p2[i]])
        ft = oracle.force_torque(prow, srow, pf=5.0) / 6.0
        gpos = P2.grad.numpy()[i, :3] / coef[i]
        worst = max(worst, np.max(np.abs(gpos - ft[:3])) / np.max(np.abs(ft[:3])))
        for k in (3, 4):
            h = 1e-7
            dq = (_frame(*(p2[i, 3:5] + h * np.eye(2)[k - 3])) - _frame(*(p2[i, 3:5] - h * np.eye(2)[k - 3]))) / (2 * h)
            W = dq @ _frame(*p2[i, 3:5]).T
            w = np.array([W[2, 1], W[0, 2], W[1, 0]])
            tw = ft[3:] @ w
            worst = max(worst, abs(P2.grad.numpy()[i, k] / coef[i] - tw) / np.max(np.abs(ft[3:])))
    print("force/torque route, max rel deviation %.2e" % worst)
    assert worst < 2e-3, worst


def test_position_gradient_against_reference_force_1024_pairs(ccoil, reference):
    """dM/d(secondary position) -- the exact derivative of the M quadrature, pair kernel
    quantity 2 -- against the reference's own force on the secondary
    (Coil::computeAllForceTorqueArrangements, CPU, src/Coil/ForceAndTorque/ComputeForceMethods.cxx)
    divided by I1 I2, on 1,024 pairs of the arrangement workload (I1 = 2, I2 = 3).

    The two are different quadratures of the same integral (the force integrates
    t x B over the secondary's nodes; the gradient differentiates the A quadrature),
    so they agree up to the quadrature error, which grows as the secondary's winding
    nears the primary's (the integrand nears a singularity).  The test asserts the
    median agreement at PF 5 (1e-7); for every pair whose windings stay at least
    5 cm apart, agreement to 1e-9 once the quadratures have converged (PF 9) and to
    1e-6 at PF 5 for 99 % of them; and that the discrepancy shrinks with the
    PrecisionFactor wherever the windings do not cross (at PF 9 the median falls
    100-fold and the 95th percentile 10-fold), i.e. that it is quadrature error."""
    from ccoil_b200 import workloads
    prim_row, sec_row, ppos, spos, py, pz, sy, sz = workloads.pair_config(arrangements=1024, seed=77,
                                                                          coaxial_fraction=0.0)
    prim_row = prim_row.copy()
    sec_row = sec_row.copy()
    prim_row[4], sec_row[4] = 2.0, 3.0
    prim = workloads.coils_from_rows(prim_row, 5.0)[0]
    sec = workloads.coils_from_rows(sec_row, 5.0)[0]
    args = (prim, sec, ppos, spos, py, pz, sy, sz)
    f_ref = reference.ft_arrangements(prim_row, sec_row, ppos, spos, py, pz, sy, sz, pf=5.0, method=0)[:, :3] / 6.0
    g5 = ccoil.Coil.compute_all_mutual_inductance_gradient_arrangements(*args, ccoil.PrecisionFactor(5.0))
    g9 = ccoil.Coil.compute_all_mutual_inductance_gradient_arrangements(*args, ccoil.PrecisionFactor(9.0))
    f5 = ccoil.Coil.compute_all_force_torque_arrangements(*args, ccoil.PrecisionFactor(5.0))[:, :3] / 6.0
    f9 = ccoil.Coil.compute_all_force_torque_arrangements(*args, ccoil.PrecisionFactor(9.0))[:, :3] / 6.0
    norm = np.linalg.norm
    # this library's FP64 force at PF 5 is the reference's to rounding
    assert np.max(norm(f5 - f_ref, axis=1) / norm(f_ref, axis=1)) < 1e-10
    e5 = norm(g5 - f_ref, axis=1) / norm(f_ref, axis=1)
    e9 = norm(g9 - f9, axis=1) / norm(f9, axis=1)
    # distance from the secondary's winding (sampled: 24 angles x 9 lengths) to the
    # primary's winding cross-section [R, R + a] x [-b/2, b/2] in the primary's frame
    R1, a1, b1 = prim_row[:3]
    R2, b2 = sec_row[0], sec_row[2]
    phi = np.linspace(0, 2 * np.pi, 24, endpoint=False)
    lz = np.linspace(-b2 / 2, b2 / 2, 9)
    ring = np.stack(np.broadcast_arrays(R2 * np.cos(phi)[:, None], R2 * np.sin(phi)[:, None], lz[None, :]),
                    -1).reshape(-1, 3)
    dist = np.zeros(len(sy))
    for i in range(len(sy)):
        A = _frame(sy[i], sz[i])  # the secondary's axes; the primary sits at the origin, unrotated
        q = ring @ A.T + spos[i]
        r, z = np.hypot(q[:, 0], q[:, 1]), q[:, 2]
        dr = np.maximum(np.maximum(R1 - r, r - (R1 + a1)), 0.0)
        dz = np.maximum(np.abs(z) - b1 / 2, 0.0)
        dist[i] = np.min(np.hypot(dr, dz))
    for lo, hi in ((0.0, 0.01), (0.01, 0.03), (0.03, 0.05), (0.05, 1.0)):
        m = (dist >= lo) & (dist < hi)
        print("windings %.2f-%.2f m apart: %4d pairs, |g - F| / |F| at PF 5 median %.1e max %.1e; PF 9 max %.1e"
              % (lo, hi, m.sum(), np.median(e5[m]) if m.any() else 0, e5[m].max(initial=0), e9[m].max(initial=0)))
    clear = dist >= 0.05
    assert np.median(e5) < 1e-7
    assert clear.sum() >= 500 and e9[clear].max() < 1e-9, np.flatnonzero(clear & (e9 >= 1e-9))
    assert np.quantile(e5[clear], 0.99) < 1e-6
    apart = dist >= 0.01  # the windings do not cross
    assert np.median(e9[apart]) < 0.01 * np.median(e5[apart])
    assert np.quantile(e9[apart], 0.95) < 0.1 * np.quantile(e5[apart], 0.95)


def test_mutual_inductance_parameter_gradient_fp32(ccoil):
    """Pair quantity 3 with the primary's quadrature in FP32 (FP32_COMPENSATED; FP64
    near the winding and in every sum) against FP64: M and its 13 derivatives on 2,048
    arrangements of the arrangement workload, each column (or group of columns of one
    scale) within 1e-5 of its largest FP64 magnitude (the FP32 path's M is within 1.2e-5 of FP64 at its worst
    arrangement, relative to 1e-3 of the batch's largest M); the float32 torch
    Function takes that path and keeps its gradients within the same bar."""
    import torch
    from ccoil_b200 import workloads
    from ccoil_b200.autograd import mutual_inductance, pair_precisions_for
    prim_row, sec_row, ppos, spos, py, pz, sy, sz = workloads.pair_config(arrangements=2048, seed=57,
                                                                          coaxial_fraction=0.05)
    prim, sec = workloads.coils_from_rows(prim_row, 5.0)[0], workloads.coils_from_rows(sec_row, 5.0)[0]
    args = (prim, sec, ppos, spos, py, pz, sy, sz, ccoil.PrecisionFactor(5.0))
    from ccoil_b200 import _lib
    from ccoil_b200.coil import _pair_arrangements
    pp, sp = ccoil.Coil._pair_args(prim, sec, 5.0)
    p1 = np.concatenate([ppos, py[:, None], pz[:, None]], axis=1)
    p2 = np.concatenate([spos, sy[:, None], sz[:, None]], axis=1)
    res = []
    for mode in (ccoil.PrecisionMode.FP64, ccoil.PrecisionMode.FP32_COMPENSATED):
        out, _ = _pair_arrangements([prim.struct(pp)], sec.struct(sp), [sp.to_struct()], p1, p2,
                                    _lib.PAIR_MUTUAL_INDUCTANCE_PARAMETER_GRADIENT, precision_mode=mode)
        res.append(out)
    d64, d32 = res
    # columns in groups that share a scale: M; each geometry parameter; both angles of a
    # coil (the primary sits at y angle 0 here, where dM/dz angle vanishes); the position
    groups = [[0], [1], [2], [3], [4, 5], [6], [7], [8], [9, 10, 11], [12, 13]]
    err = np.array([np.max(np.abs(d32[:, g] - d64[:, g])) / np.max(np.abs(d64[:, g])) for g in groups])
    print("FP32 parameter gradient, max error per column group relative to its largest value:",
          " ".join("%.1e" % e for e in err))
    assert err.max() < 1e-5, err
    # the float32 torch Function
    g1 = np.array([0.1, 0.05, 0.1, 200.0])
    g2 = np.array([0.05, 0.0, 0.2, 100.0])
    precs = pair_precisions_for(g1, g2, 5.0)
    grads = []
    for dt in (torch.float64, torch.float32):
        G1 = torch.tensor(g1, dtype=dt, requires_grad=True)
        G2 = torch.tensor(g2, dtype=dt, requires_grad=True)
        P1 = torch.tensor(p1[:256], dtype=dt, requires_grad=True)
        P2 = torch.tensor(p2[:256], dtype=dt, requires_grad=True)
        mutual_inductance(G1, G2, P1, P2, precs).sum().backward()
        grads.append([x.grad.double().numpy() for x in (G1, G2, P1, P2)])
    for a, b in zip(*grads):
        assert np.max(np.abs(b - a)) <= 1e-5 * np.max(np.abs(a)), (np.max(np.abs(b - a)), np.max(np.abs(a)))
