"""Size-independent properties at the benchmark sizes, where the oracle would take
too long: the 128-coil group at 2^20 points and 2^18 pair arrangements.

* superposition: the group's field equals the sum of the fields of its two
  halves (FP64, 1e-12 of the batch scale);
* translation invariance: moving every coil and point by the same offset leaves
  the field unchanged (FP64: median below 1e-14; maximum below 1e-8, set by the
  points closest to a winding, where the 1e-16 rounding of the shifted
  coordinates is amplified by the field's steep gradient);
* the FP32-compensated field and arrangements against FP64: median below 1e-7,
  99th percentile below 5e-7 (the statistics bench.py reports);
* bitwise reproducibility of the FP64 arrangement kernel."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

POINTS = 1 << 20
ARRANGEMENTS = 1 << 18


@pytest.fixture(scope="module")
def group_case():
    import torch
    from ccoil_b200 import workloads
    rows, _ = workloads.group_config(coils=128, points=1)
    pts = workloads.points_cube(POINTS, seed=4242)
    return rows, pts, torch.from_numpy(pts).cuda()


def field(cc, rows, pts_dev, f, mode):
    from ccoil_b200 import workloads
    plan = cc.FieldPlan([c.struct() for c in workloads.coils_from_rows(rows, 5.0)], f, mode)
    try:
        return plan(pts_dev).cpu().numpy()
    finally:
        plan.close()


def test_superposition(ccoil, group_case):
    rows, _, d = group_case
    full = field(ccoil, rows, d, 1, ccoil.PrecisionMode.FP64)
    halves = field(ccoil, rows[:64], d, 1, ccoil.PrecisionMode.FP64) + field(ccoil, rows[64:], d, 1,
                                                                          ccoil.PrecisionMode.FP64)
    assert rel_err(halves, full, floor_frac=1e-3).max() < 1e-12


def test_translation_invariance(ccoil, group_case):
    import torch
    rows, pts, d = group_case
    shift = np.array([0.125, -0.25, 0.5])
    moved = rows.copy()
    moved[:, 6:9] += shift
    a = field(ccoil, rows, d[:1 << 18], 1, ccoil.PrecisionMode.FP64)
    b = field(ccoil, moved, torch.from_numpy(pts[:1 << 18] + shift).cuda(), 1, ccoil.PrecisionMode.FP64)
    e = rel_err(b, a, floor_frac=1e-3)
    assert np.median(e) < 1e-14 and e.max() < 1e-8, (np.median(e), e.max())


@pytest.mark.parametrize("f", [0, 1])
def test_fp32c_against_fp64(ccoil, group_case, f):
    rows, _, d = group_case
    e = rel_err(field(ccoil, rows, d, f, ccoil.PrecisionMode.FP32_COMPENSATED),
                field(ccoil, rows, d, f, ccoil.PrecisionMode.FP64))
    assert np.median(e) < 1e-7 and np.percentile(e, 99) < 5e-7, (np.median(e), np.percentile(e, 99))


def test_arrangements_at_full_size(ccoil):
    import torch
    import sys
    import os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from ccoil_b200 import workloads
    from ccoil_b200.coil import pair_arrangements_device
    _, _, ps, ss, spre, pp, sp, _ = bench.pair_setup(ccoil, workloads, ARRANGEMENTS, 11)
    dp, ds = torch.from_numpy(pp).cuda(), torch.from_numpy(sp).cuda()
    outs = []
    for mode in (ccoil.PrecisionMode.FP64, ccoil.PrecisionMode.FP64, ccoil.PrecisionMode.FP32_COMPENSATED):
        out = torch.empty((ARRANGEMENTS, 1), dtype=torch.float64, device="cuda")
        pair_arrangements_device([ps], ss, [spre], dp, ds, 0, out, precision_mode=mode)
        outs.append(out.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    e = rel_err(outs[2], outs[0])
    assert np.median(e) < 1e-7 and np.percentile(e, 99) < 5e-7 * 2, (np.median(e), np.percentile(e, 99))
