"""Batched persistent launch of independent systems (one launch, CUDA graph,
autotuner) against per-system plans of the same precision."""
import numpy as np
import pytest

from conftest import gradient_band, rel_err

pytestmark = pytest.mark.gpu


def systems(cc, n=24, seed=7):
    from ccoil_b200 import workloads
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        k = int(np.floor(np.exp(rng.uniform(0, np.log(24))))) + 1
        npts = int(np.floor(np.exp(rng.uniform(np.log(16), np.log(3000)))))
        rows = workloads.coil_rows_mixed(k, seed=1000 + i)
        out.append((rows, workloads.coils_from_rows(rows, 5.0), workloads.points_cube(npts, seed=2000 + i)))
    out.append((np.zeros((0, 11)), [], workloads.points_cube(10, seed=1)))     # empty system
    out.append((out[0][0], out[0][1], np.zeros((0, 3))))                       # no points
    return out


def per_system(cc, coils, pts, field, mode):
    if len(coils) == 0:
        return np.zeros((len(pts), 9 if field == 3 else 3))
    plan = cc.FieldPlan([c.struct() for c in coils], field, mode)
    try:
        return plan(pts)
    finally:
        plan.close()


@pytest.mark.parametrize("mode", ["FP64", "FP32_COMPENSATED"])
def test_batched_matches_per_system(ccoil, mode):
    m = getattr(ccoil.PrecisionMode, mode)
    sy = systems(ccoil)
    plan = ccoil.BatchPlan([(c, p) for _, c, p in sy], fields=("B", "G"), precision=m)
    out = plan.run()
    got = {f: [t.cpu().numpy() for t in plan.split(out[f])] for f in ("B", "G")}
    errs = {"B": [], "G": []}
    for i, (rows, coils, pts) in enumerate(sy):
        if len(pts) == 0:
            continue
        for f, fid in (("B", 1), ("G", 3)):
            ref = per_system(ccoil, coils, pts, fid, ccoil.PrecisionMode.FP64)
            e = rel_err(got[f][i].reshape(len(pts), -1), ref)
            if fid == 3 and len(rows):
                e = e[~gradient_band(rows, pts)]
            errs[f].append(e)
    for f in errs:
        e = np.concatenate(errs[f])
        if mode == "FP64":
            assert e.max() < 1e-12, (f, e.max())
        else:
            # the FP32 bars of test_fields32_gpu.py, over the whole batch
            assert np.median(e) < 3e-7 and np.quantile(e, 0.99) < 2e-6 and e.max() < 1e-5, (f, e.max())
    plan.close()


def test_graph_replay_and_tuner(ccoil):
    sy = systems(ccoil, n=16, seed=11)
    plan = ccoil.BatchPlan([(c, p) for _, c, p in sy], fields=("A", "B"), precision=ccoil.PrecisionMode.FP64)
    first = {f: t.clone() for f, t in plan.run().items()}
    again = plan.run()
    for f in first:
        assert bool((first[f] == again[f]).all())
    split, ms = plan.tune()
    assert split in (2, 8, 32, 128) and ms > 0
    tuned = plan.run()
    for f in first:
        assert rel_err(tuned[f].cpu().numpy(), first[f].cpu().numpy()).max() < 1e-12
    plan.close()
