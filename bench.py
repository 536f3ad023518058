"""Benchmark of the field hot path on the coil-group workload.

One step = A, B and G of a 128-coil mixed group (25% each RECTANGULAR, THIN,
FLAT, FILAMENT; R ~ U[0.02, 0.3] m, a, b ~ U[0, 0.1] m, N ~ U{1..500},
I ~ U[-5, 5] A, centres in a 1 m cube, random axes) at 2^20 points per GPU
(uniform in a 2 m cube), PrecisionFactor 5, every coil at its CPU
PrecisionArguments.  Seeded synthetic data; no dataset is involved.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|fp32c|fp32r|both|all]
    python bench.py --impl reference        # the reference's own CPU_MT code on this host
    python bench.py --workload refine-sweep # FP32_REFINED: cost and error over its fraction (fields, arrangements)

The headline configuration (fp32r) is the FP32 one whose maximum error away
from windings stays below 1e-7: FP32_REFINED for A and B, FP32_COMPENSATED
for G; fp64 and fp32c (FP32_COMPENSATED for every field) are timed beside it.
    python bench.py --workload batched      # 2,048 independent systems, one persistent launch per step
    python bench.py --workload adjoint      # forward + backward of a B-field loss (64 coils)
    python bench.py --workload pf-sweep     # the group at PrecisionFactor 1, 3, 5, 7, 9

Under torchrun every rank evaluates its own 2^20 points (weak scaling, no
collective on the data path); times are device times (CUDA events), max over
ranks.  Rank 0 prints one JSON line.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "c-coil_b200"))

METRIC = "coil-point field evals/s & M arrangements/s: FP32-comp vs FP64 at 1e-7 rel err"
UNIT = "coil-point evals/s"
FIELDS = (("A", 0), ("B", 1), ("G", 3))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="all", choices=["fp64", "fp32c", "fp32r", "both", "all"],
                    help="fp32r: FP32_REFINED for A and B, FP32_COMPENSATED for G (the configuration at "
                         "<= 1e-7); both: fp64 + fp32c; all: fp64 + fp32c + fp32r (headline fp32r)")
    ap.add_argument("--points", type=int, default=1 << 20)
    ap.add_argument("--coils", type=int, default=128)
    ap.add_argument("--pf", type=float, default=5.0)
    ap.add_argument("--cpu-sample-points", type=int, default=32768)
    ap.add_argument("--arrangements", type=int, default=1 << 18,
                    help="coil-pair arrangements per GPU for the M and F/T part (0 skips it)")
    ap.add_argument("--cpu-sample-arrangements", type=int, default=4096)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="group", choices=["group", "batched", "adjoint", "pf-sweep", "refine-sweep"],
                    help="group: the headline coil-group fields + pair arrangements; batched: many independent "
                         "systems in one persistent launch; adjoint: forward + backward of the B-field loss; "
                         "pf-sweep: the group at PrecisionFactor 1, 3, 5, 7, 9 (2^18 points); refine-sweep: "
                         "FP32_REFINED's time and error per fraction, fields and pair arrangements")
    ap.add_argument("--systems", type=int, default=2048, help="independent systems of the batched workload")
    return ap.parse_args()


def workload_config(a, world):
    return {"workload": "coil group: %d mixed coils (RECT/THIN/FLAT/FILAMENT), %d points per GPU in a 2 m cube, "
                        "A+B+G, PrecisionFactor %g" % (a.coils, a.points, a.pf),
            "coils": a.coils, "points_per_gpu": a.points, "precision_factor": a.pf, "fields": ["A", "B", "G"],
            "l2": "flushed between timed steps (256 MiB write)",
            "parallelism": "points sharded over %d rank(s), no data-path collective" % world}


# ---------------------------------------------------------------------------
# reference arm: the reference's own CPU code (oracle/_ref), CPU_MT on all cores
# ---------------------------------------------------------------------------
def cpu_reference_rate(a, sample_points):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Reference
    from ccoil_b200 import workloads
    cores = os.cpu_count() or 1
    ref = Reference(threads=cores)
    rows, _ = workloads.group_config(coils=a.coils, points=1)
    pts = workloads.points_cube(sample_points, seed=1000 + 2)
    t0 = time.perf_counter()
    for _, f in FIELDS:
        ref.group_fields(rows, pts, f, pf=a.pf, method=1)
    dt = time.perf_counter() - t0
    units = len(FIELDS) * a.coils * sample_points
    return units / dt, cores, dt, "%d coils x %d points x A,B,G (CPU_MT, per-member MT path)" % (a.coils,
                                                                                               sample_points)


def reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Reference
    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libccoil_ref.so was not built"}))
        return
    rates = []
    sample = max(64, a.cpu_sample_points // 2)
    for _ in range(a.warmup):
        cpu_reference_rate(a, 64)
    for _ in range(a.steps):
        r, cores, dt, desc = cpu_reference_rate(a, sample)
        rates.append((r, dt))
    value = float(np.median([r for r, _ in rates]))
    ms = float(np.mean([dt for _, dt in rates]) * 1e3)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": workload_config(a, world), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def pair_setup(cc, workloads, n, seed):
    """The pair workload: RECTANGULAR primary (0.1, 0.05, 0.1, N=200), THIN secondary
    (0.05, 0, 0.2, N=100), both moving per arrangement; CPU pair arguments at PF 5."""
    prim_row, sec_row, ppos, spos, py, pz, sy, sz = workloads.pair_config(arrangements=n, seed=seed)
    prim, sec = workloads.coils_from_rows(prim_row, 5.0)[0], workloads.coils_from_rows(sec_row, 5.0)[0]
    pp, sp = cc.Coil._pair_args(prim, sec, 5.0)
    pposes = np.concatenate([ppos, py[:, None], pz[:, None]], axis=1)
    sposes = np.concatenate([spos, sy[:, None], sz[:, None]], axis=1)
    return prim_row, sec_row, prim.struct(pp), sec.struct(sp), sp.to_struct(), pposes, sposes, (pp, sp)


def rel_err_stats(got, ref, mask=None):
    """Relative error per row (norm-wise), the denominator floored at 1e-3 x the
    batch's largest reference norm; median, 99th percentile and maximum, over all
    rows or over `mask`."""
    import torch
    got = got.reshape(len(got), -1)
    ref = ref.reshape(len(ref), -1)
    nb = ref.norm(dim=1)
    e = (got - ref).norm(dim=1) / torch.clamp(nb, min=1e-3 * float(nb.max()))
    if mask is not None:
        e = e[mask]
    if e.numel() == 0:
        return None
    q = torch.quantile(e[:1 << 24].float(), torch.tensor([0.5, 0.99], device=e.device)).tolist()
    return {"median": q[0], "p99": q[1], "max": float(e.max()), "rows": int(e.numel())}


def winding_masks(rows, pts):
    """Boolean masks over points (numpy, on the host): `near` = inside some coil's
    near-field box (its winding cross-section in (r, z) inflated by 0.1 R), `band` =
    radius, in some coil's frame, within [0.9 R, R + a + 0.1 R] at any z, where the
    reference's gradient RZ integrand is ill-conditioned (its own FP64 result
    carries ~1e-7 relative error there, so FP32 is judged outside it)."""
    near = np.zeros(len(pts), dtype=bool)
    band = np.zeros(len(pts), dtype=bool)
    for row in rows:
        R, a_, b_ = row[0], row[1], row[2]
        yA, zA = row[9], row[10]
        cY, sY, cZ, sZ = np.cos(yA), np.sin(yA), np.cos(zA), np.sin(zA)
        Ti = np.array([[cZ * cZ * cY - sZ * sZ, sZ * cZ * cY + sZ * cZ, -cZ * sY],
                       [-sZ * cZ * cY - sZ * cZ, cZ * cZ - sZ * sZ * cY, sZ * sY],
                       [sY * cZ, sY * sZ, cY]])
        d = (pts - row[6:9]) @ Ti.T
        r = np.hypot(d[:, 0], d[:, 1])
        inr = (r > 0.9 * R) & (r < R + a_ + 0.1 * R)
        band |= inr
        near |= inr & (np.abs(d[:, 2]) < 0.5 * b_ + 0.1 * R)
    return near, band


def bench_arrangements(a, cc, workloads, dev, rank, max_over_ranks, barrier, modes):
    import torch
    from ccoil_b200.coil import pair_arrangements_device
    _, _, pstruct, sstruct, spre, pposes, sposes, (pp, sp) = pair_setup(cc, workloads, a.arrangements,
                                                                        3 + 7919 * rank)
    dp = torch.from_numpy(pposes).to(dev)
    ds = torch.from_numpy(sposes).to(dev)
    res = {}

    def timed(q, w, mode):
        out = torch.empty((a.arrangements, w), dtype=torch.float64, device=dev)
        pair_arrangements_device([pstruct], sstruct, [spre], dp, ds, q, out, precision_mode=mode)  # warm-up
        torch.cuda.synchronize()
        barrier()
        ms = 0.0
        for _ in range(a.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            zc = pair_arrangements_device([pstruct], sstruct, [spre], dp, ds, q, out, precision_mode=mode)
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        ms = max_over_ranks(ms / a.steps)
        return {"ms": ms, "arrangements_per_s": a.arrangements / (ms * 1e-3), "z_axis_cases": zc, "out": out}

    for mode in modes:
        key = {0: "fp64", 1: "fp32c", 2: "fp32r"}[int(mode)]
        res[key] = {name: timed(q, w, mode) for name, q, w in (("M", 0, 1), ("FT", 1, 6))}
    if "fp64" in res:
        m64, f64 = res["fp64"]["M"]["out"], res["fp64"]["FT"]["out"]
        for key in ("fp32c", "fp32r"):
            if key in res:
                m32, f32 = res[key]["M"]["out"], res[key]["FT"]["out"]
                res[key + "_errors"] = {"M": rel_err_stats(m32, m64), "F": rel_err_stats(f32[:, :3], f64[:, :3]),
                                        "T": rel_err_stats(f32[:, 3:], f64[:, 3:])}
        if "fp32r" in res:
            # the arrangements at max error <= 1e-7: FP32_REFINED at the fraction that
            # reaches it on this workload (M 0.01, F/T 0.005) and at fraction 0 (every
            # node in the FP64 refinement forms, no FP32 pass), each checked here
            # against FP64; the faster passing one is reported (FP64 where none passes)
            import ctypes
            L = cc.lib()
            default = L.ccoil_refine_fraction()
            at = {}
            try:
                for name, q, w, fractions in (("M", 0, 1, (0.01, 0.0)), ("FT", 1, 6, (0.005, 0.0))):
                    ref = res["fp64"][name]["out"]
                    cands = {}
                    for fr in fractions:
                        L.ccoil_set_refine_fraction(ctypes.c_double(fr))
                        r = timed(q, w, cc.PrecisionMode.FP32_REFINED)
                        errs = ({"M": rel_err_stats(r["out"], ref)} if name == "M" else
                                {"F": rel_err_stats(r["out"][:, :3], ref[:, :3]),
                                 "T": rel_err_stats(r["out"][:, 3:], ref[:, 3:])})
                        cands["%g" % fr] = {"ms": r["ms"], "arrangements_per_s": r["arrangements_per_s"],
                                            "max_error": {k: e["max"] for k, e in errs.items()},
                                            "passes": all(e["max"] <= 1e-7 for e in errs.values())}
                    passing = [f for f, c in cands.items() if c["passes"]]
                    if passing:
                        best = min(passing, key=lambda f: cands[f]["ms"])
                        src = cands[best]
                        mode = "FP32_REFINED, fraction %s" % best + (" (every node in FP64)" if float(best) == 0 else "")
                    else:
                        src, mode = res["fp64"][name], "FP64"
                    at[name] = {"precision_mode": mode, "arrangements_per_s": src["arrangements_per_s"],
                                "ms": src["ms"], "refined_max_error": src.get("max_error"), "candidates": cands}
            finally:
                L.ccoil_set_refine_fraction(ctypes.c_double(default))
            res["at_1e-7"] = at
    aB, tB, lB, aI, tI, lI = sp.as_tuple()
    res["secondary_nodes"] = aB * aI * tB * tI * lB * lI
    res["primary_nodes"] = pp.angular_blocks * pp.angular_increments * pp.thickness_blocks * pp.thickness_increments
    return res


def cpu_arrangement_rate(a, sample):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Reference
    from ccoil_b200 import workloads
    cores = os.cpu_count() or 1
    ref = Reference(threads=cores)
    prim, sec, ppos, spos, py, pz, sy, sz = workloads.pair_config(arrangements=sample, seed=3)
    t0 = time.perf_counter()
    ref.m_arrangements(prim, sec, ppos, spos, py, pz, sy, sz, pf=5.0, method=1)
    dt = time.perf_counter() - t0
    return sample / dt, cores, dt


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    COLS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
            "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
            "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.COLS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def flush_l2(torch, dev):
    buf = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def flush():
        buf.fill_(1)
    return flush


def bench_batched(a):
    """Independent coil systems (group size log-uniform in [1, 256], point count log-uniform in
    [256, 65536], coils as the group workload) evaluated by one persistent launch per step, B and G,
    replayed from a captured CUDA graph, split chosen by the autotuner; FP64 and FP32c."""
    import torch
    import ccoil_b200 as cc
    from ccoil_b200 import workloads
    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    raw = workloads.batched_config(groups=a.systems, seed=4)
    systems = [(workloads.coils_from_rows(r, a.pf), p) for r, p in raw]
    build_s = time.perf_counter() - t0
    coil_points = sum(len(c) * len(p) for c, p in systems)
    units = 2 * coil_points  # B and G
    flush = flush_l2(torch, dev)
    res = {}
    for mode in (cc.PrecisionMode.FP64, cc.PrecisionMode.FP32_COMPENSATED):
        plan = cc.BatchPlan(systems, fields=("B", "G"), precision=mode, device=dev)
        split, _ = plan.tune()
        for _ in range(max(a.warmup, 3)):
            plan.run()
        torch.cuda.synchronize()
        ms = 0.0
        with ClockSampler(0) as clk:
            for _ in range(a.steps):
                flush()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                plan.run()
                e1.record()
                torch.cuda.synchronize()
                ms += e0.elapsed_time(e1)
        ms /= a.steps
        res["fp64" if int(mode) == 0 else "fp32c"] = {"ms_per_step": ms, "value": units / (ms * 1e-3),
                                                      "autotuned_split": split, "clocks": clk.summary()}
        plan.close()
    head = res["fp32c"]
    line = {"metric": "batched coil-point field evals/s (B+G, many independent systems)", "value": head["value"],
            "unit": UNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": head["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (compensated) + f64",
            "data": "synthetic (seeded)",
            "config": {"workload": "%d independent systems: group size log-uniform in [1, 256], points log-uniform "
                                   "in [256, 65536], mixed coil types, B and G in one persistent launch (CUDA graph)"
                                   % a.systems, "coils": sum(len(c) for c, _ in systems),
                       "points": sum(len(p) for _, p in systems), "coil_points_per_field": coil_points,
                       "precision_factor": a.pf, "l2": "flushed between timed steps (256 MiB write)"},
            "precision_mode": "fp32c", "fp64": res["fp64"], "fp32c": res["fp32c"], "clocks": head["clocks"],
            "gpu_launches": 2 * a.steps, "host_build_s": build_s}
    print(json.dumps(line))


def bench_adjoint(a):
    """Forward + backward of a B-field loss over 64 RECTANGULAR coils at 4,096 points in a 5 cm
    ball (the adjoint kernel: dL/d(R, a, b, N I, position, orientation) of every coil)."""
    import torch
    from ccoil_b200 import workloads
    from ccoil_b200.autograd import b_field, precisions_for
    dev = torch.device("cuda", 0)
    rows, pts = workloads.adjoint_config(coils=64, points=4096, seed=5)
    params = np.stack([rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3] * rows[:, 4], rows[:, 6], rows[:, 7],
                       rows[:, 8], rows[:, 9], rows[:, 10]], axis=1)
    precs = precisions_for(params)
    X = torch.tensor(pts, dtype=torch.float64, device=dev)
    res = {}
    for dtype in (torch.float64, torch.float32):
        Xd = X.to(dtype)

        def step():
            P = torch.tensor(params, dtype=dtype, requires_grad=True)
            B = b_field(P, Xd, precs)
            loss = ((B[:, 2] - 1e-3) ** 2 + B[:, 0] ** 2 + B[:, 1] ** 2).mean()
            loss.backward()
            return P.grad
        for _ in range(max(a.warmup, 3)):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record()
        for _ in range(a.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.steps
        res["fp64" if dtype == torch.float64 else "fp32c_forward"] = {
            "ms_per_step": ms, "wall_ms_per_step": (time.perf_counter() - t0) * 1e3 / a.steps,
            "value": 64 * 4096 / (ms * 1e-3)}
    line = {"metric": "adjoint coil-point evals/s (B forward + parameter gradient backward)",
            "value": res["fp64"]["value"], "unit": "coil-point evals/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": res["fp64"]["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": "64 RECTANGULAR coils, 4096 points in a 5 cm ball, loss |B - (0, 0, 1e-3)|^2 "
                                   "mean, gradient w.r.t. 9 parameters per coil", "precision_factor": 5.0,
                       "l2": "inputs and tables are L2-resident (a small workload; not flushed)"},
            "fp64": res["fp64"], "fp32c_forward": res["fp32c_forward"], "gpu_launches": 2 * a.steps}
    print(json.dumps(line))


def bench_pf_sweep(a):
    """The coil group at PrecisionFactor 1, 3, 5, 7 and 9: throughput of A, B and G in FP64 and
    FP32-compensated, and the FP32c error against FP64, at 2^18 points."""
    import torch
    import ccoil_b200 as cc
    from ccoil_b200 import opcount, workloads
    dev = torch.device("cuda", 0)
    npts = 1 << 18
    rows, _ = workloads.group_config(coils=a.coils, points=1)
    pts_host = workloads.points_cube(npts, seed=1002)
    pts = torch.from_numpy(pts_host).to(dev)
    near, band = (torch.from_numpy(m).to(dev) for m in winding_masks(rows, pts_host))
    flush = flush_l2(torch, dev)
    sweep = []
    for pf in (1.0, 3.0, 5.0, 7.0, 9.0):
        coils = workloads.coils_from_rows(rows, pf)
        group = cc.CoilGroup(coils, cc.PrecisionFactor(pf))
        entry = {"precision_factor": pf, "nodes_per_point": opcount.group_nodes_per_point(coils)}
        outs = {}
        for mode in (cc.PrecisionMode.FP64, cc.PrecisionMode.FP32_COMPENSATED):
            key = "fp64" if int(mode) == 0 else "fp32c"
            step_ms = 0.0
            for name, f in FIELDS:
                plan = group.plan(f, mode)
                out = plan(pts)
                for _ in range(max(a.warmup, 3) - 1):
                    plan(pts, out=out)
                torch.cuda.synchronize()
                ms = 0.0
                for _ in range(a.steps):
                    flush()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    plan(pts, out=out)
                    e1.record()
                    torch.cuda.synchronize()
                    ms += e0.elapsed_time(e1)
                step_ms += ms / a.steps
                outs[(key, name)] = out.clone()
                plan.close()
            entry[key] = {"ms_per_step": step_ms, "value": len(FIELDS) * a.coils * npts / (step_ms * 1e-3)}
        entry["fp32c_speedup_vs_fp64"] = entry["fp64"]["ms_per_step"] / entry["fp32c"]["ms_per_step"]
        entry["fp32c_rel_err_vs_fp64_away"] = {
            name: rel_err_stats(outs[("fp32c", name)], outs[("fp64", name)], ~band if f == 3 else ~near)
            for name, f in FIELDS}
        sweep.append(entry)
    head = [e for e in sweep if e["precision_factor"] == 5.0][0]
    line = {"metric": "coil-point field evals/s over the PrecisionFactor sweep (A+B+G, FP32c)",
            "value": head["fp32c"]["value"], "unit": UNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": head["fp32c"]["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (compensated) + f64", "data": "synthetic (seeded)",
            "config": {"workload": "coil group: 128 mixed coils, 262144 points in a 2 m cube, A+B+G, "
                                   "PrecisionFactor 1, 3, 5, 7, 9 (value: PF 5)", "coils": a.coils,
                       "points": npts, "l2": "flushed between timed launches (256 MiB write)"},
            "sweep": sweep, "gpu_launches": (field_launches(0, npts, 1, 0) + field_launches(1, npts, 1, 0)) * len(FIELDS) * a.steps * 5}
    print(json.dumps(line))


def bench_refine_sweep(a):
    """Cost curve of FP32_REFINED on the group workload: per field and refinement
    fraction, the share of (point, coil segment) pairs re-evaluated in FP64, the
    time of the whole evaluation and its error against FP64 (away from windings),
    beside plain FP32_COMPENSATED and FP64."""
    import ctypes
    import torch
    import ccoil_b200 as cc
    from ccoil_b200 import workloads
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rows, _ = workloads.group_config(coils=a.coils, points=1)
    coils = workloads.coils_from_rows(rows, a.pf)
    group = cc.CoilGroup(coils, cc.PrecisionFactor(a.pf))
    pts_host = workloads.points_cube(a.points, seed=1000 + 2)
    pts = torch.from_numpy(pts_host).to(dev)
    near, band = (torch.from_numpy(m).to(dev) for m in winding_masks(rows, pts_host))
    flush = flush_l2(torch, dev)
    L = cc.lib()
    default_fraction = L.ccoil_refine_fraction()
    fractions = [0.5, 0.2, 0.1, 0.05, 0.02]

    def timed(plan, out):
        for _ in range(max(a.warmup, 1)):
            plan(pts, out=out)
        ms = 0.0
        for _ in range(a.steps):
            flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            plan(pts, out=out)
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        return ms / a.steps

    curve = {}
    for name, f in FIELDS:
        w = 9 if f == 3 else 3
        away = ~band if f == 3 else ~near
        outs = {}
        res = {}
        for label, mode in (("fp64", cc.PrecisionMode.FP64), ("fp32c", cc.PrecisionMode.FP32_COMPENSATED)):
            plan = group.plan(f, mode)
            outs[label] = torch.empty((a.points, w), dtype=torch.float64, device=dev)
            res[label] = {"ms": timed(plan, outs[label])}
            plan.close()
        res["fp32c"]["err"] = rel_err_stats(outs["fp32c"], outs["fp64"], away)
        for fr in fractions:
            L.ccoil_set_refine_fraction(ctypes.c_double(fr))
            plan = group.plan(f, cc.PrecisionMode.FP32_REFINED)
            out = torch.empty((a.points, w), dtype=torch.float64, device=dev)
            ms = timed(plan, out)
            res["fraction_%g" % fr] = {"ms": ms, "refined_pairs_per_point": plan.refined_pairs() / a.points,
                                       "err": rel_err_stats(out, outs["fp64"], away),
                                       "speedup_vs_fp64": res["fp64"]["ms"] / ms}
            plan.close()
        res["fp32c"]["speedup_vs_fp64"] = res["fp64"]["ms"] / res["fp32c"]["ms"]
        curve[name] = res
    L.ccoil_set_refine_fraction(ctypes.c_double(default_fraction))
    pair_curve = refine_sweep_arrangements(a, cc, workloads, dev, L, default_fraction) if a.arrangements > 0 else None
    print(json.dumps({"workload": "refine-sweep", "default_fraction": default_fraction, "config": workload_config(a, 1),
                      "steps": a.steps, "coils": a.coils, "l2": "flushed between timed evaluations", "curve": curve,
                      "arrangements": pair_curve}))


def refine_sweep_arrangements(a, cc, workloads, dev, L, default_fraction):
    """The same curve for the pair arrangements: M and F/T in FP64, FP32_COMPENSATED
    and FP32_REFINED at each fraction, time and error against FP64 over all
    arrangements (F and T separately)."""
    import ctypes
    import torch
    from ccoil_b200.coil import pair_arrangements_device
    _, _, pstruct, sstruct, spre, pposes, sposes, _ = pair_setup(cc, workloads, a.arrangements, 3)
    dp = torch.from_numpy(pposes).to(dev)
    ds = torch.from_numpy(sposes).to(dev)
    fractions = [0.1, 0.03, 0.01, 0.005, 0.003, 0.0]  # 0: every node in FP64, no FP32 pass

    def timed(q, w, mode):
        out = torch.empty((a.arrangements, w), dtype=torch.float64, device=dev)
        for _ in range(max(a.warmup, 1)):
            pair_arrangements_device([pstruct], sstruct, [spre], dp, ds, q, out, precision_mode=mode)
        torch.cuda.synchronize()
        ms = 0.0
        for _ in range(a.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            pair_arrangements_device([pstruct], sstruct, [spre], dp, ds, q, out, precision_mode=mode)
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        return ms / a.steps, out

    def errors(name, got, ref):
        if name == "M":
            return {"M": rel_err_stats(got, ref)}
        return {"F": rel_err_stats(got[:, :3], ref[:, :3]), "T": rel_err_stats(got[:, 3:], ref[:, 3:])}

    curve = {}
    try:
        for name, q, w in (("M", 0, 1), ("FT", 1, 6)):
            ms64, ref = timed(q, w, cc.PrecisionMode.FP64)
            res = {"fp64": {"ms": ms64}}
            ms, out = timed(q, w, cc.PrecisionMode.FP32_COMPENSATED)
            res["fp32c"] = {"ms": ms, "speedup_vs_fp64": ms64 / ms, "err": errors(name, out, ref)}
            for fr in fractions:
                L.ccoil_set_refine_fraction(ctypes.c_double(fr))
                ms, out = timed(q, w, cc.PrecisionMode.FP32_REFINED)
                res["fraction_%g" % fr] = {"ms": ms, "speedup_vs_fp64": ms64 / ms, "err": errors(name, out, ref)}
            curve[name] = res
    finally:
        L.ccoil_set_refine_fraction(ctypes.c_double(default_fraction))
    return {"count": a.arrangements, "curve": curve}


def main():
    a = parse()
    if a.impl == "reference":
        reference_arm(a)
        return
    if a.workload == "batched":
        bench_batched(a)
        return
    if a.workload == "adjoint":
        bench_adjoint(a)
        return
    if a.workload == "pf-sweep":
        bench_pf_sweep(a)
        return
    if a.workload == "refine-sweep":
        bench_refine_sweep(a)
        return

    import torch
    import torch.distributed as dist

    import ccoil_b200 as cc
    from ccoil_b200 import opcount, workloads

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    from ccoil_b200 import distributed as D
    barrier = D.barrier

    def max_over_ranks(x):
        return D.max_over_ranks(x, dev)

    rows, _ = workloads.group_config(coils=a.coils, points=1)
    coils = workloads.coils_from_rows(rows, a.pf)
    group = cc.CoilGroup(coils, cc.PrecisionFactor(a.pf))
    pts_host = workloads.points_cube(a.points, seed=1000 + 2 + 7919 * rank)
    pts = torch.from_numpy(pts_host).to(dev)
    PM = cc.PrecisionMode
    # precision configurations: one mode per field.  fp32r is the one whose maximum
    # error away from windings stays below 1e-7: FP32_REFINED for A and B, whose FP32
    # errors the coils' cancellation magnifies past it, FP32_COMPENSATED for G, whose
    # FP32 error is two orders lower
    configs = {"fp64": {"A": PM.FP64, "B": PM.FP64, "G": PM.FP64},
               "fp32c": {"A": PM.FP32_COMPENSATED, "B": PM.FP32_COMPENSATED, "G": PM.FP32_COMPENSATED},
               "fp32r": {"A": PM.FP32_REFINED, "B": PM.FP32_REFINED, "G": PM.FP32_COMPENSATED}}
    selected = {"fp64": ["fp64"], "fp32c": ["fp32c"], "fp32r": ["fp32r"], "both": ["fp64", "fp32c"],
                "all": ["fp64", "fp32c", "fp32r"]}[a.precision]
    headline = "fp32r" if "fp32r" in selected else ("fp32c" if "fp32c" in selected else "fp64")
    # arrangement precisions: FP64, FP32_COMPENSATED and FP32_REFINED as selected
    modes = [m for m, key in ((PM.FP64, "fp64"), (PM.FP32_COMPENSATED, "fp32c"), (PM.FP32_REFINED, "fp32r"))
             if key in selected]

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    results = {}
    launches = {}
    for key in selected:
        cfg = configs[key]
        plans = {name: group.plan(f, cfg[name]) for name, f in FIELDS}
        launches[key] = sum(field_launches(cfg[name], a.points, plans[name].segment_count(), f)
                            for name, f in FIELDS)
        outs = {name: torch.empty((a.points, 9 if f == 3 else 3), dtype=torch.float64, device=dev)
                for name, f in FIELDS}
        for _ in range(max(a.warmup, 3)):
            for name, _f in FIELDS:
                plans[name](pts, out=outs[name])
        torch.cuda.synchronize()
        field_ms = {name: 0.0 for name, _ in FIELDS}
        step_ms = 0.0
        barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            for _ in range(a.steps):
                flush.fill_(1)  # evict L2 between steps (not timed)
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(FIELDS) + 1)]
                ev[0].record()
                for i, (name, _f) in enumerate(FIELDS):
                    plans[name](pts, out=outs[name])
                    ev[i + 1].record()
                torch.cuda.synchronize()
                for i, (name, _f) in enumerate(FIELDS):
                    field_ms[name] += ev[i].elapsed_time(ev[i + 1])
                step_ms += ev[0].elapsed_time(ev[-1])
        torch.cuda.synchronize()
        barrier()
        step_ms = max_over_ranks(step_ms / a.steps)
        field_ms = {k: max_over_ranks(v / a.steps) for k, v in field_ms.items()}
        results[key] = {"step_ms": step_ms, "field_ms": field_ms, "clocks": clk.summary(),
                        "outs": {k: v.clone() for k, v in outs.items()}}

        # end to end through the public API: pinned host points in, pinned host results out
        pin_pts = torch.from_numpy(pts_host).pin_memory()
        pin_out = {name: torch.empty((a.points, 9 if f == 3 else 3), dtype=torch.float64).pin_memory()
                   for name, f in FIELDS}
        plans["A"](pin_pts.numpy(), out=pin_out["A"].numpy())  # warm the staging buffers
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for _ in range(a.steps):
            for name, _f in FIELDS:
                plans[name](pin_pts.numpy(), out=pin_out[name].numpy())
        e2e_s = max_over_ranks((time.perf_counter() - t0) / a.steps)
        results[key]["e2e_s"] = e2e_s
        for p in plans.values():
            p.close()
        # one-shot calls, the reference glue's pattern (ccoil_compute_fields): every call
        # builds and uploads the node tables, copies the points in and the results out
        api = {"A": group.compute_all_A_potential_vectors, "B": group.compute_all_B_field_vectors,
               "G": group.compute_all_B_gradient_matrices}
        api["A"](pin_pts.numpy(), precision_mode=cfg["A"])
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for _ in range(a.steps):
            for name, _f in FIELDS:
                api[name](pin_pts.numpy(), precision_mode=cfg[name])
        results[key]["e2e_oneshot_s"] = max_over_ranks((time.perf_counter() - t0) / a.steps)

    units_per_step = len(FIELDS) * a.coils * a.points * world
    r = results[headline]
    value = units_per_step / (r["step_ms"] * 1e-3)
    e2e_value = units_per_step / r["e2e_s"]
    # the roofline's kernel: the longest single launch, the FP32-compensated field
    # kernel of the slowest field (FP32_REFINED splits its work over chunks and passes)
    roof_key = "fp32c" if "fp32c" in results else headline
    headline_mode = 0 if roof_key == "fp64" else 1
    rr = results[roof_key]

    # roofline of the dominant kernel: its algorithmic work (the reference's operations
    # per node, each add, multiply, divide, square root or logarithm one flop) over its
    # CUDA-event time, against the measured FMA peak (2 flops per FMA) of the pipe it
    # runs on; the instruction-issue and MUFU models are reported beside it
    rates = ctypes_rates(cc)
    dom = max(rr["field_ms"], key=rr["field_ms"].get)
    fidx = dict(FIELDS)[dom]
    t_dom = rr["field_ms"][dom] * 1e-3
    flops_launch = opcount.group_flops_per_point(fidx, coils) * a.points
    model = {"algorithmic_flops_per_launch": flops_launch}
    if rates is None:
        bound, achieved, peak, unit = "unmeasured", None, None, "TFLOP/s"
    elif headline_mode == 0:
        bound, unit = "fp64-pipe", "TFLOP/s"
        achieved, peak = flops_launch / t_dom / 1e12, 2.0 * rates[0] / 1e12
        slots = opcount.fp64_slots_per_point(fidx, coils, rates) * a.points
        model.update({"fp64_pipe_slots_per_launch": slots, "fp64_pipe_model_frac": slots / t_dom / rates[0],
                      "dfma_slots_per_op": {"div": rates[0] / rates[1], "sqrt": rates[0] / rates[2],
                                            "log": rates[0] / rates[3]}})
    else:
        bound, unit = "fp32-pipe", "TFLOP/s"
        achieved, peak = flops_launch / t_dom / 1e12, 2.0 * rates[4] / 1e12
    clk = r["clocks"] or {}
    if clk.get("sm_mhz"):
        # nominal B200 per-SM rates at the sampled clock: FP64 64 and FP32 128 FMA per clock,
        # MUFU 16 per clock, 148 SMs
        f = clk["sm_mhz"] * 1e6
        model["nominal_at_sampled_clock"] = {"fp64_fma_tflops": 2 * 148 * 64 * f / 1e12,
                                             "fp32_fma_tflops": 2 * 148 * 128 * f / 1e12,
                                             "mufu_tops": 148 * 16 * f / 1e12, "sm_mhz": clk["sm_mhz"]}
    prof = read_profile(dom, headline_mode)
    traffic = prof.get("traffic") if prof else None

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": r["step_ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if headline_mode == 0 else "f32 (compensated) + f64",
            "data": "synthetic (seeded)", "config": workload_config(a, world),
            "precision_mode": {"fp64": "fp64", "fp32c": "fp32c (FP32_COMPENSATED, every field)",
                               "fp32r": "fp32r: FP32_REFINED for A and B (fraction %g), FP32_COMPENSATED for G"
                                        % cc.lib().ccoil_refine_fraction()}[headline],
            "per_field_ms": r["field_ms"],
            "node_evals_per_s": opcount.group_nodes_per_point(coils) * a.points * world * len(FIELDS) /
            (r["step_ms"] * 1e-3),
            "gpu_launches": a.steps * launches[headline],
            "clocks": r["clocks"],
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": len(FIELDS) * a.points * 24,
                    "d2h_bytes_per_step": sum(a.points * 8 * (9 if f == 3 else 3) for _, f in FIELDS),
                    "path": "prepared plans (ccoil_field_plan_execute), pinned host points and results"},
            "e2e_one_shot": {"value": units_per_step / r["e2e_oneshot_s"], "unit": UNIT,
                             "path": "CoilGroup.compute_all_* (ccoil_compute_fields): node tables built and "
                                     "uploaded, points copied in and results out on every call"},
            "roofline": {"bound": bound, "kernel": "field %s, %s" % (dom, configs[roof_key][dom].name),
                         "achieved": achieved, "peak": peak,
                         "unit": unit, "frac": (achieved / peak) if peak else None, "traffic": traffic,
                         "peak_source": "measured on this GPU by ccoil_measure_op_rates (FMA = 2 flops); "
                                        "achieved counts the reference's operations, one flop each",
                         "model": model,
                         "ncu": prof,
                         "rates_measured": None if rates is None else {
                             "fp64_fma_tflops": 2 * rates[0] / 1e12, "fp32_fma_tflops": 2 * rates[4] / 1e12,
                             "mufu_tops": rates[5] / 1e12, "ddiv_gops": rates[1] / 1e9,
                             "dsqrt_gops": rates[2] / 1e9, "dlog_gops": rates[3] / 1e9}}}
    for key in selected:
        rk = results[key]
        line[key] = {"value": units_per_step / (rk["step_ms"] * 1e-3), "ms_per_step": rk["step_ms"],
                     "per_field_ms": rk["field_ms"], "e2e": units_per_step / rk["e2e_s"],
                     "e2e_one_shot": units_per_step / rk["e2e_oneshot_s"],
                     "modes": {name: configs[key][name].name for name, _f in FIELDS}}
    if "fp64" in results:
        r64 = results["fp64"]
        near, band = (torch.from_numpy(m).to(dev) for m in winding_masks(rows, pts_host))
        for key in ("fp32c", "fp32r"):
            if key not in results:
                continue
            line[key + "_speedup_vs_fp64"] = r64["step_ms"] / results[key]["step_ms"]
            errs = {"definition": "norm-wise relative error per point, denominator floored at 1e-3 x the batch's "
                                  "largest FP64 norm; 'away' = outside every coil's winding box inflated by 0.1 R "
                                  "(for G also outside every coil's radial band [0.9 R, R + a + 0.1 R], where the "
                                  "reference's FP64 gradient is itself ill-conditioned)",
                    "away_fraction": {"A_B": float((~near).float().mean()), "G": float((~band).float().mean())}}
            for name, f in FIELDS:
                away = ~band if f == 3 else ~near
                errs[name] = {"all": rel_err_stats(results[key]["outs"][name], r64["outs"][name]),
                              "away": rel_err_stats(results[key]["outs"][name], r64["outs"][name], away)}
            line[key + "_rel_err_vs_fp64"] = errs
    if a.arrangements > 0:
        arr = bench_arrangements(a, cc, workloads, dev, rank, max_over_ranks, barrier, modes)
        head = "fp32c" if "fp32c" in arr else ("fp32r" if "fp32r" in arr else "fp64")
        line["arrangements"] = {"workload": "RECTANGULAR primary (0.1, 0.05, 0.1 m, N=200) x THIN secondary "
                                            "(0.05, 0, 0.2 m, N=100), %d arrangements per GPU, offsets in a "
                                            "0.6 m cube, random orientations, 5%% near-coaxial, PF 5"
                                            % a.arrangements,
                                "precision_mode": head,
                                "M_arrangements_per_s": arr[head]["M"]["arrangements_per_s"] * world,
                                "FT_arrangements_per_s": arr[head]["FT"]["arrangements_per_s"] * world,
                                "secondary_nodes": arr["secondary_nodes"], "primary_nodes": arr["primary_nodes"],
                                "z_axis_cases": arr[head]["M"]["z_axis_cases"]}
        for key in ("fp64", "fp32c", "fp32r"):
            if key in arr:
                line["arrangements"][key] = {
                    "M_arrangements_per_s": arr[key]["M"]["arrangements_per_s"] * world,
                    "FT_arrangements_per_s": arr[key]["FT"]["arrangements_per_s"] * world,
                    "M_ms": arr[key]["M"]["ms"], "FT_ms": arr[key]["FT"]["ms"]}
            if key + "_errors" in arr:
                line["arrangements"][key + "_speedup_vs_fp64"] = {
                    q: arr["fp64"][q]["ms"] / arr[key][q]["ms"] for q in ("M", "FT")}
                line["arrangements"][key + "_rel_err_vs_fp64"] = arr[key + "_errors"]
        if "at_1e-7" in arr:
            at = arr["at_1e-7"]
            line["arrangements"]["at_1e-7"] = {
                "M": dict(at["M"], arrangements_per_s=at["M"]["arrangements_per_s"] * world),
                "FT": dict(at["FT"], arrangements_per_s=at["FT"]["arrangements_per_s"] * world),
                "speedup_vs_fp64": {q: arr["fp64"][q]["ms"] / at[q]["ms"] for q in ("M", "FT")}}
        elif "fp64" in arr:
            line["arrangements"]["at_1e-7"] = {
                "precision_mode": "fp64",
                "M_arrangements_per_s": arr["fp64"]["M"]["arrangements_per_s"] * world,
                "FT_arrangements_per_s": arr["fp64"]["FT"]["arrangements_per_s"] * world}
        if rates is not None and "fp64" in arr:
            # FP64 pipe model of the arrangement kernels: every (secondary node, primary
            # node) pair evaluates the reference's A (M) or B (F/T) fast node
            pairs_per_arr = arr["secondary_nodes"] * arr["primary_nodes"]
            roof = {}
            for q, fidx in (("M", 0), ("FT", 1)):
                am, dv, sq, lg = opcount.OPS_PER_NODE_64[(fidx, True)]
                slots = pairs_per_arr * (am + dv * rates[0] / rates[1] + sq * rates[0] / rates[2] +
                                         lg * rates[0] / rates[3]) * a.arrangements
                t = arr["fp64"][q]["ms"] * 1e-3
                roof[q] = {"achieved": 2.0 * slots / t / 1e12, "peak": 2.0 * rates[0] / 1e12, "unit": "TFLOP/s",
                           "frac": slots / t / rates[0]}
            line["arrangements"]["fp64_roofline"] = roof
        # timed launches: M and F/T per precision mode, and per candidate of the 1e-7 configuration
        line["gpu_launches"] += 2 * a.steps * (len(modes) + (2 if "at_1e-7" in arr else 0))
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        rate, cores, dt, desc = cpu_reference_rate(a, a.cpu_sample_points)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                                "sample": desc, "seconds": dt}
        if a.arrangements > 0 and a.cpu_sample_arrangements > 0:
            arate, acores, adt = cpu_arrangement_rate(a, a.cpu_sample_arrangements)
            line["cpu_baseline"]["M_arrangements_per_s"] = arate
            line["cpu_baseline"]["arrangement_sample"] = ("%d arrangements of the pair workload, "
                                                          "Coil::computeAllMutualInductanceArrangements CPU_MT"
                                                          % a.cpu_sample_arrangements)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def ctypes_rates(cc):
    import ctypes
    L = cc.lib()
    L.ccoil_measure_op_rates.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    v = (ctypes.c_double * 6)()
    if L.ccoil_measure_op_rates(v, 6) != 0:
        return None
    return list(v)


def field_launches(mode, points, segments, field):
    """Kernel launches of one field-plan evaluation: FP64 one field kernel; FP32c the field
    kernel and its near-field FP64 pass, and from 16,384 to 2^30 points also the point
    ordering (bounds, Morton keys, the radix sort's 6 kernels, gather) and the scatter of
    the results; FP32_REFINED per chunk of points (contributions of at most 4 GiB, at most
    2^28 listed pairs) the field kernel, the near-field pass and the selection (count,
    scan, select) and FP64 pair passes."""
    mode = int(mode)
    if mode == 0:
        return 1
    ordering = 10 if (1 << 14) <= points <= (1 << 30) else 0
    if mode == 1:
        return 2 + ordering
    width = 9 if field == 3 else 3
    per_chunk = min((1 << 32) // (segments * width * 8), (1 << 28) // segments)
    chunks = -(-points // max(1, per_chunk))
    return ordering + 6 * chunks


def read_profile(field, mode):
    """The committed ncu figures of the field kernel (DRAM traffic per 2^20-point
    launch, pipe utilisation), or None."""
    path = os.path.join(ROOT, "profiles", "kernels.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get("%s_%s" % ("fp64" if mode == 0 else "fp32c", field))
    except Exception:
        return None


if __name__ == "__main__":
    main()
