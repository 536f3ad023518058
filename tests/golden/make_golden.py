"""Generates tests/golden/golden.npz from the reference's own CPU code.

Run in a container where the reference is mounted and oracle/_ref is built
(`make -C oracle ref`):

    python tests/golden/make_golden.py

Every value comes from the compiled reference (oracle/_ref/libccoil_ref.so,
CPU_ST, double precision).  The cases restate the deterministic geometries of
the reference's print-tests and comparisons, plus seeded cases with the
benchmark configurations' shapes:

  test_fields     src/Test/Other/TestFields.cxx:5-77 (10-coil group, 20 points, PF 4)
  arrangements    src/Test/MInductanceAndForce/TestArrangements.cxx:5-107 (20 configs, PF 5)
  group_arr       src/Test/MInductanceAndForce/TestArrangements.cxx:109-217 (secondary = member 0)
  comp_precision  src/Compare/Other/CompMiscellaneous.cxx:8-50 (Coil(0.03, 0.03, 0.12, 3600), PF 6;
                  the points follow vec3::Vector3::getFromSphericalCoords as the reference
                  defines it, i.e. z = r cos(phi) with phi = 0)
  rotation        src/Test/Other/TestMiscellaneous.cxx:32-72 (on-axis points, rotated coil)
  parallel_axes   data/values_MInductance_general.txt inputs as read by
                  src/Compare/MInductanceAndForce/CompMInductanceGeneral.cxx:138-160
  single_rect     the single RECTANGULAR coil configuration, 512 points, PF 5
  group_mixed     12 mixed-type coils, 96 points, PF 1, 3, 5, 7, 9
  pairs           24 RECTANGULAR/THIN arrangements of the pair configuration, PF 5
  z_axis          coaxial arrangements of every coil-type combination (the reference's
                  z-axis formulas, src/Coil/MInductance/CalculateMInductanceZAxis.cxx,
                  src/Coil/ForceAndTorque/CalculateForceZAxis.cxx), a coaxial group, and
                  self inductances (CalculateMInductanceZAxis.cxx:233-319)
  precision       precision arguments of 400 seeded coils at 6 PrecisionFactors, CPU and GPU
  pair_precision  pair arguments of 100 seeded pairs, CPU and pure-GPU
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "c-coil_b200"))

from oracle import Reference, coil_row  # noqa: E402
from ccoil_b200 import workloads  # noqa: E402

# the reference checkout: CCOIL_REFERENCE (default: where the build container mounts it)
REF_ROOT = os.environ.get("CCOIL_REFERENCE", "/root/reference")
REF_DATA = os.path.join(REF_ROOT, "data", "values_MInductance_general.txt")


def main():
    R = Reference()
    g = {}

    # --- TestFields: 10 coils along z, 20 points, PF 4 ------------------------------------
    coils = np.array([coil_row(0.1, 0.1, 0.1, 10000, 10.0, 50.0, (0.0, 0.0, 0.2 * i)) for i in range(10)])
    pts = np.array([[0.5, 0.0, 0.1 * i] for i in range(20)])
    g["test_fields_coils"] = coils
    g["test_fields_points"] = pts
    for q, name in enumerate("ABEG"):
        g["test_fields_" + name] = R.group_fields(coils, pts, q, pf=4.0)

    # --- TestArrangements: prim = sec = Coil(0.1, 0.1, 0.1, 10000), 20 configs, PF 5 -------
    n = 20
    prim = coil_row(0.1, 0.1, 0.1, 10000)
    sec = coil_row(0.1, 0.1, 0.1, 10000)
    ppos = np.zeros((n, 3))
    spos = np.array([[0.0, 0.1, 0.2 + 0.01 * i] for i in range(n)])
    py, pz, sy, sz = np.full(n, 0.5), np.full(n, 0.5), np.full(n, 0.6), np.full(n, 0.6)
    g["arr_prim"], g["arr_sec"] = prim, sec
    g["arr_prim_pos"], g["arr_sec_pos"] = ppos, spos
    g["arr_angles"] = np.stack([py, pz, sy, sz])
    g["arr_M"] = R.m_arrangements(prim, sec, ppos, spos, py, pz, sy, sz, pf=5.0)
    g["arr_FT"] = R.ft_arrangements(prim, sec, ppos, spos, py, pz, sy, sz, pf=5.0)

    # --- group arrangements: 10 coils (I = 10) along z, secondary = member 0, PF 4 ---------
    gcoils = np.array([coil_row(0.1, 0.1, 0.1, 10000, 10.0, 50.0, (0.0, 0.0, 0.2 * i)) for i in range(10)])
    gspos = np.array([[0.5, 0.0, 0.1 * i] for i in range(n)])
    gsy, gsz = np.full(n, 0.5), np.full(n, 0.6)
    g["garr_coils"], g["garr_sec_pos"], g["garr_angles"] = gcoils, gspos, np.stack([gsy, gsz])
    g["garr_M"] = R.group_m_arrangements(gcoils, gcoils[0], gspos, gsy, gsz, pf=4.0, sec_member=0)
    g["garr_FT"] = R.group_ft_arrangements(gcoils, gcoils[0], gspos, gsy, gsz, pf=4.0, sec_member=0)

    # --- CompMiscellaneous::fieldsPrecisionCPUvsGPU, 200 of its 2000 points ---------------
    ccoil = coil_row(0.03, 0.03, 0.12, 3600, 1.0, 50.0)
    r = 0.075
    th = np.arange(0, 2000, 10) * np.pi / 2000
    cpts = np.stack([r * np.sin(th), np.zeros_like(th), np.full_like(th, r * np.cos(0.0))], axis=1)
    g["comp_coil"], g["comp_points"] = ccoil, cpts
    g["comp_A"] = R.coil_fields(ccoil, cpts, 0, pf=6.0)
    g["comp_B"] = R.coil_fields(ccoil, cpts, 1, pf=6.0)

    # --- TestMiscellaneous::testCoilPositionAndRotation ------------------------------------
    rc1 = coil_row(0.03, 0.03, 0.12, 3600)
    rc3 = coil_row(0.03, 0.03, 0.12, 3600, 1.0, 50.0, (0.0, 0.0, 0.0), np.pi / 2, np.pi / 2)
    p1 = np.array([[0.0, 0.0, 0.001 * i] for i in range(100)])
    p2 = np.array([[0.0, 0.001 * i, 0.0] for i in range(100)])
    g["rot_coil1"], g["rot_coil3"], g["rot_p1"], g["rot_p2"] = rc1, rc3, p1, p2
    g["rot_B1"] = R.coil_fields(rc1, p1, 1, pf=5.0)
    g["rot_B3"] = R.coil_fields(rc3, p2, 1, pf=5.0)
    g["rot_G1"] = R.coil_fields(rc1, p1, 3, pf=5.0)

    # --- parallel axes mutual inductance (data file inputs), PF 3 and 5 --------------------
    if os.path.exists(REF_DATA):
        rows = np.loadtxt(REF_DATA)
        pa_prim, pa_sec, pa_M = [], [], []
        for row in rows:
            R1, a1, b1, N1, R2, a2, b2, N2, dz, dr = row
            p_ = coil_row(R1, a1, b1, int(N1))
            s_ = coil_row(R2, a2, b2, int(N2), 1.0, 50.0, (dr, 0.0, dz))
            pa_prim.append(p_)
            pa_sec.append(s_)
            pa_M.append([R.mutual_inductance(p_, s_, pf=pf) for pf in (3.0, 5.0)])
        g["pa_prim"], g["pa_sec"], g["pa_M"] = np.array(pa_prim), np.array(pa_sec), np.array(pa_M)

    # --- single RECTANGULAR coil, 512 points, PF 5 ------------------------------------------
    c1, p1 = workloads.single_rect_config(points=512, seed=11)
    g["single_coil"], g["single_points"] = c1, p1
    for q, name in enumerate("ABEG"):
        g["single_" + name] = R.coil_fields(c1[0], p1, q, pf=5.0)

    # --- mixed group at several PF ----------------------------------------------------------
    mc = workloads.coil_rows_mixed(12, seed=21)
    mp = workloads.points_cube(96, seed=22)
    g["mixed_coils"], g["mixed_points"] = mc, mp
    for pf in (1, 3, 5, 7, 9):
        for q, name in enumerate("ABEG"):
            g["mixed_%s_pf%d" % (name, pf)] = R.group_fields(mc, mp, q, pf=float(pf))

    # --- pair configuration arrangements (general and near-coaxial) ------------------------
    prim, sec, ppos, spos, py, pz, sy, sz = workloads.pair_config(arrangements=24, seed=31, coaxial_fraction=0.0)
    g["pairs_prim"], g["pairs_sec"] = prim, sec
    g["pairs_prim_pos"], g["pairs_sec_pos"] = ppos, spos
    g["pairs_angles"] = np.stack([py, pz, sy, sz])
    g["pairs_M"] = R.m_arrangements(prim, sec, ppos, spos, py, pz, sy, sz, pf=5.0)
    g["pairs_FT"] = R.ft_arrangements(prim, sec, ppos, spos, py, pz, sy, sz, pf=5.0)

    # --- coaxial pairs: the reference's z-axis formulas (every coil-type combination) ------------
    # 6 arrangements per combination: 4 coaxial (both y angles 0, centres on the z axis, any z
    # angles) and 2 off-axis ones that take the general formula; PF 3 and 5
    ztypes = [(0.1, 0.05, 0.1, 200), (0.08, 0.0, 0.12, 150), (0.12, 0.04, 0.0, 120), (0.06, 0.0, 0.0, 80)]
    zr = np.random.default_rng(51)
    zp_, zs_, zpp, zsp, zang, zm3, zm5, zft = [], [], [], [], [], [], [], []
    for pd in ztypes:
        for sd in ztypes:
            prim_row = coil_row(*pd[:3], pd[3], 2.0)
            sec_row = coil_row(*sd[:3], sd[3], 3.0)
            ppos = np.zeros((6, 3))
            ppos[:, 2] = zr.uniform(-0.1, 0.1, 6)
            dz = zr.choice([-1.0, 1.0], 6) * zr.uniform(0.15, 0.4, 6)
            spos = ppos + np.stack([np.zeros(6), np.zeros(6), dz], axis=1)
            spos[4:, 0] += zr.uniform(0.01, 0.05, 2)
            py, sy = np.zeros(6), np.zeros(6)
            sy[5] = 0.3
            pz, sz = zr.uniform(0, 2 * np.pi, 6), zr.uniform(0, 2 * np.pi, 6)
            zp_.append(prim_row)
            zs_.append(sec_row)
            zpp.append(ppos)
            zsp.append(spos)
            zang.append(np.stack([py, pz, sy, sz]))
            zm3.append(R.m_arrangements(prim_row, sec_row, ppos, spos, py, pz, sy, sz, pf=3.0))
            zm5.append(R.m_arrangements(prim_row, sec_row, ppos, spos, py, pz, sy, sz, pf=5.0))
            zft.append(R.ft_arrangements(prim_row, sec_row, ppos, spos, py, pz, sy, sz, pf=5.0))
    g["zax_prim"], g["zax_sec"], g["zax_prim_pos"], g["zax_sec_pos"] = map(np.array, (zp_, zs_, zpp, zsp))
    g["zax_angles"], g["zax_M_pf3"], g["zax_M_pf5"], g["zax_FT_pf5"] = map(np.array, (zang, zm3, zm5, zft))

    # coaxial group: 4 stacked coils of different types, a RECTANGULAR secondary moving along
    # the axis (first 5 arrangements) and off it (last 3), PF 4
    zg = np.array([coil_row(*ztypes[i][:3], ztypes[i][3], 1.5, 0.0, (0.0, 0.0, 0.3 * i - 0.45)) for i in range(4)])
    zsec = coil_row(0.05, 0.02, 0.06, 90, 2.5)
    zgs = np.zeros((8, 3))
    zgs[:, 2] = [-0.75, -0.6, 0.6, 0.75, 0.9, -0.7, 0.65, 0.8]
    zgs[5:, 1] = [0.02, 0.04, 0.01]
    zgy = np.zeros(8)
    zgz = np.linspace(0.0, 1.0, 8)
    g["zgrp_coils"], g["zgrp_sec"], g["zgrp_sec_pos"], g["zgrp_angles"] = zg, zsec, zgs, np.stack([zgy, zgz])
    g["zgrp_M"] = R.group_m_arrangements(zg, zsec, zgs, zgy, zgz, pf=4.0)
    g["zgrp_FT"] = R.group_ft_arrangements(zg, zsec, zgs, zgy, zgz, pf=4.0)

    # self inductance (Coil::computeAndSetSelfInductance) of RECTANGULAR, THIN and FLAT coils
    sic = np.array([coil_row(0.1, 0.05, 0.1, 200), coil_row(0.03, 0.03, 0.12, 3600), coil_row(0.08, 0.0, 0.12, 150),
                    coil_row(0.12, 0.04, 0.0, 120), coil_row(0.5, 0.1, 0.05, 10)])
    g["self_coils"] = sic
    g["self_L"] = np.array([[R.self_inductance(c, pf=pf) for pf in (3.0, 5.0)] for c in sic])

    # --- precision arguments ------------------------------------------------------------------
    rng = np.random.default_rng(41)
    pc, pfs, cpu, gpu = [], [], [], []
    for _ in range(400):
        Rr = rng.uniform(0.005, 0.5)
        a = 0.0 if rng.uniform() < 0.3 else rng.uniform(0, 0.3)
        b = 0.0 if rng.uniform() < 0.3 else rng.uniform(0, 0.3)
        c = coil_row(Rr, a, b, int(rng.integers(1, 2000)))
        for pf in (1.0, 2.5, 5.0, 7.0, 9.0, 12.0):
            pc.append(c)
            pfs.append(pf)
            cpu.append(R.precision_args(c, pf, gpu=False))
            gpu.append(R.precision_args(c, pf, gpu=True))
    g["prec_coils"], g["prec_pf"] = np.array(pc), np.array(pfs)
    g["prec_cpu"], g["prec_gpu"] = np.array(cpu), np.array(gpu)

    pp, ps, ppf, pcpu, pgpu = [], [], [], [], []
    for _ in range(100):
        rows = workloads.coil_rows_mixed(2, seed=int(rng.integers(1 << 30)))
        for pf in (1.0, 5.0, 9.0):
            pp.append(rows[0])
            ps.append(rows[1])
            ppf.append(pf)
            pcpu.append(R.pair_args(rows[0], rows[1], pf, gpu=False))
            pgpu.append(R.pair_args(rows[0], rows[1], pf, gpu=True, pure_gpu=True))
    g["pprec_prim"], g["pprec_sec"], g["pprec_pf"] = np.array(pp), np.array(ps), np.array(ppf)
    g["pprec_cpu"], g["pprec_gpu"] = np.array(pcpu), np.array(pgpu)

    out = os.path.join(HERE, "golden.npz")
    np.savez_compressed(out, **g)
    print(out, os.path.getsize(out), "bytes,", len(g), "arrays")


if __name__ == "__main__":
    main()
