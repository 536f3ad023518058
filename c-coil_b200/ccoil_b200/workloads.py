"""Seeded synthetic workloads with the shapes and value distributions of the
benchmark configurations (no public dataset is involved).

Coils are returned as rows {R, a, b, N, I, f, x, y, z, yAxisAngle, zAxisAngle}
(numpy float64, one row per coil); `coils_from_rows` turns them into Coil objects.
"""
import numpy as np

TYPE_NAMES = ("RECTANGULAR", "THIN", "FLAT", "FILAMENT")


def rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def coil_rows_mixed(count, seed, types=None, centre_box=1.0, frequency=50.0):
    """Coil group: type = i mod 4 (or the given list), R ~ U[0.02, 0.3], a, b ~ U[0, 0.1]
    with the type's thin dimensions set to 0, N ~ U{1..500}, I ~ U[-5, 5], centres
    uniform in [0, centre_box]^3, axis uniform on the sphere
    (yAxisAngle = arccos(1 - 2U), zAxisAngle = 2 pi U)."""
    g = rng(seed)
    rows = np.zeros((count, 11))
    for i in range(count):
        t = (i % 4) if types is None else types[i % len(types)]
        R = g.uniform(0.02, 0.3)
        a = g.uniform(0.0, 0.1)
        b = g.uniform(0.0, 0.1)
        if t in (1, 3):
            a = 0.0
        if t in (2, 3):
            b = 0.0
        N = int(g.integers(1, 501))
        I = g.uniform(-5.0, 5.0)
        pos = g.uniform(0.0, centre_box, 3)
        ya = np.arccos(1.0 - 2.0 * g.uniform())
        za = 2.0 * np.pi * g.uniform()
        rows[i] = [R, a, b, N, I, frequency, pos[0], pos[1], pos[2], ya, za]
    return rows


def points_cube(count, seed, half=1.0):
    return rng(seed).uniform(-half, half, (count, 3))


def points_cylinder(count, seed, radius=0.5, half_height=0.5):
    """r = radius sqrt(U), phi = 2 pi U, z = U[-h, h]."""
    g = rng(seed)
    r = radius * np.sqrt(g.uniform(size=count))
    phi = 2.0 * np.pi * g.uniform(size=count)
    z = g.uniform(-half_height, half_height, count)
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


def points_ball(count, seed, radius=0.05):
    g = rng(seed)
    v = g.normal(size=(count, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v * radius * np.cbrt(g.uniform(size=(count, 1)))


def single_rect_config(points=65536, seed=1):
    """One RECTANGULAR coil R = a = b = 0.1 m, N = 100, I = 1 A at the origin; points in
    the cylinder r <= 0.5 m, |z| <= 0.5 m; PrecisionFactor 5."""
    coil = np.array([[0.1, 0.1, 0.1, 100, 1.0, 50.0, 0, 0, 0, 0, 0]], dtype=np.float64)
    return coil, points_cylinder(points, seed)


def group_config(coils=128, points=1 << 20, seed=2):
    """128 mixed coils in a 1 m cube, points uniform in the 2 m cube."""
    return coil_rows_mixed(coils, seed), points_cube(points, seed + 1000)


def pair_config(arrangements=1 << 18, seed=3, coaxial_fraction=0.05):
    """Primary RECTANGULAR (0.1, 0.05, 0.1, N=200), secondary THIN (0.05, 0, 0.2, N=100);
    offsets uniform in a 0.6 m cube, random orientations; a fraction of near-coaxial
    overlapping pairs (offset along the primary axis by a few mm, angles < 1e-3)."""
    g = rng(seed)
    prim = np.array([0.1, 0.05, 0.1, 200, 1.0, 50.0, 0, 0, 0, 0, 0], dtype=np.float64)
    sec = np.array([0.05, 0.0, 0.2, 100, 1.0, 50.0, 0, 0, 0, 0, 0], dtype=np.float64)
    n = arrangements
    prim_pos = np.zeros((n, 3))
    sec_pos = g.uniform(-0.3, 0.3, (n, 3))
    py = np.zeros(n)
    pz = np.zeros(n)
    sy = np.arccos(1.0 - 2.0 * g.uniform(size=n))
    sz = 2.0 * np.pi * g.uniform(size=n)
    m = int(round(coaxial_fraction * n))
    if m:
        idx = g.choice(n, m, replace=False)
        sec_pos[idx, 0] = g.uniform(-2e-3, 2e-3, m)
        sec_pos[idx, 1] = g.uniform(-2e-3, 2e-3, m)
        sec_pos[idx, 2] = g.uniform(-5e-3, 5e-3, m)
        sy[idx] = g.uniform(0.0, 1e-3, m)
    return prim, sec, prim_pos, sec_pos, py, pz, sy, sz


def batched_config(groups=2048, seed=4, min_points=256, max_points=65536, max_group=256):
    """Independent systems: group size log-uniform in [1, 256], point count log-uniform
    in [256, 65536], coil parameters as in the group configuration."""
    g = rng(seed)
    sizes = np.floor(np.exp(g.uniform(0.0, np.log(max_group), groups))).astype(int)
    sizes = np.clip(sizes, 1, max_group)
    npts = np.floor(np.exp(g.uniform(np.log(min_points), np.log(max_points), groups))).astype(int)
    systems = []
    for i in range(groups):
        rows = coil_rows_mixed(int(sizes[i]), seed * 100003 + i)
        pts = points_cube(int(npts[i]), seed * 100019 + i)
        systems.append((rows, pts))
    return systems


def adjoint_config(coils=64, points=4096, seed=5, types=(0,)):
    """64 RECTANGULAR coils (parameters as the group configuration), points in a ball of 5 cm;
    `types` cycles other coil types instead."""
    return coil_rows_mixed(coils, seed, types=list(types)), points_ball(points, seed + 7)


def coils_from_rows(rows, precision_factor=5.0):
    from .coil import Coil, PrecisionFactor
    out = []
    for r in np.atleast_2d(rows):
        out.append(Coil(r[0], r[1], r[2], int(r[3]), r[4], r[5], PrecisionFactor(precision_factor), 8,
                        (r[6], r[7], r[8]), r[9], r[10]))
    return out
