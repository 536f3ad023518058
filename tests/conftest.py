import os
import re
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "c-coil_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.npz")
HEADER = os.path.join(ROOT, "include", "ccoil_gpu.h")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _cuda_available()


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle, ORACLE_SO
    if not os.path.exists(ORACLE_SO):
        import subprocess
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True, capture_output=True)
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference
    if not Reference.available():
        pytest.skip("oracle/_ref/libccoil_ref.so not built (needs the reference sources)")
    return Reference()


@pytest.fixture(scope="session")
def ccoil():
    import ccoil_b200
    ccoil_b200.lib()  # fails loudly if the library is not built
    return ccoil_b200


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|long long|const char \*)\s*\**\s*(\w+)\s*\(", text, flags=re.M)))


def rel_err(a, b, floor=0.0, floor_frac=1e-3):
    """Norm-wise relative error per row (vectors and flattened matrices).

    The denominator is floored at floor_frac times the largest reference norm in
    the batch, so points where the field vanishes by symmetry (A on the axis) are
    judged against the batch's scale instead of against rounding noise."""
    a = np.asarray(a).reshape(len(a), -1)
    b = np.asarray(b).reshape(len(b), -1)
    num = np.linalg.norm(a - b, axis=1)
    nb = np.linalg.norm(b, axis=1)
    den = np.maximum(nb, max(floor, floor_frac * (nb.max() if nb.size else 0.0)))
    with np.errstate(invalid="ignore", divide="ignore"):
        e = np.where(den > 0, num / den, num)
    return e


def coil_frame(row, pts):
    """(r, z) of points in the frame of a coil row {R, a, b, N, I, f, x, y, z, yA, zA}."""
    yA, zA = row[9], row[10]
    cY, sY, cZ, sZ = np.cos(yA), np.sin(yA), np.cos(zA), np.sin(zA)
    Ti = np.array([[cZ * cZ * cY - sZ * sZ, sZ * cZ * cY + sZ * cZ, -cZ * sY],
                   [-sZ * cZ * cY - sZ * cZ, cZ * cZ - sZ * sZ * cY, sZ * sY],
                   [sY * cZ, sY * sZ, cY]])
    d = (np.asarray(pts) - row[6:9]) @ Ti.T
    return np.hypot(d[:, 0], d[:, 1]), d[:, 2]


def gradient_band(rows, pts, widen=0.1):
    """Points whose radius, in the frame of any coil, lies within that coil's radial
    winding range widened by widen*R.  There the reference's gradient RZ integrand
    (src/Coil/Fields/CalculateFieldsFast.cxx:240-253) divides by (D - 2 r r' cos)^2
    and cancels a near-zero bracket: its result is ill-conditioned and differs
    between two correct double-precision evaluations well above 1e-12."""
    rows = np.atleast_2d(rows)
    band = np.zeros(len(pts), dtype=bool)
    for row in rows:
        r, _ = coil_frame(row, pts)
        R, a = row[0], row[1]
        band |= (r > R - widen * R) & (r < R + a + widen * R)
    return band


def winding_near(rows, pts, margin=0.1):
    """Points inside any coil's winding cross-section box in its (r, z) frame,
    inflated by margin*R: the near field, where the FP32 paths evaluate in FP64 and
    the FP32 error statistics are taken away from."""
    rows = np.atleast_2d(rows)
    near = np.zeros(len(pts), dtype=bool)
    for row in rows:
        r, z = coil_frame(row, pts)
        R, a, b = row[0], row[1], row[2]
        near |= (r > R - margin * R) & (r < R + a + margin * R) & (np.abs(z) < 0.5 * b + margin * R)
    return near
