"""Builds libccoil_b200.so in-tree for sm_100a with nvcc.

    python c-coil_b200/build.py            # build if any source is newer
    python c-coil_b200/build.py --force    # rebuild

The library lands next to the Python package (c-coil_b200/ccoil_b200/) so it
travels with the repository snapshot; nothing is installed into site-packages.
"""
import argparse
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT = os.path.join(HERE, "ccoil_b200", "libccoil_b200.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(INCLUDE, "*.h")))


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(f) <= t for f in sources() + headers() + [__file__])


def build(force=False, verbose=False, ptxas_info=False, out=None, defines=()):
    """Compile every source and link the library (out: alternative output path,
    defines: extra -D macros for a variant build)."""
    target = out or OUT
    if not force and out is None and not defines and up_to_date():
        return OUT
    build_dir = BUILD if out is None and not defines else BUILD + "_variant"
    os.makedirs(build_dir, exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(build_dir, os.path.basename(src) + ".o")
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-D" + d for d in defines] + ["-I", INCLUDE, "-I", CSRC, "-c", src,
                                                                            "-o", obj]
        if src.endswith(".cpp"):
            cmd += ["-x", "cu"]
        if ptxas_info and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed on " + src)
        if (verbose or ptxas_info) and (r.stdout or r.stderr):
            sys.stderr.write(r.stdout + r.stderr)
        objs.append(obj)
    tmp = target + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-cudart", "shared"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, target)
    return target


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    ap.add_argument("--out", default=None, help="alternative output path")
    ap.add_argument("-D", dest="defines", action="append", default=[], help="extra preprocessor macro")
    a = ap.parse_args()
    print(build(force=a.force or a.ptxas_info, verbose=a.verbose, ptxas_info=a.ptxas_info, out=a.out,
                defines=a.defines))
