"""Build libedp_b200.so in-tree with nvcc for sm_100a.

    python exact-depth-peeling_b200/build.py [--force]

Every .cu file under csrc/ is compiled for compute_100a / sm_100a with
binary64 contraction disabled (-fmad=false: predicates are plain IEEE and a
CPU restatement of an expression gives the same bits) and linked into
peel_b200/libedp_b200.so, next to the Python package that loads it.  The
host-only exact intersection resolver (csrc/edp_resolve.cpp) is compiled
with g++ into peel_b200/libedp_resolve.so.
"""

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIBRARY = HERE / "peel_b200" / "libedp_b200.so"
RESOLVER = HERE / "peel_b200" / "libedp_resolve.so"  # host C++ (exact resolver)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
         "--expt-relaxed-constexpr", "-I", str(HERE.parent / "include")]


def nvcc():
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found; the CUDA 12.9 toolkit is required")
    return found


def sources():
    return sorted(CSRC.glob("*.cu"))


def headers():
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [HERE.parent / "include/edp.h"]


def stale(target, deps):
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def compile_one(src, extra):
    obj = BUILD / (src.stem + ".o")
    deps = [src] + headers()
    if stale(obj, deps):
        cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stderr}")
        if r.stderr.strip():
            sys.stderr.write(r.stderr)
    return obj


def build_resolver(force=False):
    """The exact intersection resolver: host C++ (g++), no CUDA."""
    src = CSRC / "edp_resolve.cpp"
    deps = [src, HERE.parent / "include/edp_resolve.h"]
    if force or stale(RESOLVER, deps):
        cxx = shutil.which("g++") or "g++"
        cmd = [cxx, "-std=c++17", "-O3", "-fPIC", "-shared", "-pthread", "-Wall",
               "-I", str(HERE.parent / "include"), str(src), "-o", str(RESOLVER)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"g++ failed on {src.name}:\n{r.stderr}")
    return RESOLVER


def build(force=False, verbose_ptxas=False):
    BUILD.mkdir(exist_ok=True)
    if force:
        for o in BUILD.glob("*.o"):
            o.unlink()
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        objects = list(pool.map(lambda s: compile_one(s, extra), sources()))
    if force or stale(LIBRARY, objects):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIBRARY), *map(str, objects), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    build_resolver(force)
    return LIBRARY


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register/spill usage")
    a = ap.parse_args()
    print(build(a.force, a.ptxas))
