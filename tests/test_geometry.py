"""The kernels' polygon helpers (clean, split_edge, separated in
csrc/edp_device.cuh) run on the CPU from a host build of the same source.

Restates the reference's numeric regressions of its device geometry
(tests/gpu/test_peeler.py:331-375): cleaning must not erase a polygon whose
boundary backtracks by a round-off step, and splitting by a very short
clipping edge must keep the edge's position (two equal halves).  Binary64
without contraction rounds the same on the host as on the device.
"""

import ctypes
import shutil
import subprocess

import numpy as np
import pytest
from conftest import ROOT

KMAX = 32


def shoelace(v):
    """Signed area relative to the first vertex (translation-stable, as the
    reference's shapely areas are), so tiny polygons far from the origin
    keep their digits."""
    x, y = v[:, 0] - v[0, 0], v[:, 1] - v[0, 1]
    return 0.5 * float(np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y))


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    out = tmp_path_factory.mktemp("geometry") / "libgeometry.so"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17",
                    "-fmad=false", "--expt-relaxed-constexpr", "-Xcompiler",
                    "-fPIC,-ffp-contract=off", "-shared", "-o", str(out),
                    str(ROOT / "tests/native/geometry_harness.cu")], check=True)
    handle = ctypes.CDLL(str(out))
    P, I = ctypes.c_void_p, ctypes.c_int
    handle.geometry_clean.argtypes = [P, I]
    handle.geometry_clean.restype = I
    handle.geometry_split_edge.argtypes = [P, I, P, P, P, P, P]
    handle.geometry_separated.argtypes = [P, I, P, I]
    handle.geometry_separated.restype = I
    return handle


def clean(lib, points):
    buf = np.zeros((KMAX, 2))
    buf[: len(points)] = points
    n = lib.geometry_clean(buf.ctypes.data, len(points))
    return buf[:n]


def split_edge(lib, points, a, b):
    poly = np.ascontiguousarray(points, dtype=np.float64)
    ab = np.array([*a, *b], dtype=np.float64)
    inside, outside = np.zeros((KMAX, 2)), np.zeros((KMAX, 2))
    ni, no = ctypes.c_int(0), ctypes.c_int(0)
    lib.geometry_split_edge(poly.ctypes.data, len(poly), ab.ctypes.data, inside.ctypes.data,
                            ctypes.addressof(ni), outside.ctypes.data, ctypes.addressof(no))
    return inside[: ni.value], outside[: no.value]


def test_roundoff_edge_does_not_erase_polygon(lib):
    """kernels.py clean() on a square whose bottom edge steps back by 2e-12."""
    p = clean(lib, [(0.0, 0.0), (1.0, 0.0), (1.0 - 2e-12, 0.0), (1.0, 1.0), (0.0, 1.0)])
    assert len(p) >= 3
    assert abs(shoelace(p) - 1.0) < 1e-10


def test_short_clipping_edge_keeps_its_position(lib):
    """A 2e-6 square split by an edge of length ~2e-12 through its centre."""
    a = np.array([0.3, 0.3])
    h = 1e-6
    square = a + np.array([(-h, -h), (h, -h), (h, h), (-h, h)])
    inside, outside = split_edge(lib, square, a, a + np.array([1e-12, 2e-12]))
    areas = [shoelace(inside), shoelace(outside)]
    assert abs(areas[0] - areas[1]) < 1e-20
    assert abs(sum(areas) - 4e-12) < 1e-20


def test_clean_merges_and_collapses(lib):
    # Points within EPS / 100 = 1e-12 merge, the closing duplicate too.
    p = clean(lib, [(0.0, 0.0), (5e-13, 0.0), (1.0, 0.0), (1.0, 1.0), (0.0, 1.0), (0.0, 4e-13)])
    assert len(p) == 4 and abs(shoelace(p) - 1.0) < 1e-15
    # A sliver narrower than about EPS collapses.
    assert len(clean(lib, [(0.0, 0.0), (1.0, 0.0), (0.5, 1e-11)])) == 0
    # Too few distinct points collapse.
    assert len(clean(lib, [(0.0, 0.0), (1e-13, 0.0), (1.0, 1.0)])) == 0


def test_split_edge_partitions_area(lib):
    rng = np.random.default_rng(0)
    for _ in range(200):
        angles = np.sort(rng.random(7) * 2 * np.pi)
        poly = np.stack([np.cos(angles), np.sin(angles)], axis=1) * 0.4 + 0.5
        a, b = rng.random(2), rng.random(2)
        inside, outside = split_edge(lib, poly, a, b)
        total = shoelace(poly)
        parts = (shoelace(inside) if len(inside) else 0.0) + (
            shoelace(outside) if len(outside) else 0.0)
        assert abs(parts - total) < 1e-12
        d = b - a
        for v in inside:  # the inside is left of a->b
            assert d[0] * (v[1] - a[1]) - d[1] * (v[0] - a[0]) >= -1e-15


def test_separated(lib):
    square = np.array([(0.0, 0.0), (1.0, 0.0), (1.0, 1.0), (0.0, 1.0)])
    far = square + 2.0
    touching = square + np.array([1.0, 0.0])
    overlap = square + 0.5
    call = lambda a, b: lib.geometry_separated(np.ascontiguousarray(a).ctypes.data, len(a),
                                               np.ascontiguousarray(b).ctypes.data, len(b))
    assert call(square, far) and call(square, touching) and not call(square, overlap)
