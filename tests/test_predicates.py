"""Escalating sign predicates (csrc/edp_predicates.cuh) on the CPU.

The header is built for the host with g++ (no floating-point contraction)
and every sign it returns is compared with exact rational arithmetic, on
well-separated inputs (decided in binary32), near-degenerate ones (binary64)
and exactly degenerate ones (the exact stage), including coordinates far from
the origin and magnitudes outside binary32's range.
"""

import ctypes
import subprocess
from fractions import Fraction as Q

import numpy as np
import pytest
from conftest import ROOT

BINARY32, BINARY64, EXACT = 0, 1, 2


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("predicates") / "libpredicates.so"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-std=c++17", "-shared", "-fPIC",
                    "-o", str(out), str(ROOT / "tests/native/predicates_harness.cpp")],
                   check=True)
    handle = ctypes.CDLL(str(out))
    P = ctypes.c_void_p
    handle.orient2d_batch.argtypes = [P, ctypes.c_long, P, P]
    handle.orient2d_lean_batch.argtypes = [P, ctypes.c_long, P, P]
    handle.dot_sign_batch.argtypes = [P, P, ctypes.c_int, ctypes.c_long, P, P]
    handle.orient2d_filter_batch.argtypes = [P, ctypes.c_long, P]
    handle.dot_sign_filter_batch.argtypes = [P, P, ctypes.c_int, ctypes.c_long, P]
    return handle


def orient(lib, points):
    points = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 6)
    signs = np.zeros(len(points), dtype=np.int32)
    stages = np.zeros(len(points), dtype=np.int32)
    lib.orient2d_batch(points.ctypes.data, len(points), signs.ctypes.data, stages.ctypes.data)
    return signs, stages


def exact_orient(row):
    ax, ay, bx, by, cx, cy = map(Q, row)
    d = (bx - ax) * (cy - ay) - (by - ay) * (cx - ax)
    return (d > 0) - (d < 0)


def dots(lib, p, q):
    p = np.ascontiguousarray(p, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    signs = np.zeros(len(p), dtype=np.int32)
    stages = np.zeros(len(p), dtype=np.int32)
    lib.dot_sign_batch(p.ctypes.data, q.ctypes.data, p.shape[1], len(p), signs.ctypes.data,
                       stages.ctypes.data)
    return signs, stages


def exact_dot(p, q):
    s = sum(Q(a) * Q(b) for a, b in zip(p, q))
    return (s > 0) - (s < 0)


def check_orient(lib, points):
    signs, stages = orient(lib, points)
    expected = np.array([exact_orient(r) for r in np.asarray(points).reshape(-1, 6)])
    np.testing.assert_array_equal(signs, expected)
    return stages


def test_separated_points_decide_in_binary32(lib):
    rng = np.random.default_rng(1)
    stages = check_orient(lib, rng.random((4000, 6)))
    assert np.mean(stages == BINARY32) > 0.99


def test_nearly_collinear_points_escalate_and_stay_exact(lib):
    rng = np.random.default_rng(2)
    a, b = rng.random((3000, 2)), rng.random((3000, 2))
    t = rng.random((3000, 1))
    c = a + t * (b - a)  # collinear up to rounding
    stages = check_orient(lib, np.hstack([a, b, c]))
    assert np.any(stages == BINARY64) and np.any(stages == EXACT)
    assert np.mean(stages == BINARY32) < 0.05


def test_exactly_collinear_points_give_zero(lib):
    rng = np.random.default_rng(3)
    a = rng.integers(-2**20, 2**20, (500, 2)) / 2.0**20
    d = rng.integers(-2**20, 2**20, (500, 2)) / 2.0**20
    k = 2.0 ** rng.integers(-3, 4, (500, 1))
    points = np.hstack([a, a + d, a + k * d])
    signs, stages = orient(lib, points)
    assert np.all(signs == 0)
    # A zero is never certified in binary32; binary64 decides it when a product
    # is exactly zero, else the exact stage does.
    assert not np.any(stages == BINARY32) and np.any(stages == EXACT)


def test_ulp_grid_around_a_point(lib):
    """The classic stress: points a few ulps apart near (0.5, 0.5) against a
    line through far-away points."""
    base = 0.5
    ulp = np.spacing(base)
    rows = [[base + i * ulp, base + j * ulp, 12.0, 12.0, 24.0, 24.0]
            for i in range(-16, 17) for j in range(-16, 17)]
    stages = check_orient(lib, rows)
    assert np.any(stages == EXACT)


def test_far_from_origin_and_tiny_scales(lib):
    rng = np.random.default_rng(4)
    offset = 1.0e6
    a = offset + rng.random((1000, 2)) * 1e-6
    b = offset + rng.random((1000, 2)) * 1e-6
    c = a + rng.random((1000, 1)) * (b - a) + rng.normal(size=(1000, 2)) * 1e-20
    check_orient(lib, np.hstack([a, b, c]))
    tiny = rng.random((500, 6)) * 1e-30  # differences below binary32's range
    stages = check_orient(lib, tiny)
    assert not np.any(stages == BINARY32)
    huge = rng.random((500, 6)) * 1e25  # differences above it
    stages = check_orient(lib, huge)
    assert not np.any(stages == BINARY32)


def test_depth_order_signs(lib):
    """Two planes compared at a point: sum of p q over (a1 - a2, b1 - b2,
    c1 - c2) against (x, y, 1), as random, nearly equal and equal depths."""
    rng = np.random.default_rng(5)
    n = 3000
    p = rng.normal(size=(n, 4))
    q = rng.normal(size=(n, 4))
    signs, stages = dots(lib, p, q)
    np.testing.assert_array_equal(signs, [exact_dot(a, b) for a, b in zip(p, q)])
    assert np.mean(stages == BINARY32) > 0.95
    # Nearly cancelling: the last term set to minus the rounded rest.
    q[:, 3] = -(p[:, :3] * q[:, :3]).sum(axis=1) / p[:, 3]
    signs, stages = dots(lib, p, q)
    np.testing.assert_array_equal(signs, [exact_dot(a, b) for a, b in zip(p, q)])
    assert np.any(stages == EXACT) and np.mean(stages == BINARY32) < 0.05
    # Exactly zero: (1, 1, -2) . (x, x, x).
    x = rng.integers(-2**30, 2**30, (200, 1)) / 2.0**10
    signs, stages = dots(lib, np.tile([1.0, 1.0, -2.0], (200, 1)), np.hstack([x, x, x]))
    assert np.all(signs == 0) and np.all(stages == EXACT)


@pytest.mark.parametrize("terms", [1, 2, 5, 8])
def test_every_term_count(lib, terms):
    rng = np.random.default_rng(6 + terms)
    p = rng.normal(size=(500, terms)) * 10.0 ** rng.integers(-8, 8, (500, terms))
    q = rng.normal(size=(500, terms))
    q[:, -1] = -(p[:, :-1] * q[:, :-1]).sum(axis=1) / p[:, -1] if terms > 1 else q[:, -1]
    signs, _ = dots(lib, p, q)
    np.testing.assert_array_equal(signs, [exact_dot(a, b) for a, b in zip(p, q)])


def test_lean_filter_gives_the_same_signs(lib):
    """orient2d_lean (the binary64 filter as one bound test, then exact) agrees
    with the exact sign on random, nearly collinear and exactly collinear
    points, and escalates only where the filter cannot certify."""
    rng = np.random.default_rng(7)
    a = rng.uniform(-1, 1, size=(500, 2))
    b = rng.uniform(-1, 1, size=(500, 2))
    t_ = rng.uniform(-2, 2, size=(500, 1))
    on_line = a + t_ * (b - a)
    near = on_line + rng.normal(scale=1e-15, size=on_line.shape)
    for c in (rng.uniform(-1, 1, size=(500, 2)), on_line, near):
        rows = np.hstack([a, b, c])
        rows = np.ascontiguousarray(rows, dtype=np.float64)
        signs = np.zeros(len(rows), dtype=np.int32)
        stages = np.zeros(len(rows), dtype=np.int32)
        lib.orient2d_lean_batch(rows.ctypes.data, len(rows), signs.ctypes.data,
                                stages.ctypes.data)
        np.testing.assert_array_equal(signs, [exact_orient(r) for r in rows])
        assert set(stages.tolist()) <= {BINARY64, EXACT}
    grid = np.array([[0.0, 0.0, 1.0, 1.0, 0.5, 0.5], [0.0, 0.0, 0.0, 0.0, 1.0, 2.0]])
    signs = np.zeros(2, dtype=np.int32)
    stages = np.zeros(2, dtype=np.int32)
    lib.orient2d_lean_batch(grid.ctypes.data, 2, signs.ctypes.data, stages.ctypes.data)
    assert signs.tolist() == [0, 0]


UNDECIDED = 2


def test_filter_only_stages_decide_or_defer(lib):
    """The first pass of the two-pass form (orient2d_filter, dot_sign_filter)
    gives the exact sign wherever it decides and kUndecided otherwise; it
    defers exactly where orient2d_lean and dot_sign reach their exact stage."""
    rng = np.random.default_rng(8)
    a = rng.uniform(-1, 1, size=(400, 2))
    b = rng.uniform(-1, 1, size=(400, 2))
    on_line = a + rng.uniform(-2, 2, size=(400, 1)) * (b - a)
    near = on_line + rng.normal(scale=1e-15, size=on_line.shape)
    for c in (rng.uniform(-1, 1, size=(400, 2)), on_line, near):
        rows = np.ascontiguousarray(np.hstack([a, b, c]), dtype=np.float64)
        got = np.zeros(len(rows), dtype=np.int32)
        lib.orient2d_filter_batch(rows.ctypes.data, len(rows), got.ctypes.data)
        lean = np.zeros(len(rows), dtype=np.int32)
        stages = np.zeros(len(rows), dtype=np.int32)
        lib.orient2d_lean_batch(rows.ctypes.data, len(rows), lean.ctypes.data,
                                stages.ctypes.data)
        np.testing.assert_array_equal(got == UNDECIDED, stages == EXACT)
        decided = got != UNDECIDED
        np.testing.assert_array_equal(got[decided], lean[decided])
    p = rng.normal(size=(300, 6))
    q = rng.normal(size=(300, 6))
    q[:150, -1] = -(p[:150, :-1] * q[:150, :-1]).sum(axis=1) / p[:150, -1]
    p, q = np.ascontiguousarray(p), np.ascontiguousarray(q)
    got = np.zeros(len(p), dtype=np.int32)
    lib.dot_sign_filter_batch(p.ctypes.data, q.ctypes.data, 6, len(p), got.ctypes.data)
    signs, stages = dots(lib, p, q)
    np.testing.assert_array_equal(got == UNDECIDED, stages == EXACT)
    decided = got != UNDECIDED
    np.testing.assert_array_equal(got[decided], signs[decided])
    assert (~decided).any() and decided.any()
