"""The exact vertex auditor (peel_b200.audit.vertex_audit) on the CPU.

The oracle's exact extraction of every resolved reference fixture, rounded to
binary64, must be explained vertex by vertex: each vertex lies on two exact
source-edge, window or equal-depth lines, and its error against their rational
intersection is the rounding alone (one ulp of a normalised coordinate: the
rounding of the vertex, plus that of scene numbers that binary64 does not hold
exactly, such as decimal strings).  A vertex moved off its lines is measured
by the amount it moved.
"""

import numpy as np
import pytest
import parity

from oracle import exact as ex


def exact_peel(name):
    """(float polygons in the normalised window, their face indices, outlines)."""
    from peel_b200.audit import ExactOutlines
    from peel_b200.io import load_scene

    data = parity.fixture(name)
    arrays, _, _ = load_scene(data, "cpu")
    scene = ex.read_scene(data, resolved_mesh=True)
    layers, _ = ex.extract(scene)
    xmin, ymin, xmax, ymax = scene.window
    polygons, sources = [], []
    for layer in layers:
        for patch in layer:
            polygons.append(np.array([[float((x - xmin) / (xmax - xmin)),
                                       float((y - ymin) / (ymax - ymin))]
                                      for x, y in patch.points]))
            sources.append(scene.sources[patch.source].index)
    return polygons, sources, ExactOutlines(*[a.numpy() for a in arrays])


@pytest.mark.parametrize("name", parity.RESOLVED)
def test_exact_peel_vertices_are_explained(name):
    from peel_b200.audit import vertex_audit

    polygons, sources, outlines = exact_peel(name)
    report = vertex_audit(polygons, sources, outlines, samples=10 ** 6)
    assert report["unexplained_vertices"] == 0, report
    assert report["vertices_measured"] >= 3 * len(polygons) - report["collinear_vertices"]
    assert report["max_abs_error"] <= 2.0 ** -52, report


def test_moved_vertex_is_measured():
    from peel_b200.audit import vertex_audit

    polygons, sources, outlines = exact_peel("holes")
    moved = [p.copy() for p in polygons]
    moved[3][1] += np.array([3e-9, -2e-9])
    report = vertex_audit(moved, sources, outlines, samples=10 ** 6)
    assert report["unexplained_vertices"] == 0
    assert 2.9e-9 <= report["max_abs_error"] <= 3.1e-9, report
    assert report["worst"]["polygon"] == 3 and report["worst"]["vertex"] == 1


def test_vertex_off_every_line_is_unexplained():
    from peel_b200.audit import vertex_audit

    polygons, sources, outlines = exact_peel("holes")
    moved = [p.copy() for p in polygons]
    moved[0][0] += np.array([1e-4, 1e-4])
    report = vertex_audit(moved, sources, outlines, samples=10 ** 6)
    assert report["unexplained_vertices"] >= 1
