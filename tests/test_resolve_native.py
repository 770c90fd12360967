"""The C++ intersection resolver (libedp_resolve.so, include/edp_resolve.h).

It implements the construction of peel_b200/resolve.py on binary64 inputs
with exact integer arithmetic; these CPU checks hold it to the rational code:

* the library exports every entry point its header declares;
* on binary64 versions of the crossing fixtures, on random triangle soups
  (some snapped to a coarse grid, full of exact ties) and on a small packing of
  overlapping spheres and tori, both give the identical resolved scene, text
  for text, and the same summary counts;
* its binary64 output is the correct rounding of its exact output;
* a coplanar overlap fails with the same message on both paths;
* rational (non-binary64) inputs take the rational code;
* resolve_mesh welds a resolved soup into an indexed mesh whose area and
  provenance match the pieces.
"""

import json
import re
from fractions import Fraction as Q
from pathlib import Path

import numpy as np
import pytest

from peel_b200 import resolve, scenefile, scenes

ROOT = Path(__file__).resolve().parents[1]
FIXTURES = ROOT / "tests/golden/fixtures"

pytestmark = pytest.mark.skipif(resolve.native_library() is None,
                                reason="libedp_resolve.so is not built")


def binary64_scene(data):
    out = dict(data)
    out["triangles"] = [dict(t, vertices=[[float(scenefile.rational(c)) for c in p]
                                          for p in t["vertices"]]) for t in data["triangles"]]
    return out


def both(data):
    a, sa = resolve.resolve(data, native=False)
    b, sb = resolve.resolve(data, native=True)
    assert sa["implementation"] == "python" and sb["implementation"] == "native"
    return a, sa, b, sb


def assert_same(data):
    a, sa, b, sb = both(data)
    assert a["triangles"] == b["triangles"]
    for key in ("output_triangles", "intersection_segments", "cut_triangles"):
        assert sa[key] == sb[key], key
    return sb


def test_exports_every_declared_entry_point():
    header = (ROOT / "include/edp_resolve.h").read_text()
    names = set(re.findall(r"\b(edp_\w+)\s*\(", header))
    assert len(names) >= 8
    lib = resolve.native_library()
    for name in sorted(names):
        assert hasattr(lib, name), name


CROSSING = sorted(p.name for p in FIXTURES.glob("random_*.json")) + ["perspective_crossing.json",
                                                                     "crossing.json"]


@pytest.mark.parametrize("name", CROSSING)
def test_crossing_fixtures_identical(name):
    data = binary64_scene(json.loads((FIXTURES / name).read_text()))
    summary = assert_same(data)
    assert summary["intersection_segments"] >= 0


@pytest.mark.parametrize("seed", range(4))
def test_random_soups_identical(seed):
    rng = np.random.default_rng(seed)
    tri = rng.uniform(-1, 1, size=(14, 3, 3))
    if seed % 2:
        tri = np.round(tri * 4) / 4  # shared coordinates, exact ties and touching edges
    data = {"triangles": [{"id": i, "vertices": t.tolist()} for i, t in enumerate(tri)]}
    try:
        assert_same(data)
    except scenefile.SceneFormatError:
        # Snapped soups may hold coplanar overlaps; then both must reject.
        with pytest.raises(scenefile.SceneFormatError) as a:
            resolve.resolve(data, native=False)
        with pytest.raises(scenefile.SceneFormatError) as b:
            resolve.resolve(data, native=True)
        assert str(a.value) == str(b.value)


def test_overlapping_primitives_identical():
    v, f, _, _ = scenes.overlapping_primitives(total_faces=600, count=5, seed=14)
    data = {"triangles": [{"id": i, "vertices": v[t].tolist()} for i, t in enumerate(f)]}
    summary = assert_same(data)
    assert summary["cut_triangles"] > 0


def test_binary64_output_is_the_rounded_exact_output():
    v, f, _, _ = scenes.overlapping_primitives(total_faces=1500, count=6, seed=11)
    with resolve.NativeResolution(v[f], exact_text=True) as r:
        assert r.status == 0
        info = r.summary()
        tris, parents = r.arrays()
        corners = r.exact()
    assert info["cut_triangles"] > 0
    assert len(corners) == 3 * len(tris)
    den_shift = info["scale_exponent"]
    flat = tris.reshape(-1, 3)
    constructed = 0
    for k, (x, y, z, w) in enumerate(corners):
        if w == 1 and k % 7:
            continue  # input vertices: a sample; every constructed point is checked
        constructed += w != 1
        exact = [float(Q(c, w << den_shift)) for c in (x, y, z)]
        assert flat[k].tolist() == exact, k
    assert constructed > 100
    assert parents.min() >= 0 and parents.max() < len(f)
    assert np.all(np.diff(parents) >= 0)  # pieces in input order


def test_coplanar_overlap_message_matches():
    data = binary64_scene(json.loads((FIXTURES / "tie.json").read_text()))
    with pytest.raises(scenefile.SceneFormatError) as a:
        resolve.resolve(data, native=False)
    with pytest.raises(scenefile.SceneFormatError) as b:
        resolve.resolve(data, native=True)
    assert str(a.value) == str(b.value)


def test_rational_inputs_take_the_rational_code():
    data = json.loads((FIXTURES / "random_00.json").read_text())
    _, summary = resolve.resolve(data)
    assert summary["implementation"] == "python"
    _, summary = resolve.resolve(binary64_scene(data))
    assert summary["implementation"] == "native"


def test_resolve_mesh_welds_and_conserves_area():
    v, f, _, _ = scenes.overlapping_primitives(total_faces=3000, count=8, seed=13)
    rv, rf, parents, summary = scenes.resolve_mesh(v, f)
    assert summary["intersection_segments"] > 0
    assert rf.min() >= 0 and rf.max() < len(rv)
    assert len(np.unique(rv, axis=0)) == len(rv)

    def areas(vertices, faces):
        t = vertices[faces]
        return 0.5 * np.linalg.norm(np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]), axis=1)

    per_parent = np.bincount(parents, weights=areas(rv, rf), minlength=len(f))
    np.testing.assert_allclose(per_parent, areas(v, f), rtol=1e-9, atol=1e-15)
