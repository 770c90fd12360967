"""The exact oracle pinned against the reference's own golden vectors.

The goldens in ``tests/golden`` come from the reference checkout
(``tests/golden/make_golden.py``): its CC0 fixture scenes with their
accept/reject manifest, and the exact CGAL arrangement outputs it recorded for
nine of them.  Everything here runs on the CPU.
"""

import json
from fractions import Fraction as Q

import pytest
from conftest import GOLDEN

from oracle import exact as ex

MANIFEST = json.loads((GOLDEN / "fixtures/manifest.json").read_text())["fixtures"]
EXPECTED = json.loads((GOLDEN / "exact_regions.json").read_text())
ACCEPTED = [f["name"] for f in MANIFEST if f["expected"] == "accept"]
REJECTED = [f["name"] for f in MANIFEST if f["expected"] != "accept"]


def scene(name, resolved=True):
    return ex.read_scene(json.loads((GOLDEN / f"fixtures/{name}.json").read_text()), resolved)


@pytest.mark.parametrize("name", sorted(EXPECTED))
@pytest.mark.parametrize("resolved", [True, False])
def test_import_matches_reference_planes_and_polygons(name, resolved):
    s = scene(name, resolved)
    byid = s.by_id()
    for src in EXPECTED[name]["sources"]:
        mine = byid[src["id"]]
        assert (mine.score.a, mine.score.b, mine.score.c) == tuple(Q(x) for x in src["score"])
        ring = [(Q(x), Q(y)) for x, y in src["polygon"]]
        assert ex.area2(ring) == ex.area2(mine.poly)
        assert all(ex.strictly_inside(ring, p) >= 0 for p in mine.poly)


@pytest.mark.parametrize("name", sorted(EXPECTED))
@pytest.mark.parametrize("resolved", [True, False])
def test_exact_regions_equal_reference_arrangement(name, resolved):
    """Per (layer, source) exact doubled area equals the CGAL arrangement's."""
    s = scene(name, resolved)
    layers, residual = ex.extract(s)
    assert not residual
    expected = {(r["layer"], r["source"]): Q(r["area2"]) for r in EXPECTED[name]["regions"]}
    assert ex.region_area2(s, layers) == expected
    assert len(layers) == EXPECTED[name]["layers"]


@pytest.mark.parametrize("name", REJECTED)
def test_positive_area_ties_rejected(name):
    with pytest.raises(ex.SceneError, match="positive-area depth tie"):
        scene(name)


@pytest.mark.parametrize("name", ACCEPTED)
def test_every_patch_has_its_exact_ray_rank(name):
    """Independent audit: the exact rank at each patch centroid is its layer."""
    s = scene(name, resolved=False)
    layers, residual = ex.extract(s)
    assert not residual
    index = ex.RankIndex(s)
    for k, layer in enumerate(layers):
        for p in layer:
            assert index.polygon_rank(p.source, p.points) == k


def test_prefix_keeps_residual():
    s = scene("holes")
    layers, residual = ex.extract(s, layers=1)
    assert len(layers) == 1 and residual


def test_stack_known_answer():
    """Identical footprints at distinct depths: layer == source index."""
    tri = [["-3/4", "-3/4", "0"], ["3/4", "-3/4", "0"], ["0", "3/4", "0"]]
    data = {
        "window": [-1, -1, 1, 1],
        "camera": {"type": "orthographic"},
        "triangles": [
            {"id": i, "vertices": [[v[0], v[1], str(i + 1)] for v in tri[i % 3:] + tri[:i % 3]]}
            for i in range(16)
        ],
    }
    s = ex.read_scene(data)
    layers, _ = ex.extract(s)
    assert [[s.sources[p.source].id for p in layer] for layer in layers] == [[i] for i in range(16)]
