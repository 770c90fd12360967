"""The rational ray auditor (peel_b200.audit) on exact oracle regions.

The oracle's exact extraction of a fixture, rounded to binary64 window
coordinates, must pass the audit with no rank mismatch, and a planted wrong
layer must be found (the reference's scripts/audit_gpu.py is the model)."""

import numpy as np
import pytest
import parity
from oracle import exact as ex

AUDITED = ["holes", "partial", "closed_object", "stacked", "components", "perspective_torus"]


def regions(data):
    scene = ex.read_scene(data, resolved_mesh=True)
    layers, residual = ex.extract(scene)
    assert not residual
    xmin, ymin, xmax, ymax = scene.window
    polys, sources, ranks = [], [], []
    for k, layer in enumerate(layers):
        for p in layer:
            polys.append(np.array([[float((x - xmin) / (xmax - xmin)),
                                    float((y - ymin) / (ymax - ymin))] for x, y in p.points]))
            sources.append(scene.sources[p.source].id)
            ranks.append(k)
    return polys, np.array(sources), np.array(ranks)


@pytest.mark.parametrize("name", AUDITED)
def test_oracle_regions_pass(name):
    from peel_b200.audit import audit_regions

    data = parity.fixture(name)
    polys, sources, ranks = regions(data)
    report = audit_regions(polys, sources, ranks, data)
    assert report["rank_mismatches"] == 0, report["examples"][:3]
    assert report["checked_rays"] > 0


def test_planted_rank_error_is_found():
    from peel_b200.audit import audit_regions

    data = parity.fixture("stacked")
    polys, sources, ranks = regions(data)
    wrong = ranks.copy()
    wrong[int(np.argmax(ranks))] += 1
    report = audit_regions(polys, sources, wrong, data)
    assert report["rank_mismatches"] > 0
