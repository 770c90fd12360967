"""Crossing scenes through the contour route on the GPU.

The EventPeeler needs resolved meshes, so each crossing fixture is first
resolved on the CPU (peel_b200.resolve, the preprocessing the reference runs
before its resolved-mesh tests, tests/gpu/test_events.py:19-45), uploaded as
binary64 and peeled.  Per (layer, original source) areas must equal the
oracle's arrangement of the unresolved input, and every output polygon's
layer must be the exact rank of its parent triangle at an interior point.
"""

import numpy as np
import pytest
import parity

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


@pytest.mark.parametrize("name", sorted(parity.CROSSING))
def test_resolved_crossing_fixture(name):
    from oracle import exact as ex
    from peel_b200 import EventPeeler
    from peel_b200.io import load_scene
    from peel_b200.resolve import resolve

    data = parity.fixture(name)
    resolved, _ = resolve(data)
    arrays, _, _ = load_scene(resolved)
    p = EventPeeler(*arrays)
    p.run()
    polys = parity.polygons(p)
    original = np.array([t["original_source_id"] for t in resolved["triangles"]])
    scene = ex.read_scene(data, resolved_mesh=False)
    layers, residual = ex.extract(scene)
    assert not residual
    parity.assert_areas(parity.gpu_areas(polys, original), parity.oracle_areas(scene, layers))
    index = {t.get("id", i): i for i, t in enumerate(data["triangles"])}
    parents = [(layer, index[int(original[s])], v) for layer, s, v in polys]
    assert parity.assert_exact_ranks(scene, parents) == len(parents)
