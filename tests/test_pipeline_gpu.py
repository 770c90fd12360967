"""PeelStream (peel_b200.pipeline) on the GPU: a stream of meshes of one
shape, uploaded from host memory and read back while the next extracts,
gives each mesh the triangles of a single EventPeeler and download_mesh."""

from collections import defaultdict

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def area_by_key(uv, sources, layers):
    a, b = uv[:, 1] - uv[:, 0], uv[:, 2] - uv[:, 0]
    cross = a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]
    out = defaultdict(float)
    for s, l, c in zip(sources, layers, cross):
        out[(int(l), int(s))] += 0.5 * c
    return out


def test_stream_matches_single_extractions():
    from peel_b200 import EventPeeler, scenes
    from peel_b200.io import download_mesh
    from peel_b200.pipeline import PeelStream, as_numpy

    vertices, faces, camera, settings = scenes.nested_icospheres()
    meshes = []
    for shift in (0.0, 0.05, -0.1, 0.2):
        cam = camera.copy()
        cam[0, 3] += shift
        meshes.append([torch.as_tensor(a).pin_memory() for a in (vertices, faces, cam, settings)])
    stream = PeelStream(scenes.to_device((vertices, faces, camera, settings)))
    results = []
    for host in meshes:
        got = stream.submit(host)
        if got is not None:
            results.append(as_numpy(got))
    results.append(as_numpy(stream.finish()))
    assert len(results) == len(meshes)
    for host, (status, mesh) in zip(meshes, results):
        single = EventPeeler(*[h.cuda() for h in host])
        single.run()
        expected = download_mesh(single)
        assert status["triangles"] == expected["status"]["triangles"]
        got = area_by_key(mesh["triangles_uv"], mesh["triangle_sources"], mesh["triangle_layers"])
        want = area_by_key(expected["uv"], expected["sources"], expected["layers"])
        assert got.keys() == want.keys()
        assert max(abs(got[k] - want[k]) for k in want) <= 1e-12
