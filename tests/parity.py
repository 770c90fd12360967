"""Helpers shared by the GPU parity tests: compare a peeler's device output with
the exact oracle.  Mirrors the reference's checks in
tests/gpu/test_peeler.py:24-136 without shapely: per (layer, source) region
areas, an exact ray rank at a generic interior point of every output polygon,
triangle orientation and area conservation, world reprojection and source-plane
distance.
"""

import json
from collections import defaultdict
from fractions import Fraction as Q

import numpy as np
from conftest import GOLDEN

from oracle import exact as ex

CROSSING = {"crossing", "perspective_crossing"} | {f"random_{i:02}" for i in range(12)}
MANIFEST = json.loads((GOLDEN / "fixtures/manifest.json").read_text())["fixtures"]
ACCEPTED = [f["name"] for f in MANIFEST if f["expected"] == "accept"]
RESOLVED = [n for n in ACCEPTED if n not in CROSSING]


def fixture(name):
    return json.loads((GOLDEN / f"fixtures/{name}.json").read_text())


def polygons(peeler):
    """[(layer, dense source, (n, 2) float64 vertices)] of the live output."""
    info = peeler.read_status()
    count = info["polygons"]
    verts = peeler.output.vertices[:count].cpu().numpy()
    sizes = peeler.output.sizes[:count].cpu().numpy()
    sources = peeler.output_sources[:count].cpu().numpy()
    layers = peeler.output_layers[:count].cpu().numpy()
    return [(int(layers[i]), int(sources[i]), verts[i, : sizes[i]]) for i in range(count)
            if sizes[i] >= 3]


def shoelace(v):
    x, y = v[:, 0], v[:, 1]
    return 0.5 * float(np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y))


def gpu_areas(polys, labels):
    """{(layer, external id): normalised window area}."""
    out = defaultdict(float)
    for layer, source, v in polys:
        out[(layer, int(labels[source]))] += shoelace(v)
    return dict(out)


def oracle_areas(scene, layers):
    """{(layer, external id): normalised window area} of an exact extraction."""
    xmin, ymin, xmax, ymax = scene.window
    scale = (xmax - xmin) * (ymax - ymin)
    return {k: float(a / 2 / scale) for k, a in ex.region_area2(scene, layers).items()}


def assert_areas(actual, expected, tolerance=1e-9):
    """Symmetric per-key area agreement (the reference's 1e-9 normalised bound)."""
    for key in actual.keys() | expected.keys():
        a, b = actual.get(key, 0.0), expected.get(key, 0.0)
        assert abs(a - b) <= tolerance, (key, a, b)


def assert_exact_ranks(scene, polys, skip_ambiguous=False):
    """Every output polygon's layer equals the exact rank of its source at a
    generic interior point (bit-for-bit rank parity).  Returns polygons checked."""
    index = ex.RankIndex(scene)
    dense = {s.index: i for i, s in enumerate(scene.sources)}
    checked = 0
    for layer, source, v in polys:
        ring = [ex.to_window(scene, float(x), float(y)) for x, y in v]
        rank = index.polygon_rank(dense[source], ring)
        if rank is None and skip_ambiguous:
            continue
        assert rank == layer, (source, layer, rank, v.tolist())
        checked += 1
    return checked


def assert_mesh(peeler, labels, expected_areas):
    """Triangles: positive orientation, areas equal to the regions, world
    positions reproject to uv and lie on their source planes
    (tests/gpu/test_peeler.py:101-133)."""
    info = peeler.read_status()
    t = info["triangles"]
    tris = peeler.triangles_uv[:t].cpu().numpy()
    sources = peeler.triangle_sources[:t].cpu().numpy()
    layers = peeler.triangle_layers[:t].cpu().numpy()
    area = defaultdict(float)
    for i, tri in enumerate(tris):
        a, b = tri[1] - tri[0], tri[2] - tri[0]
        cross = a[0] * b[1] - a[1] * b[0]
        assert cross > 0, (i, tri)
        area[(int(layers[i]), int(labels[sources[i]]))] += 0.5 * cross
    assert_areas(dict(area), expected_areas)
    if t == 0:
        return
    world = peeler.triangles_world[:t].cpu().numpy()
    camera = peeler.camera.reshape(4, 4).cpu().numpy()
    settings = peeler.settings.cpu().numpy()
    transformed = world @ camera[:3, :3].T + camera[:3, 3]
    uv = transformed[:, :, :2].copy()
    if settings[4]:
        uv /= transformed[:, :, 2, None]
    uv = (uv - settings[:2]) / (settings[2:4] - settings[:2])
    np.testing.assert_allclose(uv, tris, atol=2e-9, rtol=0)
    vertices = peeler.vertices.cpu().numpy()
    faces = peeler.faces.cpu().numpy()
    inputs = vertices[faces[sources]]
    normals = np.cross(inputs[:, 1] - inputs[:, 0], inputs[:, 2] - inputs[:, 0])
    normals /= np.linalg.norm(normals, axis=1)[:, None]
    distances = np.sum((world - inputs[:, :1]) * normals[:, None], axis=2)
    np.testing.assert_allclose(distances, 0, atol=2e-8, rtol=0)


def check_against_oracle(peeler, data, labels):
    """Full comparison of one extraction with the exact oracle."""
    scene = ex.read_scene(data, resolved_mesh=True)
    layers, residual = ex.extract(scene)
    assert not residual
    expected = oracle_areas(scene, layers)
    polys = polygons(peeler)
    assert_areas(gpu_areas(polys, labels), expected)
    assert_exact_ranks(scene, polys)
    assert_mesh(peeler, labels, expected)
    return expected


def stack_arrays(n, device="cuda"):
    """n congruent triangles at z = 1..n with cyclic vertex order
    (tests/gpu/test_events.py:59-71)."""
    import torch

    vertices = np.array([[-0.75, -0.75, 0], [0.75, -0.75, 0], [0, 0.75, 0]], dtype=np.float64)
    mesh = np.stack([np.roll(vertices, i % 3, axis=0) for i in range(n)])
    mesh[:, :, 2] = np.arange(1, n + 1)[:, None]
    return [
        torch.as_tensor(mesh.reshape(-1, 3), device=device),
        torch.as_tensor(np.arange(3 * n, dtype=np.int32).reshape(-1, 3), device=device),
        torch.as_tensor(np.eye(4), device=device),
        torch.as_tensor([-1.0, -1.0, 1.0, 1.0, 0.0, 0.01], dtype=torch.float64, device=device),
    ]


def exact_scene_of(vertices, faces, camera, settings):
    """A scene dict for the oracle from host arrays (floats are exact in it)."""
    cam = {"type": "perspective" if settings[4] else "orthographic",
           "near": float(settings[5]),
           "world_to_camera": [[float(x) for x in row] for row in camera[:3]]}
    return {
        "window": [float(x) for x in settings[:4]],
        "camera": cam,
        "triangles": [
            {"id": i, "vertices": [[float(c) for c in vertices[j]] for j in f]}
            for i, f in enumerate(faces)
        ],
    }


__all__ = ["Q"]
