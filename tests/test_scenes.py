"""The seeded synthetic workloads: sizes and topology (CPU only)."""

import numpy as np


def closed_genus(vertices, faces):
    edges = np.sort(np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]]), 1)
    unique, counts = np.unique(edges, axis=0, return_counts=True)
    assert (counts == 2).all(), "every edge of a closed surface has two faces"
    return (2 - (len(vertices) - len(unique) + len(faces))) // 2


def test_genus3_surface():
    from peel_b200 import scenes

    v, f = scenes.genus3_surface()
    assert 15000 < len(f) < 17500
    assert closed_genus(v, f) == 3
    # Outward winding: the signed volume is positive.
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    assert np.einsum("ij,ij->i", a, np.cross(b, c)).sum() > 0


def test_batched_workload():
    from peel_b200 import scenes

    batch = scenes.batched_scenes()
    assert len(batch) == 128
    views, meshes = batch[:64], batch[64:]
    assert all(v[0] is views[0][0] for v in views)  # one surface, 64 cameras
    assert len({tuple(v[2].ravel()) for v in views}) == 64
    sizes = [len(m[1]) for m in meshes]
    assert min(sizes) >= 900 and max(sizes) <= 36000
    for v, f, camera, settings in batch:
        assert f.dtype == np.int32 and camera.shape == (4, 4) and settings[4] == 1.0
        # Every vertex is in front of the near plane.
        z = v @ camera[2, :3] + camera[2, 3]
        assert z.min() > settings[5]
