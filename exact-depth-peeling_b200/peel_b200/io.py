"""Optional host serialisation adapters around the device extraction.

``load_scene`` follows warp_peel/io.py:11-48 (scene JSON to float64 device
tensors, one vertex copy per triangle, faces = arange, exact rational strings
rounded once to binary64); ``download_mesh`` follows io.py:51-72.
"""

import json
from fractions import Fraction
from pathlib import Path

import numpy as np


def _number(x):
    return float(Fraction(x)) if isinstance(x, str) else float(x)


def scene_arrays(data):
    """Host numpy arrays (vertices, faces, camera, settings, labels) of a scene."""
    triangles = data["triangles"]
    vertices = np.array(
        [[[_number(x) for x in p] for p in t["vertices"]] for t in triangles], dtype=np.float64
    ).reshape((-1, 3))
    faces = np.arange(3 * len(triangles), dtype=np.int32).reshape((-1, 3))
    camera = np.eye(4, dtype=np.float64)
    cam = data.get("camera", {})
    if cam.get("type", "orthographic") not in ("orthographic", "perspective"):
        raise ValueError("Unknown camera type")
    if "world_to_camera" in cam:
        camera[:3] = [[_number(x) for x in row] for row in cam["world_to_camera"]]
    settings = np.array(
        [_number(x) for x in data["window"]]
        + [int(cam.get("type") == "perspective"), _number(cam.get("near", 0.01))],
        dtype=np.float64,
    )
    if (not np.isfinite(vertices).all() or not np.isfinite(camera).all()
            or not np.isfinite(settings).all()):
        raise ValueError("Input must be finite")
    if settings[2] <= settings[0] or settings[3] <= settings[1] or settings[5] <= 0:
        raise ValueError("Invalid image window or near plane")
    labels = np.array([t.get("id", i) for i, t in enumerate(triangles)], dtype=np.int64)
    if len(set(labels.tolist())) != len(labels):
        raise ValueError("Source IDs must be unique")
    return vertices, faces, camera, settings, labels


def scene_data(vertices, faces, camera, settings):
    """Scene JSON (as a dict) of host or device arrays: the inverse of
    ``scene_arrays``, one triangle per face with id = face index.  Binary64
    values are written as JSON numbers, whose shortest repr reads back exactly."""
    host = [np.asarray(a.cpu() if hasattr(a, "cpu") else a) for a in
            (vertices, faces, camera, settings)]
    v, f, cam, st = host
    tri = v[f.astype(np.int64)]
    return {
        "window": [float(x) for x in st[:4]],
        "camera": {"type": "perspective" if st[4] else "orthographic", "near": float(st[5]),
                   "world_to_camera": cam[:3].tolist()},
        "triangles": [{"id": i, "vertices": tri[i].tolist()} for i in range(len(tri))],
    }


def load_scene(path, device="cuda:0"):
    """Upload a scene JSON; returns ([vertices, faces, camera, settings], labels, data)."""
    import torch

    data = json.loads(Path(path).read_text()) if not isinstance(path, dict) else path
    vertices, faces, camera, settings, labels = scene_arrays(data)
    arrays = [
        torch.as_tensor(vertices, device=device),
        torch.as_tensor(faces, device=device),
        torch.as_tensor(camera, device=device),
        torch.as_tensor(settings, device=device),
    ]
    return arrays, labels, data


def download_mesh(peeler, labels=None):
    """Explicit host transfer for serialisation; not part of the GPU pipeline."""
    info = peeler.read_status()
    n = info["triangles"]
    if n == 0:
        return {
            "uv": np.empty((0, 3, 2)),
            "world": np.empty((0, 3, 3)),
            "sources": np.empty(0, dtype=np.int64),
            "layers": np.empty(0, dtype=np.int32),
            "status": info,
        }
    sources = peeler.triangle_sources[:n].cpu().numpy().astype(np.int64)
    if labels is not None:
        sources = np.asarray(labels)[sources]
    return {
        "uv": peeler.triangles_uv[:n].cpu().numpy(),
        "world": peeler.triangles_world[:n].cpu().numpy(),
        "sources": sources,
        "layers": peeler.triangle_layers[:n].cpu().numpy(),
        "status": info,
    }
