"""Host adapters around a device-resident extraction: scene upload and mesh
download.  The reference's module of the same name (warp_peel/io.py) defines
the interface kept here: ``load_scene`` returns the four input arrays, the
external ids and the scene dict; ``download_mesh`` returns the ``layers.npz``
arrays plus the decoded status.  Nothing here is part of the extraction.
"""

import numpy as np

from .scenefile import SceneFile, scene_dict

# The layers.npz arrays: name -> (peeler attribute, host dtype).
MESH_ARRAYS = {
    "uv": ("triangles_uv", np.float64),
    "world": ("triangles_world", np.float64),
    "sources": ("triangle_sources", np.int64),
    "layers": ("triangle_layers", np.int32),
}


def scene_arrays(data):
    """Host (vertices, faces, camera, settings, labels) of a scene dict."""
    scene = SceneFile(data)
    return (*scene.arrays(), scene.labels)


def scene_data(vertices, faces, camera, settings):
    """Scene dict of host or device arrays (``SceneFile`` reads it back)."""
    return scene_dict(vertices, faces, camera, settings)


def load_scene(path, device="cuda:0"):
    """Read a scene (path or dict) and put its arrays on ``device`` as torch
    tensors; returns ([vertices, faces, camera, settings], labels, data)."""
    import torch

    scene = SceneFile(path)
    tensors = [torch.from_numpy(a).to(device) for a in scene.arrays()]
    return tensors, scene.labels, scene.data


def download_mesh(peeler, labels=None):
    """Copy the finished extraction's triangles to the host.

    Returns the ``layers.npz`` arrays (``uv`` [T,3,2], ``world`` [T,3,3],
    ``sources`` as external ids when ``labels`` is given, zero-based
    ``layers``) and ``status``, the decoded status.  Synchronises the
    workspace stream (through ``read_status``)."""
    status = peeler.read_status()
    count = status["triangles"]
    mesh = {name: getattr(peeler, attribute)[:count].cpu().numpy().astype(dtype, copy=False)
            for name, (attribute, dtype) in MESH_ARRAYS.items()}
    if labels is not None:
        mesh["sources"] = np.asarray(labels, dtype=np.int64)[mesh["sources"]]
    mesh["status"] = status
    return mesh
