"""Scene JSON files: one reader for the peelers, the resolver and the auditor.

A scene is the reference's JSON format (warp_peel/io.py:11-48 reads it for
the GPU route, src/exact_geometry.cpp:5-39 and src/camera.cpp:74-229 for the
exact solvers):

    {"window": [xmin, ymin, xmax, ymax],
     "camera": {"type": "orthographic" | "perspective", "near": n,
                "world_to_camera": [[...4...], [...4...], [...4...]]},
     "triangles": [{"id": k, "vertices": [[x, y, z], [x, y, z], [x, y, z]]}, ...]}

Numbers are JSON numbers or strings.  Two readings exist and both are kept:

* ``binary64`` is the GPU route's: a JSON number is taken as is, a string is
  read as an exact fraction and rounded once to the nearest double;
* ``rational`` is the exact solvers': a JSON number exactly (its binary64
  value), a string only as an integer or "numerator/denominator".

``SceneFile`` parses a scene once and validates it with the reference's
messages; ``arrays()`` gives the four binary64 arrays the peelers take (one
vertex per triangle corner, faces 0..3N-1) and ``labels`` the external ids.
"""

import json
import math
from fractions import Fraction
from pathlib import Path

import numpy as np


class SceneFormatError(ValueError):
    """A scene number or record the exact reader does not accept."""


def binary64(value):
    """A scene number as the GPU route reads it (the nearest double)."""
    if isinstance(value, str):
        return float(Fraction(value))
    return float(value)


def exact(value):
    """The exact value of a scene number before the GPU route rounds it: a
    JSON number's binary64 value, a string read as a fraction."""
    if isinstance(value, str):
        return Fraction(value)
    if isinstance(value, float):
        return Fraction(value)
    return Fraction(int(value))


def _is_integer_text(text):
    digits = text[1:] if text[:1] in "+-" else text
    return digits.isascii() and digits.isdigit()


def rational(value):
    """A scene number as the exact solvers read it: JSON numbers exactly,
    strings as integers or "numerator/denominator" only."""
    if isinstance(value, bool):
        raise SceneFormatError(f"Expected integer or rational string: {value}")
    if isinstance(value, float):
        if not math.isfinite(value):
            raise SceneFormatError("Nonfinite coordinate")
        return Fraction(value)
    if isinstance(value, int):
        return Fraction(value)
    text = str(value)
    numerator, slash, denominator = text.partition("/")
    if not _is_integer_text(numerator) or (slash and not _is_integer_text(denominator)):
        raise SceneFormatError(f"Expected integer or rational string: {text}")
    if slash and int(denominator) == 0:
        raise SceneFormatError("Zero rational denominator")
    return Fraction(int(numerator), int(denominator) if slash else 1)


def read_json(source):
    """A scene dict from a dict, a path, or JSON text in a path-like string."""
    if isinstance(source, dict):
        return source
    return json.loads(Path(source).read_text())


class SceneFile:
    """A parsed, validated scene.

    Attributes: ``data`` (the dict), ``labels`` (int64 external ids, the
    triangle's "id" or its position), ``perspective``, and the binary64
    ``corners`` [N, 3, 3], ``world_to_camera`` [4, 4] (identity rows unless
    given) and ``settings`` [6] (window, perspective flag, near plane).
    Raises ValueError with the GPU route's messages (warp_peel/io.py:27-44)."""

    CAMERA_TYPES = ("orthographic", "perspective")

    def __init__(self, source):
        self.data = read_json(source)
        triangles = self.data["triangles"]
        camera = self.data.get("camera", {})
        kind = camera.get("type", "orthographic")
        if kind not in self.CAMERA_TYPES:
            raise ValueError("Unknown camera type")
        self.perspective = kind == "perspective"
        self.corners = np.array([[[binary64(x) for x in corner] for corner in t["vertices"]]
                                 for t in triangles], dtype=np.float64).reshape(-1, 3, 3)
        self.world_to_camera = np.eye(4, dtype=np.float64)
        if "world_to_camera" in camera:
            self.world_to_camera[:3] = [[binary64(x) for x in row]
                                        for row in camera["world_to_camera"]]
        window = [binary64(x) for x in self.data["window"]]
        self.settings = np.array(window + [1.0 if self.perspective else 0.0,
                                           binary64(camera.get("near", 0.01))], dtype=np.float64)
        finite = (np.isfinite(self.corners).all() and np.isfinite(self.world_to_camera).all()
                  and np.isfinite(self.settings).all())
        if not finite:
            raise ValueError("Input must be finite")
        xmin, ymin, xmax, ymax, _, near = self.settings
        if xmax <= xmin or ymax <= ymin or near <= 0:
            raise ValueError("Invalid image window or near plane")
        self.labels = np.array([t.get("id", i) for i, t in enumerate(triangles)], dtype=np.int64)
        if np.unique(self.labels).size != self.labels.size:
            raise ValueError("Source IDs must be unique")

    def __len__(self):
        return len(self.corners)

    def arrays(self):
        """(vertices [3N, 3] f64, faces [N, 3] i32, camera [4, 4] f64, settings [6] f64)."""
        faces = np.arange(3 * len(self), dtype=np.int32).reshape(-1, 3)
        return self.corners.reshape(-1, 3).copy(), faces, self.world_to_camera.copy(), \
            self.settings.copy()


def scene_dict(vertices, faces, camera, settings):
    """Scene JSON (as a dict) of host or device arrays, one triangle per face
    with id = face index.  Binary64 values are written as JSON numbers, whose
    shortest repr reads back to the same double."""
    host = [np.asarray(a.cpu() if hasattr(a, "cpu") else a) for a in
            (vertices, faces, camera, settings)]
    v, f, cam, st = host
    corners = v[f.astype(np.int64)]
    return {
        "window": [float(x) for x in st[:4]],
        "camera": {"type": "perspective" if st[4] else "orthographic", "near": float(st[5]),
                   "world_to_camera": cam[:3].tolist()},
        "triangles": [{"id": i, "vertices": c.tolist()} for i, c in enumerate(corners)],
    }
