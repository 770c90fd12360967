"""Independent rational-ray audit of an extraction's labelled regions.

    python -m peel_b200.audit scene.json [--method events] [--samples 512]

Restates the reference's large-scene audit (scripts/audit_gpu.py:22-137,
scripts/check_rays.py): query points are a 32 x 32 grid of the normalised
window plus an interior point of sampled output polygons.  At each point the
extraction's answer is the sorted (layer, source id) list of the output
polygons that contain it; the expected answer casts one ray through every
scene triangle with exact rational arithmetic (Moller-Trumbore in
``fractions.Fraction``), orders the hits by depth and numbers them from 0.
Points within 1e-11 of an output polygon's boundary, rays that touch a
triangle edge and equal-depth hits are skipped.  It is a sampled check of
ranks and labels, not a certificate of the regions, and it shares no code with
the extraction.
"""

import argparse
import json
import sys
from fractions import Fraction as Q
from pathlib import Path

import numpy as np

SCOPE = ("Sampled source-labelled ranks using independent rational ray/triangle tests, "
         "padded floating input bounds, and downloaded output polygons; not a region "
         "certificate. Grid plus output interior samples; boundary-near samples skipped.")


def _sub(a, b):
    return tuple(x - y for x, y in zip(a, b))


def _dot(a, b):
    return sum(x * y for x, y in zip(a, b))


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


class RationalScene:
    """A scene JSON in exact arithmetic: camera-space triangles and padded
    binary64 bounds of their projections (audit_gpu.py:32-68)."""

    def __init__(self, data):
        q = lambda x: Q(str(x))
        cam = data.get("camera", {})
        matrix = [[q(x) for x in row] for row in cam.get(
            "world_to_camera", [[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0]])]
        self.perspective = cam.get("type") == "perspective"
        self.near = q(cam.get("near", "0.01"))
        self.window = [q(x) for x in data["window"]]
        self.triangles, lower, upper = [], [], []
        for i, t in enumerate(data["triangles"]):
            camera = [tuple(_dot(row[:3], tuple(map(q, v))) + row[3] for row in matrix)
                      for v in t["vertices"]]
            if self.perspective and min(v[2] for v in camera) < self.near:
                raise ValueError("the audit needs every source vertex beyond the near plane")
            uv = [(float(v[0] / v[2]), float(v[1] / v[2])) if self.perspective
                  else (float(v[0]), float(v[1])) for v in camera]
            self.triangles.append((t.get("id", i), camera[0], _sub(camera[1], camera[0]),
                                   _sub(camera[2], camera[0])))
            lower.append(np.min(uv, axis=0))
            upper.append(np.max(uv, axis=0))
        self.lower = np.asarray(lower).reshape(-1, 2)
        self.upper = np.asarray(upper).reshape(-1, 2)

    def ranks(self, uv):
        """Exact [(rank, source id)] along the ray through normalised window
        point uv, or None when the ray touches an edge or two hits tie."""
        x = tuple(self.window[a] + Q(str(uv[a])) * (self.window[a + 2] - self.window[a])
                  for a in range(2))
        xf = np.array([float(x[0]), float(x[1])])
        selected = np.where(np.all(self.lower <= xf + 1e-9, axis=1)
                            & np.all(self.upper >= xf - 1e-9, axis=1))[0]
        if self.perspective:
            origin, direction = (Q(0), Q(0), Q(0)), (x[0], x[1], Q(1))
        else:
            origin, direction = (x[0], x[1], Q(0)), (Q(0), Q(0), Q(1))
        hits = []
        for i in selected:
            ident, v, e1, e2 = self.triangles[i]
            h = _cross(direction, e2)
            det = _dot(e1, h)
            if det == 0:
                continue
            s = _sub(origin, v)
            b = _dot(s, h) / det
            qq = _cross(s, e1)
            c = _dot(direction, qq) / det
            depth = _dot(e2, qq) / det
            if b < 0 or c < 0 or b + c > 1 or (self.perspective and depth < self.near):
                continue
            if b == 0 or c == 0 or b + c == 1:
                return None
            hits.append((depth, ident))
        hits.sort()
        if any(a[0] == b[0] for a, b in zip(hits, hits[1:])):
            return None
        return [(rank, int(ident)) for rank, (_, ident) in enumerate(hits)]


def _answers(polygons, lo, hi, point):
    """Sorted indices of the output polygons containing point, or None when the
    point lies within 1e-11 of one of their boundaries."""
    near = np.where(np.all(lo <= point + 1e-11, axis=1) & np.all(hi >= point - 1e-11, axis=1))[0]
    inside = []
    for i in near:
        v = polygons[i]
        a, b = v, np.roll(v, -1, axis=0)
        d = b - a
        cross = d[:, 0] * (point[1] - a[:, 1]) - d[:, 1] * (point[0] - a[:, 0])
        length = np.hypot(d[:, 0], d[:, 1])
        t = np.clip(((point - a) * d).sum(1) / np.maximum(length ** 2, 1e-300), 0.0, 1.0)
        distance = np.hypot(*(a + t[:, None] * d - point).T)
        if distance.min() < 1e-11:
            return None
        if (cross > 0).all():
            inside.append(i)
    return inside


def audit_regions(polygons, sources, layers, data, samples=512, queries=()):
    """Audit labelled regions: `polygons` is a list of (k, 2) arrays in the
    normalised window (counter-clockwise), `sources` their external ids,
    `layers` their zero-based layers.  Returns the report dictionary."""
    scene = RationalScene(data)
    polygons = [np.asarray(v, dtype=np.float64) for v in polygons]
    count = len(polygons)
    lo = np.array([v.min(0) for v in polygons]).reshape(-1, 2)
    hi = np.array([v.max(0) for v in polygons]).reshape(-1, 2)
    points = [((x + 0.371) / 32, (y + 0.619) / 32) for x in range(32) for y in range(32)]
    if count:
        for i in np.linspace(0, count - 1, min(samples, count), dtype=int):
            points.append(tuple(polygons[i].mean(0)))
    points.extend(queries)
    checked = skipped = mismatch = max_hits = 0
    examples = []
    for uv in points:
        inside = _answers(polygons, lo, hi, np.asarray(uv, dtype=np.float64))
        expected = scene.ranks(uv)
        if inside is None or expected is None:
            skipped += 1
            continue
        actual = sorted((int(layers[i]), int(sources[i])) for i in inside)
        if not expected and not actual:
            continue
        checked += 1
        max_hits = max(max_hits, len(expected))
        if actual != expected:
            mismatch += 1
            if len(examples) < 20:
                examples.append({"uv_normalized": list(uv), "expected": expected,
                                 "actual": actual})
    return {"scope": SCOPE, "checked_rays": checked, "skipped_boundary_rays": skipped,
            "rank_mismatches": mismatch, "maximum_hits": max_hits, "examples": examples}


def audit(peeler, labels, data, samples=512, queries=()):
    """Audit a finished extraction (EventPeeler or DevicePeeler)."""
    info = peeler.read_status()
    count = info["polygons"]
    n = peeler.output.sizes[:count].cpu().numpy()
    v = peeler.output.vertices[:count].cpu().numpy()
    keep = n >= 3
    polygons = [v[i, : n[i]] for i in np.nonzero(keep)[0]]
    sources = np.asarray(labels)[peeler.output_sources[:count].cpu().numpy()[keep]]
    layers = peeler.output_layers[:count].cpu().numpy()[keep]
    report = audit_regions(polygons, sources, layers, data, samples, queries)
    report["output"] = info
    return report


def main(argv=None):
    from . import DevicePeeler, EventPeeler
    from .io import load_scene

    parser = argparse.ArgumentParser(description=__doc__,
                                     formatter_class=argparse.RawDescriptionHelpFormatter)
    parser.add_argument("scene", type=Path)
    parser.add_argument("--method", choices=("peel", "events"), default="events")
    parser.add_argument("--samples", type=int, default=512)
    parser.add_argument("--device", default="cuda:0")
    args = parser.parse_args(argv)
    arrays, labels, data = load_scene(args.scene, args.device)
    peeler = (EventPeeler if args.method == "events" else DevicePeeler)(*arrays)
    peeler.run()
    report = audit(peeler, labels, data, args.samples)
    print(json.dumps(report))
    return 1 if report["rank_mismatches"] else 0


if __name__ == "__main__":
    sys.exit(main())
