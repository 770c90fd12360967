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

from . import scenefile

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
        q = scenefile.exact
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


VERTEX_SCOPE = ("Sampled output polygon vertices against the exact rational intersection of "
                "the two projected source-edge (or window) lines their incident edges lie on; "
                "errors in normalised window units and relative to the projected scene extent.")


class ExactOutlines:
    """Exact projected outlines of a mesh's triangles, built on demand.

    The inputs are the peeler's own binary64 arrays (vertices [V,3], faces
    [N,3], the 4x4 affine world-to-camera matrix and the six settings: window
    xmin, ymin, xmax, ymax, perspective flag, near).  Every double is taken
    exactly.  A triangle's outline is its camera-space polygon clipped to
    z >= near (perspective only), projected (x/z, y/z) or (x, y), and mapped
    to the normalised window; its edges, with the window's four borders, are
    every line a vertex of an analytic depth peel can lie on (contour cuts run
    along source edges).  Binary64 boxes of the projections, padded, select
    the triangles near a query."""

    def __init__(self, vertices, faces, camera, settings):
        self.vertices = np.asarray(vertices, dtype=np.float64).reshape(-1, 3)
        self.faces = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
        camera = np.asarray(camera, dtype=np.float64).reshape(4, 4)
        settings = np.asarray(settings, dtype=np.float64).reshape(-1)
        self.matrix = [[Q(float(x)) for x in camera[r]] for r in range(3)]
        self.perspective = bool(settings[4] != 0)
        self.near = Q(float(settings[5]))
        self.window = [Q(float(x)) for x in settings[:4]]
        self._cam = {}
        self._outline = {}
        self._plane = {}
        cam = self.vertices @ camera[:3, :3].T + camera[:3, 3]
        tri = cam[self.faces]
        if self.perspective:
            z = tri[:, :, 2]
            crosses = ~(z > settings[5]).all(axis=1)
            xy = tri[:, :, :2] / np.where(z > 0, z, 1.0)[:, :, None]
        else:
            crosses = np.zeros(len(tri), bool)
            xy = tri[:, :, :2]
        uv = (xy - settings[:2]) / (settings[2:4] - settings[:2])
        lo, hi = uv.min(axis=1), uv.max(axis=1)
        pad = 1e-7 * (1.0 + np.abs(lo).max(axis=1, initial=0) + np.abs(hi).max(axis=1, initial=0))
        self.lo = lo - pad[:, None]
        self.hi = hi + pad[:, None]
        # A triangle that reaches behind the near plane projects without a
        # finite binary64 box: it is a candidate everywhere.
        self.lo[crosses] = -np.inf
        self.hi[crosses] = np.inf
        visible = ~crosses
        if visible.any():
            self.extent = float(max(hi[visible].max(axis=0) - lo[visible].min(axis=0)))
        else:
            self.extent = 1.0

    def _camera_point(self, index):
        if index not in self._cam:
            p = [Q(float(x)) for x in self.vertices[index]]
            self._cam[index] = tuple(row[0] * p[0] + row[1] * p[1] + row[2] * p[2] + row[3]
                                     for row in self.matrix)
        return self._cam[index]

    def _normalise(self, c):
        if self.perspective:
            x, y = c[0] / c[2], c[1] / c[2]
        else:
            x, y = c[0], c[1]
        w = self.window
        return ((x - w[0]) / (w[2] - w[0]), (y - w[1]) / (w[3] - w[1]))

    def outline(self, face):
        """Exact normalised outline of `face` (a list of (u, v) Fractions)."""
        if face not in self._outline:
            ring = [self._camera_point(int(i)) for i in self.faces[face]]
            if self.perspective:
                clipped = []
                for k, a in enumerate(ring):
                    b = ring[(k + 1) % len(ring)]
                    if a[2] >= self.near:
                        clipped.append(a)
                    if (a[2] >= self.near) != (b[2] >= self.near):
                        t = (self.near - a[2]) / (b[2] - a[2])
                        clipped.append(tuple(a[j] + t * (b[j] - a[j]) for j in range(3)))
                ring = [c for c in clipped if c[2] > 0]
            self._outline[face] = [self._normalise(c) for c in ring]
        return self._outline[face]

    def plane(self, face):
        """Exact depth score of `face` as an affine function a*u + b*v + c of
        the normalised window point (the score is z for an orthographic
        camera and 1/z for a pinhole one, both affine in the projection), or
        None when the triangle projects to a segment or a point."""
        if face not in self._plane:
            ring = [self._camera_point(int(i)) for i in self.faces[face]]
            uv = [self._normalise(c) for c in ring] if all(c[2] != 0 for c in ring) \
                or not self.perspective else None
            result = None
            if uv is not None:
                score = [1 / c[2] if self.perspective else c[2] for c in ring]
                (u0, v0), (u1, v1), (u2, v2) = uv
                det = (u1 - u0) * (v2 - v0) - (u2 - u0) * (v1 - v0)
                if det != 0:
                    ds1, ds2 = score[1] - score[0], score[2] - score[0]
                    a = (ds1 * (v2 - v0) - ds2 * (v1 - v0)) / det
                    b = ((u1 - u0) * ds2 - (u2 - u0) * ds1) / det
                    result = (a, b, score[0] - a * u0 - b * v0)
            self._plane[face] = result
        return self._plane[face]

    def lines_near(self, lo, hi, face=None):
        """Exact lines (pairs of distinct exact points) of every outline whose
        box meets the box [lo, hi], plus the window borders and, with `face`,
        the lines where `face`'s depth equals each of those triangles' (the
        iterative clipping route cuts along them)."""
        hit = np.nonzero((self.lo[:, 0] <= hi[0]) & (self.hi[:, 0] >= lo[0])
                         & (self.lo[:, 1] <= hi[1]) & (self.hi[:, 1] >= lo[1]))[0]
        one, zero = Q(1), Q(0)
        lines = [((zero, zero), (one, zero)), ((one, zero), (one, one)),
                 ((one, one), (zero, one)), ((zero, one), (zero, zero))]
        own = self.plane(face) if face is not None else None
        for f in hit:
            ring = self.outline(int(f))
            for k in range(len(ring)):
                a, b = ring[k], ring[(k + 1) % len(ring)]
                if a != b:
                    lines.append((a, b))
            other = self.plane(int(f)) if own is not None and int(f) != face else None
            if other is not None:
                da, db, dc = (x - y for x, y in zip(own, other))
                if db != 0:
                    lines.append(((zero, -dc / db), (one, -(da + dc) / db)))
                elif da != 0:
                    lines.append(((-dc / da, zero), (-dc / da, one)))
        return lines


def _best_line(lines, floats, p, q):
    """Index of the line nearest to both float points p and q, and that
    distance (the larger of the two, in normalised units)."""
    a, d = floats[:, 0:2], floats[:, 2:4] - floats[:, 0:2]
    length = np.maximum(np.hypot(d[:, 0], d[:, 1]), 1e-300)
    dp = np.abs(d[:, 0] * (p[1] - a[:, 1]) - d[:, 1] * (p[0] - a[:, 0])) / length
    dq = np.abs(d[:, 0] * (q[1] - a[:, 1]) - d[:, 1] * (q[0] - a[:, 0])) / length
    worst = np.maximum(dp, dq)
    k = int(np.argmin(worst))
    return k, float(worst[k])


def _intersection(l1, l2):
    """Exact intersection point of two lines given by exact point pairs, or
    None when they are parallel."""
    (a, b), (c, d) = l1, l2
    r = (b[0] - a[0], b[1] - a[1])
    s = (d[0] - c[0], d[1] - c[1])
    den = r[0] * s[1] - r[1] * s[0]
    if den == 0:
        return None
    t = ((c[0] - a[0]) * s[1] - (c[1] - a[1]) * s[0]) / den
    return (a[0] + t * r[0], a[1] + t * r[1])


def vertex_audit(polygons, sources, outlines, samples=512, seed=0, tolerance=1e-7):
    """Exact error of sampled output polygon vertices.

    `polygons` are (k, 2) float arrays in the normalised window, `sources`
    their dense face indices into `outlines` (an ExactOutlines).  For each
    sampled polygon, every vertex's two incident edges are matched to the
    exact line nearest to both of their endpoints - a source edge, a window
    border or a line of equal depth between the polygon's source and another
    triangle whose box meets the source's; the vertex's
    exact position is those lines' rational intersection.  A vertex whose
    edges match no line within `tolerance`, or whose two edges match one line
    (a collinear vertex), is counted and not measured.  Returns a report with
    the maximum absolute error (normalised window units, per coordinate) and
    that maximum relative to the projected scene's extent."""
    count = len(polygons)
    rng = np.random.default_rng(seed)
    picks = rng.choice(count, size=min(samples, count), replace=False) if count else []
    measured = collinear = unexplained = 0
    worst = 0.0
    worst_example = None
    for i in picks:
        v = np.asarray(polygons[i], dtype=np.float64)
        n = len(v)
        if n < 3:
            continue
        face = int(sources[i])
        lines = outlines.lines_near(outlines.lo[face], outlines.hi[face], face) \
            if np.isfinite(outlines.lo[face]).all() else \
            outlines.lines_near(v.min(0) - 1e-7, v.max(0) + 1e-7, face)
        floats = np.array([[float(a[0]), float(a[1]), float(b[0]), float(b[1])]
                           for a, b in lines])
        fitted = [_best_line(lines, floats, v[k], v[(k + 1) % n]) for k in range(n)]
        for k in range(n):
            (l_in, d_in), (l_out, d_out) = fitted[k - 1], fitted[k]
            if max(d_in, d_out) > tolerance:
                unexplained += 1
                continue
            point = _intersection(lines[l_in], lines[l_out])
            if point is None:
                collinear += 1
                continue
            err = float(max(abs(Q(float(v[k, 0])) - point[0]),
                            abs(Q(float(v[k, 1])) - point[1])))
            measured += 1
            if err > worst:
                worst = err
                worst_example = {"polygon": int(i), "vertex": int(k), "source": face,
                                 "uv": v[k].tolist(),
                                 "exact": [float(point[0]), float(point[1])]}
    return {"scope": VERTEX_SCOPE, "polygons": int(len(picks)), "vertices_measured": measured,
            "collinear_vertices": collinear, "unexplained_vertices": unexplained,
            "max_abs_error": worst, "scene_extent": outlines.extent,
            "max_rel_error": worst / outlines.extent, "worst": worst_example}


def peeler_vertex_audit(peeler, samples=512, seed=0):
    """vertex_audit of a finished extraction, against its own input arrays."""
    info = peeler.read_status()
    count = info["polygons"]
    n = peeler.output.sizes[:count].cpu().numpy()
    v = peeler.output.vertices[:count].cpu().numpy()
    src = peeler.output_sources[:count].cpu().numpy()
    keep = np.nonzero(n >= 3)[0]
    outlines = ExactOutlines(peeler.vertices.cpu().numpy(), peeler.faces.cpu().numpy(),
                             peeler.camera.cpu().numpy(), peeler.settings.cpu().numpy())
    return vertex_audit([v[i, : n[i]] for i in keep], src[keep], outlines, samples, seed)


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
