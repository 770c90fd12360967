"""Exact CPU oracle for analytic depth peeling (test infrastructure only).

This module is the parity checker of the project.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it;
the product path never calls it.

It restates, with ``fractions.Fraction`` in place of CGAL's exact rationals,
the reference's exact ``bvh-peel`` route:

* rational input parsing ............ ``src/exact_geometry.cpp:5-39``
* polygon cleanup .................... ``src/exact_geometry.cpp:48-71``
* camera inverse, scene import,
  projection, depth-plane fit, window
  clip, positive-area tie rejection .. ``src/camera.cpp:12-229``
* mesh contour topology .............. ``src/peel_common.h:88-124``
* exact predicates, split, separated,
  cut ................................ ``src/bvh_peel.cpp:52-199``
* whole-source classification ........ ``src/peel_common.h:127-167`` with the
  exact policy ``src/bvh_peel.cpp:558-596``
* the all-layer scheduler ............ ``src/peel_common.h:341-460`` (the
  non-accelerated candidate order of lines 403-409; the accelerated order of
  the reference visits the same candidates, so the regions are the same)

plus an exact per-point rank (the independent ray audit of
``src/bvh_peel.cpp:739-784`` restated in projected coordinates).

Coordinates are the reference's exact camera-projected coordinates (not the
GPU's normalised window coordinates).  Pure Python: use it on small scenes
(the reference fixtures, up to a few hundred sources); for large meshes use
``exact_rank`` on sampled points.
"""

from __future__ import annotations

import json
import math
from dataclasses import dataclass, field
from fractions import Fraction as Q
from pathlib import Path


class SceneError(RuntimeError):
    pass


# --------------------------------------------------------------------------
# Parsing (src/exact_geometry.cpp:5-39)


def rational(value) -> Q:
    """Exact value of a JSON coordinate: floats exactly, strings "n" or "n/d"."""
    if isinstance(value, bool):
        raise SceneError(f"Expected integer or rational string: {value}")
    if isinstance(value, float):
        if not math.isfinite(value):
            raise SceneError("Nonfinite coordinate")
        return Q(value)
    if isinstance(value, int):
        return Q(value)
    text = str(value)
    head, slash, tail = text.partition("/")

    def integer(v):
        if not v:
            return False
        i = 1 if v[0] in "+-" else 0
        return i < len(v) and v[i:].isdigit()

    if not integer(head) or (slash and not integer(tail)):
        raise SceneError(f"Expected integer or rational string: {text}")
    if slash:
        d = int(tail)
        if d == 0:
            raise SceneError("Zero rational denominator")
        return Q(int(head), d)
    return Q(int(head))


# --------------------------------------------------------------------------
# Planar predicates (src/bvh_peel.cpp:52-79)


def side(a, b, p) -> Q:
    return (b[0] - a[0]) * (p[1] - a[1]) - (b[1] - a[1]) * (p[0] - a[0])


def sign(x) -> int:
    return (x > 0) - (x < 0)


def side_sign(a, b, p) -> int:
    if p == a or p == b:
        return 0
    return sign(side(a, b, p))


def collinear(a, b, c) -> bool:
    return side(a, b, c) == 0


@dataclass(frozen=True)
class Score:
    """Affine depth plane s(x, y) = a x + b y + c (src/geometry.h:31-34)."""

    a: Q
    b: Q
    c: Q

    def at(self, p) -> Q:
        return self.a * p[0] + self.b * p[1] + self.c

    def __sub__(self, o: Score) -> Score:
        return Score(self.a - o.a, self.b - o.b, self.c - o.c)


def area2(ring) -> Q:
    """Twice the signed area of a ring."""
    total = Q(0)
    for j in range(1, len(ring) - 1):
        total += side(ring[0], ring[j], ring[j + 1])
    return total


# --------------------------------------------------------------------------
# Polygon cleanup (src/exact_geometry.cpp:48-71)


def polygon(points):
    p = list(points)
    if len(p) > 1 and p[0] == p[-1]:
        p.pop()
    changed = True
    while changed and len(p) >= 3:
        changed = False
        for i in range(len(p)):
            a, b, c = p[i - 1], p[i], p[(i + 1) % len(p)]
            if a == b or b == c or collinear(a, b, c):
                del p[i]
                changed = True
                break
    if len(p) < 3 or area2(p) == 0:
        return []
    if area2(p) < 0:
        p.reverse()
    return p


def clip_halfplane(ring, f):
    """Sutherland-Hodgman against f(p) >= 0 (the convex window intersection)."""
    out = []
    for i in range(len(ring)):
        a, b = ring[i], ring[(i + 1) % len(ring)]
        da, db = f(a), f(b)
        if da >= 0:
            out.append(a)
        if (da > 0 and db < 0) or (da < 0 and db > 0):
            t = da / (da - db)
            out.append((a[0] + t * (b[0] - a[0]), a[1] + t * (b[1] - a[1])))
    return out


# --------------------------------------------------------------------------
# Scene import (src/camera.cpp:12-229)


@dataclass
class Camera:
    perspective: bool = False
    near: Q = Q(1, 100)
    world_to_camera: list = field(default_factory=list)  # 3x4
    camera_to_world: list = field(default_factory=list)  # 3x4


@dataclass
class Source:
    id: int
    index: int  # dense input face index (the GPU's source index)
    mesh_face: int
    world: list
    cam: list
    score: Score
    poly: list  # exact ccw convex polygon, projected camera coordinates
    clipped: bool = False


@dataclass
class Scene:
    camera: Camera
    window: tuple
    sources: list
    contours: list
    topology: dict
    input_sources: int = 0
    zero_area: int = 0
    clipped_empty: int = 0

    def by_id(self):
        return {s.id: s for s in self.sources}


def transform(m, p):
    return tuple(m[i][0] * p[0] + m[i][1] * p[1] + m[i][2] * p[2] + m[i][3] for i in range(3))


def read_camera(j) -> Camera:
    c = Camera()
    kind = j.get("type", "orthographic")
    if kind not in ("orthographic", "perspective"):
        raise SceneError("Unknown camera type")
    c.perspective = kind == "perspective"
    if "near" in j:
        c.near = rational(j["near"])
    if c.near <= 0:
        raise SceneError("Near plane must be strictly positive")
    w = [[Q(int(i == k)) for k in range(4)] for i in range(3)]
    if "world_to_camera" in j:
        a = j["world_to_camera"]
        if len(a) != 3 or any(len(r) != 4 for r in a):
            raise SceneError("world_to_camera must be 3x4 affine matrix")
        w = [[rational(x) for x in r] for r in a]
    c.world_to_camera = w
    m = [[w[i][k] for k in range(3)] + [Q(int(i == k)) for k in range(3)] for i in range(3)]
    for k in range(3):
        pivot = k
        while pivot < 3 and m[pivot][k] == 0:
            pivot += 1
        if pivot == 3:
            raise SceneError("Singular camera transform")
        m[k], m[pivot] = m[pivot], m[k]
        d = m[k][k]
        m[k] = [x / d for x in m[k]]
        for i in range(3):
            if i != k:
                v = m[i][k]
                m[i] = [m[i][t] - v * m[k][t] for t in range(6)]
    inv = [[Q(0)] * 4 for _ in range(3)]
    for i in range(3):
        for k in range(3):
            inv[i][k] = m[i][k + 3]
            inv[i][3] -= m[i][k + 3] * w[k][3]
    c.camera_to_world = inv
    return c


def fit(p, z) -> Score:
    x1, y1 = p[1][0] - p[0][0], p[1][1] - p[0][1]
    x2, y2 = p[2][0] - p[0][0], p[2][1] - p[0][1]
    det = x1 * y2 - x2 * y1
    a = ((z[1] - z[0]) * y2 - (z[2] - z[0]) * y1) / det
    b = (x1 * (z[2] - z[0]) - x2 * (z[1] - z[0])) / det
    return Score(a, b, z[0] - a * p[0][0] - b * p[0][1])


def separated_any(a, b) -> bool:
    """Some edge of convex ``a`` has no vertex of ``b`` strictly to its left."""
    for i in range(len(a)):
        u, v = a[i], a[(i + 1) % len(a)]
        if not any(side(u, v, p) > 0 for p in b):
            return True
    return False


def project_triangle(cam, window, camv):
    """Near clip, projection, depth-plane fit and window clip of one triangle
    given in exact camera coordinates (camera.cpp:108-154).

    Returns (score, ccw polygon, projected points, in_window), or the reason it
    is dropped: "clipped_empty" or "zero_area"."""
    xmin, ymin, xmax, ymax = window
    clipped = list(camv)
    if cam.perspective:
        clipped = []
        for i in range(3):
            a, b = camv[i], camv[(i + 1) % 3]
            da, db = a[2] - cam.near, b[2] - cam.near
            if da >= 0:
                clipped.append(a)
            if (da < 0 and db > 0) or (da > 0 and db < 0):
                u = da / (da - db)
                clipped.append(tuple(a[k] + (b[k] - a[k]) * u for k in range(3)))
    if len(clipped) < 3:
        return "clipped_empty"
    projected, depths = [], []
    for p in clipped:
        if cam.perspective:
            projected.append((p[0] / p[2], p[1] / p[2]))
            depths.append(-Q(1) / p[2])
        else:
            projected.append((p[0], p[1]))
            depths.append(p[2])
    k = 2
    while k < len(projected) and collinear(projected[0], projected[1], projected[k]):
        k += 1
    if k == len(projected):
        return "zero_area"
    score = fit([projected[0], projected[1], projected[k]], [depths[0], depths[1], depths[k]])
    in_window = all(xmin <= p[0] <= xmax and ymin <= p[1] <= ymax for p in projected)
    poly = polygon(projected)
    if not in_window and poly:
        for f in (
            lambda p: p[0] - xmin,
            lambda p: xmax - p[0],
            lambda p: p[1] - ymin,
            lambda p: ymax - p[1],
        ):
            poly = clip_halfplane(poly, f)
            if not poly:
                break
        poly = polygon(poly)
    if not poly:
        return "clipped_empty"
    return score, poly, projected, in_window


def read_scene(data, resolved_mesh=True) -> Scene:
    """Exact scene import; ``data`` is the parsed scene JSON (or a path)."""
    if isinstance(data, (str, Path)):
        data = json.loads(Path(data).read_text())
    cam = read_camera(data.get("camera", {}))
    w = data["window"]
    if len(w) != 4:
        raise SceneError("Window must be [xmin,ymin,xmax,ymax]")
    window = tuple(rational(x) for x in w)
    if window[0] >= window[2] or window[1] >= window[3]:
        raise SceneError("Invalid window")
    xmin, ymin, xmax, ymax = window
    s = Scene(cam, window, [], [], {})
    ids = set()
    vertex_ids: dict = {}
    edges: dict = {}
    clipped_count = 0
    for index, t in enumerate(data["triangles"]):
        sid = t.get("id", s.input_sources)
        mesh_face = t.get("mesh_face_id", sid)
        s.input_sources += 1
        if sid in ids:
            raise SceneError("Duplicate source ID")
        ids.add(sid)
        if len(t["vertices"]) != 3:
            raise SceneError("Expected three vertices")
        world, camv = [], []
        for v in t["vertices"]:
            if len(v) != 3:
                raise SceneError("Expected 3D vertex")
            pw = tuple(rational(x) for x in v)
            world.append(pw)
            camv.append(transform(cam.world_to_camera, pw))
        projected_source = project_triangle(cam, window, camv)
        if isinstance(projected_source, str):
            if projected_source == "zero_area":
                s.zero_area += 1
            else:
                s.clipped_empty += 1
            continue
        score, poly, projected, in_window = projected_source
        clipped_camera = not in_window or (
            cam.perspective and any(v[2] < cam.near for v in camv)
        )
        if resolved_mesh:
            if clipped_camera:
                for i in range(len(poly)):
                    s.contours.append((poly[i], poly[(i + 1) % len(poly)]))
                    clipped_count += 1
            else:
                vid = [vertex_ids.setdefault(world[i], len(vertex_ids)) for i in range(3)]
                facing = 1 if side(projected[0], projected[1], projected[2]) > 0 else -1
                for i in range(3):
                    a, b = vid[i], vid[(i + 1) % 3]
                    edges.setdefault((min(a, b), max(a, b)), []).append(
                        (1 if a < b else -1, facing, (projected[i], projected[(i + 1) % 3]))
                    )
        s.sources.append(
            Source(sid, index, mesh_face, world, camv, score, poly, clipped_camera)
        )
    # src/peel_common.h:100-123
    boundary = silhouette = nonmanifold = ignored = 0
    for key in sorted(edges):
        f = edges[key]
        if len(f) == 2 and f[0][0] != f[1][0] and f[0][1] == f[1][1]:
            ignored += 1
            continue
        if len(f) == 1:
            boundary += 1
        elif len(f) != 2 or f[0][0] == f[1][0]:
            nonmanifold += 1
        else:
            silhouette += 1
        s.contours.append(f[0][2])
    s.topology = {
        "resolved_mesh_contract": resolved_mesh,
        "boundary_edges": boundary,
        "silhouette_edges": silhouette,
        "nonmanifold_or_inconsistent_edges": nonmanifold,
        "same_facing_internal_edges_ignored": ignored,
        "camera_clipping_boundary_edges": clipped_count,
        "contour_segments": len(s.contours),
    }
    # Positive-area ties between sources on one exact plane (camera.cpp:181-227).
    groups: dict = {}
    for src in s.sources:
        groups.setdefault((src.score.a, src.score.b, src.score.c), []).append(src)
    for group in groups.values():
        for i in range(len(group)):
            for j in range(i + 1, len(group)):
                a, b = group[i].poly, group[j].poly
                if not separated_any(a, b) and not separated_any(b, a):
                    raise SceneError(
                        "Unsupported positive-area depth tie between sources "
                        f"{group[i].id} and {group[j].id}"
                    )
    return s


# --------------------------------------------------------------------------
# Exact bvh-peel (src/bvh_peel.cpp:80-199, src/peel_common.h:127-460)


def clean(r):
    out = []
    for p in r:
        if not out or p != out[-1]:
            out.append(p)
    if len(out) > 1 and out[0] == out[-1]:
        out.pop()
    return out if len(out) >= 3 else []


def split(r, value):
    """Partition a convex ring by value(p) >= 0 (inside) / <= 0 (outside)."""
    d = [sign(value(p)) for p in r]
    if not any(x < 0 for x in d):
        return r, []
    if not any(x > 0 for x in d):
        return [], r
    inside, outside = [], []
    for i in range(len(r)):
        j = (i + 1) % len(r)
        if d[i] >= 0:
            inside.append(r[i])
        if d[i] <= 0:
            outside.append(r[i])
        if (d[i] > 0 and d[j] < 0) or (d[i] < 0 and d[j] > 0):
            di, dj = value(r[i]), value(r[j])
            t = di / (di - dj)
            p = (r[i][0] + t * (r[j][0] - r[i][0]), r[i][1] + t * (r[j][1] - r[i][1]))
            inside.append(p)
            outside.append(p)
    return clean(inside), clean(outside)


def separated(a, b) -> bool:
    for i in range(len(a)):
        if not any(side_sign(a[i], a[(i + 1) % len(a)], p) > 0 for p in b):
            return True
    return False


def fbox(ring):
    """Float bounding box padded outward (a conservative prefilter only)."""
    xs = [float(p[0]) for p in ring]
    ys = [float(p[1]) for p in ring]
    pad = 1e-9 * (1 + max(abs(v) for v in xs + ys))
    return (min(xs) - pad, min(ys) - pad, max(xs) + pad, max(ys) + pad)


def boxes_overlap(a, b) -> bool:
    return a[0] <= b[2] and b[0] <= a[2] and a[1] <= b[3] and b[1] <= a[3]


def cut(visible, hidden, occluder, delta):
    """Subtract ``occluder`` where ``delta`` = target - occluder score > 0."""
    cb = fbox(occluder)
    out = []
    for p in visible:
        if not boxes_overlap(fbox(p), cb) or separated(p, occluder) or separated(occluder, p):
            out.append(p)
            continue
        d = [sign(delta.at(v)) for v in p]
        nearer, behind = any(x > 0 for x in d), any(x < 0 for x in d)
        if not nearer:
            out.append(p)
            continue
        inside, outside = p, []
        if behind:
            inside, rest = split(inside, delta.at)
            if rest:
                outside.append(rest)
        for j in range(len(occluder)):
            if not inside:
                break
            a, b = occluder[j], occluder[(j + 1) % len(occluder)]
            inside, rest = split(inside, lambda v, a=a, b=b: side(a, b, v))
            if rest:
                outside.append(rest)
        if not inside:
            out.append(p)
        else:
            hidden.append(inside)
            out.extend(outside)
    return out


def touches_contour(poly, e) -> bool:
    """Exact convex polygon / segment contact (src/bvh_peel.cpp:559-574)."""
    for k in range(len(poly)):
        a, b = poly[k], poly[(k + 1) % len(poly)]
        if side_sign(a, b, e[0]) < 0 and side_sign(a, b, e[1]) < 0:
            return False
    pos = neg = False
    for v in poly:
        sg = side_sign(e[0], e[1], v)
        pos |= sg >= 0
        neg |= sg <= 0
    return pos and neg


def ray_order(scene, i, j, p) -> int:
    """1 if source j is strictly nearer at p, 0 if not covering, -1 ambiguous."""
    ring = scene.sources[j].poly
    edge = False
    for k in range(len(ring)):
        sg = side_sign(ring[k], ring[(k + 1) % len(ring)], p)
        if sg < 0:
            return 0
        edge |= sg == 0
    if edge:
        return -1
    sg = sign((scene.sources[i].score - scene.sources[j].score).at(p))
    return -1 if sg == 0 else int(sg > 0)


def classify(scene):
    """Whole-source ranks, -1 where clipping is required (peel_common.h:127-167)."""
    n = len(scene.sources)
    ranks = [-1] * n
    if not scene.topology.get("resolved_mesh_contract", False):
        return ranks
    boxes = [fbox(s.poly) for s in scene.sources]
    cboxes = [fbox(list(e)) for e in scene.contours]
    for i, src in enumerate(scene.sources):
        if any(
            boxes_overlap(boxes[i], cboxes[j]) and touches_contour(src.poly, e)
            for j, e in enumerate(scene.contours)
        ):
            continue
        if len(src.poly) != 3:
            continue
        r = src.poly
        p = ((r[0][0] + r[1][0] + r[2][0]) / 3, (r[0][1] + r[1][1] + r[2][1]) / 3)
        fp = (float(p[0]), float(p[1]))
        pb = (fp[0], fp[1], fp[0], fp[1])
        rank, ambiguous = 0, False
        for j in range(n):
            if j == i or not boxes_overlap(boxes[j], pb):
                continue
            hit = ray_order(scene, i, j, p)
            ambiguous |= hit < 0
            rank += hit > 0
        if not ambiguous:
            ranks[i] = rank
    return ranks


@dataclass
class Patch:
    source: int  # dense index into scene.sources
    points: list


def extract(scene, layers=0):
    """All-layer (or prefix) exact extraction; returns (layers, residual).

    ``layers`` is a list over layers of lists of ``Patch``; residual holds the
    patches left when a prefix was requested (peel_common.h:341-460).
    """
    originals = [Patch(i, list(s.poly)) for i, s in enumerate(scene.sources)]
    ranks = classify(scene)
    residual, direct = [], []
    for i, r in enumerate(ranks):
        if r < 0:
            residual.append(originals[i])
        else:
            while len(direct) <= r:
                direct.append([])
            direct[r].append(i)
    limit = layers or len(originals)
    out = []
    obox = [fbox(p.points) for p in originals]
    k = 0
    while k < limit and (residual or k < len(direct)):
        rboxes = [fbox(p.points) for p in residual]
        visible_all, hidden_all = [], []
        for ti, target in enumerate(residual):
            tb = rboxes[ti]
            score_t = scene.sources[target.source].score
            visible, hidden = [target.points], []
            for c, cand in enumerate(originals):
                if not visible:
                    break
                if ranks[c] < k or cand.source == target.source or not boxes_overlap(obox[c], tb):
                    continue
                visible = cut(visible, hidden, cand.points, score_t - scene.sources[c].score)
            for c, cand in enumerate(residual):
                if not visible:
                    break
                if cand.source == target.source or not boxes_overlap(rboxes[c], tb):
                    continue
                visible = cut(
                    visible, hidden, cand.points, score_t - scene.sources[cand.source].score
                )
            if not visible:
                hidden = [target.points]
            visible_all.extend(Patch(target.source, v) for v in visible)
            hidden_all.extend(Patch(target.source, h) for h in hidden)
        layer = [originals[i] for i in (direct[k] if k < len(direct) else [])] + visible_all
        if not layer:
            raise SceneError("BVH peeling made no progress")
        out.append(layer)
        residual = hidden_all
        k += 1
    if not layers and residual:
        raise SceneError("Peeling exceeded source-count layer limit")
    for kk in range(len(out), len(direct)):
        residual.extend(originals[i] for i in direct[kk])
    return out, residual


def region_area2(scene, layers):
    """{(layer, external source id): exact doubled area} of an extraction."""
    areas: dict = {}
    for k, layer in enumerate(layers):
        for p in layer:
            key = (k, scene.sources[p.source].id)
            areas[key] = areas.get(key, Q(0)) + area2(p.points)
    return areas


# --------------------------------------------------------------------------
# Exact point rank (independent ray audit)


def strictly_inside(ring, p):
    """+1 strictly inside, 0 on the boundary, -1 outside (convex ccw ring)."""
    on = False
    for k in range(len(ring)):
        sg = side_sign(ring[k], ring[(k + 1) % len(ring)], p)
        if sg < 0:
            return -1
        on |= sg == 0
    return 0 if on else 1


class RankIndex:
    """Float-box grid over exact source polygons for fast candidate lookup."""

    def __init__(self, scene, cells=64):
        self.scene = scene
        self.boxes = [fbox(s.poly) for s in scene.sources]
        xs = [b[0] for b in self.boxes] + [b[2] for b in self.boxes] or [0.0, 1.0]
        ys = [b[1] for b in self.boxes] + [b[3] for b in self.boxes] or [0.0, 1.0]
        self.lo = (min(xs), min(ys))
        self.span = (max(max(xs) - self.lo[0], 1e-300), max(max(ys) - self.lo[1], 1e-300))
        self.cells = cells
        self.grid: dict = {}
        for i, b in enumerate(self.boxes):
            for cx in range(self._cx(b[0]), self._cx(b[2]) + 1):
                for cy in range(self._cy(b[1]), self._cy(b[3]) + 1):
                    self.grid.setdefault((cx, cy), []).append(i)

    def _cx(self, x):
        return min(self.cells - 1, max(0, int((x - self.lo[0]) / self.span[0] * self.cells)))

    def _cy(self, y):
        return min(self.cells - 1, max(0, int((y - self.lo[1]) / self.span[1] * self.cells)))

    def candidates(self, p):
        fx, fy = float(p[0]), float(p[1])
        out = []
        for i in self.grid.get((self._cx(fx), self._cy(fy)), []):
            b = self.boxes[i]
            if b[0] <= fx <= b[2] and b[1] <= fy <= b[3]:
                out.append(i)
        return out

    def rank(self, source, p):
        """Exact depth rank of dense source ``source`` at exact point ``p``.

        Returns None when the ray is ambiguous: ``p`` on a boundary of a
        covering source, not strictly inside ``source``, or an exact depth tie.
        """
        src = self.scene.sources[source]
        if strictly_inside(src.poly, p) != 1:
            return None
        z = src.score.at(p)
        rank = 0
        for j in self.candidates(p):
            if j == source:
                continue
            other = self.scene.sources[j]
            inside = strictly_inside(other.poly, p)
            if inside < 0:
                continue
            if inside == 0:
                return None
            zj = other.score.at(p)
            if zj == z:
                return None
            rank += zj < z
        return rank


    def polygon_rank(self, source, ring):
        """Exact rank of ``source`` inside convex ``ring`` at a generic interior point.

        Tries the vertex centroid first, then centroid-to-vertex blends, and
        returns the first unambiguous rank (None if every sample is ambiguous).
        """
        n = len(ring)
        c = (sum(v[0] for v in ring) / n, sum(v[1] for v in ring) / n)
        points = [c]
        for w in (Q(1, 3), Q(1, 7), Q(2, 5)):
            for v in ring:
                points.append((c[0] + w * (v[0] - c[0]), c[1] + w * (v[1] - c[1])))
        for p in points:
            r = self.rank(source, p)
            if r is not None:
                return r
        return None


def to_window(scene, u, v):
    """Exact camera-projected point of normalised window coordinates (u, v);
    ``u``, ``v`` are floats (taken exactly) or Fractions."""
    xmin, ymin, xmax, ymax = scene.window
    return (xmin + Q(u) * (xmax - xmin), ymin + Q(v) * (ymax - ymin))


class SparseRanks:
    """Exact ranks on large meshes: source triangles are imported exactly only
    when a query point needs them.

    The inputs are the device arrays themselves (binary64 vertices, int faces,
    a 4x4 affine camera, the six window/camera settings); the exact scene is
    the rational value of every double.  Candidate sources for a point come
    from a grid over float bounding boxes of the projected triangles, padded
    so that no source containing the point is missed; every decision is then
    exact (the same predicates as ``RankIndex``)."""

    def __init__(self, vertices, faces, camera, settings, cells=512):
        import numpy as np

        self.vertices = np.asarray(vertices, dtype=np.float64)
        self.faces = np.asarray(faces, dtype=np.int64)
        camera = np.asarray(camera, dtype=np.float64).reshape(4, 4)
        settings = np.asarray(settings, dtype=np.float64)
        self.cam = Camera(perspective=bool(settings[4] != 0), near=Q(float(settings[5])),
                          world_to_camera=[[Q(float(x)) for x in camera[r]] for r in range(3)])
        self.window = tuple(Q(float(x)) for x in settings[:4])
        self.cache: dict = {}
        # Float projection, conservative boxes in normalised window coordinates.
        cam = self.vertices @ camera[:3, :3].T + camera[:3, 3]
        tri = cam[self.faces]  # [N, 3, 3]
        w = settings
        scale = np.array([w[2] - w[0], w[3] - w[1]])
        if settings[4]:
            z = tri[:, :, 2]
            front = (z > w[5]).all(axis=1)
            xy = tri[:, :, :2] / np.where(z > 0, z, 1.0)[:, :, None]
        else:
            front = np.ones(len(tri), bool)
            xy = tri[:, :, :2]
        uv = (xy - w[:2]) / scale
        lo, hi = uv.min(axis=1), uv.max(axis=1)
        pad = 1e-9 * (1.0 + np.abs(lo).max(axis=1, initial=0) + np.abs(hi).max(axis=1, initial=0))
        lo = lo - pad[:, None]
        hi = hi + pad[:, None]
        # Triangles crossing the near plane: their projection is unbounded; every
        # query must consider them.
        self.always = np.nonzero(~front)[0].tolist()
        self.cells = cells
        self.lo, self.hi = lo, hi
        # A compressed uniform grid: the faces meeting each cell, cell by cell.
        faces = np.nonzero(front)[0]
        clo = np.clip(np.floor(lo[faces] * cells), 0, cells - 1).astype(np.int64)
        chi = np.clip(np.floor(hi[faces] * cells), 0, cells - 1).astype(np.int64)
        nx, ny = chi[:, 0] - clo[:, 0] + 1, chi[:, 1] - clo[:, 1] + 1
        per = nx * ny
        owner = np.repeat(np.arange(len(faces)), per)
        local = np.arange(int(per.sum())) - np.repeat(np.cumsum(per) - per, per)
        cx = clo[owner, 0] + local % nx[owner]
        cy = clo[owner, 1] + local // nx[owner]
        cell = cx * cells + cy
        order = np.argsort(cell, kind="stable")
        self.cell_faces = faces[owner[order]]
        self.cell_start = np.searchsorted(cell[order], np.arange(cells * cells + 1))

    def source(self, f):
        """(score, exact ccw polygon) of face f, or None if it projects to nothing."""
        if f not in self.cache:
            camv = []
            for v in self.faces[f]:
                pw = tuple(Q(float(x)) for x in self.vertices[v])
                camv.append(transform(self.cam.world_to_camera, pw))
            got = project_triangle(self.cam, self.window, camv)
            self.cache[f] = None if isinstance(got, str) else (got[0], got[1])
        return self.cache[f]

    def candidates(self, u, v):
        u, v = float(u), float(v)
        cx = min(self.cells - 1, max(0, int(u * self.cells)))
        cy = min(self.cells - 1, max(0, int(v * self.cells)))
        c = cx * self.cells + cy
        out = [int(f) for f in self.cell_faces[self.cell_start[c]:self.cell_start[c + 1]]
               if self.lo[f, 0] <= u <= self.hi[f, 0] and self.lo[f, 1] <= v <= self.hi[f, 1]]
        return out + self.always

    def rank(self, face, u, v):
        """Exact rank of `face` at normalised window point (u, v); None if ambiguous."""
        src = self.source(face)
        if src is None:
            return None
        p = to_window(self, u, v)
        if strictly_inside(src[1], p) != 1:
            return None
        z = src[0].at(p)
        rank = 0
        for j in self.candidates(u, v):
            if j == face:
                continue
            other = self.source(j)
            if other is None:
                continue
            inside = strictly_inside(other[1], p)
            if inside < 0:
                continue
            if inside == 0:
                return None
            zj = other[0].at(p)
            if zj == z:
                return None
            rank += zj < z
        return rank

    def polygon_rank(self, face, ring):
        """First unambiguous exact rank at generic interior points of a
        normalised-coordinate ring (vertex mean, then blends toward vertices)."""
        n = len(ring)
        cu = sum(Q(float(x)) for x, _ in ring) / n
        cv = sum(Q(float(y)) for _, y in ring) / n
        points = [(cu, cv)]
        for w in (Q(1, 3), Q(1, 7), Q(2, 5)):
            for x, y in ring:
                points.append((cu + w * (Q(float(x)) - cu), cv + w * (Q(float(y)) - cv)))
        for u, v in points:
            r = self.rank(face, u, v)
            if r is not None:
                return r
        return None


# --------------------------------------------------------------------------
# Parallel sampled ranks (a process pool of SparseRanks over one mesh)

_POOL_MESHES = None
_POOL_RANKS: dict = {}


def _pool_init(hosts):
    global _POOL_MESHES
    _POOL_MESHES = hosts


def _pool_rank(item):
    mesh, face, ring = item
    if mesh not in _POOL_RANKS:
        _POOL_RANKS[mesh] = SparseRanks(*_POOL_MESHES[mesh])
    return _POOL_RANKS[mesh].polygon_rank(face, ring)


def polygon_ranks_multi(hosts, items, processes=None):
    """Exact ranks of (mesh, face, ring) items, ``mesh`` indexing ``hosts``
    (each (vertices, faces, camera, settings)), each as
    ``SparseRanks.polygon_rank``, over a pool of spawned processes (spawned,
    so that the pool is safe after a CUDA context exists in the caller)."""
    import multiprocessing
    import os

    items = list(items)
    if processes is None:
        processes = min(16, os.cpu_count() or 1)
    if processes <= 1 or len(items) < 64:
        cache = {}
        out = []
        for mesh, face, ring in items:
            if mesh not in cache:
                cache[mesh] = SparseRanks(*hosts[mesh])
            out.append(cache[mesh].polygon_rank(face, ring))
        return out
    ctx = multiprocessing.get_context("spawn")
    with ctx.Pool(processes, initializer=_pool_init, initargs=(list(hosts),)) as pool:
        return pool.map(_pool_rank, items, chunksize=max(1, len(items) // (8 * processes)))


def polygon_ranks(host, items, processes=None):
    """polygon_ranks_multi on one mesh: items are (face, ring)."""
    return polygon_ranks_multi([host], [(0, f, r) for f, r in items], processes)
