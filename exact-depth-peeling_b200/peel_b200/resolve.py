"""Exact intersection splitting of a triangle scene (offline, on the CPU).

    python -m peel_b200.resolve INPUT.json OUTPUT.json

The peelers take resolved meshes: no two triangles may cross.  This is the
camera-independent preprocessing that produces one
(src/resolve_intersections.cpp:19-105): every triangle is split where other
triangles meet it, in exact rational arithmetic, and each piece keeps its
parent's provenance (`original_source_id`, `mesh_face_id`); the output scene
carries the input triangles as `original_triangles` and writes coordinates
as exact rational strings ("n/d"), like the reference.

Construction (this module's own; the reference calls CGAL's autorefine):

1. Candidate pairs come from a sweep over padded binary64 boxes; each pair's
   contact is computed exactly: the part of each triangle on the other's
   plane, intersected along the planes' common line.  Coplanar pairs must
   not overlap with positive area (outside the contract, as in the
   reference); their touching points are kept.
2. A triangle whose interior a contact segment crosses is cut by the
   segment's supporting line (in its own plane), so its pieces are convex.
3. Every point created by a contact or a cut is inserted into every piece
   edge it lies on, so pieces that meet along a contact share the same
   edges exactly.  Where two triangles cross, the four pieces along the
   crossing then share its edges, which makes them non-manifold edges: the
   contours the resolved-mesh topology keeps (src/peel_common.h:100-123).
4. A piece that stayed a triangle is written as is; any other piece is
   written as a fan, in the parent's winding: from its first corner (a
   vertex not collinear with its neighbours) whose neighbours are corners
   too, or else around the centroid of its first three corners.

Two implementations of the same construction give identical output: the host
C++ library libedp_resolve.so (include/edp_resolve.h: exact integer
arithmetic on the scene's binary64 coordinates, all host threads), used
whenever every input coordinate is a binary64 value and the library is built,
and the arbitrary-precision rational code below, used otherwise (rational
inputs, or numbers beyond the native size limit).

Unlike the reference's importer, the input need not be a manifold: any
triangle soup without coplanar overlaps is accepted.  Zero-area input
triangles pass through unchanged.
"""

import ctypes
import json
import sys
import time
from fractions import Fraction as Q
from pathlib import Path

import numpy as np

from . import scenefile


# Errors in the input scene, its numbers included (the scene reader's error).
ResolveError = scenefile.SceneFormatError


# ---------------------------------------------------------------- numbers

# A scene number as an exact rational: JSON numbers exactly, strings as
# integers or "numerator/denominator" only (src/exact_geometry.cpp:5-39).
rational = scenefile.rational


def text(q):
    """An exact rational as the reference writes it: "n/d", "/1" for integers."""
    return f"{q.numerator}/{q.denominator}"


# ---------------------------------------------------------------- vectors


def sub(a, b):
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def add(a, b):
    return (a[0] + b[0], a[1] + b[1], a[2] + b[2])


def scale(a, s):
    return (a[0] * s, a[1] * s, a[2] * s)


def dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


ZERO = (Q(0), Q(0), Q(0))


def on_open_segment(x, u, w):
    """x strictly between u and w on the segment u-w."""
    d = sub(w, u)
    r = sub(x, u)
    if cross(d, r) != ZERO:
        return None
    t = dot(r, d)
    return t / dot(d, d) if 0 < t < dot(d, d) else None


def collinear(u, w, x):
    return cross(sub(w, u), sub(x, u)) == ZERO


# ---------------------------------------------------------------- contacts


class Face:
    """One input triangle: exact vertices, plane (normal . p = offset)."""

    def __init__(self, index, record):
        self.index = index
        self.record = record
        vertices = record["vertices"]
        if len(vertices) != 3 or any(len(v) != 3 for v in vertices):
            raise ResolveError("Expected a triangle of 3D vertices")
        self.v = tuple(tuple(rational(c) for c in p) for p in vertices)
        self.normal = cross(sub(self.v[1], self.v[0]), sub(self.v[2], self.v[0]))
        self.offset = dot(self.normal, self.v[0])
        self.degenerate = self.normal == ZERO
        self.cuts = []  # (p, r): supporting lines of contact segments crossing the interior

    def plane(self, p):
        return dot(self.normal, p) - self.offset

    def on_boundary(self, p, r):
        """The segment p-r lies on the line of one of this triangle's edges."""
        return any(collinear(self.v[k], self.v[(k + 1) % 3], p)
                   and collinear(self.v[k], self.v[(k + 1) % 3], r) for k in range(3))


def plane_section(face, other):
    """Points of `face` on `other`'s plane: None (strictly one side),
    "coplanar", or a list of one or two distinct points."""
    values = [other.plane(p) for p in face.v]
    if all(v > 0 for v in values) or all(v < 0 for v in values):
        return None
    if all(v == 0 for v in values):
        return "coplanar"
    points = [face.v[k] for k in range(3) if values[k] == 0]
    for k in range(3):
        a, b = values[k], values[(k + 1) % 3]
        if (a < 0 < b) or (b < 0 < a):
            u, w = face.v[k], face.v[(k + 1) % 3]
            points.append(add(u, scale(sub(w, u), a / (a - b))))
    unique = []
    for p in points:
        if p not in unique:
            unique.append(p)
    return unique


def dominant_axes(normal):
    k = max(range(3), key=lambda i: abs(normal[i]))
    return [i for i in range(3) if i != k]


def coplanar_contact(fa, fb):
    """Touching points of two coplanar triangles; raises on a positive-area
    overlap (outside the resolved-mesh contract)."""
    ax = dominant_axes(fa.normal)
    flat = lambda p: (p[ax[0]], p[ax[1]])
    ta, tb = [flat(p) for p in fa.v], [flat(p) for p in fb.v]
    orient = lambda a, b, c: (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0])
    sa = 1 if orient(*ta) > 0 else -1
    poly = [(p, q) for p, q in zip(tb, fb.v)]
    for k in range(3):
        a, b = ta[k], ta[(k + 1) % 3]
        side = lambda p: sa * orient(a, b, p)
        out = []
        for i in range(len(poly)):
            (p, p3), (q, q3) = poly[i], poly[(i + 1) % len(poly)]
            sp, sq = side(p), side(q)
            if sp >= 0:
                out.append((p, p3))
            if (sp > 0 > sq) or (sq > 0 > sp):
                t = sp / (sp - sq)
                x3 = add(p3, scale(sub(q3, p3), t))
                out.append((flat(x3), x3))
        poly = out
        if not poly:
            return []
    area2 = sum(orient(poly[0][0], poly[i][0], poly[i + 1][0]) for i in range(1, len(poly) - 1))
    if area2 != 0:
        raise overlap_error(fa, fb)
    return [p3 for _, p3 in poly]


def contact(fa, fb):
    """Exact contact of two non-degenerate triangles: (points, segment or None)."""
    sa = plane_section(fb, fa)
    if sa is None:
        return [], None
    if sa == "coplanar":
        return coplanar_contact(fa, fb), None
    sb = plane_section(fa, fb)
    if sb is None:
        return [], None
    line = cross(fa.normal, fb.normal)
    ra = sorted((dot(line, p), p) for p in sa)
    rb = sorted((dot(line, p), p) for p in sb)
    lo = max(ra[0], rb[0])
    hi = min(ra[-1], rb[-1])
    if lo[0] > hi[0]:
        return [], None
    if lo[0] == hi[0]:
        return [lo[1]], None
    return [lo[1], hi[1]], (lo[1], hi[1])


# ---------------------------------------------------------------- pieces


def shared_contact_only(live, corners, pairs):
    """For each candidate pair, True when the two triangles can only meet in
    the vertices they share exactly: some vertex of one lies clearly off the
    other's plane, every such vertex on the same side, and the rest are
    vertices of the other (a triangle meets a plane only in its points on
    it).  False leaves the pair to the exact test.

    "Clearly" is binary64 against a margin: coordinates rounded from exact
    values (relative error u), differences, a cross product and a dot
    product stay within about 600 u M^3 of the exact side value, M the
    largest coordinate magnitude of the pair; the margin is 1e-12 M^3, and
    pairs with M outside [1e-50, 1e50] are left to the exact test."""
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    done = np.zeros(len(pairs), dtype=bool)
    for a_col, b_col in ((0, 1), (1, 0)):
        with np.errstate(over="ignore", invalid="ignore"):  # untrusted pairs are discarded
            trusted, side, tol = _sides(corners, pairs, a_col, b_col)
            clear = (side > tol) | (side < -tol)
            one_side = (np.all(~clear | (side > 0), axis=1)
                        | np.all(~clear | (side < 0), axis=1))
        for k in np.nonzero(trusted & one_side & clear.any(axis=1) & ~done)[0]:
            fa, fb = live[pairs[k, a_col]], live[pairs[k, b_col]]
            done[k] = all(clear[k, v] or fb.v[v] in fa.v for v in range(3))
    return done


def _sides(corners, pairs, a_col, b_col):
    """Binary64 side values of each pair's second triangle against the
    first one's plane, their margin, and whether the pair's range is trusted."""
    A, B = corners[pairs[:, a_col]], corners[pairs[:, b_col]]
    m = np.maximum(np.abs(A).max(axis=(1, 2)), np.abs(B).max(axis=(1, 2)))
    trusted = (m >= 1e-50) & (m <= 1e50)
    tol = (1e-12 * m ** 3)[:, None]
    normal = np.cross(A[:, 1] - A[:, 0], A[:, 2] - A[:, 0])
    side = np.einsum("kvj,kj->kv", B - A[:, :1], normal)
    return trusted, side, tol


def split(poly, p, r, normal):
    """Both sides of the convex polygon `poly` (3D, in the plane with
    `normal`) about the line p-r of that plane; parts without area dropped."""
    d = sub(r, p)
    side = [dot(cross(d, sub(v, p)), normal) for v in poly]
    if all(s >= 0 for s in side) or all(s <= 0 for s in side):
        return [poly]
    left, right = [], []
    n = len(poly)
    for i in range(n):
        u, w = poly[i], poly[(i + 1) % n]
        su, sw = side[i], side[(i + 1) % n]
        if su >= 0:
            left.append(u)
        if su <= 0:
            right.append(u)
        if (su > 0 > sw) or (sw > 0 > su):
            x = add(u, scale(sub(w, u), su / (su - sw)))
            left.append(x)
            right.append(x)
    return [part for part in (left, right) if len(part) >= 3 and area_vector(part) != ZERO]


def area_vector(poly):
    total = ZERO
    for i in range(1, len(poly) - 1):
        total = add(total, cross(sub(poly[i], poly[0]), sub(poly[i + 1], poly[0])))
    return total


def boxes(points):
    a = np.array([[float(c) for c in p] for p in points], dtype=np.float64).reshape(-1, 3)
    return a


def candidate_pairs(lo, hi):
    """Index pairs whose boxes overlap (sweep along x)."""
    order = np.argsort(lo[:, 0], kind="stable")
    slo, shi = lo[order], hi[order]
    pairs = []
    for k in range(len(order)):
        end = np.searchsorted(slo[:, 0], shi[k, 0], side="right")
        if end <= k + 1:
            continue
        rest = np.arange(k + 1, end)
        keep = rest[np.all(slo[rest, 1:] <= shi[k, 1:], axis=1)
                    & np.all(shi[rest, 1:] >= slo[k, 1:], axis=1)]
        pairs.extend((int(order[k]), int(order[j])) for j in keep)
    return pairs


def resolve(data, native=None):
    """The resolved scene (a new dict) and a summary of the preprocessing.

    `native` None picks the C++ library when every coordinate is binary64
    and the library is built; True requires it, False uses the rational
    code."""
    start = time.perf_counter()
    triangles = data["triangles"]
    faces = [Face(i, t) for i, t in enumerate(triangles)]
    import_seconds = time.perf_counter() - start
    if native is not False:
        done = _resolve_native(data, faces, import_seconds, required=bool(native))
        if done is not None:
            return done
    start = time.perf_counter()
    live = [f for f in faces if not f.degenerate]
    if live:
        corners = np.stack([boxes(f.v) for f in live])
        pad = 1e-9 * (np.abs(corners).max(axis=(1, 2)) + 1.0)
        lo = corners.min(axis=1) - pad[:, None]
        hi = corners.max(axis=1) + pad[:, None]
        pairs = candidate_pairs(lo, hi)
        skip = shared_contact_only(live, corners, pairs)
        pairs = [pq for pq, gone in zip(pairs, skip) if not gone]
    else:
        pairs = []
    points = []  # contact points and cut vertices: inserted into the edges they lie on
    segments = 0
    for a, b in pairs:
        fa, fb = live[a], live[b]
        found, segment = contact(fa, fb)
        points.extend(x for x in found if not (x in fa.v and x in fb.v))
        if segment is None:
            continue
        crossing = False
        for f in (fa, fb):
            if f.on_boundary(*segment):
                continue
            crossing = True
            if not any(collinear(p, r, segment[0]) and collinear(p, r, segment[1])
                       for p, r in f.cuts):
                f.cuts.append(segment)
        segments += crossing
    pieces = {}
    for f in live:
        parts = [list(f.v)]
        for p, r in f.cuts:
            parts = [q for part in parts for q in split(part, p, r, f.normal)]
        pieces[f.index] = parts
        if f.cuts:
            points.extend(v for part in parts for v in part if v not in f.v)
    unique = list(dict.fromkeys(points))
    cloud = boxes(unique) if unique else np.zeros((0, 3))
    out = []
    cut_faces = sum(1 for f in live if f.cuts)
    for f in faces:
        record = f.record
        source = record.get("original_source_id", record.get("id", f.index))
        mesh_face = record.get("mesh_face_id", source)
        if f.degenerate:
            polygons = [list(f.v)]
        else:
            polygons = []
            for part in pieces[f.index]:
                polygons.append(insert_points(part, unique, cloud))
        for poly in polygons:
            for tri in fan(poly):
                out.append({"id": len(out), "original_source_id": source,
                            "mesh_face_id": mesh_face,
                            "vertices": [[text(c) for c in p] for p in tri]})
    refine_seconds = time.perf_counter() - start
    summary = {
        "method": "exact rational line splitting with shared-edge insertion",
        "arithmetic": "exact rational constructions",
        "implementation": "python",
        "input_triangles": len(triangles),
        "output_triangles": len(out),
        "intersection_segments": segments,
        "cut_triangles": cut_faces,
        "import_seconds": import_seconds,
        "refinement_seconds": refine_seconds,
        "positive_area_coincident_surfaces_supported": False,
    }
    result = dict(data)
    result["triangles"] = out
    if "original_triangles" not in result:
        result["original_triangles"] = triangles
    result["intersection_preprocessing"] = summary
    return result, summary


# ---------------------------------------------------------------- native

NATIVE = Path(__file__).resolve().parent / "libedp_resolve.so"
_native_lib = None


def native_library():
    """ctypes handle of libedp_resolve.so, or None when it is not built."""
    global _native_lib
    if _native_lib is None and NATIVE.exists():
        lib = ctypes.CDLL(str(NATIVE))
        P, I64 = ctypes.c_void_p, ctypes.c_int64
        lib.edp_resolve_abi_version.restype = ctypes.c_int
        lib.edp_resolve.argtypes = [P, I64, ctypes.c_int, ctypes.c_int, ctypes.POINTER(P)]
        lib.edp_resolve.restype = ctypes.c_int
        lib.edp_resolution_triangles.argtypes = [P]
        lib.edp_resolution_triangles.restype = I64
        lib.edp_resolution_summary.argtypes = [P, P]
        lib.edp_resolution_summary.restype = None
        lib.edp_resolution_binary64.argtypes = [P, P, P]
        lib.edp_resolution_binary64.restype = ctypes.c_int
        lib.edp_resolution_exact.argtypes = [P, P, I64]
        lib.edp_resolution_exact.restype = I64
        lib.edp_resolution_overlap.argtypes = [P, P, P]
        lib.edp_resolution_overlap.restype = None
        lib.edp_resolution_free.argtypes = [P]
        lib.edp_resolution_free.restype = None
        if lib.edp_resolve_abi_version() != 1:
            raise RuntimeError(f"{NATIVE.name}: unexpected ABI version")
        _native_lib = lib
    return _native_lib


class NativeResolution:
    """One run of the C++ resolver over binary64 triangles [T, 3, 3]."""

    TOO_LARGE, BAD_INPUT = 2, 3

    def __init__(self, triangles, threads=0, exact_text=False):
        lib = native_library()
        if lib is None:
            raise RuntimeError(f"{NATIVE.name} is not built (exact-depth-peeling_b200/build.py)")
        tri = np.ascontiguousarray(triangles, dtype=np.float64).reshape(-1, 9)
        self._lib = lib
        self._handle = ctypes.c_void_p()
        self.status = lib.edp_resolve(tri.ctypes.data, tri.shape[0], int(threads),
                                      int(bool(exact_text)), ctypes.byref(self._handle))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        if self._handle:
            self._lib.edp_resolution_free(self._handle)
            self._handle = ctypes.c_void_p()

    def overlap(self):
        a, b = ctypes.c_int64(), ctypes.c_int64()
        self._lib.edp_resolution_overlap(self._handle, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def summary(self):
        s = np.zeros(6, dtype=np.int64)
        self._lib.edp_resolution_summary(self._handle, s.ctypes.data)
        keys = ("intersection_segments", "cut_triangles", "candidate_pairs", "exact_pairs",
                "points", "scale_exponent")
        return dict(zip(keys, (int(v) for v in s)))

    def arrays(self):
        """(triangles [T, 3, 3] correctly rounded, parents [T] input indices)."""
        t = int(self._lib.edp_resolution_triangles(self._handle))
        vertices = np.empty((t, 3, 3), dtype=np.float64)
        parents = np.empty(t, dtype=np.int64)
        self._lib.edp_resolution_binary64(self._handle, vertices.ctypes.data, parents.ctypes.data)
        return vertices, parents

    def exact(self):
        """Per output corner the exact coordinates as (X, Y, Z, W) integers;
        the value is (X, Y, Z) / (W 2^E)."""
        size = int(self._lib.edp_resolution_exact(self._handle, None, 0))
        buf = ctypes.create_string_buffer(size)
        self._lib.edp_resolution_exact(self._handle, buf, size)
        return [tuple(int(h, 16) for h in line.split())
                for line in buf.value.decode().split("\n") if line]


def overlap_error(fa, fb):
    return ResolveError(
        f"Triangles {fa.record.get('id', fa.index)} and {fb.record.get('id', fb.index)} "
        "overlap on one plane with positive area; coincident surfaces are outside the "
        "resolved-mesh contract")


def resolve_arrays(triangles, threads=0):
    """Resolve a binary64 triangle soup [T, 3, 3] with the C++ resolver:
    returns (triangles [T', 3, 3], the exact pieces correctly rounded to
    binary64; parents [T'], each piece's input triangle; summary)."""
    with NativeResolution(triangles, threads) as r:
        if r.status == 1:
            a, b = r.overlap()
            raise ResolveError(f"Triangles {a} and {b} overlap on one plane with positive area; "
                               "coincident surfaces are outside the resolved-mesh contract")
        if r.status:
            raise RuntimeError(f"native resolver failed with status {r.status}")
        vertices, parents = r.arrays()
        return vertices, parents, r.summary()


def _binary64(q):
    try:
        x = float(q)
    except OverflowError:
        return None
    return x if Q(x) == q else None


def _resolve_native(data, faces, import_seconds, required):
    """resolve() through the C++ library; None when it does not apply (not
    built, rational inputs, numbers beyond its limits) and not `required`."""
    if native_library() is None:
        if required:
            raise RuntimeError(f"{NATIVE.name} is not built (exact-depth-peeling_b200/build.py)")
        return None
    coords = [_binary64(c) for f in faces for p in f.v for c in p]
    if any(c is None for c in coords):
        if required:
            raise ValueError("the native resolver takes binary64 coordinates only")
        return None
    start = time.perf_counter()
    tri = np.array(coords, dtype=np.float64).reshape(-1, 3, 3)
    with NativeResolution(tri, exact_text=True) as r:
        if r.status == 1:
            a, b = r.overlap()
            raise overlap_error(faces[a], faces[b])
        if r.status in (NativeResolution.TOO_LARGE, NativeResolution.BAD_INPUT) and not required:
            return None
        if r.status:
            raise RuntimeError(f"native resolver failed with status {r.status}")
        info = r.summary()
        _, parents = r.arrays()
        corners = r.exact()
    scale = info["scale_exponent"]
    out = []
    for t, parent in enumerate(parents):
        record = faces[int(parent)].record
        source = record.get("original_source_id", record.get("id", int(parent)))
        mesh_face = record.get("mesh_face_id", source)
        vertices = []
        for x, y, z, w in corners[3 * t:3 * t + 3]:
            den = w << scale
            vertices.append([text(Q(x, den)), text(Q(y, den)), text(Q(z, den))])
        out.append({"id": len(out), "original_source_id": source, "mesh_face_id": mesh_face,
                    "vertices": vertices})
    summary = {
        "method": "exact rational line splitting with shared-edge insertion",
        "arithmetic": "exact rational constructions",
        "implementation": "native",
        "input_triangles": len(faces),
        "output_triangles": len(out),
        "intersection_segments": info["intersection_segments"],
        "cut_triangles": info["cut_triangles"],
        "import_seconds": import_seconds,
        "refinement_seconds": time.perf_counter() - start,
        "positive_area_coincident_surfaces_supported": False,
    }
    result = dict(data)
    result["triangles"] = out
    if "original_triangles" not in result:
        result["original_triangles"] = data["triangles"]
    result["intersection_preprocessing"] = summary
    return result, summary


def insert_points(poly, points, cloud):
    """`poly` with every point of `points` lying inside one of its edges
    inserted there, in order along the edge."""
    if not points:
        return poly
    corners = boxes(poly)
    pad = 1e-9 * (np.abs(corners).max() + 1.0)
    near = np.nonzero(np.all(cloud >= corners.min(0) - pad, axis=1)
                      & np.all(cloud <= corners.max(0) + pad, axis=1))[0]
    if len(near) == 0:
        return poly
    # Points clearly off an edge's line (binary64 cross product above a
    # margin far over its rounding error, as in shared_contact_only) skip the
    # exact test; outside [1e-50, 1e50] every point takes it.
    m = float(max(np.abs(corners).max(), np.abs(cloud[near]).max()))
    tol = 1e-12 * m ** 2 if 1e-50 <= m <= 1e50 else np.inf
    result = []
    n = len(poly)
    for i in range(n):
        u, w = poly[i], poly[(i + 1) % n]
        result.append(u)
        fu, fw = corners[i], corners[(i + 1) % n]
        with np.errstate(over="ignore", invalid="ignore"):  # out of range: tol is inf
            off = np.abs(np.cross(fw - fu, cloud[near] - fu)).max(axis=1)
        inside = []
        for k in near[off <= tol]:
            t = on_open_segment(points[k], u, w)
            if t is not None:
                inside.append((t, points[k]))
        result.extend(p for _, p in sorted(inside))
    return result


def fan(poly):
    """Triangles of a convex piece: itself when it is one; else a fan from its
    first corner whose two neighbours are corners too (no point inserted on
    the edges at that corner, so no fan triangle is degenerate), or, when
    every corner has an inserted neighbour, a fan around the centroid of its
    first three corners.  Corners are vertices not collinear with their
    neighbours; every boundary edge is kept, so there are no T-junctions."""
    if len(poly) == 3:
        return [poly]
    n = len(poly)
    corner = [not collinear(poly[i - 1], poly[(i + 1) % n], poly[i]) for i in range(n)]
    for v in range(n):
        if corner[v] and corner[v - 1] and corner[(v + 1) % n]:
            return [[poly[v], poly[(v + t) % n], poly[(v + t + 1) % n]] for t in range(1, n - 1)]
    corners = [poly[i] for i in range(n) if corner[i]]
    center = tuple(sum(p[c] for p in corners[:3]) / 3 for c in range(3))
    return [[center, poly[i], poly[(i + 1) % n]] for i in range(n)]


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 2:
        sys.stderr.write("python -m peel_b200.resolve INPUT.json OUTPUT.json\nExact "
                         "camera-independent intersection splitting of a triangle scene.\n")
        return 2
    try:
        with open(argv[0]) as f:
            data = json.load(f)
        result, summary = resolve(data)
        with open(argv[1], "w") as f:
            json.dump(result, f)
            f.write("\n")
    except (OSError, ValueError, KeyError, TypeError) as e:
        sys.stderr.write(f"error: {e}\n")
        return 1
    print(json.dumps(summary))
    return 0


if __name__ == "__main__":
    sys.exit(main())
