"""Seeded synthetic scenes for the benchmark configurations.

Every generator returns host numpy arrays ``(vertices float64 [V,3], faces
int32 [N,3], camera float64 [4,4], settings float64 [6])`` with shared
(welded) vertices, so the peeler sees mesh connectivity.  The shapes, sizes
and value distributions follow the benchmark's configuration text; no public
dataset is involved.
"""

import math

import numpy as np


def _ortho_down_z(vertices, margin=0.05):
    """Orthographic view along world -z (camera = diag(1, 1, -1)); the window is
    the xy bounding box grown by ``margin`` on each side."""
    camera = np.diag([1.0, 1.0, -1.0, 1.0])
    lo, hi = vertices[:, :2].min(0), vertices[:, :2].max(0)
    pad = margin * (hi - lo)
    settings = np.array([lo[0] - pad[0], lo[1] - pad[1], hi[0] + pad[0], hi[1] + pad[1], 0.0,
                         0.01])
    return camera, settings


def _pinhole(eye, target, fov_degrees=60.0, near=0.01):
    """Pinhole camera at ``eye`` looking at ``target``; camera z is depth
    (positive in front), the window is the normalised image plane +-tan(fov/2)."""
    eye, target = np.asarray(eye, float), np.asarray(target, float)
    forward = target - eye
    forward /= np.linalg.norm(forward)
    up = np.array([0.0, 1.0, 0.0]) if abs(forward[1]) < 0.9 else np.array([1.0, 0.0, 0.0])
    right = np.cross(up, forward)
    right /= np.linalg.norm(right)
    true_up = np.cross(forward, right)
    rotation = np.stack([right, true_up, forward])
    camera = np.eye(4)
    camera[:3, :3] = rotation
    camera[:3, 3] = -rotation @ eye
    h = math.tan(math.radians(fov_degrees) / 2)
    settings = np.array([-h, -h, h, h, 1.0, near])
    return camera, settings


def icosphere(subdivisions):
    """Unit icosphere: 20 * 4**subdivisions faces, outward (ccw) winding."""
    t = (1 + 5 ** 0.5) / 2
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
             (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(v, float) / np.linalg.norm(v) for v in verts]
    for _ in range(subdivisions):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nxt = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nxt += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nxt
    return np.array(verts), np.array(faces, dtype=np.int32)


def nested_icospheres(seed=0):
    """Two nested noisy icospheres (2 x 1,280 faces), orthographic view down -z.

    Outer radii lie in [0.85, 1.15], the inner copy's in [0.425, 0.575]: the
    shells cannot intersect.  About four layers."""
    v, f = icosphere(3)
    rng0, rng1 = np.random.default_rng(seed), np.random.default_rng(seed + 1)
    outer = v * (1 + rng0.uniform(-0.15, 0.15, size=(len(v), 1)))
    inner = 0.5 * v * (1 + rng1.uniform(-0.15, 0.15, size=(len(v), 1)))
    vertices = np.concatenate([outer, inner])
    faces = np.concatenate([f, f + len(v)]).astype(np.int32)
    camera, settings = _ortho_down_z(vertices)
    return vertices, faces, camera, settings


def torus_knot(t, p=3, q=7):
    r = 2 + np.cos(q * t)
    return np.stack([r * np.cos(p * t), r * np.sin(p * t), np.sin(q * t)], axis=-1)


def knot_tube(rings=256, segments=128, radius=0.3, noise=0.02, seed=2):
    """Tube swept along a (3,7) torus knot: rings x segments quads split into
    2 * rings * segments triangles (65,536 by default), radius noise N(0, noise)
    per vertex, pinhole camera with a 60 degree field of view at 3x the
    bounding radius on +z looking at the centroid.  The radius 0.3 keeps the
    knot strands 1.26 tube diameters apart (``knot_clearance``), so the tube
    has no self-intersections to resolve."""
    rng = np.random.default_rng(seed)
    t = np.linspace(0, 2 * np.pi, rings, endpoint=False)
    dt = 1e-4
    center = torus_knot(t)
    tangent = torus_knot(t + dt) - torus_knot(t - dt)
    tangent /= np.linalg.norm(tangent, axis=1, keepdims=True)
    # Rotation-minimising frame by parallel transport, closed with a twist fix.
    normal = np.zeros_like(center)
    n0 = np.cross(tangent[0], [0.0, 0.0, 1.0])
    normal[0] = n0 / np.linalg.norm(n0)
    for i in range(1, rings):
        n = normal[i - 1] - np.dot(normal[i - 1], tangent[i]) * tangent[i]
        normal[i] = n / np.linalg.norm(n)
    binormal = np.cross(tangent, normal)
    last = normal[-1] - np.dot(normal[-1], tangent[0]) * tangent[0]
    last /= np.linalg.norm(last)
    twist = math.atan2(np.dot(np.cross(last, normal[0]), tangent[0]), np.dot(last, normal[0]))
    theta = np.linspace(0, 2 * np.pi, segments, endpoint=False)
    angle = theta[None, :] + twist * (np.arange(rings) / rings)[:, None]
    r = radius * (1 + rng.normal(0.0, noise, size=(rings, segments)))
    vertices = (center[:, None, :]
                + r[..., None] * (np.cos(angle)[..., None] * normal[:, None, :]
                                  + np.sin(angle)[..., None] * binormal[:, None, :]))
    vertices = vertices.reshape(-1, 3)
    i = np.arange(rings)[:, None]
    j = np.arange(segments)[None, :]
    a = i * segments + j
    b = ((i + 1) % rings) * segments + j
    c = ((i + 1) % rings) * segments + (j + 1) % segments
    d = i * segments + (j + 1) % segments
    faces = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3),
                            np.stack([a, c, d], -1).reshape(-1, 3)]).astype(np.int32)
    centroid = vertices.mean(0)
    bound = np.linalg.norm(vertices - centroid, axis=1).max()
    camera, settings = _pinhole(centroid + np.array([0.0, 0.0, 3 * bound]), centroid,
                                near=0.01 * bound)
    return vertices, faces, camera, settings


def knot_clearance(rings=2048, radius=0.3, noise=0.02):
    """Smallest centreline distance between knot points more than one tube
    diameter apart along the curve, divided by the largest tube diameter
    (4 sigma noise); > 1 means the swept tube cannot self-intersect."""
    t = np.linspace(0, 2 * np.pi, rings, endpoint=False)
    c = torus_knot(t)
    step = np.linalg.norm(np.diff(c, axis=0), axis=1).mean()
    diameter = 2 * radius * (1 + 4 * noise)
    separation = int(np.ceil(3 * diameter / step))
    best = np.inf
    for k in range(rings):
        d = np.linalg.norm(c - c[k], axis=1)
        idx = np.arange(rings)
        gap = np.minimum(np.abs(idx - k), rings - np.abs(idx - k))
        far = gap > separation
        best = min(best, d[far].min())
    return best / diameter


def stress_stack(n=65536, jitter=1e-9, seed=3):
    """n congruent triangles at z = i * 1e-3 with per-vertex xy jitter
    U(-jitter, jitter), orthographic view (n layers)."""
    rng = np.random.default_rng(seed)
    base = np.array([[-0.75, -0.75], [0.75, -0.75], [0.0, 0.75]])
    xy = base[None] + rng.uniform(-jitter, jitter, size=(n, 3, 2)) if jitter else np.repeat(
        base[None], n, 0)
    z = (np.arange(n) * 1e-3)[:, None, None] * np.ones((n, 3, 1))
    vertices = np.concatenate([xy, z], axis=2).reshape(-1, 3)
    faces = np.arange(3 * n, dtype=np.int32).reshape(-1, 3)
    camera = np.diag([1.0, 1.0, -1.0, 1.0])
    settings = np.array([-1.0, -1.0, 1.0, 1.0, 0.0, 0.01])
    return vertices, faces, camera, settings


def uv_sphere(rings, segments, radius, noise, rng):
    """Closed noisy sphere: 2 * segments * (rings - 1) faces, outward winding."""
    theta = np.linspace(0, np.pi, rings + 1)[1:-1]
    phi = np.linspace(0, 2 * np.pi, segments, endpoint=False)
    body = np.stack([np.sin(theta)[:, None] * np.cos(phi)[None],
                     np.sin(theta)[:, None] * np.sin(phi)[None],
                     np.cos(theta)[:, None] * np.ones_like(phi)[None]], -1).reshape(-1, 3)
    vertices = np.concatenate([[[0, 0, 1]], body, [[0, 0, -1]]])
    vertices = vertices * (radius * (1 + rng.uniform(-noise, noise, size=(len(vertices), 1))))
    top, bottom = 0, len(vertices) - 1
    ring = lambda i, j: 1 + i * segments + j % segments  # noqa: E731
    faces = []
    for j in range(segments):
        faces.append((top, ring(0, j), ring(0, j + 1)))
        faces.append((bottom, ring(rings - 2, j + 1), ring(rings - 2, j)))
    for i in range(rings - 2):
        for j in range(segments):
            a, b, c, d = ring(i, j), ring(i + 1, j), ring(i + 1, j + 1), ring(i, j + 1)
            faces += [(a, b, c), (a, c, d)]
    return vertices, np.array(faces, dtype=np.int32)


def torus(major_segments, minor_segments, major, minor, noise, rng):
    """Closed noisy torus: 2 * major_segments * minor_segments faces."""
    u = np.linspace(0, 2 * np.pi, major_segments, endpoint=False)[:, None]
    v = np.linspace(0, 2 * np.pi, minor_segments, endpoint=False)[None, :]
    r = minor * (1 + rng.uniform(-noise, noise, size=(major_segments, minor_segments)))
    vertices = np.stack([(major + r * np.cos(v)) * np.cos(u), (major + r * np.cos(v)) * np.sin(u),
                         r * np.sin(v)], -1).reshape(-1, 3)
    i = np.arange(major_segments)[:, None]
    j = np.arange(minor_segments)[None, :]
    a = i * minor_segments + j
    b = ((i + 1) % major_segments) * minor_segments + j
    c = ((i + 1) % major_segments) * minor_segments + (j + 1) % minor_segments
    d = i * minor_segments + (j + 1) % minor_segments
    faces = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3),
                            np.stack([a, c, d], -1).reshape(-1, 3)]).astype(np.int32)
    return vertices, faces


def packed_primitives(total_faces=720000, count=40, noise=0.02, seed=7, direction=None):
    """``count`` noisy spheres and tori (bounding radii log-uniform in
    [0.05, 0.5], faces in proportion to surface area, about ``total_faces`` in
    all), placed without overlap by rejection sampling in a cube that grows
    until they fit, then viewed by a 60 degree pinhole camera at 3x the scene's
    bounding radius from `direction` (default (0.3, 0.4, 3)).  Disjoint
    placement stands in for resolving overlapping primitives, which needs an
    exact mesh-intersection resolver."""
    rng = np.random.default_rng(seed)
    radii = np.exp(rng.uniform(np.log(0.05), np.log(0.5), size=count))
    kinds = rng.integers(0, 2, size=count)  # 0 sphere, 1 torus
    area = np.where(kinds == 0, 4 * np.pi * radii ** 2, 4 * np.pi ** 2 * (0.7 * radii) * (0.3 * radii))
    budget = total_faces * area / area.sum()
    side, centers = 1.0, []
    while len(centers) < count:
        centers = []
        for r in radii:
            for _ in range(2000):
                c = rng.uniform(r, side - r, size=3)
                if all(np.linalg.norm(c - c2) > r + r2 for c2, r2 in zip(centers, radii)):
                    centers.append(c)
                    break
            else:
                break
        side *= 1.1
    vertices, faces = _primitives(radii, kinds, budget, centers, noise, rng)
    return vertices, faces, *_primitive_camera(vertices, direction)


def _primitives(radii, kinds, budget, centers, noise, rng):
    """One mesh of noisy spheres (kind 0) and tori (kind 1) of the given
    bounding radii, face budgets and centres."""
    parts_v, parts_f, offset = [], [], 0
    for r, kind, faces, c in zip(radii, kinds, budget, centers):
        if kind == 0:
            rings = max(3, int(round(np.sqrt(faces / 4.0))) + 1)
            v, f = uv_sphere(rings, 2 * (rings - 1), r / (1 + noise), noise, rng)
        else:
            minor_segments = max(3, int(round(np.sqrt(faces / 6.0))))
            major_segments = max(3, int(round(faces / (2 * minor_segments))))
            v, f = torus(major_segments, minor_segments, 0.7 * r, 0.3 * r / (1 + noise), noise, rng)
            v = v @ _random_rotation(rng).T
        parts_v.append(v + c)
        parts_f.append(f + offset)
        offset += len(v)
    return np.concatenate(parts_v), np.concatenate(parts_f).astype(np.int32)


def _primitive_camera(vertices, direction):
    """The 60 degree pinhole at 3x the bounding radius from `direction`
    (default (0.3, 0.4, 3))."""
    centroid = vertices.mean(0)
    bound = np.linalg.norm(vertices - centroid, axis=1).max()
    view = np.array([0.3, 0.4, 3.0]) if direction is None else np.asarray(direction, float)
    camera, settings = _pinhole(centroid + view / np.linalg.norm(view) * 3 * bound, centroid,
                                near=0.01 * bound)
    return camera, settings


def overlapping_primitives(total_faces=720000, count=40, noise=0.02, seed=7, direction=None):
    """``count`` noisy spheres and tori (bounding radii log-uniform in
    [0.05, 0.5], faces in proportion to surface area, about ``total_faces`` in
    all) with centres uniform in the unit box, free to overlap: an
    unresolved triangle soup (vertices, faces, camera, settings) whose
    surfaces cross."""
    rng = np.random.default_rng(seed)
    radii = np.exp(rng.uniform(np.log(0.05), np.log(0.5), size=count))
    kinds = rng.integers(0, 2, size=count)  # 0 sphere, 1 torus
    area = np.where(kinds == 0, 4 * np.pi * radii ** 2, 4 * np.pi ** 2 * (0.7 * radii) * (0.3 * radii))
    budget = total_faces * area / area.sum()
    centers = rng.uniform(0.0, 1.0, size=(count, 3))
    vertices, faces = _primitives(radii, kinds, budget, centers, noise, rng)
    return vertices, faces, *_primitive_camera(vertices, direction)


def resolve_mesh(vertices, faces, threads=0):
    """The resolved mesh of a triangle soup: every crossing split exactly by
    the C++ resolver (peel_b200.resolve), pieces rounded to binary64 and
    their equal corners welded.  Returns (vertices, faces, parents: each
    face's input face, summary)."""
    from .resolve import resolve_arrays

    tris, parents, summary = resolve_arrays(vertices[faces], threads)
    corners = tris.reshape(-1, 3)
    unique, index = np.unique(corners, axis=0, return_inverse=True)
    return unique, index.reshape(-1, 3).astype(np.int32), parents, summary


def resolved_primitives(total_faces=720000, count=40, noise=0.02, seed=7, direction=None):
    """The overlapping primitives (overlapping_primitives) resolved
    (resolve_mesh): about 720K input faces by default; every face of the
    result lies on one input face (resolution_info gives the map).  The
    camera is the packed primitives' one.  Returns (vertices, faces, camera,
    settings)."""
    key = (total_faces, count, noise, seed)
    if key not in _RESOLVED:
        v, f, camera, settings = overlapping_primitives(total_faces, count, noise, seed)
        rv, rf, parents, summary = resolve_mesh(v, f)
        _RESOLVED[key] = (rv, rf, camera, settings, parents, summary, v, f)
    rv, rf, camera, settings = _RESOLVED[key][:4]
    if direction is not None:
        camera, settings = _primitive_camera(_RESOLVED[key][6], direction)
    return rv, rf, camera, settings


_RESOLVED = {}  # resolved_primitives() results by arguments (the resolution takes seconds)


def resolution_info(total_faces=720000, count=40, noise=0.02, seed=7):
    """(parents, resolver summary, input vertices, input faces) of a
    resolved_primitives() call made before."""
    entry = _RESOLVED[(total_faces, count, noise, seed)]
    return entry[4], entry[5], entry[6], entry[7]


def training_mesh(seed):
    """One seeded mesh of the pool-sizing training set: packed primitives
    (4 to 40 of them, 4,096 to 65,536 faces, log-uniform) seen from a random
    direction by the 60 degree pinhole camera at 3x the bounding radius."""
    rng = np.random.default_rng(seed)
    faces = int(np.exp(rng.uniform(np.log(4096), np.log(65536))))
    count = int(rng.integers(4, 41))
    direction = rng.normal(size=3)
    return packed_primitives(total_faces=faces, count=count, seed=seed, direction=direction)


def marching_tetrahedra(field, lo, hi, cells):
    """Closed triangle mesh of the zero set of ``field`` (negative inside) over
    the box [lo, hi] split into ``cells`` grid cells per axis, each cell cut
    into six tetrahedra around its main diagonal.  A vertex is made once per
    crossed grid edge (shared by every tetrahedron on the edge), so the mesh is
    watertight; triangles face the positive side."""
    lo, hi, cells = np.asarray(lo, float), np.asarray(hi, float), np.asarray(cells, int)
    axes = [np.linspace(lo[a], hi[a], cells[a] + 1) for a in range(3)]
    points = np.stack(np.meshgrid(*axes, indexing="ij"), -1)
    values = field(points)
    values = np.where(values == 0.0, 1e-12, values)  # no grid point on the surface
    shape = values.shape
    flat_p, flat_f = points.reshape(-1, 3), values.reshape(-1)
    ci, cj, ck = (a.ravel() for a in np.meshgrid(*(np.arange(c) for c in cells), indexing="ij"))
    index = lambda d: ((ci + d[0]) * shape[1] + cj + d[1]) * shape[2] + ck + d[2]
    unit = np.eye(3, dtype=int)
    tets = []
    for order in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)):
        corner = [np.zeros(3, int)]
        for axis in order:
            corner.append(corner[-1] + unit[axis])
        tets.append(np.stack([index(c) for c in corner], 1))
    tets = np.concatenate(tets)
    inside = flat_f[tets] < 0
    crossing = (inside.sum(1) > 0) & (inside.sum(1) < 4)
    tets, inside = tets[crossing], inside[crossing]
    vertex_of, vertices, faces = {}, [], []

    def vertex(a, b):
        key = (a, b) if a < b else (b, a)
        if key not in vertex_of:
            t = flat_f[key[0]] / (flat_f[key[0]] - flat_f[key[1]])
            vertices.append(flat_p[key[0]] + t * (flat_p[key[1]] - flat_p[key[0]]))
            vertex_of[key] = len(vertices) - 1
        return vertex_of[key]

    for tet, flags in zip(tets, inside):
        ins = [v for v, f in zip(tet, flags) if f]
        out = [v for v, f in zip(tet, flags) if not f]
        if len(ins) == 1 or len(out) == 1:
            lone, rest = (ins[0], out) if len(ins) == 1 else (out[0], ins)
            polys = [[vertex(lone, r) for r in rest]]
        else:
            a, b = vertex(ins[0], out[0]), vertex(ins[0], out[1])
            c, d = vertex(ins[1], out[1]), vertex(ins[1], out[0])
            polys = [[a, b, c], [a, c, d]]
        outward = flat_p[out].mean(0) - flat_p[ins].mean(0)
        for tri in polys:
            pa, pb, pc = (vertices[k] for k in tri)
            if np.dot(np.cross(pb - pa, pc - pa), outward) < 0:
                tri = [tri[0], tri[2], tri[1]]
            faces.append(tri)
    return np.array(vertices), np.array(faces, dtype=np.int32)


def genus3_surface(cells=49, seed=4, amplitude=0.03):
    """Closed genus-3 surface of about 16K faces (16,152 at the defaults): the
    union of three tori whose centre circles touch in a row (the thickened
    chain of circles has three independent loops), its implicit field displaced
    by a seeded sum of smooth sinusoids, polygonised by marching tetrahedra.
    An implicit surface does not intersect itself."""
    rng = np.random.default_rng(seed)
    major, minor = 1.0, 0.36
    waves = [(rng.normal(size=3) * 2.0, rng.uniform(0, 2 * np.pi)) for _ in range(4)]

    def field(p):
        value = np.full(p.shape[:-1], np.inf)
        for cx in (-2 * major, 0.0, 2 * major):
            q = p - np.array([cx, 0.0, 0.0])
            torus_ = np.hypot(np.hypot(q[..., 0], q[..., 1]) - major, q[..., 2]) - minor
            value = np.minimum(value, torus_)
        for k, phase in waves:
            value = value + amplitude / len(waves) * np.sin(p @ k + phase)
        return value

    pad = minor + amplitude + 0.05
    hi = np.array([3 * major + pad, major + pad, pad])
    lo = -hi
    size = hi - lo
    counts = np.maximum(1, np.round(size / (size[0] / cells)).astype(int))
    return marching_tetrahedra(field, lo, hi, counts)


def turntable_views(vertices, count=64, seed=5, fov_degrees=60.0):
    """``count`` pinhole cameras at 3x the bounding radius around the centroid:
    azimuth uniform in [0, 2 pi), elevation uniform in [-30, 30] degrees."""
    rng = np.random.default_rng(seed)
    centroid = vertices.mean(0)
    bound = np.linalg.norm(vertices - centroid, axis=1).max()
    views = []
    for azimuth, elevation in zip(rng.uniform(0, 2 * np.pi, count),
                                  np.radians(rng.uniform(-30, 30, count))):
        direction = np.array([np.cos(elevation) * np.cos(azimuth), np.sin(elevation),
                              np.cos(elevation) * np.sin(azimuth)])
        views.append(_pinhole(centroid + 3 * bound * direction, centroid, fov_degrees,
                              near=0.01 * bound))
    return views


def batched_scenes(views=64, meshes=64, seed=6):
    """The batched workload: ``views`` turntable views of the genus-3 surface,
    then ``meshes`` packed-primitive meshes of 1K to 32K faces (log-uniform
    counts, 1 to 4 primitives each).  A list of (vertices, faces, camera,
    settings)."""
    vertices, faces = genus3_surface()
    out = [(vertices, faces, camera, settings)
           for camera, settings in turntable_views(vertices, views)]
    rng = np.random.default_rng(seed)
    for k in range(meshes):
        total = int(np.exp(rng.uniform(np.log(1024), np.log(32768))))
        out.append(packed_primitives(total, int(rng.integers(1, 5)), seed=1000 + k))
    return out


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


CONFIGS = {
    "overlap-720k": resolved_primitives,
    "primitives-720k": packed_primitives,
    "icospheres-2560": nested_icospheres,
    "knot-65536": knot_tube,
    "stack-65536": lambda: stress_stack(65536, 0.0),
    "batched-128": batched_scenes,  # a list of scenes, peeled by one graph replay
}


def to_device(arrays, device="cuda:0"):
    import torch

    return [torch.as_tensor(np.ascontiguousarray(a), device=device) for a in arrays]
