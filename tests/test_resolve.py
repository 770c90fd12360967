"""The exact intersection resolver (peel_b200.resolve) on the CPU.

Its output must peel, as a resolved mesh, to exactly the arrangement the
oracle computes for the unresolved input (per (layer, original source) exact
area); every piece must lie in its parent triangle and the pieces must
conserve the parent's vector area (the reference's own checks of resolved
scenes, scripts/validate_fast.py:150-175); and the pieces must form a
conforming mesh: two pieces meet only in a common vertex or a common edge.
The conformity checks here are written independently of the resolver.
"""

import json
import subprocess
import sys
from fractions import Fraction as Q

import numpy as np
import parity
import pytest
from conftest import ROOT

from oracle import exact as ex

CROSSING = sorted(parity.CROSSING)
RESOLVED = [n for n in parity.RESOLVED if n != "empty"]
REJECTED = [f["name"] for f in parity.MANIFEST if f["expected"] != "accept"]


def resolve(data):
    from peel_b200.resolve import resolve as run

    return run(data)


def areas_by_original(scene, layers, data):
    ids = {t["id"]: t.get("original_source_id", t["id"]) for t in data["triangles"]}
    out = {}
    for (k, sid), a in ex.region_area2(scene, layers).items():
        key = (k, ids[sid])
        out[key] = out.get(key, Q(0)) + a
    return out


def peel(data, resolved):
    scene = ex.read_scene(data, resolved_mesh=resolved)
    layers, residual = ex.extract(scene)
    assert not residual
    return len(layers), areas_by_original(scene, layers, data)


# ------------------------------------------------------------ exact helpers


def tri(record):
    return tuple(tuple(Q(c) for c in p) for p in record["vertices"])


def sub(a, b):
    return tuple(x - y for x, y in zip(a, b))


def dot(a, b):
    return sum(x * y for x, y in zip(a, b))


def cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def normal(t):
    return cross(sub(t[1], t[0]), sub(t[2], t[0]))


def barycentric(t, w):
    """(on the plane, b, c) of w in triangle t."""
    u, v, r = sub(t[1], t[0]), sub(t[2], t[0]), sub(w, t[0])
    uu, uv, vv = dot(u, u), dot(u, v), dot(v, v)
    den = uu * vv - uv * uv
    b = (dot(r, u) * vv - dot(r, v) * uv) / den
    c = (dot(r, v) * uu - dot(r, u) * uv) / den
    return dot(r, normal(t)) == 0, b, c


def inside(t, w, strict):
    plane, b, c = barycentric(t, w)
    if strict:
        return plane and b > 0 and c > 0 and b + c < 1
    return plane and b >= 0 and c >= 0 and b + c <= 1


def on_open_edge(w, a, b):
    d, r = sub(b, a), sub(w, a)
    return cross(d, r) == (0, 0, 0) and 0 < dot(r, d) < dot(d, d)


def edges(t):
    return [(t[k], t[(k + 1) % 3]) for k in range(3)]


def violation(t, u):
    """Why pieces t and u do not meet in a common vertex or edge, or None."""
    if set(t) == set(u):
        return "duplicate"
    n = normal(u)
    d = dot(n, u[0])
    for w in t:
        for a, b in edges(u):
            if on_open_edge(w, a, b):
                return "vertex on an open edge"
        if inside(u, w, strict=True):
            return "vertex inside"
    for p, q in edges(t):
        sp, sq = dot(n, p) - d, dot(n, q) - d
        if sp * sq < 0:
            x = tuple(pc + (qc - pc) * (sp / (sp - sq)) for pc, qc in zip(p, q))
            if inside(u, x, strict=False):
                return "edge crosses"
        elif sp == 0 and sq == 0:
            # An edge on u's plane: where it runs inside u, it must stay on u's boundary.
            lo, hi = Q(0), Q(1)
            for a, b in edges(u):
                side = lambda x: dot(cross(sub(b, a), sub(x, a)), n)
                s0, s1 = side(p), side(q)
                if s0 < 0 and s1 < 0:
                    lo, hi = Q(1), Q(0)
                elif s0 < 0 or s1 < 0:
                    cut = s0 / (s0 - s1)
                    lo, hi = (max(lo, cut), hi) if s0 < 0 else (lo, min(hi, cut))
            if lo < hi:
                m = tuple(pc + (qc - pc) * ((lo + hi) / 2) for pc, qc in zip(p, q))
                if inside(u, m, strict=True):
                    return "edge runs inside"
    return None


def check_conforming(pieces):
    corners = np.array([[[float(c) for c in p] for p in t] for t in pieces])
    lo, hi = corners.min(axis=1) - 1e-9, corners.max(axis=1) + 1e-9
    normals = np.cross(corners[:, 1] - corners[:, 0], corners[:, 2] - corners[:, 0])
    normals /= np.linalg.norm(normals, axis=1)[:, None]
    for i in range(len(pieces)):
        near = np.nonzero(np.all(lo <= hi[i], axis=1) & np.all(hi >= lo[i], axis=1))[0]
        near = near[near > i]
        # Pieces whose corners lie clearly on one side of piece i's plane
        # cannot meet it (a binary64 margin far above the rounding of corners).
        side = (corners[near] - corners[i, 0]) @ normals[i]
        apart = np.all(side > 1e-9, axis=1) | np.all(side < -1e-9, axis=1)
        for j in near[~apart]:
            for a, b in ((pieces[i], pieces[j]), (pieces[j], pieces[i])):
                why = violation(a, b)
                assert why is None, (why, i, j)


# ------------------------------------------------------------------ tests


@pytest.mark.parametrize("name", CROSSING)
def test_crossing_fixture_peels_to_the_unresolved_arrangement(name):
    data = parity.fixture(name)
    result, summary = resolve(data)
    assert summary["output_triangles"] == len(result["triangles"])
    assert result["original_triangles"] == data["triangles"]
    assert peel(result, resolved=True) == peel(data, resolved=False)


@pytest.mark.parametrize("name", RESOLVED)
def test_resolved_fixture_keeps_its_arrangement(name):
    data = parity.fixture(name)
    result, summary = resolve(data)
    assert summary["intersection_segments"] == 0
    assert peel(result, resolved=True) == peel(data, resolved=True)


@pytest.mark.parametrize("name", CROSSING + ["coplanar_adjacent", "shared_vertex"])
def test_pieces_lie_in_their_parent_conserve_area_and_conform(name):
    data = parity.fixture(name)
    result, _ = resolve(data)
    parents = {t.get("id", i): tri(t) for i, t in enumerate(data["triangles"])}
    total = {k: (Q(0), Q(0), Q(0)) for k in parents}
    pieces = []
    for record in result["triangles"]:
        t = tri(record)
        parent = parents[record["original_source_id"]]
        assert record["mesh_face_id"] == record["original_source_id"]
        assert all(inside(parent, w, strict=False) for w in t)
        total[record["original_source_id"]] = tuple(
            x + y for x, y in zip(total[record["original_source_id"]], normal(t)))
        pieces.append(t)
    assert total == {k: normal(t) for k, t in parents.items()}
    check_conforming(pieces)


@pytest.mark.parametrize("name", ["crossing", "random_07", "random_10"])
def test_second_pass_changes_nothing(name):
    first, _ = resolve(parity.fixture(name))
    second, summary = resolve(first)
    assert summary["intersection_segments"] == 0
    key = lambda r: (r["original_source_id"], tuple(map(tuple, r["vertices"])))
    assert sorted(map(key, second["triangles"])) == sorted(map(key, first["triangles"]))
    assert second["original_triangles"] == first["original_triangles"]


def test_interpenetrating_icospheres():
    """Two icosahedra crossing each other along closed curves."""
    from peel_b200 import scenes

    v, f = scenes.icosphere(0)
    v = np.asarray(v, dtype=np.float64)
    f = np.asarray(f)
    vertices = np.concatenate([v, v * 0.8 + np.array([1.3, 0.1, 0.05])])
    faces = np.concatenate([f, f + len(v)])
    data = parity.exact_scene_of(vertices, faces, np.diag([1.0, 1.0, -1.0, 1.0]),
                                 [-1.5, -1.5, 3.0, 1.5, 0.0, 0.01])
    result, summary = resolve(data)
    assert summary["intersection_segments"] > 0 and summary["cut_triangles"] > 0
    assert peel(result, resolved=True) == peel(data, resolved=False)
    check_conforming([tri(r) for r in result["triangles"]])


@pytest.mark.parametrize("name", REJECTED)
def test_coplanar_overlap_rejected(name):
    from peel_b200.resolve import ResolveError

    with pytest.raises(ResolveError, match="positive area"):
        resolve(parity.fixture(name))


@pytest.mark.parametrize("exponent", [500, -500])
def test_extreme_scales_resolve_exactly(exponent):
    """Coordinates scaled by 2^500 or 2^-500 (outside the range the binary64
    pre-tests trust) resolve to exactly the scaled pieces."""
    import warnings

    k = Q(2) ** exponent
    for name in ("crossing", "random_07"):
        data = parity.fixture(name)
        scaled = dict(data, triangles=[
            dict(t, vertices=[[str(Q(c) * k) for c in v] for v in t["vertices"]])
            for t in data["triangles"]])
        with warnings.catch_warnings():
            warnings.simplefilter("error")
            big, _ = resolve(scaled)
        small, _ = resolve(data)
        grow = lambda r: sorted((t["original_source_id"], tuple(
            tuple(Q(c) * k for c in p) for p in tri(t))) for t in r["triangles"])
        same = lambda r: sorted((t["original_source_id"], tri(t)) for t in r["triangles"])
        assert same(big) == grow(small)


def test_duplicate_triangle_rejected():
    """A triangle listed twice overlaps itself on one plane: it is an error,
    not a pair whose shared vertices are its only contact."""
    from peel_b200.resolve import ResolveError

    data = parity.fixture("single")
    twice = dict(data, triangles=data["triangles"] + [dict(data["triangles"][0], id=99)])
    with pytest.raises(ResolveError, match="positive area"):
        resolve(twice)


def test_numbers_parse_like_the_reference():
    from peel_b200.resolve import ResolveError, rational, text

    assert rational("3/4") == Q(3, 4) and rational("-2") == -2 and rational("+5/10") == Q(1, 2)
    assert rational(0.1) == Q(0.1) and rational(7) == 7
    for bad in ("1.5", "1/0", "1/", "/2", "x", "", "1e3"):
        with pytest.raises(ResolveError):
            rational(bad)
    with pytest.raises(ResolveError):
        rational(float("nan"))
    assert text(Q(-3)) == "-3/1" and text(Q(6, 4)) == "3/2"


def test_command_line(tmp_path):
    source = ROOT / "tests/golden/fixtures/crossing.json"
    out = tmp_path / "resolved.json"
    cmd = [sys.executable, "-m", "peel_b200.resolve"]
    env_path = str(ROOT / "exact-depth-peeling_b200")
    run = lambda args: subprocess.run(cmd + args, capture_output=True, text=True,
                                      cwd=env_path, timeout=120)
    done = run([str(source), str(out)])
    assert done.returncode == 0, done.stderr
    summary = json.loads(done.stdout)
    written = json.loads(out.read_text())
    assert summary["output_triangles"] == len(written["triangles"]) == 4
    assert written["intersection_preprocessing"] == summary
    assert run([str(source)]).returncode == 2
    bad = tmp_path / "bad.json"
    bad.write_text(json.dumps({"window": [0, 0, 1, 1],
                               "triangles": [{"vertices": [[0, 0, "1.5"]] * 3}]}))
    failed = run([str(bad), str(out)])
    assert failed.returncode == 1 and failed.stderr.startswith("error:")
