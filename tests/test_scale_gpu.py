"""Parity at the benchmark configurations' full sizes.

The exact Fraction oracle cannot peel tens of thousands of faces, so these tests
check size-independent properties instead:

* exact ranks at sampled output polygons (oracle.exact.SparseRanks imports only
  the source triangles near each sample, exactly);
* conservation: the output regions of each source, summed over all layers,
  cover exactly its projected area;
* the triangle mesh covers exactly the same area per (layer, source) as the
  polygons (a checksum of the noding and fan emission);
* the identical-footprint stack's known answers (layer = source, work counts).
"""

from collections import defaultdict

import numpy as np
import pytest
import parity

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def projected_areas(vertices, faces, camera, settings):
    """Float area of each face's projection in normalised window coordinates
    (for scenes that neither the near plane nor the window clips)."""
    cam = vertices @ camera[:3, :3].T + camera[:3, 3]
    tri = cam[faces]
    xy = tri[:, :, :2] / tri[:, :, 2:3] if settings[4] else tri[:, :, :2]
    uv = (xy - settings[:2]) / (settings[2:4] - settings[:2])
    assert (uv >= 0).all() and (uv <= 1).all(), "scene must lie inside the window"
    a, b = uv[:, 1] - uv[:, 0], uv[:, 2] - uv[:, 0]
    return 0.5 * np.abs(a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0])


def check_conservation(p, host, polys):
    expected = projected_areas(*host)
    got = np.zeros(len(expected))
    for _, source, v in polys:
        got[source] += parity.shoelace(v)
    np.testing.assert_allclose(got, expected, rtol=0, atol=1e-12)


def check_mesh_checksum(p, polys):
    info = p.read_status()
    t = info["triangles"]
    uv = p.triangles_uv[:t].cpu().numpy()
    src = p.triangle_sources[:t].cpu().numpy()
    lay = p.triangle_layers[:t].cpu().numpy()
    a, b = uv[:, 1] - uv[:, 0], uv[:, 2] - uv[:, 0]
    cross = a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]
    assert (cross > 0).all()
    mesh, poly = defaultdict(float), defaultdict(float)
    for s_, l_, c in zip(src, lay, cross):
        mesh[(int(l_), int(s_))] += 0.5 * c
    for layer, source, v in polys:
        poly[(layer, source)] += parity.shoelace(v)
    parity.assert_areas(dict(mesh), dict(poly), tolerance=1e-11)


def check_sampled_ranks(host, polys, samples, seed=0):
    from oracle import exact as ex

    oracle = ex.SparseRanks(*host)
    rng = np.random.default_rng(seed)
    picks = rng.choice(len(polys), size=min(samples, len(polys)), replace=False)
    checked = 0
    for k in picks:
        layer, source, v = polys[k]
        rank = oracle.polygon_rank(source, [tuple(x) for x in v])
        if rank is None:  # every generic sample ambiguous: a sliver on a boundary
            continue
        assert rank == layer, (source, layer, rank, v.tolist())
        checked += 1
    assert checked >= 0.95 * len(picks)


def run(peeler_cls, host, **kw):
    from peel_b200 import scenes

    arrays = scenes.to_device(host)
    if peeler_cls == "events":
        from peel_b200.sizing import fit_event_capacities

        p, _ = fit_event_capacities(arrays, **kw)
    else:
        from peel_b200 import DevicePeeler

        p = DevicePeeler(*arrays, **kw)
        p.run()
    p.read_status()
    return p


@pytest.mark.parametrize("method", ["events", "device"])
def test_nested_icospheres_every_polygon(method):
    """Config 1 (2 x 1,280 faces): the exact rank of every output polygon."""
    from peel_b200 import scenes

    host = scenes.nested_icospheres()
    p = run(method, host)
    polys = parity.polygons(p)
    check_conservation(p, host, polys)
    check_mesh_checksum(p, polys)
    check_sampled_ranks(host, polys, samples=len(polys))


def test_knot_tube_sampled_ranks_and_conservation():
    """Config 2 (65,536-face knot tube): 1,500 sampled exact ranks,
    conservation of every source and the mesh checksum."""
    from peel_b200 import scenes

    host = scenes.knot_tube()
    p = run("events", host)
    polys = parity.polygons(p)
    info = p.read_status()
    assert info["layers"] >= 15
    check_conservation(p, host, polys)
    check_mesh_checksum(p, polys)
    check_sampled_ranks(host, polys, samples=1500)


def test_identical_stack_65536():
    """Config 3's control: 65,536 identical footprints at distinct depths."""
    from peel_b200 import scenes

    host = scenes.stress_stack(65536, 0.0)
    p = run("events", host)
    info = p.read_status()
    n = 65536
    assert info["polygons"] == n and info["layers"] == n
    assert info["splits"] == 0 and info["unique_contours"] == 3
    assert info["ray_groups"] == 1 and info["ray_hits"] == n
    # Viewed down -z: the largest z (the last source) is nearest.
    order = np.argsort(p.output_layers[:n].cpu().numpy())
    np.testing.assert_array_equal(p.output_sources[:n].cpu().numpy()[order], np.arange(n)[::-1])
