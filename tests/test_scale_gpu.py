"""Parity at the benchmark configurations' full sizes.

The exact Fraction oracle cannot peel tens of thousands of faces, so these tests
check size-independent properties instead:

* exact ranks at sampled output polygons, drawn per layer (stratified) and
  re-drawn when a sample is ambiguous (oracle.exact.SparseRanks imports only
  the source triangles near each sample, exactly; a pool of spawned processes
  evaluates them);
* exact vertex error: sampled polygon vertices against the rational
  intersection of the source-edge lines they lie on (peel_b200.audit), at most
  1e-9 of the projected scene's extent;
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


def stratified_order(polys, seed):
    """Per layer, the indices of that layer's polygons in a seeded random order."""
    rng = np.random.default_rng(seed)
    by_layer = defaultdict(list)
    for i, (layer, _, _) in enumerate(polys):
        by_layer[layer].append(i)
    return {layer: [idx[k] for k in rng.permutation(len(idx))]
            for layer, idx in sorted(by_layer.items())}


def sample_quotas(order, samples, minimum=16):
    """Samples per layer: in proportion to the layer's polygons, at least
    `minimum` (or the whole layer), `samples` in all (about)."""
    total = sum(len(v) for v in order.values())
    return {layer: min(len(idx), max(minimum, int(round(samples * len(idx) / total))))
            for layer, idx in order.items()}


def check_sampled_ranks_multi(hosts, meshes, samples, seed=0, max_ambiguous=0.02):
    """Exact ranks of stratified samples of every mesh's output polygons.

    `meshes` holds each mesh's polygon list (parity.polygons).  Each layer
    of each mesh gets its quota of unambiguous samples: an ambiguous sample
    (every generic interior point on a boundary or a depth tie) is replaced
    by the next polygon of the same layer, and at most `max_ambiguous` of
    the evaluated samples may be ambiguous.  Returns the ranks checked."""
    from oracle import exact as ex

    plans = []
    for m, polys in enumerate(meshes):
        order = stratified_order(polys, seed + m)
        for layer, quota in sample_quotas(order, samples[m] if isinstance(samples, list)
                                          else samples).items():
            plans.append([m, layer, order[layer], quota, 0, 0])  # next index, checked
    evaluated = ambiguous = checked = 0
    while True:
        batch, owners = [], []
        for plan in plans:
            m, layer, idx, quota, nxt, done = plan
            want = quota - done
            take = idx[nxt:nxt + want + (want + 19) // 20] if want > 0 else []
            for k in take:
                _, source, v = meshes[m][k]
                batch.append((m, source, [tuple(x) for x in v]))
                owners.append((plan, k))
            plan[4] = nxt + len(take)
        if not batch:
            break
        ranks = ex.polygon_ranks_multi(hosts, batch)
        for (plan, k), rank in zip(owners, ranks):
            m, layer = plan[0], plan[1]
            evaluated += 1
            if rank is None:
                ambiguous += 1
                continue
            if plan[5] >= plan[3]:
                continue
            assert rank == layer, (m, meshes[m][k][1], layer, rank, meshes[m][k][2].tolist())
            plan[5] += 1
            checked += 1
    for m, layer, idx, quota, nxt, done in plans:
        assert done == quota or nxt == len(idx), (m, layer, done, quota)
    assert ambiguous <= max_ambiguous * evaluated, (ambiguous, evaluated)
    return checked


def check_sampled_ranks(host, polys, samples, seed=0):
    return check_sampled_ranks_multi([host], [polys], samples, seed)


def check_vertex_error(p, samples, seed=0):
    """Sampled output vertices within 1e-9 of the scene extent of their exact
    rational position (every vertex explained by two exact lines)."""
    from peel_b200.audit import peeler_vertex_audit

    report = peeler_vertex_audit(p, samples=samples, seed=seed)
    assert report["unexplained_vertices"] == 0, report
    assert report["vertices_measured"] > 0
    assert report["max_rel_error"] <= 1e-9, report
    return report


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
    assert check_sampled_ranks(host, polys, samples=len(polys)) >= 0.98 * len(polys)
    if method == "events":
        check_vertex_error(p, samples=len(polys))


def test_knot_tube_sampled_ranks_and_conservation():
    """Config 2 (65,536-face knot tube): 20,000 exact ranks drawn per layer,
    exact vertex error, conservation of every source and the mesh checksum."""
    from peel_b200 import scenes

    host = scenes.knot_tube()
    p = run("events", host)
    polys = parity.polygons(p)
    info = p.read_status()
    assert info["layers"] >= 15
    check_conservation(p, host, polys)
    check_mesh_checksum(p, polys)
    assert check_sampled_ranks(host, polys, samples=20000) >= 19600
    check_vertex_error(p, samples=2000)


def test_primitives_720k_sampled_ranks_and_conservation():
    """Config 5 (720,916 faces of 40 packed spheres and tori): 10,000 exact
    ranks drawn per layer, exact vertex error, conservation of every source
    and the mesh checksum."""
    from peel_b200 import scenes

    host = scenes.packed_primitives()
    p = run("events", host)
    polys = parity.polygons(p)
    info = p.read_status()
    assert info["layers"] >= 10
    check_conservation(p, host, polys)
    check_mesh_checksum(p, polys)
    assert check_sampled_ranks(host, polys, samples=10000) >= 9800
    check_vertex_error(p, samples=1000)


def test_overlap_720k_sampled_ranks_and_conservation():
    """Config 5 as named: the 40 primitives placed with overlap (720,916
    faces) and resolved exactly on the host (1,218,926 faces, every crossing a
    shared edge): 3,000 exact ranks drawn per layer, exact vertex error,
    conservation of every source and the mesh checksum."""
    from peel_b200 import scenes

    host = scenes.resolved_primitives()
    assert scenes.resolution_info()[1]["intersection_segments"] > 10000
    p = run("events", host)
    polys = parity.polygons(p)
    info = p.read_status()
    assert info["layers"] >= 10
    check_conservation(p, host, polys)
    check_mesh_checksum(p, polys)
    assert check_sampled_ranks(host, polys, samples=3000) >= 2940
    check_vertex_error(p, samples=1000)


def test_batched_128_every_scene_sampled():
    """Config 4: one graph replay of all 128 scenes (64 turntable views of the
    genus-3 surface, 64 packed-primitive meshes); in every scene 160 exact
    ranks drawn per layer, conservation and the mesh checksum."""
    from peel_b200 import BatchPeeler, scenes

    hosts = scenes.batched_scenes()
    batch = BatchPeeler([scenes.to_device(h) for h in hosts], fit=True)
    batch.run()
    infos = batch.read_status()
    assert len(infos) == 128
    meshes = [parity.polygons(p) for p in batch.peelers]
    for host, p, polys in zip(hosts, batch.peelers, meshes):
        check_conservation(p, host, polys)
        check_mesh_checksum(p, polys)
    checked = check_sampled_ranks_multi(hosts, meshes, samples=160)
    assert checked >= 100 * len(hosts)


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
