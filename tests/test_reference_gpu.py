"""The reference's remaining GPU tests, restated through the C ABI.

* the graph contract (tests/gpu/test_peeler.py:155-202): an external capture
  of enqueue() does no host read or synchronisation, and the captured graph
  holds a conditional node and no memcpy or allocation node;
* no T-junctions in either peeler's mesh (test_peeler.py:255-280,
  test_events.py:113-116), checked without shapely;
* the EventPeeler replays a camera moved on the device (test_events.py:119-121);
* rank components on a shared grid scene, with and without half cover
  (test_components.py:13-61);
* the identical stack of 4,096 keeps the edge hash bounded
  (test_components.py:81-93);
* one captured graph replays 1025, 127, 0, 257, 256 and 1025 live polygons
  (test_components.py:96-114).
"""

import numpy as np
import pytest
import parity

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def load(name):
    from peel_b200.io import load_scene

    return load_scene(parity.fixture(name))


def peeler_type(method):
    from peel_b200 import DevicePeeler, EventPeeler

    return EventPeeler if method == "events" else DevicePeeler


@pytest.mark.parametrize("method", ["events", "peel"])
def test_capture_contract(tmp_path, monkeypatch, method):
    """enqueue() inside an external capture reads nothing back and never
    synchronises; the graph has a conditional node and no copy or
    allocation node (cudaGraphDebugDotPrint through torch's debug dump)."""
    arrays, labels, data = load("partial")
    p = peeler_type(method)(*arrays)
    p.warmup()
    p.stream.synchronize()
    graph = torch.cuda.CUDAGraph(keep_graph=True)  # keep the cudaGraph_t to print it
    graph.enable_debug_mode()

    def forbidden(*_a, **_k):
        pytest.fail("host read or synchronisation during capture")

    # torch.cuda.graph synchronises on entry, so the host calls are forbidden
    # only inside the capture, around enqueue() itself.
    with torch.cuda.graph(graph, stream=p.stream):
        with monkeypatch.context() as m:
            for owner, name in ((torch.Tensor, "cpu"), (torch.Tensor, "numpy"),
                                (torch.Tensor, "item"), (torch.Tensor, "tolist"),
                                (torch.cuda, "synchronize"), (torch.cuda.Stream, "synchronize"),
                                (torch.cuda.Event, "synchronize")):
                m.setattr(owner, name, forbidden)
            p.enqueue()
    graph.instantiate()
    graph.replay()
    parity.check_against_oracle(p, data, labels)
    dot = tmp_path / "graph.dot"
    graph.debug_dump(str(dot))
    text = dot.read_text().upper()
    assert "CONDITIONAL" in text
    for kind in ("MEMCPY", "DTOH", "HTOD", "ALLOC"):
        assert kind not in text, kind


def assert_no_t_junctions(uv, layers):
    """No triangle vertex of a layer lies in the interior of another
    triangle edge of that layer (within 1e-11, the reference's bound)."""
    for layer in np.unique(layers):
        tris = uv[layers == layer]
        points = np.unique(tris.reshape(-1, 2), axis=0)
        for a, b in ((tris[:, 0], tris[:, 1]), (tris[:, 1], tris[:, 2]), (tris[:, 2], tris[:, 0])):
            d = b - a
            lo, hi = np.minimum(a, b) - 1e-10, np.maximum(a, b) + 1e-10
            for k in range(len(tris)):
                near = points[np.all((points >= lo[k]) & (points <= hi[k]), axis=1)]
                if not len(near):
                    continue
                t = (near - a[k]) @ d[k] / (d[k] @ d[k])
                dist = np.abs(d[k, 0] * (near[:, 1] - a[k, 1])
                              - d[k, 1] * (near[:, 0] - a[k, 0])) / np.linalg.norm(d[k])
                assert not np.any((t > 1e-8) & (t < 1 - 1e-8) & (dist < 1e-11)), (layer, k)


@pytest.mark.parametrize("method", ["events", "peel"])
@pytest.mark.parametrize("name", ["partial", "holes", "closed_object"])
def test_mesh_has_no_t_junctions(name, method):
    arrays, _, _ = load(name)
    p = peeler_type(method)(*arrays)
    p.run()
    t = p.read_status()["triangles"]
    assert t > 0
    assert_no_t_junctions(p.triangles_uv[:t].cpu().numpy(), p.triangle_layers[:t].cpu().numpy())


def test_event_camera_update():
    """The camera moved on the device between replays of one graph."""
    from oracle import exact as ex
    from peel_b200 import EventPeeler

    arrays, labels, data = load("partial")
    p = EventPeeler(*arrays)
    p.run()
    before = parity.gpu_areas(parity.polygons(p), labels)
    with torch.cuda.stream(p.stream):
        arrays[2][0, 3] += 0.5
    p.run()
    after = parity.gpu_areas(parity.polygons(p), labels)
    assert before != after
    data = dict(data)
    data["camera"] = {"type": "orthographic",
                      "world_to_camera": [[1, 0, 0, 0.5], [0, 1, 0, 0], [0, 0, 1, 0]]}
    scene = ex.read_scene(data)
    layers, _ = ex.extract(scene)
    parity.assert_areas(after, parity.oracle_areas(scene, layers))


def grid_scene(half_cover):
    """Two 4 x 4 grids of unit squares (two triangles each) at z = 1 and 2;
    with half_cover the near grid keeps only its x < 2 half."""
    triangles = []
    for z in (1, 2):
        for y in range(4):
            for x in range(4):
                if half_cover and z == 1 and x >= 2:
                    continue
                a, b, c, d = [x, y, z], [x + 1, y, z], [x + 1, y + 1, z], [x, y + 1, z]
                for corners in ([a, b, c], [a, c, d]):
                    triangles.append({"id": len(triangles), "vertices": corners})
    return {"window": [-1, -1, 5, 5], "camera": {"type": "orthographic"},
            "triangles": triangles}


@pytest.mark.parametrize("half_cover", [False, True])
def test_mesh_rank_components(half_cover):
    from oracle import exact as ex
    from peel_b200 import EventPeeler
    from peel_b200.io import load_scene

    data = grid_scene(half_cover)
    arrays, labels, _ = load_scene(data)
    p = EventPeeler(*arrays, share_regions=False)
    p.run()
    info = p.read_status()
    assert info["rank_connections"] > 0
    assert info["rank_components"] <= 3
    assert info["ray_groups"] <= 3
    assert info["merged_polygons"] == 0
    assert info["polygons"] == len(labels)
    parity.check_against_oracle(p, data, labels)
    baseline = EventPeeler(*arrays, share_regions=False, propagate_ranks=False,
                           merge_regions=False)
    baseline.run()
    parity.assert_areas(parity.gpu_areas(parity.polygons(p), labels),
                        parity.gpu_areas(parity.polygons(baseline), labels))
    assert baseline.read_status()["ray_groups"] >= 16
    # Deform both grids and replay the same graphs: the old adjacency must
    # not survive, and the patches are no longer coplanar.
    with torch.cuda.stream(p.stream):
        xyz = arrays[0]
        xyz[:, 2] += 0.05 * xyz[:, 0] * xyz[:, 1]
    baseline.stream.wait_stream(p.stream)
    p.run()
    baseline.run()
    parity.assert_areas(parity.gpu_areas(parity.polygons(p), labels),
                        parity.gpu_areas(parity.polygons(baseline), labels))
    deformed = parity.exact_scene_of(arrays[0].cpu().numpy(), arrays[1].cpu().numpy(),
                                     arrays[2].cpu().numpy(), arrays[3].cpu().numpy())
    scene = ex.read_scene(deformed)
    layers, _ = ex.extract(scene)
    parity.assert_areas(parity.gpu_areas(parity.polygons(p), labels),
                        parity.oracle_areas(scene, layers))


def test_stack_hash_is_bounded():
    from peel_b200 import EventPeeler

    p = EventPeeler(*parity.stack_arrays(4096))
    p.run()
    info = p.read_status()
    assert info["edge_hash_misses"] == 0
    assert info["matched_patch_edges"] == 0
    assert info["rank_components"] == 4096
    assert info["ray_groups"] == 1
    np.testing.assert_array_equal(p.output_layers[:4096].cpu().numpy(),
                                  p.output_sources[:4096].cpu().numpy())


def test_live_count_replay():
    """One captured graph over 1025 stacked triangles, of which only `count`
    stay in the window: every live count peels to the same identity ranks."""
    from peel_b200 import EventPeeler

    arrays = parity.stack_arrays(1025)
    original = arrays[0].clone().reshape(1025, 3, 3)
    p = EventPeeler(*arrays)
    p.capture()
    for count in (1025, 127, 0, 257, 256, 1025):
        changed = original.clone()
        changed[count:, :, 0] += 10.0
        with torch.cuda.stream(p.stream):
            arrays[0].copy_(changed.reshape(-1, 3))
        p.run()
        info = p.read_status()
        assert info["polygons"] == count and info["layers"] == count
        assert info["ray_groups"] == int(count > 0)
        np.testing.assert_array_equal(p.output_sources[:count].cpu().numpy(),
                                      p.output_layers[:count].cpu().numpy())
