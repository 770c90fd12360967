"""EventPeeler on the GPU, through the C ABI, against the exact oracle.

Restates the reference's tests/gpu/test_peeler.py and test_events.py checks
for the contour-subdivision route.  Every test needs a CUDA device.
"""

from dataclasses import replace

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


@pytest.mark.parametrize("name", parity.RESOLVED)
def test_complete_oracle(name):
    from peel_b200 import EventPeeler

    arrays, labels, data = load(name)
    p = EventPeeler(*arrays)
    p.run()
    parity.check_against_oracle(p, data, labels)
    # Replay resets all counters and emits the same labelled regions.
    first = parity.gpu_areas(parity.polygons(p), labels)
    p.run()
    parity.assert_areas(parity.gpu_areas(parity.polygons(p), labels), first)


@pytest.mark.parametrize("limit", [1, 2])
def test_prefix(limit):
    from oracle import exact as ex
    from peel_b200 import EventPeeler

    arrays, labels, data = load("holes")
    p = EventPeeler(*arrays, layers=limit)
    p.run()
    scene = ex.read_scene(data)
    layers, _ = ex.extract(scene)
    expected = {k: v for k, v in parity.oracle_areas(scene, layers).items() if k[0] < limit}
    parity.assert_areas(parity.gpu_areas(parity.polygons(p), labels), expected)


@pytest.mark.parametrize("n", [16, 33, 65, 128, 257, 1024])
def test_shared_stack(n):
    """Work-count known answers (tests/gpu/test_events.py:74-88)."""
    from peel_b200 import EventPeeler

    p = EventPeeler(*parity.stack_arrays(n))
    p.run()
    info = p.read_status()
    assert info["polygons"] == n
    assert info["splits"] == 0
    assert info["unique_contours"] == 3
    assert info["ray_groups"] == 1
    assert info["ray_candidate_tests"] == n
    assert info["ray_hits"] == n
    assert info["contour_tests"] <= 3 * n
    np.testing.assert_array_equal(p.output_layers[:n].cpu().numpy(),
                                  p.output_sources[:n].cpu().numpy())


@pytest.mark.parametrize("field,match", [
    ("hits", "shared ray hit"),
    ("rounds", "subdivision round"),
    ("frontier", "residual pool"),
    ("regions", "output polygon"),
])
def test_capacity(field, match):
    from peel_b200 import EventCapacities, EventPeeler

    arrays, _, _ = load("holes")
    cap = replace(EventCapacities.for_mesh(arrays[1].shape[0]), **{field: 1})
    p = EventPeeler(*arrays, capacities=cap)
    for _ in range(2):
        p.run()
        with pytest.raises(RuntimeError, match=match):
            p.read_status()


@pytest.mark.parametrize("invalid", ["index", "camera"])
def test_invalid_device_input(invalid):
    from peel_b200 import EventPeeler

    arrays, _, _ = load("single")
    p = EventPeeler(*arrays)
    p.run()
    p.read_status()
    with torch.cuda.stream(p.stream):
        if invalid == "index":
            arrays[1][0] = torch.tensor([-1, 0, 1000000], dtype=torch.int32, device="cuda")
        else:
            arrays[2].zero_()
    p.run()
    with pytest.raises(RuntimeError, match="invalid input"):
        p.read_status()


def test_external_capture_and_changed_input():
    """enqueue() inside a torch CUDA graph capture, then replay after an
    on-device translation of the vertices (tests/gpu/test_peeler.py:155-202)."""
    from oracle import exact as ex
    from peel_b200 import EventPeeler

    arrays, labels, data = load("partial")
    p = EventPeeler(*arrays)
    p.warmup()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=p.stream):
        p.enqueue()
    graph.replay()
    before = parity.gpu_areas(parity.polygons(p), labels)
    with torch.cuda.stream(p.stream):
        arrays[0] += torch.tensor([0.5, 0.25, 0.0], dtype=torch.float64, device="cuda")
    graph.replay()
    after = parity.gpu_areas(parity.polygons(p), labels)
    assert any(abs(before[k] - after.get(k, 0.0)) > 1e-4 for k in before) or before != after
    shifted = parity.exact_scene_of(arrays[0].cpu().numpy(), arrays[1].cpu().numpy(),
                                    arrays[2].cpu().numpy(), arrays[3].cpu().numpy())
    scene = ex.read_scene(shifted)
    layers, _ = ex.extract(scene)
    parity.assert_areas(after, parity.oracle_areas(scene, layers))
    # Another workspace does not invalidate this graph.
    arrays2, _, _ = load("perspective_torus")
    q = EventPeeler(*arrays2)
    q.run()
    q.read_status()
    graph.replay()
    parity.assert_areas(parity.gpu_areas(parity.polygons(p), labels), after)


def test_device_welding_signed_zero():
    from peel_b200 import EventPeeler

    vertices = np.array([[0, 2, 1], [-0.0, 1, 1], [0, 1, 1], [-0.0, 2, 1]], dtype=np.float64)
    p = EventPeeler(
        torch.as_tensor(vertices, device="cuda"),
        torch.zeros((0, 3), dtype=torch.int32, device="cuda"),
        torch.eye(4, dtype=torch.float64, device="cuda"),
        torch.tensor([-5.0, -5.0, 5.0, 5.0, 0.0, 1.0], dtype=torch.float64, device="cuda"),
    )
    p.run()
    p.read_status()
    ids = p.canonical.cpu().numpy()
    assert ids[0] == ids[3] and ids[1] == ids[2] and ids[0] != ids[1]


def test_empty_download():
    from peel_b200 import EventPeeler
    from peel_b200.io import download_mesh

    arrays, _, _ = load("empty")
    p = EventPeeler(*arrays)
    p.run()
    data = download_mesh(p)
    assert data["world"].shape == (0, 3, 3)


def test_foreground_unsplit():
    """A foreground source stays one polygon (tests/gpu/test_events.py:126-133)."""
    from peel_b200 import EventPeeler

    arrays, _, _ = load("cover_2")
    p = EventPeeler(*arrays)
    p.run()
    info = p.read_status()
    ids = p.output_sources[: info["polygons"]].cpu().numpy()
    ranks = p.output_layers[: info["polygons"]].cpu().numpy()
    assert np.count_nonzero((ids == 0) & (ranks == 0)) == 1


def test_nonmanifold_edge():
    from peel_b200 import EventPeeler
    from peel_b200.io import load_scene

    a, b = [-1, 0, 2], [1, 0, 2]
    data = {
        "window": [-2, -2, 2, 2],
        "camera": {"type": "orthographic"},
        "triangles": [{"id": i, "vertices": [a, b, c]}
                      for i, c in enumerate([[0, 1, 1], [0, -1, 1], [0, 1, 3]])],
    }
    arrays, labels, _ = load_scene(data)
    p = EventPeeler(*arrays)
    p.run()
    parity.check_against_oracle(p, data, labels)


@pytest.mark.parametrize("slanted", [False, True])
def test_certified_distinct_samples(slanted):
    """Nested footprints: one certified rectangle and one shared ray
    (tests/gpu/test_events.py:154-190)."""
    from peel_b200 import EventCapacities, EventPeeler

    n = 128
    arrays = parity.stack_arrays(n)
    xyz = arrays[0].cpu().numpy().reshape(n, 3, 3)
    t = np.arange(n) / n
    xyz[:, :, :2] *= (1 - 0.1 * t)[:, None, None]
    xyz[:, :, 0] += 0.01 * t[:, None]
    if slanted:
        xyz[:, :, 2] = 10 + 0.001 * np.arange(n)[:, None] + 10 * xyz[:, :, 0]
    arrays[0] = torch.as_tensor(xyz.reshape(-1, 3), device="cuda")
    p = EventPeeler(*arrays)
    p.run()
    info = p.read_status()
    assert info["splits"] == 0
    assert info["polygons"] == n
    assert info["certified_beams"] == 1
    assert info["ray_groups"] == 1
    assert info["ray_candidate_tests"] == n
    assert info["beam_candidate_tests"] == n
    np.testing.assert_array_equal(p.output_sources[:n].cpu().numpy(),
                                  p.output_layers[:n].cpu().numpy())
    baseline = EventPeeler(*arrays, share_regions=False,
                           capacities=replace(EventCapacities.for_mesh(n), hits=n * n))
    baseline.run()
    control = baseline.read_status()
    assert control["ray_groups"] == n
    assert control["ray_candidate_tests"] == n * n
    np.testing.assert_array_equal(baseline.output_sources[:n].cpu().numpy(),
                                  baseline.output_layers[:n].cpu().numpy())


def test_heavy_disjoint_groups():
    from peel_b200 import EventPeeler

    arrays = parity.stack_arrays(130)
    xyz = arrays[0].cpu().numpy().reshape(130, 3, 3)
    xyz[:, :, 0] *= 0.25
    xyz[:, :, 0] += np.where(np.arange(130) % 2, 0.5, -0.5)[:, None]
    arrays[0] = torch.as_tensor(xyz.reshape(-1, 3), device="cuda")
    p = EventPeeler(*arrays)
    p.run()
    info = p.read_status()
    assert info["ray_groups"] == info["heavy_ray_groups"] == 2
    assert info["ray_hits"] == 130
    np.testing.assert_array_equal(p.output_sources[:130].cpu().numpy() // 2,
                                  p.output_layers[:130].cpu().numpy())


def test_replay_changes_sort_bucket():
    """One captured graph serves different live hit counts (test_events.py:209-238)."""
    from peel_b200 import EventCapacities, EventPeeler

    n = 64
    arrays = parity.stack_arrays(n)
    cap = replace(EventCapacities.for_mesh(n), hits=n * n)
    p = EventPeeler(*arrays, capacities=cap, share_regions=False)
    p.run()
    assert p.read_status()["ray_hits"] == n
    xyz = arrays[0].cpu().numpy().reshape(n, 3, 3)
    xyz[:, :, :2] *= (1 - 0.1 * np.arange(n) / n)[:, None, None]
    xyz[:, :, 0] += (0.01 * np.arange(n) / n)[:, None]
    changed = torch.as_tensor(xyz.reshape(-1, 3), device="cuda")
    with torch.cuda.stream(p.stream):
        p.stream.wait_stream(torch.cuda.default_stream())
        arrays[0].copy_(changed)
    p.run()
    assert p.read_status()["ray_hits"] == n * n
    np.testing.assert_array_equal(p.output_sources[:n].cpu().numpy(),
                                  p.output_layers[:n].cpu().numpy())
    with torch.cuda.stream(p.stream):
        arrays[0].copy_(parity.stack_arrays(n)[0])
    p.run()
    assert p.read_status()["ray_hits"] == n
