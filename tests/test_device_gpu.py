"""DevicePeeler (iterative clipping) on the GPU, through the C ABI, against the
exact oracle.  Restates the reference's tests/gpu/test_peeler.py, which runs
this route on every accepted fixture, unresolved crossings included."""

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


@pytest.mark.parametrize("name", parity.ACCEPTED)
def test_oracle(name):
    from peel_b200 import DevicePeeler

    arrays, labels, data = load(name)
    p = DevicePeeler(*arrays)
    p.run()
    parity.check_against_oracle(p, data, labels)
    first = parity.gpu_areas(parity.polygons(p), labels)
    p.run()
    parity.assert_areas(parity.gpu_areas(parity.polygons(p), labels), first)


@pytest.mark.parametrize("limit", [1, 2])
def test_prefix(limit):
    from oracle import exact as ex
    from peel_b200 import DevicePeeler

    arrays, labels, data = load("holes")
    p = DevicePeeler(*arrays, layers=limit)
    p.run()
    scene = ex.read_scene(data)
    layers, _ = ex.extract(scene)
    expected = {k: v for k, v in parity.oracle_areas(scene, layers).items() if k[0] < limit}
    parity.assert_areas(parity.gpu_areas(parity.polygons(p), labels), expected)


@pytest.mark.parametrize("field,bit", [
    ("residual", 4),
    ("polygons", 8),
    ("vertices", 16),
    ("triangles", 32),
    ("layers", 64),
    ("pieces_per_worker", 2),
])
def test_overflow(field, bit):
    """Each capacity set to 1 raises its error bit, also on a second replay
    (tests/gpu/test_peeler.py:216-238)."""
    from peel_b200 import Capacities, DevicePeeler

    arrays, _, _ = load("holes")
    cap = replace(Capacities.for_mesh(arrays[1].shape[0]), **{field: 1})
    p = DevicePeeler(*arrays, capacities=cap)
    for _ in range(2):
        p.run()
        with pytest.raises(RuntimeError, match="GPU extraction failed"):
            p.read_status()
        assert int(p.status[9].item()) & bit


@pytest.mark.parametrize("invalid", ["index", "camera"])
def test_invalid_device_input(invalid):
    from peel_b200 import DevicePeeler

    arrays, _, _ = load("single")
    p = DevicePeeler(*arrays)
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


def test_device_camera_update():
    """Changing the camera on the device between replays (test_peeler.py:290-302)."""
    from oracle import exact as ex
    from peel_b200 import DevicePeeler

    arrays, labels, data = load("partial")
    p = DevicePeeler(*arrays)
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


def test_stack_ranks():
    from peel_b200 import DevicePeeler

    p = DevicePeeler(*parity.stack_arrays(64))
    p.run()
    info = p.read_status()
    assert info["polygons"] == 64 and info["layers"] == 64
    np.testing.assert_array_equal(np.sort(p.output_layers[:64].cpu().numpy()), np.arange(64))
    order = np.argsort(p.output_layers[:64].cpu().numpy())
    np.testing.assert_array_equal(p.output_sources[:64].cpu().numpy()[order], np.arange(64))
