"""BatchPeeler: many scenes in one CUDA graph replay, each with the results of
its own EventPeeler (the batched configuration's contract)."""

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


def test_batch_matches_single_peelers():
    from peel_b200 import BatchPeeler, EventPeeler, scenes

    fixtures = [load(name) for name in ("holes", "partial", "closed_object", "stacked")]
    generated = [scenes.to_device(scenes.nested_icospheres()),
                 scenes.to_device(scenes.stress_stack(512, 0.0))]
    views = scenes.turntable_views(scenes.nested_icospheres()[0], count=3, seed=11)
    ico = scenes.nested_icospheres()
    generated += [scenes.to_device((ico[0], ico[1], c, s)) for c, s in views]
    all_scenes = [f[0] for f in fixtures] + generated
    batch = BatchPeeler(all_scenes)
    batch.run()
    infos = batch.read_status()
    for k, (arrays, info) in enumerate(zip(all_scenes, infos)):
        single = EventPeeler(*arrays)
        single.run()
        control = single.read_status()
        assert info["polygons"] == control["polygons"] and info["layers"] == control["layers"], k
        labels = range(arrays[1].shape[0])
        parity.assert_areas(parity.gpu_areas(parity.polygons(batch.peelers[k]), labels),
                            parity.gpu_areas(parity.polygons(single), labels))
    for (arrays, labels, data), p in zip(fixtures, batch.peelers):
        parity.check_against_oracle(p, data, labels)


def test_batch_replay_with_changed_input():
    from peel_b200 import BatchPeeler

    arrays = [parity.stack_arrays(64), parity.stack_arrays(128)]
    batch = BatchPeeler(arrays)
    batch.run()
    assert [i["layers"] for i in batch.read_status()] == [64, 128]
    shifted = arrays[1][0].clone().reshape(128, 3, 3)
    shifted[1::2, :, 0] += 0.25  # every other layer moves: two overlapping footprints
    shifted = shifted.reshape(-1, 3)
    with torch.cuda.stream(batch.stream):
        batch.stream.wait_stream(torch.cuda.default_stream())
        arrays[1][0].copy_(shifted)
    batch.run()
    first, second = batch.read_status()
    assert first["layers"] == 64 and first["polygons"] == 64
    assert second["polygons"] > 128
    np.testing.assert_array_equal(batch.peelers[0].output_layers[:64].cpu().numpy(),
                                  batch.peelers[0].output_sources[:64].cpu().numpy())


def test_empty_batch_rejected():
    from peel_b200 import BatchPeeler

    with pytest.raises(ValueError):
        BatchPeeler([])
