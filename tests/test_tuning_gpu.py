"""Work-distribution knobs and the autotuner on the GPU: extreme settings of
every knob give the same extraction as the defaults (the oracle's regions on
fixtures), a replay after re-tuning records the graph again, and the
autotuner's choice keeps the output counts."""

import pytest
import parity

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

EXTREME = [
    {"step_budget": 1},
    {"step_budget": 100000, "subdivide_blocks": 1},
    {"heavy_noding_work": 1},
    {"heavy_noding_work": 1 << 30, "subdivide_blocks": 32},
]


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def load(name):
    from peel_b200.io import load_scene

    return load_scene(parity.fixture(name))


@pytest.mark.parametrize("knobs", EXTREME)
@pytest.mark.parametrize("name", ["holes", "closed_object", "perspective_torus"])
def test_knobs_keep_the_oracle_regions(name, knobs):
    from peel_b200 import EventPeeler

    arrays, labels, data = load(name)
    p = EventPeeler(*arrays)
    p.set_tuning(**knobs)
    p.run()
    parity.check_against_oracle(p, data, labels)
    assert all(p.tuning()[k] == v for k, v in knobs.items())


@pytest.mark.parametrize("budget", [1, 4, 1000])
def test_clip_budget_keeps_the_oracle_regions(budget):
    from peel_b200 import DevicePeeler

    arrays, labels, data = load("cover_2")
    p = DevicePeeler(*arrays)
    p.set_tuning(clip_budget=budget)
    p.run()
    parity.check_against_oracle(p, data, labels)


def test_retuning_records_the_graph_again():
    from peel_b200 import EventPeeler, scenes

    arrays = scenes.to_device(scenes.nested_icospheres())
    p = EventPeeler(*arrays)
    p.run()
    first = p.read_status()
    p.set_tuning(step_budget=8, heavy_noding_work=64)
    assert p.graph is None
    p.run()
    second = p.read_status()
    for key in ("polygons", "triangles", "layers", "splits"):
        assert first[key] == second[key], key
    labels = range(arrays[1].shape[0])
    base = EventPeeler(*arrays)
    base.run()
    parity.assert_areas(parity.gpu_areas(parity.polygons(p), labels),
                        parity.gpu_areas(parity.polygons(base), labels), 1e-12)


def test_autotune_keeps_the_counts():
    from peel_b200 import EventPeeler, scenes
    from peel_b200.autotune import tune

    arrays = scenes.to_device(scenes.nested_icospheres())
    space = {"step_budget": (16, 48), "heavy_noding_work": (256, 1024)}
    best, default_ms, best_ms, trials = tune(lambda: EventPeeler(*arrays), space=space,
                                             replays=3)
    assert set(best) == set(space) and best_ms <= default_ms
    assert len(trials) == 3
