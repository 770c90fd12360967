"""Optional convex merging (merge_regions) on the GPU, through the C ABI.

Restates the reference's tests/gpu/test_components.py checks of the merge
switch: the merged extraction keeps every (layer, source) region of the exact
oracle, exact ranks and a conforming mesh, with or without rank propagation,
and a captured graph replays it after the input changes.
"""

import pytest
import parity

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SWITCHED = ["holes", "partial", "closed_object", "coplanar_adjacent"]


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def load(name):
    from peel_b200.io import load_scene

    return load_scene(parity.fixture(name))


@pytest.mark.parametrize("propagate,merge", [(True, False), (False, True), (True, True)])
@pytest.mark.parametrize("name", SWITCHED)
def test_component_switches(name, propagate, merge):
    """Regions, ranks and mesh against the oracle (test_components.py:70-84)."""
    from peel_b200 import EventPeeler

    arrays, labels, data = load(name)
    p = EventPeeler(*arrays, propagate_ranks=propagate, merge_regions=merge)
    p.run()
    parity.check_against_oracle(p, data, labels)
    info = p.read_status()
    assert info["edge_hash_misses"] == 0
    if not merge:
        assert info["merged_polygons"] == 0


def test_merge_counts_are_consistent():
    """Each merge removes one polygon from the unmerged extraction."""
    from peel_b200 import EventPeeler, scenes

    cases = [load(name)[:2] for name in parity.RESOLVED]
    icospheres = scenes.to_device(scenes.nested_icospheres())
    cases.append((icospheres, list(range(icospheres[1].shape[0]))))
    merged_any = 0
    for arrays, labels in cases:
        name = len(labels)
        p = EventPeeler(*arrays, merge_regions=True)
        control = EventPeeler(*arrays)
        p.run()
        control.run()
        info, base = p.read_status(), control.read_status()
        assert info["polygons"] == base["polygons"] - info["merged_polygons"], name
        polys = parity.polygons(p)
        assert all(len(v) >= 3 for _, _, v in polys)
        parity.assert_areas(parity.gpu_areas(polys, labels),
                            parity.gpu_areas(parity.polygons(control), labels))
        merged_any += info["merged_polygons"]
    assert merged_any > 0


def test_merge_replay_changed_input():
    """One graph replays the merge after the input changes, and separated
    triangles bypass the adjacency (test_components.py:110-130)."""
    from peel_b200 import EventPeeler

    arrays, labels, _ = load("partial")
    original = arrays[0].clone()
    separated = parity.stack_arrays(2)[0]
    assert separated.shape == original.shape
    p = EventPeeler(*arrays, merge_regions=True)
    control = EventPeeler(*arrays, propagate_ranks=False, merge_regions=False)
    p.capture()
    control.capture()
    for xyz in (original, separated, original, separated):
        for peeler in (p, control):
            with torch.cuda.stream(peeler.stream):
                peeler.stream.wait_stream(torch.cuda.default_stream())
                arrays[0].copy_(xyz)
            peeler.run()
        parity.assert_areas(parity.gpu_areas(parity.polygons(p), labels),
                            parity.gpu_areas(parity.polygons(control), labels))
        if xyz is separated:
            info = p.read_status()
            assert info["splits"] == 0
            assert info["matched_patch_edges"] == 0
            assert info["polygons"] == 2
            assert info["rank_components"] == 2
