"""The kernels' sign predicates in their three forms on the GPU: the plain
binary64 expressions of the reference's kernels, the filtered exact signs
(binary32 with a static error bound, binary64, then expansion arithmetic),
and the filtered form with per-class tallies of the deciding stage."""

import numpy as np
import pytest
import parity

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FORMS = ["filtered", "binary64", "counted", "filtered64"]


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def load(name):
    from peel_b200.io import load_scene

    return load_scene(parity.fixture(name))


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("name", ["holes", "closed_object", "cover_2", "cyclic",
                                  "perspective_torus", "shared_vertex", "coplanar_adjacent"])
def test_every_form_matches_the_oracle(name, form):
    from peel_b200 import EventPeeler

    arrays, labels, data = load(name)
    p = EventPeeler(*arrays, predicates=form)
    p.run()
    parity.check_against_oracle(p, data, labels)


def test_counted_tallies_every_class():
    """Nested icospheres: each class of the contour route is evaluated, most
    calls are decided by the first filter, and the forms give the same
    regions."""
    from peel_b200 import EventPeeler, scenes

    arrays = scenes.to_device(scenes.nested_icospheres())
    counted = EventPeeler(*arrays, predicates="counted")
    counted.run()
    counts = counted.predicate_counts()
    for cls in ("side", "segment", "depth", "contain", "order"):
        total = sum(counts[cls].values())
        assert total > 0, (cls, counts)
        # The depth test's filter is a binary64 bound on the two planes'
        # magnitudes; the others start in binary32.
        decided = counts[cls]["binary32"] + (counts[cls]["binary64"] if cls == "depth" else 0)
        assert decided >= 0.5 * total, (cls, counts)
    assert sum(counts["clip"].values()) == 0
    plain = EventPeeler(*arrays, predicates="binary64")
    plain.run()
    # Where rounding decided a sign the forms may cut differently (the
    # subdivision is not canonical), so compare the regions, not the pieces.
    a, b = counted.read_status(), plain.read_status()
    assert a["layers"] == b["layers"]
    labels = range(arrays[1].shape[0])
    parity.assert_areas(parity.gpu_areas(parity.polygons(counted), labels),
                        parity.gpu_areas(parity.polygons(plain), labels))
    uncounted = EventPeeler(*arrays)
    uncounted.run()
    assert sum(sum(v.values()) for v in uncounted.predicate_counts().values()) == 0


def test_exact_degeneracy_is_never_decided_in_binary32():
    """Identical footprints: the patch vertices lie exactly on the contour
    lines.  The binary32 filter never certifies a zero; these zeros are
    decided later (binary64 sees the exactly zero products) and the ranks are
    the stack order."""
    from peel_b200 import EventPeeler

    p = EventPeeler(*parity.stack_arrays(1024), predicates="counted")
    p.run()
    info = p.read_status()
    assert info["polygons"] == 1024 and info["layers"] == 1024
    np.testing.assert_array_equal(p.output_layers[:1024].cpu().numpy(),
                                  p.output_sources[:1024].cpu().numpy())
    counts = p.predicate_counts()
    assert counts["side"]["binary64"] + counts["side"]["exact"] > 0, counts


def test_form_is_fixed_once_captured():
    from peel_b200 import EventPeeler

    arrays, _, _ = load("holes")
    with pytest.raises(ValueError):
        EventPeeler(*arrays, predicates="exact")
    p = EventPeeler(*arrays)
    p.capture()
    with pytest.raises(RuntimeError):
        p._set_predicates("binary64")
