"""Learned pool sizing on the CPU: the float64 reference network against
finite differences, BF16 rounding, and the capacity rule (sums of predicted
tile counts with margins, never above the worst-case layer count)."""

import numpy as np

import mlp_reference as ref


def small_network(seed):
    from peel_b200 import learned

    return learned.unpack(learned.init_params(seed))


def test_reference_gradient_matches_finite_differences():
    w = {k: v.copy() for k, v in small_network(1).items()}
    rng = np.random.default_rng(2)
    x = rng.normal(size=(9, 16))
    t = rng.normal(size=(9, 3))
    mask = (rng.random((9, 3)) < 0.8).astype(float)
    _, g = ref.loss_and_gradient(w, x, t, mask, 0.5)
    # Differentiate through the biases (weights enter rounded to BF16, so
    # their finite differences are steps of the rounding, not the gradient).
    for name in ("b1", "b2", "b3"):
        for i in range(0, w[name].size, 7):
            step = 1e-6
            w[name].flat[i] += step
            up, _ = ref.loss_and_gradient(w, x, t, mask, 0.5)
            w[name].flat[i] -= 2 * step
            down, _ = ref.loss_and_gradient(w, x, t, mask, 0.5)
            w[name].flat[i] += step
            numeric = 0.5 * (up - down) / (2 * step)
            assert abs(numeric - g[name].flat[i]) <= 1e-6 * max(1.0, abs(numeric)), (name, i)


def test_bf16_rounding_is_to_nearest_even():
    v = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, -2.5])
    r = ref.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0  # a tie goes to the even mantissa
    assert r[2] == 1.0 + 2.0 ** -7 and r[3] == -2.5


def test_capacities_from_counts():
    from peel_b200 import learned
    from peel_b200.events import EventCapacities

    counts = np.zeros((learned.TILES, 3))
    counts[:10] = [100.0, 300.0, 4.0]
    margins = {"fragments": 1.5, "triangles": 1.2, "hits": 2.0, "layers": 1.25}
    cap = learned.capacities_from_counts(counts, margins, 65536)
    assert cap.regions == cap.frontier == int(1.5 * 1000) + 256
    assert cap.triangles == int(1.2 * 3000) + 1024
    assert cap.vertices == cap.triangles + 2 * cap.regions
    assert cap.hits == int(2.0 * 4000) + 1024
    assert cap.layers == int(1.25 * 4) + 8
    base = EventCapacities.for_mesh(65536)
    assert cap.regions < base.regions and cap.hits < base.hits
    huge = learned.capacities_from_counts(counts * 1e6, margins, 65536)
    assert (huge.regions, huge.hits, huge.triangles) == (base.regions, base.hits, base.triangles)
    few = np.zeros_like(counts)
    few[0] = [10.0, 30.0, 40.0]
    assert learned.capacities_from_counts(few, margins, 4).layers == EventCapacities.for_mesh(4).layers


def test_training_meshes_are_seeded_and_in_range():
    from peel_b200 import scenes

    a, b = scenes.training_mesh(1000), scenes.training_mesh(1000)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    for seed in (1000, 1001, 1002):
        v, f, camera, settings = scenes.training_mesh(seed)
        assert 3000 <= len(f) <= 70000
        assert settings[4] == 1.0


def test_counts_per_faces_round_trip():
    from peel_b200 import learned

    counts = np.array([[100.0, 300.0, 4.0], [0.0, 0.0, 0.0]])
    scaled = learned.per_faces(counts, 8192)
    assert scaled[0].tolist() == [50.0, 150.0, 4.0]
    np.testing.assert_array_equal(learned.per_faces(scaled, 8192, inverse=True), counts)
