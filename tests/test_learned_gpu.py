"""Learned pool sizing on the GPU.

* The training kernel's gradient equals the float64 numpy reference's
  (tests/mlp_reference.py) on the same BF16 weights.
* The tensor-core inference equals the reference with BF16 inputs and hidden
  activations (the operands the MMA takes).
* Adam steps of the project's kernels lower the loss of a small regression.
* The tile features count every triangle once.
* Ablation (with the trained weights): on held-out meshes the learned pools
  take less memory than the worst-case sizing and give the same extraction, and
  a forced under-estimate falls back to the worst-case sizing with the same
  result.
"""

import numpy as np
import pytest
import parity

import mlp_reference as ref

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def batch(rows, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(rows, 16))
    t = rng.normal(size=(rows, 3))
    mask = (rng.random((rows, 3)) < 0.9).astype(float)
    return x, t, mask


def dev(a):
    return torch.tensor(np.asarray(a), dtype=torch.float32, device="cuda")


@pytest.mark.parametrize("rows", [1, 63, 200, 1000])
def test_gradient_matches_float64_reference(rows):
    from peel_b200 import learned

    params = learned.init_params(3)
    x, t, mask = batch(rows, rows)
    scale = 1.0 / (rows * 3)
    grad, loss = learned.gradient(dev(params), dev(x), dev(t), dev(mask), scale)
    # The reference takes the float32 values the kernel sees.
    f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
    w = learned.unpack(f32(params))
    expected_loss, g = ref.loss_and_gradient(w, f32(x), f32(t), mask, scale)
    flat = np.zeros(learned.PARAMS)
    for name, (at, shape) in learned.SLICES.items():
        flat[at:at + int(np.prod(shape))] = g[name].ravel()
    got = grad.cpu().numpy().astype(np.float64)
    assert abs(float(loss.item()) - expected_loss) <= 1e-4 * max(1.0, expected_loss)
    err = np.abs(got - flat)
    assert err.max() <= 1e-4 * max(1.0, np.abs(flat).max()), (err.max(), np.abs(flat).max())


def test_tensor_core_inference_matches_reference():
    from peel_b200 import learned

    params = learned.init_params(5)
    x, _, _ = batch(333, 9)
    y = learned.infer(dev(params), dev(x)).cpu().numpy()
    f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
    _, _, expected = ref.forward(learned.unpack(f32(params)), f32(x), round_activations=True)
    np.testing.assert_allclose(y, expected, rtol=1e-4, atol=1e-4)


def test_adam_training_lowers_the_loss():
    from peel_b200 import learned

    rng = np.random.default_rng(11)
    features = rng.normal(size=(40, learned.TILES, 16))
    hidden = rng.normal(size=(16, 3))
    targets = np.expm1(np.abs(np.tanh(features @ hidden)) * 3.0)
    _, _, _, history = learned.train(features, targets, epochs=30, batch=1024, lr=3e-3)
    assert history[-1] < 0.2 * history[0], history


def test_tile_features_cover_every_triangle():
    from peel_b200 import learned, scenes

    host = scenes.knot_tube()
    f = learned.tile_features(scenes.to_device(host)).cpu().numpy()
    assert f.shape == (learned.TILES, 16)
    assert np.isfinite(f).all()
    # Counts are taken per 4,096 faces, so the tile counts sum to 4,096.
    np.testing.assert_allclose(np.expm1(f[:, 0]).sum(), learned.PER_FACES, rtol=1e-5)
    occupied = np.expm1(f[:, 0]) * len(host[1]) / learned.PER_FACES > 0.5
    assert (f[:, 8] <= f[:, 9] + 1e-6)[occupied].all()
    assert ((f[:, 12] >= 0.0) & (f[:, 12] <= 1.0)).all()


HELD_OUT = [5000, 5001, 5002, 5003]


def trained():
    from peel_b200 import learned

    if not learned.WEIGHTS.exists():
        pytest.skip("no trained weights (python -m peel_b200.learned train)")


@pytest.mark.parametrize("seed", HELD_OUT)
def test_learned_pools_against_worst_case(seed):
    """Held-out meshes (seeds outside the training range): the learned pools
    hold the extraction, take under three quarters of the worst-case memory
    (about 60% measured), and give the same regions and mesh."""
    from peel_b200 import EventPeeler, learned, scenes

    trained()
    arrays = scenes.to_device(scenes.training_mesh(seed))
    p, cap, fell_back = learned.peel(arrays)
    base = EventPeeler(*arrays)
    base.run()
    a, b = p.read_status(), base.read_status()
    for key in ("polygons", "triangles", "layers"):
        assert a[key] == b[key], key
    labels = range(arrays[1].shape[0])
    parity.assert_areas(parity.gpu_areas(parity.polygons(p), labels),
                        parity.gpu_areas(parity.polygons(base), labels))
    assert not fell_back
    assert learned.workspace_bytes(p) < 0.75 * learned.workspace_bytes(base)


def test_under_estimate_falls_back():
    from peel_b200 import EventPeeler, learned, scenes

    trained()
    arrays = scenes.to_device(scenes.training_mesh(HELD_OUT[0]))
    p, cap, fell_back = learned.peel(arrays, scale=0.01)
    assert fell_back
    base = EventPeeler(*arrays)
    base.run()
    assert p.read_status()["polygons"] == base.read_status()["polygons"]
