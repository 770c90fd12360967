"""edp_weld_noalloc: welding for callers that cannot allocate device memory.

A plugin whose host framework owns all device memory through its own arena,
or a real-time loop that must not allocate after start-up, cannot create a
workspace (edp_event_create allocates its pools).  This entry point welds a
vertex buffer with a fixed, preallocated scratch array instead.  The test
calls it through the C ABI and checks its ids against two references on two
calls in a row (the second call must not see the first call's table
contents): a host computation in numpy (the smallest index with an equal
position, signed zeros equal) and the `canonical` ids of the existing
workspace path on the same vertices.  This file is collected last so that a
failure here comes after every other test ran.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def noalloc():
    from peel_b200 import _lib

    return _lib.load().edp_weld_noalloc


def host_canonical(vertices):
    """The smallest index j with vertices[j] == vertices[i], signed zeros
    equal (adding 0.0 turns -0.0 into +0.0 and changes nothing else)."""
    v = np.ascontiguousarray(vertices + 0.0)
    _, first, inverse = np.unique(v, axis=0, return_index=True, return_inverse=True)
    return first[inverse.reshape(-1)].astype(np.int32)


def workspace_canonical(vertices, faces):
    """Canonical ids from the existing entry point (an EventPeeler extraction)."""
    from peel_b200 import EventPeeler

    camera = torch.eye(4, dtype=torch.float64, device="cuda")
    settings = torch.tensor([-10.0, -10.0, 10.0, 10.0, 0.0, 0.01], dtype=torch.float64,
                            device="cuda")
    p = EventPeeler(vertices, faces, camera, settings)
    p.run()
    # Welding is the first stage; its ids are final whether or not the random
    # overlapping triangles later fit the default pools.
    p.stream.synchronize()
    return p.canonical[: vertices.shape[0]].cpu().numpy()


def scene(seed, nv):
    """Vertices with many exact repeats, signed zeros among them."""
    rng = np.random.default_rng(seed)
    base = rng.integers(-3, 4, size=(nv // 3, 3)).astype(np.float64)
    vertices = base[rng.integers(0, len(base), size=nv)]
    vertices = np.where((vertices == 0) & (rng.random(vertices.shape) < 0.5), -0.0, vertices)
    faces = np.arange(3 * (nv // 3), dtype=np.int32).reshape(-1, 3)
    return vertices, faces


def test_host_reference_welds_signed_zeros():
    v = np.array([[0.0, 1.0, -0.0], [1.0, 1.0, 1.0], [-0.0, 1.0, 0.0], [1.0, 1.0, 1.0]])
    np.testing.assert_array_equal(host_canonical(v), [0, 1, 0, 1])


@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_noalloc_weld_matches_host_and_workspace_on_two_calls_in_a_row():
    fn = noalloc()
    stream = torch.cuda.current_stream().cuda_stream
    for seed, nv in ((0, 30000), (1, 3000)):  # the second, smaller call reuses the table
        host_v, host_f = scene(seed, nv)
        vertices = torch.as_tensor(host_v, device="cuda")
        faces = torch.as_tensor(host_f, device="cuda")
        expected = host_canonical(host_v)
        np.testing.assert_array_equal(workspace_canonical(vertices, faces), expected)
        out = torch.full((nv,), -7, dtype=torch.int32, device="cuda")
        assert fn(vertices.data_ptr(), nv, out.data_ptr(), stream) == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), expected)


@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_noalloc_weld_rejects_sizes_beyond_its_scratch():
    fn = noalloc()
    limit = 262144
    vertices = torch.zeros((limit + 1, 3), dtype=torch.float64, device="cuda")
    out = torch.zeros(limit + 1, dtype=torch.int32, device="cuda")
    assert fn(vertices.data_ptr(), limit + 1, out.data_ptr(),
              torch.cuda.current_stream().cuda_stream) == 1
