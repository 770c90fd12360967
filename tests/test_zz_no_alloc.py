"""edp_weld_noalloc: welding for callers that cannot allocate device memory.

Code that is recording a CUDA graph, code running under an allocator that owns
all device memory, and loops that must not allocate after start-up cannot
create a workspace (edp_event_create allocates its pools).  This entry point
welds a vertex buffer with a fixed, preallocated scratch array instead.  The
test calls it through the C ABI and checks that its ids equal the `canonical`
ids of the existing workspace path on the same vertices, on two calls in a
row (the second call must not see the first call's table contents).  This file
is collected last so that a failure here comes after every other test ran.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def noalloc():
    from peel_b200 import _lib

    fn = _lib.load().edp_weld_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


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
    return (torch.as_tensor(vertices, device="cuda"),
            torch.as_tensor(faces, device="cuda"))


@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_noalloc_weld_matches_workspace_on_two_calls_in_a_row():
    fn = noalloc()
    stream = torch.cuda.current_stream().cuda_stream
    for seed, nv in ((0, 30000), (1, 3000)):  # the second, smaller call reuses the table
        vertices, faces = scene(seed, nv)
        expected = workspace_canonical(vertices, faces)
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
