"""Edge noding on the GPU against the exact oracle.

A large triangle's long edge meets a triangulated half-square of m x m
cells at the same depth: m - 1 T-junctions on that edge, which the resolved
mesh must node (warp_peel/kernels.py:1009-1125), and every point of the
small triangles inside the large triangle's box.  For small m the large
triangle is noded by a thread (k_mesh_polygons); for larger m its grid cells
hold enough candidates that a whole warp nodes it (k_mesh_heavy).  Both must
give the oracle's regions and the same fan: m + 2 triangles.
"""

from dataclasses import replace

import numpy as np
import pytest
import parity

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SETTINGS = [-1.0, -1.0, 1.0, 1.0, 0.0, 0.01]


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def fan_scene(m, s=0.75):
    """Lattice points (m - 2j, m - 2i) * s / m of the half-square above
    x + y = 0, two triangles per cell, then the large triangle below that
    line (the last face).  Points on the line are exact negatives, so they
    lie on the large triangle's long edge exactly."""
    points, index = [], {}
    for i in range(m + 1):
        for j in range(m + 1 - i):
            index[(i, j)] = len(points)
            points.append([(m - 2 * j) * s / m, (m - 2 * i) * s / m, 1.0])
    faces = []
    for i in range(m):
        for j in range(m - i):
            faces.append([index[(i, j)], index[(i + 1, j)], index[(i, j + 1)]])
            if i + j + 1 < m:
                faces.append([index[(i + 1, j)], index[(i + 1, j + 1)], index[(i, j + 1)]])
    k = len(points)
    points += [[-s, -s, 1.0], [s, -s, 1.0], [-s, s, 1.0]]
    faces.append([k, k + 1, k + 2])
    return np.array(points), np.array(faces, dtype=np.int32)


def device_arrays(vertices, faces):
    return [torch.as_tensor(vertices, device="cuda"), torch.as_tensor(faces, device="cuda"),
            torch.as_tensor(np.eye(4), device="cuda"),
            torch.as_tensor(SETTINGS, dtype=torch.float64, device="cuda")]


@pytest.mark.parametrize("m,heavy", [(4, False), (8, False), (26, True)])
def test_t_junctions_noded(m, heavy):
    from peel_b200 import EventPeeler

    vertices, faces = fan_scene(m)
    p = EventPeeler(*device_arrays(vertices, faces))
    p.run()
    info = p.read_status()
    assert (info["heavy_noded_polygons"] > 0) == heavy
    data = parity.exact_scene_of(vertices, faces, np.eye(4), SETTINGS)
    parity.check_against_oracle(p, data, range(len(faces)))
    t = info["triangles"]
    sources = p.triangle_sources[:t].cpu().numpy()
    large = sources == len(faces) - 1
    assert large.sum() == m + 2
    # Every T-junction is a vertex of the large triangle's fan (placed at its
    # parameter along the edge, so within rounding of the lattice point).
    uv = p.triangles_uv[:t].cpu().numpy()[large].reshape(-1, 2)
    window = (vertices[:, :2] - np.array(SETTINGS[:2])) / 2.0
    on_edge = np.unique(window[vertices[:, 0] + vertices[:, 1] == 0.0], axis=0)
    assert len(on_edge) == m + 1
    for x in on_edge:
        assert np.any(np.all(np.abs(uv - x) < 1e-12, axis=1)), x


@pytest.mark.parametrize("m", [8, 26])
def test_edge_noding_capacity(m):
    """m - 1 split points on one edge overflow an edge capacity of m - 2."""
    from peel_b200 import EventCapacities, EventPeeler

    vertices, faces = fan_scene(m)
    cap = replace(EventCapacities.for_mesh(len(faces)), edge_vertices=m - 2)
    p = EventPeeler(*device_arrays(vertices, faces), capacities=cap)
    p.run()
    with pytest.raises(RuntimeError, match="edge noding capacity"):
        p.read_status()
    ok = EventPeeler(*device_arrays(vertices, faces),
                     capacities=replace(cap, edge_vertices=m - 1))
    ok.run()
    assert ok.read_status()["triangles"] > 0
