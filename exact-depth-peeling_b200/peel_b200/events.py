"""EventPeeler: contour subdivision and shared-ray ranks on one B200.

Same call surface as the reference's ``warp_peel.EventPeeler``
(warp_peel/events.py:36-845) over torch CUDA tensors: construct, then
``capture()``/``run()`` (asynchronous graph replay on ``peeler.stream``), and
``read_status()`` for an explicit host check.  The whole extraction runs in
hand-written CUDA kernels inside one CUDA graph whose subdivision loop is a
device-side conditional WHILE node; there is no host loop, transfer or
allocation during replay.
"""

import ctypes
from dataclasses import dataclass

from . import _lib
from .solver import METRIC_COUNT, _Peeler, _Workspace, _check_inputs, _decode_status


@dataclass(frozen=True)
class EventCapacities:
    frontier: int
    regions: int
    hits: int
    vertices: int
    triangles: int
    rounds: int = 4096
    layers: int = 4096
    edge_vertices: int = 128

    @classmethod
    def for_mesh(cls, n):
        """4N frontier, 8N regions, 32N hits/vertices/triangles (events.py:30-33)."""
        n = max(16, n)
        return cls(4 * n, 8 * n, 32 * n, 32 * n, 32 * n, layers=n)


METRIC_NAMES = (
    "target_visits", "contour_tests", "splits", "ray_groups", "ray_candidate_tests",
    "ray_hits", "rounds", "unique_contours", "heavy_ray_groups", "beam_attempts",
    "certified_beams", "beam_candidate_tests", "heavy_beams", "rank_components",
    "rank_connections", "connection_contour_tests", "merged_polygons", "matched_patch_edges",
    "edge_hash_misses", "heavy_noded_polygons", "parked_patches", "deferred_contain_tests",
    "deferred_hit_groups", "deferred_polygons",
)
assert len(METRIC_NAMES) == METRIC_COUNT


class EventPeeler(_Peeler):
    """All-layer contour subdivision followed by shared sorted ray hits.

    vertices: float64 [V, 3]; faces: int32 [N, 3]; camera: float64 [4, 4]
    (or [1, 4, 4]) affine world-to-camera with last row [0, 0, 0, 1];
    settings: float64 [6] = xmin, ymin, xmax, ymax, perspective (0/1), near.
    All on one CUDA device.  The caller owns the inputs and may change their
    values (not addresses or sizes) between replays on ``peeler.stream``.
    Inputs must have resolved surface intersections.

    ``predicates`` (not in the reference, whose kernels are plain binary64)
    selects the sign predicates: "filtered64" (the default: exact signs
    through a binary64 filter and expansion arithmetic), "filtered" (exact
    signs through binary32, then binary64 filters, then expansions),
    "binary64" (the reference's plain expressions) or "counted" ("filtered",
    with per-class tallies of the deciding stage, read by
    ``predicate_counts()``).
    """

    def __init__(self, vertices, faces, camera, settings, *, capacities=None, layers=0,
                 share_regions=True, propagate_ranks=True, merge_regions=False,
                 predicates="filtered64"):
        import torch

        self.device = _check_inputs(vertices, faces, camera, settings)
        ec = capacities or EventCapacities.for_mesh(faces.shape[0])
        if min(vars(ec).values()) < 1:
            raise ValueError("Event capacities must be positive")
        if ec.edge_vertices > 128:
            raise ValueError("Capacities must be positive; edge_vertices must be <= 128")
        if layers < 0 or layers > ec.layers:
            raise ValueError("layers must be zero (all), or fit in the layer capacity")
        self.event_cap = ec
        self.cap = ec
        self.share_regions = share_regions
        self.propagate_ranks = propagate_ranks
        self.merge_regions = merge_regions
        self.vertices, self.faces = vertices, faces
        self.camera, self.settings = camera, settings
        self.n = faces.shape[0]
        self.nv = vertices.shape[0]
        self.limit = layers or ec.layers
        self.all_layers = int(layers == 0)
        self.stream = torch.cuda.Stream(self.device)
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        lib = _lib.load()
        c = _lib.EventCapacitiesC(*[int(getattr(ec, f)) for f, _ in _lib.EventCapacitiesC._fields_])
        o = _lib.EventOptionsC(int(layers), int(share_regions), int(propagate_ranks),
                               int(merge_regions))
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(
                lib.edp_event_create(
                    vertices.data_ptr(), self.nv, faces.data_ptr(), self.n, camera.data_ptr(),
                    settings.data_ptr(), ctypes.byref(c), ctypes.byref(o),
                    self.stream.cuda_stream, ctypes.byref(handle)),
                "EventPeeler")
        self._ws = _Workspace(handle, self.device, (vertices, faces, camera, settings))
        self._ws.expose(self)
        self._set_predicates(predicates)
        self.graph = None
        self.warmed = False

    def read_status(self):
        """Synchronise the workspace stream and decode status and counters."""
        status, metrics = self._ws.read()
        if status[9] & 1024:
            raise RuntimeError("GPU extraction failed: shared ray hit capacity")
        if status[9] & 2048:
            raise RuntimeError("GPU extraction failed: subdivision round capacity")
        info = _decode_status(status)
        for name in ("peeling_passes", "max_hidden_pieces"):
            info.pop(name)
        info.update(zip(METRIC_NAMES, map(int, metrics)))
        return info
