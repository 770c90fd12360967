"""Workspace plumbing shared by both peelers, plus ``Capacities``/``DevicePeeler``.

Mirrors warp_peel/solver.py:10-519.  Device buffers owned by the native
workspace are exposed as torch tensors (zero-copy views through
``__cuda_array_interface__``) under the reference's attribute names.
"""

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib

METRIC_COUNT = 24  # EDP_METRICS: workspace counters (include/edp.h)

_ERROR_LABELS = {
    1: "polygon vertices",
    2: "per-worker pieces",
    4: "residual pool",
    8: "output polygon pool",
    16: "boundary vertex pool",
    32: "triangle pool",
    64: "layer limit",
    128: "edge noding capacity",
    256: "invalid input",
}


@dataclass(frozen=True)
class Capacities:
    """DevicePeeler pools (warp_peel/solver.py:10-31).  residual: patches
    left for the next layer; polygons, vertices, triangles: outputs.  The
    clipping queue shares polygons + residual piece slots among all targets;
    pieces_per_worker bounds the visible and the hidden pieces of one target
    (the reference's per-worker pool error); workers is kept for the
    interface."""

    residual: int
    polygons: int
    vertices: int
    triangles: int
    workers: int = 4096
    pieces_per_worker: int = 512
    layers: int = 128
    edge_vertices: int = 128

    @classmethod
    def for_mesh(cls, triangles: int):
        """Reference defaults (solver.py:21-31)."""
        n = max(triangles, 16)
        return cls(4 * n, 16 * n, 96 * n, 64 * n, workers=min(4096, n),
                   pieces_per_worker=512 if n <= 8192 else 2048)


def _decode_status(values):
    """Raise on sticky device errors; return the reference's status dictionary
    (solver.py:488-519)."""
    if values[9]:
        raise RuntimeError(
            "GPU extraction failed: "
            + ", ".join(v for b, v in _ERROR_LABELS.items() if values[9] & b)
        )
    return {
        "residual_patches": int(values[0]),
        "polygons": int(values[2]),
        "triangles": int(values[3]),
        "layers": int(values[4]),
        "peeling_passes": int(values[5]),
        "boundary_vertices": int(values[6]),
        "depth_ties": int(values[8]),
        "error": int(values[9]),
        "max_hidden_pieces": int(values[10]),
        "peak_residual_patches": int(values[12]),
    }


def _check_inputs(vertices, faces, camera, settings):
    """Validate tensors like solver.py:114-128; return the CUDA device."""
    import torch

    for t in (vertices, faces, camera, settings):
        if not isinstance(t, torch.Tensor):
            raise ValueError("Expected torch tensors on a CUDA device")
    device = vertices.device
    if device.type != "cuda":
        raise ValueError("Peelers require a CUDA device")
    spec = [
        (vertices, torch.float64, lambda s: len(s) == 2 and s[1] == 3, "float64 [V, 3] vertices"),
        (faces, torch.int32, lambda s: len(s) == 2 and s[1] == 3, "int32 [N, 3] faces"),
        (camera, torch.float64, lambda s: tuple(s) in ((4, 4), (1, 4, 4)), "float64 [4, 4] camera"),
        (settings, torch.float64, lambda s: tuple(s) == (6,), "float64 [6] settings"),
    ]
    for t, dtype, shape_ok, what in spec:
        if t.device != device or t.dtype != dtype or not shape_ok(t.shape):
            raise ValueError(f"Expected a {what} tensor on {device}")
        if not t.is_contiguous():
            raise ValueError(f"Expected a contiguous {what} tensor")
    return device


class _DeviceArray:
    """__cuda_array_interface__ over workspace memory; keeps the workspace alive."""

    def __init__(self, ptr, shape, typestr, owner):
        self._owner = owner
        self.__cuda_array_interface__ = {
            "shape": tuple(int(s) for s in shape),
            "typestr": typestr,
            "data": (int(ptr), False),
            "version": 3,
            "strides": None,
            "stream": None,
        }


class PolygonArray:
    """Output polygons: ``vertices`` [R, 32, 2] float64 and ``sizes`` [R] int32.

    ``numpy()`` returns the reference's structured layout with fields ``v``
    (32 x 2 binary64) and ``n``, so ``p.output.numpy()[i]["v"][:n]`` works.
    """

    DTYPE = np.dtype([("v", np.float64, (32, 2)), ("n", np.int32)])

    def __init__(self, vertices, sizes):
        self.vertices = vertices
        self.sizes = sizes

    def __len__(self):
        return self.sizes.shape[0]

    def numpy(self):
        out = np.zeros(len(self), dtype=self.DTYPE)
        out["v"] = self.vertices.cpu().numpy()
        out["n"] = self.sizes.cpu().numpy()
        return out


class _Workspace:
    """Owner of one native workspace handle."""

    def __init__(self, handle, device, inputs):
        self.handle = handle
        self.device = device
        self.inputs = inputs  # keep the caller's input tensors alive with the graph

    def view(self, ptr, shape, torch_dtype, typestr):
        import torch

        count = int(np.prod(shape)) if len(shape) else 1
        if count == 0:
            return torch.empty(shape, dtype=torch_dtype, device=self.device)
        return torch.as_tensor(_DeviceArray(ptr, shape, typestr, self), device=self.device)

    def expose(self, peeler):
        import torch

        lib = _lib.load()
        o = _lib.OutputsC()
        _lib.check(lib.edp_get_outputs(self.handle, ctypes.byref(o)), "outputs")
        R, T = int(o.regions), int(o.triangles)
        i32, f64 = (torch.int32, "<i4"), (torch.float64, "<f8")
        peeler.status = self.view(o.status, (16,), *i32)
        peeler.metrics = self.view(o.metrics, (METRIC_COUNT,), torch.int64, "<i8")
        peeler.output = PolygonArray(self.view(o.output_vertices, (R, 32, 2), *f64),
                                     self.view(o.output_sizes, (R,), *i32))
        peeler.output_sources = self.view(o.output_sources, (R,), *i32)
        peeler.output_layers = self.view(o.output_layers, (R,), *i32)
        peeler.triangles_uv = self.view(o.triangles_uv, (T, 3, 2), *f64)
        peeler.triangles_world = self.view(o.triangles_world, (T, 3, 3), *f64)
        peeler.triangle_sources = self.view(o.triangle_sources, (T,), *i32)
        peeler.triangle_layers = self.view(o.triangle_layers, (T,), *i32)
        peeler.canonical = self.view(o.canonical, (max(1, peeler.nv),), *i32)

    def call(self, name, what):
        import torch

        with torch.cuda.device(self.device):
            _lib.check(getattr(_lib.load(), name)(self.handle), what)

    def call_args(self, name, what, *args):
        import torch

        with torch.cuda.device(self.device):
            _lib.check(getattr(_lib.load(), name)(self.handle, *args), what)

    def read(self):
        status = np.zeros(16, dtype=np.int32)
        metrics = np.zeros(METRIC_COUNT, dtype=np.int64)
        _lib.check(
            _lib.load().edp_read_status(self.handle, status.ctypes.data, metrics.ctypes.data),
            "read_status")
        return status, metrics

    def __del__(self):
        h, self.handle = getattr(self, "handle", None), None
        if h and _lib._lib is not None:
            _lib._lib.edp_destroy(h)


class _Peeler:
    """Execution methods shared by both peelers (solver.py:447-486, events.py:782-806)."""

    def warmup(self):
        """One eager extraction before any capture (host-driven loop control)."""
        import torch

        if torch.cuda.is_current_stream_capturing():
            raise RuntimeError("Warm-up must run before graph capture")
        self._ws.call("edp_warmup", "warm-up")
        self.warmed = True

    def enqueue(self):
        """Record the complete pipeline into the caller's capture on ``self.stream``."""
        import torch

        if not self.warmed or not torch.cuda.is_current_stream_capturing():
            raise RuntimeError("Call warmup(), then enqueue() inside a CUDA graph capture")
        if torch.cuda.current_stream(self.device).cuda_stream != self.stream.cuda_stream:
            raise RuntimeError("Capture on the workspace stream (peeler.stream)")
        _lib.check(_lib.load().edp_enqueue(self._ws.handle, self.stream.cuda_stream), "enqueue")

    def capture(self):
        """Capture and instantiate the workspace's own graph (warm-up first)."""
        if not self.warmed:
            self.warmup()
        self._ws.call("edp_capture", "capture")
        self.graph = self._ws.handle
        return self.graph

    def run(self):
        """Asynchronously replay; results and the error flag remain on device."""
        if self.graph is None:
            self.capture()
        self._ws.call("edp_run", "run")

    def set_tuning(self, **knobs):
        """Work-distribution knobs (edp_tuning in edp.h: step_budget,
        subdivide_blocks, heavy_noding_work, clip_budget); none changes a
        result.  The peeler's graph is recorded again by the next run()."""
        unknown = set(knobs) - {f for f, _ in _lib.TuningC._fields_}
        if unknown:
            raise ValueError(f"unknown tuning knobs: {sorted(unknown)}")
        t = _lib.TuningC(*[int(knobs.get(f, 0)) for f, _ in _lib.TuningC._fields_])
        self._ws.call_args("edp_set_tuning", "tuning", ctypes.byref(t))
        self.graph = None  # the workspace dropped its graph; run() records it again

    def tuning(self):
        """The knobs the workspace uses (dict)."""
        t = _lib.TuningC()
        _lib.check(_lib.load().edp_get_tuning(self._ws.handle, ctypes.byref(t)), "tuning")
        return {f: int(getattr(t, f)) for f, _ in _lib.TuningC._fields_}

    def _set_predicates(self, predicates):
        if predicates not in _lib.PREDICATE_MODES:
            raise ValueError(f"predicates must be one of {sorted(_lib.PREDICATE_MODES)}")
        self._ws.call_args("edp_set_predicates", "predicates", _lib.PREDICATE_MODES[predicates])
        self.predicates = predicates

    def predicate_counts(self):
        """{class: {stage: calls}} of the last extraction when the peeler was
        made with predicates="counted" (zeros otherwise); waits for it."""
        counts = np.zeros(3 * len(_lib.PREDICATE_CLASSES), dtype=np.int64)
        _lib.check(_lib.load().edp_predicate_counts(self._ws.handle, counts.ctypes.data),
                   "predicate counts")
        rows = counts.reshape(-1, 3)
        return {c: dict(zip(_lib.PREDICATE_STAGES, map(int, row)))
                for c, row in zip(_lib.PREDICATE_CLASSES, rows)}

    def stage_times(self):
        """{stage: device ms} of the last replay of this peeler's own graph
        (run() / capture()), from timing events the graph records at each
        stage's end; waits for that replay.  The values sum to its time."""
        ms = np.zeros(len(_lib.STAGE_NAMES), dtype=np.float32)
        _lib.check(_lib.load().edp_stage_times(self._ws.handle, ms.ctypes.data), "stage times")
        return dict(zip(_lib.STAGE_NAMES, map(float, ms)))


class DevicePeeler(_Peeler):
    """Iterative per-layer clipping (warp_peel/solver.py:92-519).

    Same inputs, outputs and graph lifetime as ``EventPeeler``; handles input
    that still has unresolved surface crossings.
    """

    def __init__(self, vertices, faces, camera, settings, *, capacities=None, layers=0,
                 predicates="filtered64"):
        import torch

        self.device = _check_inputs(vertices, faces, camera, settings)
        self.n = faces.shape[0]
        self.nv = vertices.shape[0]
        self.cap = capacities or Capacities.for_mesh(self.n)
        if min(vars(self.cap).values()) < 1 or self.cap.edge_vertices > 128:
            raise ValueError("Capacities must be positive; edge_vertices must be <= 128")
        if layers < 0 or layers > self.cap.layers:
            raise ValueError("layers must be zero (all), or fit in the layer capacity")
        self.vertices, self.faces, self.camera, self.settings = vertices, faces, camera, settings
        self.limit = layers or self.cap.layers
        self.all_layers = int(layers == 0)
        self.stream = torch.cuda.Stream(self.device)
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        lib = _lib.load()
        c = _lib.DeviceCapacitiesC(*[int(getattr(self.cap, f)) for f, _ in
                                     _lib.DeviceCapacitiesC._fields_])
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(
                lib.edp_device_create(
                    vertices.data_ptr(), self.nv, faces.data_ptr(), self.n, camera.data_ptr(),
                    settings.data_ptr(), ctypes.byref(c), int(layers), self.stream.cuda_stream,
                    ctypes.byref(handle)),
                "DevicePeeler")
        self._ws = _Workspace(handle, self.device, (vertices, faces, camera, settings))
        self._ws.expose(self)
        self._set_predicates(predicates)
        self.graph = None
        self.warmed = False

    def read_status(self):
        status, _ = self._ws.read()
        return _decode_status(status)

