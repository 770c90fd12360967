"""ctypes binding of libedp_b200.so (the C ABI declared in include/edp.h).

The shared library is built in-tree by ``exact-depth-peeling_b200/build.py``.
There is no fallback: a missing library raises immediately.
"""

import ctypes
from pathlib import Path

LIBRARY = Path(__file__).resolve().parent / "libedp_b200.so"
ABI_VERSION = 5  # EDP_ABI_VERSION in include/edp.h

I64 = ctypes.c_int64
I32 = ctypes.c_int32
P = ctypes.c_void_p


class EventCapacitiesC(ctypes.Structure):
    _fields_ = [(n, I64) for n in (
        "frontier", "regions", "hits", "vertices", "triangles", "rounds", "layers",
        "edge_vertices")]


class EventOptionsC(ctypes.Structure):
    _fields_ = [(n, I32) for n in ("layers", "share_regions", "propagate_ranks", "merge_regions")]


class DeviceCapacitiesC(ctypes.Structure):
    _fields_ = [(n, I64) for n in (
        "residual", "polygons", "vertices", "triangles", "workers", "pieces_per_worker",
        "layers", "edge_vertices")]


class TuningC(ctypes.Structure):
    _fields_ = [(n, I32) for n in (
        "step_budget", "subdivide_blocks", "heavy_noding_work", "clip_budget")]


class OutputsC(ctypes.Structure):
    _fields_ = [
        ("status", P), ("metrics", P), ("output_vertices", P), ("output_sizes", P),
        ("output_sources", P), ("output_layers", P), ("triangles_uv", P),
        ("triangles_world", P), ("triangle_sources", P), ("triangle_layers", P),
        ("canonical", P), ("regions", I64), ("triangles", I64), ("vertices", I64),
    ]


EXPORTS = (
    "edp_event_create", "edp_device_create", "edp_event_default_capacities",
    "edp_device_default_capacities", "edp_warmup", "edp_enqueue", "edp_capture", "edp_run",
    "edp_read_status", "edp_get_outputs", "edp_destroy", "edp_status_string",
    "edp_last_cuda_error", "edp_abi_version", "edp_run_stage", "edp_graph_kernels",
    "edp_last_error_site", "edp_weld_noalloc", "edp_stage_times", "edp_set_predicates",
    "edp_predicate_counts", "edp_workspace_bytes", "edp_tile_features", "edp_mlp_infer",
    "edp_mlp_grad", "edp_adam_step", "edp_set_tuning", "edp_get_tuning",
)

# enum edp_predicates and enum edp_predicate_class in include/edp.h.
PREDICATE_MODES = {"binary64": 0, "filtered": 1, "counted": 2, "filtered64": 3}
PREDICATE_CLASSES = ("side", "segment", "depth", "contain", "order", "clip")
PREDICATE_STAGES = ("binary32", "binary64", "exact")

# enum edp_stage in include/edp.h, in order (edp_stage_times fills one float each).
STAGE_NAMES = (
    "prepare", "subdivide", "rank_order", "rank_connectivity", "rank_samples",
    "rank_query_groups", "rank_certify", "rank_ray_grid", "rank_ray_primary", "rank_ray_heavy",
    "rank_hit_sort", "rank_assign", "rank_merge", "mesh_vertices", "mesh_index", "mesh_emit",
)

_lib = None


def load():
    """Load the library once; raise if it is missing or incomplete."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY.exists():
        raise RuntimeError(
            f"{LIBRARY.name} is not built; run exact-depth-peeling_b200/build.py "
            "(nvcc for sm_100a). There is no CPU fallback."
        )
    lib = ctypes.CDLL(str(LIBRARY))
    for name in EXPORTS:
        if not hasattr(lib, name):
            raise RuntimeError(f"{LIBRARY.name} lacks {name}")
    pp = ctypes.POINTER(P)
    lib.edp_event_create.argtypes = [P, I64, P, I64, P, P, ctypes.POINTER(EventCapacitiesC),
                                     ctypes.POINTER(EventOptionsC), P, pp]
    lib.edp_device_create.argtypes = [P, I64, P, I64, P, P, ctypes.POINTER(DeviceCapacitiesC),
                                      I32, P, pp]
    lib.edp_event_default_capacities.argtypes = [I64, ctypes.POINTER(EventCapacitiesC)]
    lib.edp_event_default_capacities.restype = None
    lib.edp_device_default_capacities.argtypes = [I64, ctypes.POINTER(DeviceCapacitiesC)]
    lib.edp_device_default_capacities.restype = None
    for name in ("edp_warmup", "edp_capture", "edp_run"):
        getattr(lib, name).argtypes = [P]
    lib.edp_enqueue.argtypes = [P, P]
    lib.edp_read_status.argtypes = [P, P, P]
    lib.edp_get_outputs.argtypes = [P, ctypes.POINTER(OutputsC)]
    lib.edp_run_stage.argtypes = [P, I32]
    lib.edp_graph_kernels.argtypes = [P, P, P]
    lib.edp_stage_times.argtypes = [P, P]
    lib.edp_set_predicates.argtypes = [P, I32]
    lib.edp_predicate_counts.argtypes = [P, P]
    lib.edp_workspace_bytes.argtypes = [P, P]
    lib.edp_set_tuning.argtypes = [P, ctypes.POINTER(TuningC)]
    lib.edp_get_tuning.argtypes = [P, ctypes.POINTER(TuningC)]
    lib.edp_tile_features.argtypes = [P, I64, P, I64, P, P, P, P, P]
    lib.edp_mlp_infer.argtypes = [P, P, I64, P, P]
    lib.edp_mlp_grad.argtypes = [P, P, P, P, I64, ctypes.c_float, P, P, P]
    lib.edp_adam_step.argtypes = [P, P, P, P, I64] + [ctypes.c_float] * 4 + [I32, P]
    lib.edp_weld_noalloc.argtypes = [P, I64, P, P]
    lib.edp_weld_noalloc.restype = ctypes.c_int
    lib.edp_destroy.argtypes = [P]
    lib.edp_destroy.restype = None
    lib.edp_status_string.argtypes = [ctypes.c_int]
    lib.edp_status_string.restype = ctypes.c_char_p
    lib.edp_last_cuda_error.restype = ctypes.c_int
    lib.edp_last_error_site.restype = ctypes.c_char_p
    lib.edp_abi_version.restype = ctypes.c_int
    if lib.edp_abi_version() != ABI_VERSION:
        raise RuntimeError(f"{LIBRARY.name} has ABI version {lib.edp_abi_version()}, this "
                           f"package needs {ABI_VERSION}: rebuild it (build.py)")
    _lib = lib
    return lib


class NativeError(RuntimeError):
    pass


def check(code, what):
    """Map a non-zero edp_status to the reference's exception types."""
    if code == 0:
        return
    lib = load()
    text = lib.edp_status_string(code).decode()
    if code == 1:
        raise ValueError(f"{what}: {text}")
    if code == 3:
        site = lib.edp_last_error_site().decode()
        raise NativeError(f"{what}: {text} (cudaError {lib.edp_last_cuda_error()} at {site})")
    raise RuntimeError(f"{what}: {text}")
