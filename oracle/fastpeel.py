"""ctypes wrapper of the fast-bvh-peel restatement (benchmark infrastructure).

``run`` imports a scene from host arrays once, then times ``repeat``
extractions (classification, all layers' clipping and meshing) with
``threads`` OpenMP threads, as the reference's
``geometric_peel --method fast-bvh-peel --resolved-mesh --metrics-only``
times ``algorithm_seconds`` (src/fast_peel.cpp:659-664).
"""

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "libfastpeel.so"


def build():
    source = HERE / "fast_peel.cpp"
    if not LIBRARY.exists() or LIBRARY.stat().st_mtime < source.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE), "libfastpeel.so"], check=True)
    return LIBRARY


def _lib():
    if not LIBRARY.exists():
        build()
    lib = ctypes.CDLL(str(LIBRARY))
    P = ctypes.c_void_p
    lib.fastpeel_run.argtypes = [P, P, ctypes.c_int64, P, P] + [ctypes.c_int32] * 5 + [P, P]
    lib.fastpeel_max_threads.restype = ctypes.c_int
    lib.fastpeel_regions.argtypes = [P, P, ctypes.c_int64, P, P] + [ctypes.c_int32] * 4 + \
        [ctypes.c_int64, ctypes.c_int64, P, P, P]
    return lib


def max_threads():
    return _lib().fastpeel_max_threads()


def run(vertices, faces, camera, settings, threads=1, repeat=1, bits=30, resolved=True, layers=0):
    """Returns (per-repetition seconds, {layers, patches, triangles, residual})."""
    v = np.ascontiguousarray(vertices, dtype=np.float64)
    f = np.ascontiguousarray(faces, dtype=np.int32)
    c = np.ascontiguousarray(camera, dtype=np.float64).reshape(4, 4)
    s = np.ascontiguousarray(settings, dtype=np.float64)
    seconds = np.zeros(repeat, dtype=np.float64)
    out = np.zeros(4, dtype=np.int64)
    rc = _lib().fastpeel_run(v.ctypes.data, f.ctypes.data, len(f), c.ctypes.data, s.ctypes.data,
                             threads, repeat, bits, int(resolved), layers, seconds.ctypes.data,
                             out.ctypes.data)
    if rc != 0:
        raise RuntimeError("fast-bvh-peel restatement failed (no progress or layer limit)")
    return seconds.tolist(), dict(zip(("layers", "patches", "triangles", "residual"),
                                      map(int, out)))


def regions(vertices, faces, camera, settings, threads=1, bits=30, resolved=True, layers=0):
    """One extraction's regions: a list of (layer, input face, (k, 2) float
    array in the normalised window), and the layer count."""
    v = np.ascontiguousarray(vertices, dtype=np.float64)
    f = np.ascontiguousarray(faces, dtype=np.int32)
    c = np.ascontiguousarray(camera, dtype=np.float64).reshape(4, 4)
    s = np.ascontiguousarray(settings, dtype=np.float64)
    out = np.zeros(3, dtype=np.int64)
    capacity = [max(1024, 8 * len(f)), max(8192, 64 * len(f))]
    lib = _lib()
    for _ in range(2):
        meta = np.zeros((capacity[0], 3), dtype=np.int64)
        coords = np.zeros((capacity[1], 2), dtype=np.int64)
        rc = lib.fastpeel_regions(v.ctypes.data, f.ctypes.data, len(f), c.ctypes.data,
                                  s.ctypes.data, threads, bits, int(resolved), layers,
                                  capacity[0], capacity[1], meta.ctypes.data, coords.ctypes.data,
                                  out.ctypes.data)
        if rc < 0:
            raise RuntimeError("fast-bvh-peel restatement failed (no progress or layer limit)")
        if rc == 0:
            break
        capacity = [int(out[0]), int(out[1])]
    grid = float(1 << bits)
    result, start = [], 0
    for layer, face, n in meta[: out[0]]:
        result.append((int(layer), int(face), coords[start:start + n].astype(np.float64) / grid))
        start += n
    return result, int(out[2])
