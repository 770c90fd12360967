"""Host-to-host extraction of a stream of meshes, with transfers overlapped.

``PeelStream`` keeps two EventPeeler workspaces (or more) over input buffers
of one shape, each on its own CUDA stream.  ``submit(host_arrays)`` uploads
the mesh from host memory into the next workspace's inputs, replays its
graph, and then collects the previous submission: it waits for that
extraction, reads its status, and copies its triangles into pinned host
buffers on that workspace's stream.  So the device-to-host copy of mesh i
runs while mesh i + 1 is extracted, and a stream of meshes costs about
max(extraction, transfers) each instead of their sum.  ``finish()`` collects
the last submission.  The reference downloads after each extraction
(warp_peel/io.py:51-72, ``download_mesh``); this class is the same download,
pipelined.
"""

import numpy as np

from . import EventPeeler

MESH_ATTRIBUTES = ("triangles_uv", "triangles_world", "triangle_sources", "triangle_layers")


class PeelStream:
    """``template``: (vertices, faces, camera, settings) device tensors that
    fix the shapes (copied, so each workspace owns its inputs);
    ``capacities``: EventCapacities for every workspace; ``depth``: how many
    workspaces take turns.  Other keyword options go to every EventPeeler."""

    def __init__(self, template, capacities=None, depth=2, tuning=None, **options):
        import torch

        if depth < 2:
            raise ValueError("a stream needs at least two workspaces")
        self.inputs = [[t.clone() for t in template] for _ in range(depth)]
        self.peelers = [EventPeeler(*a, capacities=capacities, **options) for a in self.inputs]
        for p in self.peelers:
            if tuning:
                p.set_tuning(**tuning)
            p.capture()
        self.host = [{name: torch.empty(tuple(getattr(p, name).shape), dtype=getattr(p, name).dtype
                                        ).pin_memory() for name in MESH_ATTRIBUTES}
                     for p in self.peelers]
        self.turn = 0
        self.pending = None  # index of the workspace whose results are not collected

    def _collect(self, k):
        """Wait for workspace k's extraction, then queue the copy of its
        triangles to the host; returns (status, {name: pinned tensor view},
        an event that completes with the copy)."""
        import torch

        p = self.peelers[k]
        status = p.read_status()
        count = status["triangles"]
        views = {}
        with torch.cuda.stream(p.stream):
            for name in MESH_ATTRIBUTES:
                dst = self.host[k][name][:count]
                dst.copy_(getattr(p, name)[:count], non_blocking=True)
                views[name] = dst
            done = torch.cuda.Event()
            done.record(p.stream)
        return status, views, done

    def submit(self, host_arrays):
        """Start the extraction of one mesh (host arrays, pinned for overlap)
        and return the previous submission's (status, triangles, event), or
        None for the first.  The returned host views are valid once the event
        has completed and until this workspace is reused (``depth``
        submissions later)."""
        import torch

        k = self.turn
        p = self.peelers[k]
        with torch.cuda.stream(p.stream):
            for dst, src in zip(self.inputs[k], host_arrays):
                dst.copy_(torch.as_tensor(src).reshape(dst.shape), non_blocking=True)
        p.run()
        previous = self._collect(self.pending) if self.pending is not None else None
        self.pending = k
        self.turn = (k + 1) % len(self.peelers)
        return previous

    def finish(self):
        """Collect the last submission and wait for every queued copy."""
        result = None
        if self.pending is not None:
            result = self._collect(self.pending)
            self.pending = None
        for p in self.peelers:
            p.stream.synchronize()
        return result


def as_numpy(result):
    """(status, {name: numpy array}) of a collected result: waits for its
    copy and copies the arrays out of the pinned buffers, which the stream
    reuses ``depth`` submissions later."""
    status, views, done = result
    done.synchronize()
    return status, {name: v.numpy().copy() for name, v in views.items()}
