"""Many meshes or camera views peeled by one CUDA graph replay.

Each scene keeps its own ``EventPeeler`` workspace (pools, outputs, stream).
``capture()`` records every workspace's complete extraction into a single CUDA
graph: each one on its own branch, forked from the batch's capture stream and
joined back, so independent extractions of small meshes run side by side on
the GPU's 148 SMs, and one ``run()`` replays the whole batch with no host
work in between.  Outputs are read per workspace, as for a single peeler.
"""

from .events import EventPeeler


class BatchPeeler:
    """``scenes``: (vertices, faces, camera, settings) device tensors per mesh
    or view (views of one mesh may share its vertex and face tensors).
    ``capacities``: one ``EventCapacities`` for all, a list with one per
    scene, or None for ``EventCapacities.for_mesh``; ``fit=True`` sizes each
    workspace from a trial extraction (``sizing.fit_event_capacities``)
    instead.  ``tuning``: work-distribution knobs (``autotune``) for every
    workspace.  Other keyword options go to every ``EventPeeler``."""

    def __init__(self, scenes, *, capacities=None, fit=False, tuning=None, **options):
        import torch

        scenes = list(scenes)
        if not scenes:
            raise ValueError("A batch needs at least one scene")
        if isinstance(capacities, (list, tuple)):
            if len(capacities) != len(scenes):
                raise ValueError("One capacity set per scene")
            caps = list(capacities)
        else:
            caps = [capacities] * len(scenes)
        if fit:
            from .sizing import fit_event_capacities

            self.peelers = [fit_event_capacities(s, c, **options)[0] for s, c in zip(scenes, caps)]
        else:
            self.peelers = [EventPeeler(*s, capacities=c, **options) for s, c in zip(scenes, caps)]
        self.tuning = dict(tuning or {})
        if self.tuning:
            for p in self.peelers:
                p.set_tuning(**self.tuning)
        self.device = self.peelers[0].device
        self.stream = torch.cuda.Stream(self.device)
        self.graph = None

    def __len__(self):
        return len(self.peelers)

    def capture(self):
        """Warm every workspace up, then record all extractions into one graph."""
        import torch

        for p in self.peelers:
            if not p.warmed:
                p.warmup()
        for p in self.peelers:
            p.stream.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=self.stream):
            # Every branch forks from the start of the capture and joins at its
            # end; joining one before forking the next would chain them.
            for p in self.peelers:
                p.stream.wait_stream(self.stream)
            for p in self.peelers:
                with torch.cuda.stream(p.stream):
                    p.enqueue()
            for p in self.peelers:
                self.stream.wait_stream(p.stream)
        self.graph = graph
        return graph

    def run(self):
        """Asynchronously replay the batch on ``self.stream``."""
        import torch

        if self.graph is None:
            self.capture()
        with torch.cuda.stream(self.stream):
            self.graph.replay()

    def read_status(self):
        """Wait for the batch, then each workspace's decoded status and counters."""
        self.stream.synchronize()
        return [p.read_status() for p in self.peelers]
