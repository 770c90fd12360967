"""Autotuner for the peeler's work-distribution knobs.

The knobs (``edp_tuning`` in include/edp.h) decide how work is spread over
rounds, blocks and warps, never which regions or triangles come out:

* ``step_budget``: subdivision walk steps a patch spends per round (the
  queue granularity of the subdivision loop);
* ``subdivide_blocks``: subdivision blocks of four warps per SM (the tile
  width of the persistent subdivision grid);
* ``heavy_noding_work``: candidate x edge tests above which a polygon is
  noded by a warp instead of one thread;
* ``clip_budget``: DevicePeeler candidate tests per piece and clipping round.

``tune`` runs a coordinate search: starting from the defaults, each knob in
turn takes each of its values with the others fixed, and the value with the
lowest median replay time (CUDA events on the workspace stream, L2 flushed
before each replay) is kept.  Every trial's extraction must produce the same
polygon, triangle and layer counts as the first, or tuning stops with an
error.  The reference has no counterpart (its kernels fix these choices).
"""

import statistics

SPACE = {
    "step_budget": (16, 32, 48, 96, 256),
    "subdivide_blocks": (4, 8, 16),
    "heavy_noding_work": (256, 1024, 4096),
}
DEVICE_SPACE = {"clip_budget": (8, 32, 128)}


def time_replays(peeler, replays, flush):
    """Median device ms of `replays` replays of the peeler's own graph."""
    import torch

    times = []
    for _ in range(replays):
        with torch.cuda.stream(peeler.stream):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(peeler.stream)
        peeler.run()
        b.record(peeler.stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    return statistics.median(times)


def trial(make, knobs, replays, flush):
    """(median ms, output counts) of one configuration."""
    p = make()
    p.set_tuning(**knobs)
    p.capture()
    for _ in range(2):
        p.run()
    info = p.read_status()
    ms = time_replays(p, replays, flush)
    counts = (info["polygons"], info["triangles"], info["layers"])
    del p
    return ms, counts


def tune(make, space=SPACE, replays=5, log=None):
    """Coordinate search over `space` for the peeler that `make()` builds
    (uncaptured, same inputs each time).  Returns (best knobs, default ms,
    best ms, trials)."""
    import torch

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    probe = make()
    best = {k: v for k, v in probe.tuning().items() if k in space}
    del probe
    best_ms, expected = trial(make, best, replays, flush)
    default_ms = best_ms
    trials = [{"knobs": dict(best), "ms": best_ms}]
    tried = {tuple(sorted(best.items()))}
    for knob, values in space.items():
        for value in values:
            knobs = dict(best, **{knob: value})
            key = tuple(sorted(knobs.items()))
            if key in tried:
                continue
            tried.add(key)
            ms, counts = trial(make, knobs, replays, flush)
            trials.append({"knobs": knobs, "ms": ms})
            if log:
                log(f"{knobs}: {ms:.3f} ms")
            if counts != expected:
                raise RuntimeError(f"tuning changed the extraction: {knobs} gave {counts}, "
                                   f"expected {expected}")
            if ms < best_ms:
                best, best_ms = knobs, ms
    return best, default_ms, best_ms, trials
