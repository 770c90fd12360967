"""Conservative pool sizing: grow exactly the pools that overflowed.

The reference leaves overflow handling to the caller ("Reallocate/recapture
explicitly with larger capacities", warp_peel/README.md:167-173; ``--pool-scale``
in warp_peel/__main__.py:96-124).  ``fit_event_capacities`` automates that
host-side: run, read the sticky error bits, double the pools they name, repeat.
Outputs never depend on the capacities, only whether they fit.
"""

from dataclasses import replace

from .events import EventCapacities, EventPeeler

# Error bit -> EventCapacities field that it names (events.py:808-814, kernels.py:17-21).
_POOL_OF_BIT = {4: "frontier", 8: "regions", 16: "vertices", 32: "triangles", 64: "layers",
                1024: "hits", 2048: "rounds"}


def _usage(p):
    """Observed use of each pool by the last extraction (status/metrics slots).
    The caller has synchronised the workspace stream."""
    status = p.status.cpu().numpy()
    metrics = p.metrics.cpu().numpy()
    return {"frontier": int(status[12]), "regions": int(status[2]), "vertices": int(status[6]),
            "triangles": int(status[3]), "hits": int(metrics[5]), "rounds": int(metrics[6])}


def fit_event_capacities(arrays, capacities=None, attempts=8, headroom=2.0, **options):
    """Return (peeler, capacities) whose extraction of ``arrays`` does not
    overflow, with ``headroom`` x the observed use of every pool.

    Atomic appends make the polygon order, and with it the query grouping and
    the hit count, vary slightly between replays, hence the headroom.  Bits
    that no capacity can fix (invalid input, polygon vertices, edge noding)
    raise immediately."""
    cap = capacities or EventCapacities.for_mesh(arrays[1].shape[0])
    for _ in range(attempts):
        p = EventPeeler(*arrays, capacities=cap, **options)
        p.run()
        p.stream.synchronize()  # the views live on the workspace stream
        error = int(p.status[9].item())
        if error == 0:
            used = _usage(p)
            tight = {f: max(getattr(cap, f) * 2, int(headroom * used[f]))
                     for f in used if used[f] * headroom > getattr(cap, f)}
            if not tight:
                return p, cap
            del p
            cap = replace(cap, **tight)
            continue
        grow = {f: getattr(cap, f) * 2 for b, f in _POOL_OF_BIT.items() if error & b}
        if not grow or error & ~sum(_POOL_OF_BIT):
            p.read_status()  # raises with the reference's message
        del p
        cap = replace(cap, **grow)
    raise RuntimeError(f"pools still overflow after {attempts} doublings: {cap}")
