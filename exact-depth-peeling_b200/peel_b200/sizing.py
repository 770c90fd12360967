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


def fit_event_capacities(arrays, capacities=None, attempts=8, **options):
    """Return (peeler, capacities) whose extraction of ``arrays`` does not overflow.

    Bits that no capacity can fix (invalid input, polygon vertices, edge noding)
    raise immediately."""
    cap = capacities or EventCapacities.for_mesh(arrays[1].shape[0])
    for _ in range(attempts):
        p = EventPeeler(*arrays, capacities=cap, **options)
        p.run()
        error = int(p.status[9].item())  # synchronising read of the sticky error bits
        if error == 0:
            return p, cap
        grow = {f: getattr(cap, f) * 2 for b, f in _POOL_OF_BIT.items() if error & b}
        if not grow or error & ~sum(_POOL_OF_BIT):
            p.read_status()  # raises with the reference's message
        del p
        cap = replace(cap, **grow)
    raise RuntimeError(f"pools still overflow after {attempts} doublings: {cap}")
