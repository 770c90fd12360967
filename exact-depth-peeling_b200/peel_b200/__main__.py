"""Peel a scene JSON on the GPU and write its triangle layers.

    python -m peel_b200 scene.json --out layers.npz [--method peel|events]
                        [--layers K] [--pool-scale S] [--pieces P] [--device cuda:0]

``layers.npz`` holds ``uv``, ``world``, ``sources`` (external ids) and
zero-based ``layers``; ``layers.json`` beside it records the method, the
scene and the decoded status.  Flags, file names and sidecar keys are the
reference's command line (warp_peel/__main__.py), which readers of these
files depend on.
"""

import argparse
import json
from dataclasses import replace
from pathlib import Path

import numpy as np

from . import Capacities, DevicePeeler, EventCapacities, EventPeeler
from .io import download_mesh, load_scene

SIDECAR_FORMAT = "warp-peel-approximate-v1"

# Per method: the peeler, its capacity type, and the pools --pool-scale grows.
METHODS = {
    "peel": (DevicePeeler, Capacities, ("residual", "polygons", "vertices", "triangles")),
    "events": (EventPeeler, EventCapacities,
               ("frontier", "regions", "hits", "vertices", "triangles")),
}


def parse(argv):
    parser = argparse.ArgumentParser(prog="python -m peel_b200", description=__doc__,
                                     formatter_class=argparse.RawDescriptionHelpFormatter)
    parser.add_argument("scene", type=Path)
    parser.add_argument("--out", type=Path, required=True)
    parser.add_argument("--layers", type=int, default=0, help="0 means all layers")
    parser.add_argument("--method", choices=tuple(METHODS), default="peel",
                        help="peel: iterative per-layer clipping; events: contour "
                             "subdivision with shared ray ranks")
    parser.add_argument("--pieces", type=int, help="piece budget per clipping task (peel)")
    parser.add_argument("--pool-scale", type=int, default=1,
                        help="multiply the output and work pools by this factor")
    parser.add_argument("--device", default="cuda:0")
    args = parser.parse_args(argv)
    if args.pieces is not None and args.method != "peel":
        parser.error("--pieces applies only to --method peel")
    return args


def capacities(args, faces):
    """The method's default capacities for `faces` sources, scaled and
    overridden as the flags ask."""
    _, kind, scaled = METHODS[args.method]
    base = kind.for_mesh(faces)
    changes = {name: getattr(base, name) * args.pool_scale for name in scaled}
    if args.pieces:  # 0 keeps the default, as in the reference
        changes["pieces_per_worker"] = args.pieces
    return replace(base, **changes)


def sidecar(args, status):
    return {"format": SIDECAR_FORMAT, "zero_based_layers": True, "exact_geometry": False,
            "method": args.method, "scene": str(args.scene), "output": status}


def main(argv=None):
    args = parse(argv)
    arrays, labels, _ = load_scene(args.scene, args.device)
    peeler_type = METHODS[args.method][0]
    peeler = peeler_type(*arrays, capacities=capacities(args, arrays[1].shape[0]),
                         layers=args.layers)
    peeler.run()
    mesh = download_mesh(peeler, labels)
    status = mesh.pop("status")
    args.out.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(args.out, **mesh)
    args.out.with_suffix(".json").write_text(json.dumps(sidecar(args, status), indent=2) + "\n")
    print(json.dumps(status))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
